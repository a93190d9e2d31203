"""QGGMRFDenoiser: the qGGMRF proximal-map image denoiser (denoising.py of
mbirtorch, v0.0.2).

The denoiser is MBIR with the IDENTITY forward model: the residual image
plays the error sinogram and the forward Hessian is 1, so one subset update
is the qGGMRF direction, a closed-form step and an update of the image and
the residual at the subset's voxels (vcd_subset_denoiser,
denoising.py:35-83).  One fixed partition (granularity 16 by default) is
swept in its stored order every iteration; the denoiser never reshuffles,
so a seeded partition makes the whole sweep deterministic.

The host side mirrors the reference: the noise estimate and the
auto-regularization look at strided subsamples on the host, and the sweep
runs on the device through ``mbir_denoise_pass`` (one call per iteration,
no host synchronization per subset).
"""

import datetime

import numpy as np
import torch

from . import _lib, vcd_utils
from . import qggmrf as _qggmrf
from ._lib import ptr, require_cuda, stream_of
from ._utils import recon_param_names
from .tomography_model import TomographyModel
from .vcd_engine import make_vcd_params


def _subsample_to_host(image, row_step=1, col_step=1, slice_step=1):
    """``image[::row_step, ::col_step, ::slice_step]`` as a host numpy array;
    a tensor is strided on its own device first (denoising.py:101-163)."""
    if torch.is_tensor(image):
        return image[::row_step, ::col_step, ::slice_step].detach().contiguous().cpu().numpy()
    return np.asarray(image)[::row_step, ::col_step, ::slice_step]


class QGGMRFDenoiser(TomographyModel):
    """MAP denoiser for additive white Gaussian noise with the 3D qGGMRF
    prior (denoising.py:166-446).  The primary interface is :meth:`denoise`.

    Args:
        image_shape (tuple of int): shape of the images to denoise
            (3-dimensional).  To denoise a 2D image, use shape (1, m, n).
        compile_mode (str, optional): accepted for signature compatibility.
    """

    def __init__(self, image_shape, compile_mode='auto'):
        if len(image_shape) != 3:
            raise ValueError('image_shape must be 3-dimensional. Got image_shape={}. '
                             'To denoise a 2D image, use shape (1, m, n).'.format(image_shape))
        super().__init__(image_shape, compile_mode=compile_mode, view_params_name='None',
                         sigma_noise=None)
        self.set_params(use_ror_mask=False)
        self.set_params(sharpness=0)
        self.set_params(granularity=[16], partition_sequence=[0])

    # ── model hooks ──────────────────────────────────────────────────────
    def get_magnification(self):
        return 1.0

    def get_psf_radius(self):
        raise NotImplementedError('get_psf_radius is not implemented for QGGMRFDenoiser.')

    def verify_valid_params(self):
        super().verify_valid_params()
        sinogram_shape = self.get_params('sinogram_shape')
        image_shape = self.get_params('recon_shape')
        if tuple(image_shape) != tuple(sinogram_shape):
            raise ValueError('image_shape and sinogram_shape must be the same. \n'
                             f'Got {image_shape} for image_shape and '
                             f'{sinogram_shape} for sinogram_shape')

    def auto_set_recon_geometry(self, no_compile=False, no_warning=False):
        self.set_params(no_compile=no_compile, no_warning=no_warning,
                        recon_shape=self.get_params('sinogram_shape'))

    def auto_set_sigma_y(self, sinogram, sino_indicator, weights=1):
        self.set_params(no_warning=True, sigma_y=self.get_params('sigma_noise'),
                        auto_regularize_flag=True)

    def _check_lateral_truncation(self, sino_indicator):
        return

    def _get_sino_indicator(self, noisy_image, sigma_noise=None, verbose=1):
        """Support indicator: a small fraction of the mean magnitude plus the
        noise floor (denoising.py:295-303)."""
        if sigma_noise is None:
            sigma_noise = self.get_params('sigma_noise')
        threshold = 0.05 * np.mean(np.fabs(noisy_image)) + sigma_noise
        threshold = min(threshold, np.amax(noisy_image))
        return np.int8(noisy_image >= threshold)

    def _get_estimate_of_recon_std(self, noisy_image, support_indicator):
        """Mean over the support of the std of each voxel and its three
        backward neighbours (denoising.py:284-293)."""
        inds = np.where(support_indicator)
        vals = np.stack([noisy_image[inds[0], inds[1], inds[2]],
                         noisy_image[inds[0] - 1, inds[1], inds[2]],
                         noisy_image[inds[0], inds[1] - 1, inds[2]],
                         noisy_image[inds[0], inds[1], inds[2] - 1]], axis=0)
        return np.mean(np.std(vals, axis=0))

    def estimate_image_noise_std(self, image):
        """Noise std from a strided subsample of at most ~5 million points:
        two passes of support indicator + neighbour-difference std
        (denoising.py:256-282)."""
        num_rows, num_cols, num_slices = (int(n) for n in tuple(image.shape))
        num_elements = num_rows * num_cols * num_slices
        num_pts_to_use = np.minimum(5_000_000, num_elements)
        stride = round((num_elements / num_pts_to_use) ** (1 / 3))
        small = _subsample_to_host(image, stride, stride, stride)
        indicator = self._get_sino_indicator(small, sigma_noise=0.0)
        sigma_noise = self._get_estimate_of_recon_std(small, indicator)
        indicator = self._get_sino_indicator(small, sigma_noise=sigma_noise)
        return self._get_estimate_of_recon_std(small, indicator)

    def recon(self, *args, **kwargs):
        raise NotImplementedError('recon is not implemented for QGGMRFDenoiser.  '
                                  'Use `denoise` instead.')

    # ── denoising ────────────────────────────────────────────────────────
    def denoise(self, image, sigma_noise=None, use_ror_mask=False, init_image=None,
                max_iterations=15, stop_threshold_change_pct=0.2, first_iteration=0,
                logfile_path='~/.mbirtorch/logs/recon.log', print_logs=True,
                output_sharded=False):
        """MAP denoising of ``image`` (AWGN, qGGMRF prior).  ``sigma_noise``
        None estimates it from the image.  The pixel partition is drawn from
        numpy's global random generator.  Returns (denoised_image,
        denoiser_dict) as the reference does (denoising.py:316-446)."""
        self.setup_logger(logfile_path=logfile_path, print_logs=print_logs)
        self._require_cuda()
        self.set_params(no_warning=True, use_ror_mask=use_ror_mask)
        if sigma_noise is None:
            sigma_noise = self.estimate_image_noise_std(image)
        self.set_params(no_warning=True, sigma_noise=sigma_noise)
        self.logger.info('Initializing QGGMRFDenoiser')

        num_rows = int(tuple(image.shape)[0])
        sampled_rows = self.subsample_views(np.arange(num_rows))
        row_step = int(sampled_rows[1] - sampled_rows[0]) if sampled_rows.size > 1 else 1
        small = _subsample_to_host(image, row_step=row_step)
        verbose = self.get_params('verbose')
        self.set_params(no_warning=True, verbose=0)
        regularization_params = self.auto_set_regularization_params(small)
        self.set_params(no_warning=True, verbose=verbose)

        image_shape, granularity = self.get_params(['recon_shape', 'granularity'])
        partition_sequence = self.get_params('partition_sequence')
        partition = vcd_utils.gen_set_of_pixel_partitions(
            image_shape, [granularity[partition_sequence[0]]], device=self.torch_device,
            use_ror_mask=self.get_params('use_ror_mask'))[0]

        fm_constant = 1.0 / (self.get_params('sigma_y') ** 2.0)
        nbr, sigma_x, p, q, T = self.get_params(['qggmrf_nbr_wts', 'sigma_x', 'p', 'q', 'T'])
        prm = make_vcd_params(fm_constant, sigma_x, p, q, T, _qggmrf.get_b_from_nbr_wts(nbr),
                              1.5, False, _lib.MBIR_F32)
        stop_thresh = stop_threshold_change_pct / 100.0

        image_t = self._recon_device(image)
        init_t = image_t if init_image is None else self._recon_device(init_image)
        S = int(image_shape[2])
        flat = init_t.clone().reshape(-1, S).contiguous()
        flat_err = (image_t.reshape(-1, S) - flat).contiguous()
        require_cuda(flat, flat_err, partition)
        K, n = partition.shape
        ws = torch.empty(int(_lib.query(flat.device, 'mbir_denoise_workspace_size', S, n)),
                         dtype=torch.uint8, device=flat.device)
        accum = torch.zeros(2, dtype=torch.float64, device=flat.device)
        host = torch.empty(3, dtype=torch.float64, pin_memory=True)
        nmae_update = np.zeros(max_iterations)
        alpha_values = np.zeros(max_iterations)
        num_iters = 0
        self.logger.info('Starting VCD iterations')
        with torch.no_grad():
            for i in range(max_iterations):
                accum.zero_()
                _lib.call(flat.device, 'mbir_denoise_pass', int(image_shape[0]),
                          int(image_shape[1]), S, prm, ptr(flat), ptr(flat_err), ptr(partition),
                          K, n, ptr(accum), ptr(ws), ws.numel(), stream_of(flat.device))
                l1 = torch.sum(torch.abs(flat)).to(torch.float64)
                host.copy_(torch.cat([accum, l1.reshape(1)]), non_blocking=True)
                torch.cuda.current_stream(flat.device).synchronize()
                ell1, alpha_sum, image_l1 = (float(v) for v in host.numpy())
                nmae = ell1 / image_l1
                nmae_update[i] = nmae
                alpha_values[i] = alpha_sum / K
                num_iters += 1
                if verbose >= 1 and (i % 5) == 0:
                    self.logger.info('After iteration {} of a max of {}: Pct change={:.4f}'
                                     .format(i + first_iteration, max_iterations, 100 * nmae))
                if nmae < stop_thresh:
                    break
        denoised = flat.reshape(tuple(image_shape))
        recon_params = dict(zip(recon_param_names, [
            int(num_iters), granularity, partition_sequence, None, None, regularization_params,
            [100 * float(v) for v in nmae_update[:num_iters]],
            [float(v) for v in alpha_values[:num_iters]], None]))
        self.close_log_file()
        notes = 'Reconstruction completed: {}\n\n'.format(datetime.datetime.now())
        denoiser_dict = self.get_recon_dict(recon_params, notes=notes)
        return self._out(denoised, output_sharded), denoiser_dict
