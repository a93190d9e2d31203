"""TomographyModel: the reference's public model API over the sm_100a path.

Public surface kept from mbirtorch (reference v0.0.2, tomography_model.py):
constructor, ``get_params``/``set_params``, ``forward_project``,
``back_project``, ``sparse_forward_project``, ``sparse_back_project``,
``compute_hessian_diagonal``, ``recon``, ``initialize_recon``,
``auto_set_regularization_params``, ``get_forward_model_loss``,
``create_vcd_subset_updater``, ``vcd_partition_iterator``, ``recon_direct``
(geometry subclasses), ``get_recon_dict``, ``scale_recon_shape``,
``full_indices_device``.  Public inputs may be numpy arrays or tensors;
outputs are numpy unless ``output_sharded=True`` (a device tensor; there is
one device per model, so "sharded" is the single-device case).

What differs by design:

* All compute runs in libmbir_b200.so on one CUDA device; a model on a
  machine without one can be built and configured but raises on compute.
* ``compile_mode`` and ``view_batch_size`` are accepted for signature
  compatibility and have no effect: the kernels hold no per-view transient.
* The VCD loop state is resident on the device in the channel-major layout
  (vcd_engine.py); ``storage_dtype`` ('float32', 'bfloat16', 'float16')
  picks the precision of the error sinogram, weights and delta sinogram.
"""

import datetime
import os
import warnings

import numpy as np
import torch

from . import tomography_utils, vcd_utils
from . import qggmrf as _qggmrf
from ._utils import AUTO_REGULARIZATION_PARAM_NAMES, Param, recon_param_names
from .kernels import DeviceProjector
from .parameter_handler import ParameterHandler
from .vcd_engine import (ResidentSinogram, VcdEngine, make_vcd_params, order_array,
                         storage_code)

_F32_EPS = float(np.finfo(np.float32).eps)


def _default_device():
    if torch.cuda.is_available():
        return torch.device('cuda', torch.cuda.current_device())
    return torch.device('cpu')


class _DeferredPartitions:
    """The pixel partitions of a recon, one per granularity, drawn from
    numpy's global generator (gen_pixel_partition, in granularity order) at
    the first access rather than at construction."""

    def __init__(self, recon_shape, granularity, use_ror_mask):
        self._args = (tuple(recon_shape), list(granularity), use_ror_mask)
        self._parts = None

    def _get(self):
        if self._parts is None:
            shape, gran, ror = self._args
            self._parts = [vcd_utils.gen_pixel_partition(shape, n, use_ror_mask=ror)
                           for n in gran]
        return self._parts

    def __len__(self):
        return len(self._args[1])

    def __getitem__(self, k):
        return self._get()[k]

    def __iter__(self):
        return iter(self._get())


class TomographyModel(ParameterHandler):
    """Base class of the geometry models (see ParallelBeamModel,
    ConeBeamModel)."""

    def __init__(self, sinogram_shape, view_batch_size=None, compile_mode='auto', **kwargs):
        super().__init__()
        self.view_batch_size = view_batch_size
        self.compile_mode = compile_mode
        self.storage_dtype = 'float32'
        # With 16-bit storage the resident error sinogram is re-formed from
        # the measured one every this many iterations.  None picks: never for
        # float32; every 5 iterations for float16, whose 11-bit significand
        # keeps the drift of in-place updates below the quantization error
        # over 5 iterations; every iteration for bfloat16 (8 bits).
        self.error_refresh_interval = None
        # bfloat16 storage: the last iterations run with the error sinogram
        # re-formed in float16 (same bytes, 3 more significand bits)
        self.bf16_finish_iterations = 3
        self._torch_device = None
        self._projector = None
        self._full_indices_cache = None
        self.prox_data = None
        for key, val in kwargs.items():
            self.params[key] = Param(val, True)
        self.set_params(no_compile=True, no_warning=True,
                        sinogram_shape=tuple(int(s) for s in sinogram_shape))
        self.auto_set_recon_geometry(no_compile=True, no_warning=True)
        self.verify_valid_params()

    # ── device ──────────────────────────────────────────────────────────────
    @property
    def torch_device(self):
        if self._torch_device is None:
            self._torch_device = _default_device()
        return self._torch_device

    @torch_device.setter
    def torch_device(self, value):
        self._torch_device = torch.device(value)
        self.refresh_device_bindings()

    def configure_devices(self, devices=None, num_devices=None, like=None):
        """Pin the model to ONE device.  The sm_100a path runs one model per
        GPU (independent jobs on other GPUs are separate models); a request
        for several devices raises."""
        if like is not None:
            devices = [like.torch_device]
        if num_devices is not None and int(num_devices) != 1:
            raise ValueError('mbirtorch_b200 runs each model on one device; '
                             f'got num_devices={num_devices}')
        if devices is not None:
            devices = list(devices)
            if len(devices) != 1:
                raise ValueError('mbirtorch_b200 runs each model on one device; '
                                 f'got {len(devices)} devices')
            self.torch_device = devices[0]

    def refresh_device_bindings(self):
        self._projector = None
        self._full_indices_cache = None

    @property
    def projector(self):
        """The device projector pair of the current geometry."""
        if self._projector is None:
            self._require_cuda()
            self._projector = DeviceProjector(self._geometry(), self._view_params_array(),
                                              self.torch_device)
        return self._projector

    def _require_cuda(self):
        if self.torch_device.type != 'cuda':
            raise RuntimeError('mbirtorch_b200 computes with sm_100a CUDA kernels only; no CUDA '
                               'device is available (there is no CPU fallback).')

    def set_storage_precision(self, storage_dtype):
        """Precision of the resident error sinogram, weights and delta
        sinogram in recon(): 'float32' (default), 'bfloat16' or 'float16'."""
        storage_code(storage_dtype)
        self.storage_dtype = storage_dtype

    # ── geometry hooks ──────────────────────────────────────────────────────
    def get_magnification(self):
        raise NotImplementedError

    def get_psf_radius(self):
        raise NotImplementedError

    def auto_set_recon_geometry(self, no_compile=False, no_warning=False):
        raise NotImplementedError

    def _geometry(self):
        raise NotImplementedError

    def _view_params_array(self):
        raise NotImplementedError

    def _dc_damping_profile(self):
        return None

    def recon_direct(self, sinogram, filter_name="ramp", output_sharded=False):
        raise NotImplementedError

    # ── helpers ─────────────────────────────────────────────────────────────
    def _full_indices(self):
        recon_shape, use_ror_mask = self.get_params(['recon_shape', 'use_ror_mask'])
        return vcd_utils.gen_full_indices(recon_shape, use_ror_mask=use_ror_mask)

    def full_index_count(self):
        return int(np.shape(self._full_indices())[0])

    def full_indices_device(self):
        recon_shape, use_ror_mask = self.get_params(['recon_shape', 'use_ror_mask'])
        key = (tuple(recon_shape), use_ror_mask if isinstance(use_ror_mask, bool) else None,
               str(self.torch_device))
        if key[1] is None:
            return torch.as_tensor(self._full_indices(), dtype=torch.int64,
                                   device=self.torch_device)
        if self._full_indices_cache is None or self._full_indices_cache[0] != key:
            idx = torch.as_tensor(self._full_indices(), dtype=torch.int64,
                                  device=self.torch_device)
            self._full_indices_cache = (key, idx)
        return self._full_indices_cache[1]

    def _to_device(self, array):
        return torch.as_tensor(array, dtype=torch.float32, device=self.torch_device)

    def _sino_device(self, sinogram):
        self._require_cuda()
        sino = self._to_device(sinogram)
        num_views = self.get_params('sinogram_shape')[0]
        if sino.shape[0] != num_views:
            raise ValueError(f'Cannot place the sinogram: its view axis has size {sino.shape[0]}, '
                             f'but the model expects {num_views} views.')
        return sino

    def _recon_device(self, recon):
        self._require_cuda()
        recon = self._to_device(recon)
        num_slices = self.get_params('recon_shape')[2]
        if recon.shape[-1] != num_slices:
            raise ValueError(f'Cannot place the reconstruction: its slice axis has size '
                             f'{recon.shape[-1]}, but the model expects {num_slices} slices.')
        return recon

    @staticmethod
    def _out(t, output_sharded):
        if output_sharded:
            return t
        t = t.detach()
        if not t.is_cuda:
            return t.numpy()
        # Through a pinned staging buffer (reused by torch's host caching
        # allocator): one DMA at link speed and one host copy, where a
        # pageable copy stages through the driver at a fraction of the rate.
        host = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        host.copy_(t)
        return host.numpy().copy()

    # ── projections ─────────────────────────────────────────────────────────
    def sparse_forward_project(self, voxel_values, pixel_indices):
        """Cylinders (P, S) at ``pixel_indices`` -> (V, R, C) device tensor."""
        vals = self._recon_device(voxel_values)
        idx = torch.as_tensor(pixel_indices, dtype=torch.int64, device=self.torch_device)
        return self.projector.forward(vals, idx)

    def sparse_back_project(self, sinogram, pixel_indices, coeff_power=1):
        """(V, R, C) sinogram -> (P, S) cylinders at ``pixel_indices``."""
        sino = self._sino_device(sinogram)
        idx = torch.as_tensor(pixel_indices, dtype=torch.int64, device=self.torch_device)
        return self.projector.back(sino, idx, coeff_power=coeff_power)

    def forward_project(self, recon, output_sharded=False):
        """Full forward projection of a (rows, cols, slices) volume (over the
        ROR pixels when use_ror_mask is set)."""
        recon = self._recon_device(recon)
        idx = self.full_indices_device()
        flat = recon.reshape(-1, recon.shape[-1])
        return self._out(self.projector.forward_volume(flat, idx), output_sharded)

    def back_project(self, sinogram, output_sharded=False):
        """Full back projection to a (rows, cols, slices) volume (zero outside
        the ROR when use_ror_mask is set)."""
        recon_shape = self.get_params('recon_shape')
        cyl = self.sparse_back_project(sinogram, self.full_indices_device())
        vol = torch.zeros((recon_shape[0] * recon_shape[1], cyl.shape[-1]),
                          dtype=torch.float32, device=self.torch_device)
        vol[self.full_indices_device()] = cyl
        return self._out(vol.reshape(tuple(recon_shape[:2]) + (cyl.shape[-1],)), output_sharded)

    def compute_hessian_diagonal(self, weights=None, output_sharded=False, indices=None):
        """Back projection of the weights with squared coefficients
        (tomography_model.py:1951-2032)."""
        sinogram_shape, recon_shape = self.get_params(['sinogram_shape', 'recon_shape'])
        if weights is None:
            self._require_cuda()
            w = torch.ones(tuple(sinogram_shape), dtype=torch.float32, device=self.torch_device)
        else:
            if tuple(weights.shape) != tuple(sinogram_shape):
                raise ValueError('Weights must be constant or an array compatible with sinogram'
                                 f'\nGot weights.shape = {tuple(weights.shape)}, but '
                                 f'sinogram.shape = {tuple(sinogram_shape)}')
            w = self._sino_device(weights)
        num_grid = int(recon_shape[0] * recon_shape[1])
        dense = indices is None
        idx = (torch.arange(num_grid, dtype=torch.int64, device=self.torch_device) if dense
               else torch.as_tensor(indices, dtype=torch.int64, device=self.torch_device))
        cyl = self.projector.back(w, idx, coeff_power=2)
        if dense:
            vol = cyl
        else:
            vol = torch.zeros((num_grid, cyl.shape[-1]), dtype=torch.float32,
                              device=self.torch_device)
            vol.index_copy_(0, idx, cyl)
        return self._out(vol.reshape(tuple(recon_shape[:2]) + (cyl.shape[-1],)), output_sharded)

    def get_voxels_at_indices(self, recon, indices):
        return recon.reshape((-1, recon.shape[-1]))[indices]

    # ── direct recon (filtered back projection) ────────────────────────────
    def _apply_direct_recon_filter(self, sinogram, filter_name, filter_scale,
                                   output_sharded=False, row_weight=None):
        sino = self._sino_device(sinogram)
        num_views, _, num_channels = self.get_params('sinogram_shape')
        filt = tomography_utils.generate_direct_recon_filter(num_channels, filter_name)
        filt = filt * np.float32(filter_scale * (np.pi / num_views))
        ft = torch.as_tensor(filt, device=self.torch_device)
        out = tomography_utils.apply_row_filter(sino, ft, row_weight=row_weight)
        return self._out(out, output_sharded)

    # ── auto-regularization (host numpy, tomography_model.py:2057-2276) ────
    def auto_set_regularization_params(self, sinogram, weights=None):
        # Only a ~20-view subsample reaches the host (subsample_views takes
        # it on the device for a tensor).
        if self.get_params('auto_regularize_flag'):
            small = self.subsample_views(sinogram)
            small_w = 1 if weights is None else self.subsample_views(weights)
            indicator = self._get_sino_indicator(small, verbose=self.get_params('verbose'))
            self._check_lateral_truncation(indicator)
            self.auto_set_sigma_y(small, indicator, small_w)
            recon_std = self._get_estimate_of_recon_std(small, indicator)
            self.auto_set_sigma_x(recon_std)
            self.auto_set_sigma_prox(recon_std)
        vals = [float(v) for v in self.get_params(list(AUTO_REGULARIZATION_PARAM_NAMES))]
        return dict(zip(AUTO_REGULARIZATION_PARAM_NAMES, vals))

    def _check_lateral_truncation(self, indicator):
        if np.all(indicator):
            return
        edge = float(np.mean(np.logical_or(indicator[:, :, 0], indicator[:, :, -1])))
        if edge > 0.02 and self.get_params('verbose') > 0:
            warnings.warn(f"Lateral FoV truncation detected: the object support reaches the "
                          f"detector's edge channels in {edge:.0%} of the sampled view-rows.  "
                          f"Consider using scale_recon_shape(s, s) where s >= 1.1 to improve "
                          f"image quality.")

    def auto_set_sigma_y(self, sinogram, sino_indicator, weights=1):
        if torch.is_tensor(sinogram):
            sinogram = sinogram.detach().cpu().numpy()
        if torch.is_tensor(weights):
            weights = weights.detach().cpu().numpy()
        snr_db = self.get_params('snr_db')
        magnification = self.get_magnification()
        delta_voxel, delta_det_channel = self.get_params(['delta_voxel', 'delta_det_channel'])
        signal_rms = float(np.average(weights * np.asarray(sinogram) ** 2, None,
                                      sino_indicator) ** 0.5)
        rel_noise_std = 10 ** (-snr_db / 20)
        pitch_rel = delta_voxel / (delta_det_channel / magnification)
        sigma_y = np.float32(rel_noise_std * signal_rms * (pitch_rel ** 0.5))
        self.set_params(no_warning=True, sigma_y=float(sigma_y), auto_regularize_flag=True)

    def auto_set_sigma_x(self, recon_std):
        sigma_x = np.float32(0.2 * (2 ** self.get_params('sharpness')) * recon_std)
        self.set_params(no_warning=True, sigma_x=float(sigma_x), auto_regularize_flag=True)

    def auto_set_sigma_prox(self, recon_std):
        sigma_prox = np.float32(0.2 * (2 ** self.get_params('sharpness')) * recon_std)
        self.set_params(no_warning=True, sigma_prox=float(sigma_prox), auto_regularize_flag=True)

    @staticmethod
    def subsample_views(array, max_views_to_use=20):
        if torch.is_tensor(array):
            array = array.detach()
            n = array.shape[0]
            step = max(n // min(max_views_to_use, n), 1)
            return array[::step].cpu().numpy()
        n = array.shape[0]
        step = max(n // min(max_views_to_use, n), 1)
        return np.array(array[::step])

    @staticmethod
    def _get_sino_indicator(sinogram, verbose=1):
        sinogram = np.asarray(sinogram)
        if np.iscomplexobj(sinogram):
            raise TypeError("sinogram must be real-valued; got complex dtype.")
        if not np.isfinite(sinogram).all():
            raise ValueError("sinogram contains NaN and/or Inf values.")
        left, right = vcd_utils.estimate_background_cluster_boundaries(sinogram)
        threshold = right + (right - left)
        max_sino = np.max(sinogram)
        if max_sino <= 0:
            if verbose > 0:
                warnings.warn("Sinogram contains no positive values. This may lead to a "
                              "contrast reversed reconstruction.")
            return np.ones_like(sinogram, dtype=np.int8)
        if max_sino < threshold:
            if verbose > 0:
                warnings.warn('\nUnable to determine sinogram background. This may affect '
                              'regularization.\n')
            return np.ones_like(sinogram, dtype=np.int8)
        object_median = np.median(sinogram[sinogram >= threshold])
        return np.int8(sinogram >= 0.25 * object_median)

    def _get_estimate_of_recon_std(self, sinogram, sino_indicator):
        delta_det_channel, delta_voxel = self.get_params(['delta_det_channel', 'delta_voxel'])
        recon_shape = self.get_params('recon_shape')
        magnification = self.get_magnification()
        num_det_channels = sinogram.shape[-1]
        typical_value = np.average(np.abs(sinogram), weights=sino_indicator)
        path_space = (2 * recon_shape[0] * recon_shape[1]) / (recon_shape[0] + recon_shape[1]) \
            * delta_voxel
        path_sino = num_det_channels * delta_det_channel / magnification
        return typical_value / np.minimum(path_space, path_sino)

    # ── losses ──────────────────────────────────────────────────────────────
    @staticmethod
    def get_forward_model_loss(error_sinogram, sigma_y, weights=None, normalize=True):
        if weights is None:
            weights, avg_weight = 1, 1
        elif np.ndim(weights) == 0:
            avg_weight = weights
        else:
            weights = torch.as_tensor(weights, dtype=torch.float32, device=error_sinogram.device)
            avg_weight = torch.mean(weights)
        if normalize:
            wsq = torch.sum(error_sinogram * error_sinogram * weights)
            return torch.sqrt(wsq / (avg_weight * float(error_sinogram.numel()))) / sigma_y
        return (1.0 / (2 * sigma_y ** 2)) * torch.sum((error_sinogram * error_sinogram) * weights)

    # ── the VCD engine seam ─────────────────────────────────────────────────
    def _vcd_params(self, storage, prox_flat=None):
        nbr, sigma_x, p, q, T = self.get_params(['qggmrf_nbr_wts', 'sigma_x', 'p', 'q', 'T'])
        b = _qggmrf.get_b_from_nbr_wts(nbr)
        fm_constant = 1.0 / (self.get_params('sigma_y') ** 2.0)
        prox_constant, prox_ptr = 0.0, None
        if prox_flat is not None:
            # 1 / sigma_prox^2 in double precision, rounded once to float32 as
            # the reference's python-scalar * float32-tensor product does.
            prox_constant = 1.0 / (self.get_params('sigma_prox') ** 2.0)
            prox_ptr = prox_flat.data_ptr()
        return make_vcd_params(fm_constant, sigma_x, p, q, T, b, self.get_params('max_alpha'),
                               self.get_params('positivity_flag') is True, storage,
                               prox_constant, prox_ptr)

    def _prox_flat(self, prox_input):
        """The proximal-map input as a contiguous (N*N, S) float32 device
        array (tomography_model.py:2842-2860: shape checked before
        flattening)."""
        if prox_input is None:
            return None
        recon_shape = tuple(self.get_params('recon_shape'))
        if tuple(prox_input.shape) != recon_shape:
            raise ValueError('prox_input does not have the correct size. \n'
                             f'Expected {recon_shape}, got shape '
                             f'{tuple(prox_input.shape)} for prox_input shape.')
        return self._recon_device(prox_input).reshape(-1, recon_shape[2]).contiguous()

    def _make_engine(self, fm_hessian_flat, weights_res, storage, max_subset_pixels=1,
                     prox_flat=None):
        dc = self._dc_damping_profile()
        dc_t = None if dc is None else torch.as_tensor(dc, dtype=torch.float32,
                                                       device=self.torch_device)
        engine = VcdEngine(self._geometry(), self.projector.view_params,
                           self._vcd_params(storage, prox_flat), fm_hessian_flat,
                           weights=weights_res, dc_profile=dc_t,
                           max_subset_pixels=max_subset_pixels)
        engine.prox_flat = prox_flat  # the parameters point at it
        return engine

    def create_vcd_subset_updater(self, fm_hessian, weights, prox_input=None):
        """The subset updater of tomography_model.py:2434-2660: returns
        ``vcd_subset_updater(flat_recon, error_sinogram, pixel_indices)``
        updating both in place and returning
        ``(flat_recon, error_sinogram, ell1, alpha, delta_sumsq)`` as device
        values.  ``error_sinogram`` may be the resident form
        (:class:`ResidentSinogram`) or a (V, R, C) float32 CUDA tensor
        (converted in and out around the update).  With ``prox_input``
        (the recon's shape) the prior is the proximal map's instead of
        qGGMRF."""
        const_weights = not torch.is_tensor(weights) and not isinstance(weights,
                                                                       ResidentSinogram)
        if const_weights and abs(weights - 1) > 1e-5:
            raise ValueError('Constant weights must have value 1.')
        storage = storage_code(self.storage_dtype)
        H = self._recon_device(fm_hessian)
        H = H.reshape(-1, H.shape[-1]).contiguous()
        w_res = None
        if not const_weights:
            w_res = (weights if isinstance(weights, ResidentSinogram)
                     else ResidentSinogram.from_vrc(self._sino_device(weights), storage))
        engine = self._make_engine(H, w_res, storage, prox_flat=self._prox_flat(prox_input))

        def vcd_subset_updater(flat_recon, error_sinogram, pixel_indices):
            plain = torch.is_tensor(error_sinogram)
            err = (ResidentSinogram.from_vrc(error_sinogram, storage) if plain
                   else error_sinogram)
            ell1, alpha, sumsq = engine.subset_update(flat_recon, err, pixel_indices)
            if plain:
                error_sinogram.copy_(err.to_vrc())
            return flat_recon, error_sinogram, ell1, alpha, sumsq

        vcd_subset_updater.engine = vcd_subset_updater.engine_ = engine
        return vcd_subset_updater

    def vcd_partition_iterator(self, vcd_subset_updater, flat_recon, error_sinogram, partition):
        """One VCD iteration over ``partition`` (tomography_model.py:2662-2697):
        one np.random.permutation of the subset order, then every subset.
        Returns (flat_recon, error_sinogram, ell1, mean alpha, delta_sumsq)."""
        order = order_array(partition.shape[0])
        engine = getattr(vcd_subset_updater, 'engine', None)
        if engine is not None and isinstance(error_sinogram, ResidentSinogram):
            acc = torch.zeros(2 + self.get_params('recon_shape')[2], dtype=torch.float64,
                              device=self.torch_device)
            engine.partition_pass(flat_recon, error_sinogram, partition, order, acc)
            return (flat_recon, error_sinogram, acc[0], acc[1] / partition.shape[0], acc[2:])
        ell1, alpha_sum, sumsq = 0, 0, 0
        for k in order:
            flat_recon, error_sinogram, e1, a, s = vcd_subset_updater(
                flat_recon, error_sinogram, partition[int(k)])
            ell1, alpha_sum, sumsq = ell1 + e1, alpha_sum + a, sumsq + s
        return flat_recon, error_sinogram, ell1, alpha_sum / partition.shape[0], sumsq

    # ── reconstruction ──────────────────────────────────────────────────────
    def initialize_recon(self, sinogram, weights=None, init_recon=None, max_iterations=15,
                         first_iteration=0, logfile_path='~/.mbirtorch/logs/recon.log',
                         print_logs=True, _defer_partitions=False):
        """Partitions (np.random, reference order), partition sequence, input
        checks and auto-regularization (tomography_model.py:3015-3095).
        ``_defer_partitions`` (internal): return the partitions as a
        _DeferredPartitions list, drawn from the global generator at first
        use; recon() uses it so that the host draws them while the device
        runs the initial reconstruction and the Hessian.  Nothing between
        the two points draws random numbers, so the partitions are the
        same."""
        if first_iteration == 0 or self.log_buffer is None:
            self.setup_logger(logfile_path=logfile_path, print_logs=print_logs)
        from . import __version__
        self.logger.info(f'MBIRTorch-B200 Version = {__version__}')
        recon_shape, granularity, use_ror_mask = self.get_params(
            ['recon_shape', 'granularity', 'use_ror_mask'])
        if _defer_partitions:
            partitions = _DeferredPartitions(recon_shape, granularity, use_ror_mask)
        else:
            partitions = [vcd_utils.gen_pixel_partition(recon_shape, n, use_ror_mask=use_ror_mask)
                          for n in granularity]
        seq = vcd_utils.gen_partition_sequence(self.get_params('partition_sequence'),
                                               max_iterations=max_iterations)
        seq = seq[first_iteration:]
        on_device = self.torch_device.type == 'cuda'
        if not torch.is_tensor(sinogram):
            s_np = np.asarray(sinogram)
            if np.iscomplexobj(s_np):
                raise TypeError("sinogram must be real-valued; got complex dtype.")
            if on_device:
                # The host array goes to the device once; the checks and the
                # recon then read the device copy.
                sinogram = self._sino_device(s_np)
            elif not np.isfinite(s_np).all():
                raise ValueError("sinogram contains NaN and/or Inf values.")
        if torch.is_tensor(sinogram):
            if sinogram.is_complex():
                raise TypeError("sinogram must be real-valued; got complex dtype.")
            if on_device and not sinogram.is_cuda:
                # A host tensor (pinned or not) goes to the device before the
                # checks, which then run there instead of on the host cores.
                sinogram = self._sino_device(sinogram)
            if not bool(torch.isfinite(sinogram).all()):
                raise ValueError("sinogram contains NaN and/or Inf values.")
        if weights is not None:
            if not torch.is_tensor(weights) and on_device and np.ndim(weights) > 0:
                weights = self._sino_device(np.asarray(weights))
            elif (torch.is_tensor(weights) and on_device and not weights.is_cuda
                  and weights.ndim > 0):
                weights = self._sino_device(weights)
            if torch.is_tensor(weights):
                if not bool(torch.isfinite(weights).all()):
                    raise ValueError("weights contains NaN and/or Inf values.")
                if bool((weights < 0).any()):
                    raise ValueError("weights contain negative values.")
                if bool((weights == 0).all()):
                    raise ValueError("all weights are zero.")
            else:
                w_np = np.asarray(weights)
                if not np.isfinite(w_np).all():
                    raise ValueError("weights contains NaN and/or Inf values.")
                if (w_np < 0).any():
                    raise ValueError("weights contain negative values.")
                if (w_np == 0).all():
                    raise ValueError("all weights are zero.")
        reg = self.auto_set_regularization_params(sinogram, weights=weights)
        return sinogram, weights, init_recon, partitions, seq, granularity, reg

    def recon(self, sinogram, weights=None, init_recon=None, max_iterations=15,
              stop_threshold_change_pct=0.2, first_iteration=0,
              logfile_path='~/.mbirtorch/logs/recon.log', print_logs=True,
              output_sharded=False):
        """MBIR reconstruction by multi-granular VCD (tomography_model.py:
        3097-3204).  Returns (recon, recon_dict)."""
        (sinogram, weights, init_recon, partitions, seq, granularity,
         reg) = self.initialize_recon(sinogram, weights, init_recon, max_iterations,
                                      first_iteration, logfile_path=logfile_path,
                                      print_logs=print_logs, _defer_partitions=True)
        with torch.no_grad():
            recon, losses = self._vcd_recon(sinogram, partitions, seq, stop_threshold_change_pct,
                                            weights=weights, init_recon=init_recon,
                                            first_iteration=first_iteration)
        fm_rmse = [float(v) for v in losses[0]]
        recon_params = dict(zip(recon_param_names, [
            len(fm_rmse), granularity, [int(v) for v in seq], fm_rmse, [0], reg,
            [100 * float(v) for v in losses[2]], [float(v) for v in losses[3]],
            [[float(x) for x in row] for row in losses[4]]]))
        if logfile_path:
            self.logger.info('Logs written to {}'.format(
                os.path.abspath(os.path.expanduser(logfile_path))))
        for h in list(self.logger.handlers):
            h.flush()
        self.close_log_file()
        notes = 'Reconstruction completed: {}\n\n'.format(datetime.datetime.now())
        recon_dict = self.get_recon_dict(recon_params, notes=notes)
        return self._out(recon, output_sharded), recon_dict

    def _vcd_recon(self, sinogram, partitions, partition_sequence, stop_threshold_change_pct,
                   weights=None, init_recon=None, prox_input=None, compute_prior_loss=False,
                   first_iteration=0, init_error_sinogram=None, fm_hessian=None,
                   return_checkpoint=False):
        """The device VCD loop (tomography_model.py:2699-3013).  The loop
        state -- recon, resident error sinogram, Hessian -- stays on the
        device; one host synchronization per iteration reads the stats."""
        from .vcd_run import VcdRun
        run = VcdRun(self, sinogram, partitions, partition_sequence, stop_threshold_change_pct,
                     weights=weights, init_recon=init_recon,
                     init_error_sinogram=init_error_sinogram, fm_hessian=fm_hessian,
                     first_iteration=first_iteration, prox_input=prox_input).run()
        if return_checkpoint:
            return run.recon3d(), run.losses(), run.checkpoint()
        return run.recon3d(), run.losses()

    def prox_map(self, prox_input, sinogram, sigma_prox=None, weights=None, init_recon=None,
                 do_initialization=True, stop_threshold_change_pct=0.2, max_iterations=3,
                 first_iteration=0, logfile_path='~/.mbirtorch/logs/prox.log', print_logs=True,
                 output_sharded=False):
        """Proximal map for Plug-and-Play (tomography_model.py:3251-3373): a
        reconstruction whose prior is Gaussian with mean ``prox_input`` and
        standard deviation ``sigma_prox`` (automatic from the sinogram when
        None).  ``do_initialization=False`` reuses the partitions and
        regularization of the previous call on this model.  The pixel
        partitions are drawn from numpy's global random generator.  Returns
        (recon, recon_dict)."""
        if do_initialization or self.prox_data is None:
            (sinogram, weights, init_recon, partitions, seq, granularity,
             reg) = self.initialize_recon(sinogram, weights, init_recon, max_iterations,
                                          first_iteration, logfile_path=logfile_path,
                                          print_logs=print_logs)
            self.prox_data = (partitions, seq, granularity, reg)
        else:
            partitions, seq, granularity, reg = self.prox_data
            if self.log_buffer is None:
                self.setup_logger(logfile_path=logfile_path, print_logs=print_logs)
        own_sigma_prox = self.get_params('sigma_prox')
        if sigma_prox is not None:
            reg = dict(reg, sigma_prox=sigma_prox)
            self.set_params(no_warning=True, sigma_prox=sigma_prox,
                            auto_regularize_flag=self.get_params('auto_regularize_flag'))
        try:
            with torch.no_grad():
                recon, losses = self._vcd_recon(sinogram, partitions, seq,
                                                stop_threshold_change_pct, weights=weights,
                                                init_recon=init_recon, prox_input=prox_input,
                                                first_iteration=first_iteration)
        finally:
            self.set_params(no_warning=True, sigma_prox=own_sigma_prox)
        fm_rmse = [float(v) for v in losses[0]]
        recon_params = dict(zip(recon_param_names, [
            len(fm_rmse), granularity, [int(v) for v in seq], fm_rmse, [0], reg,
            [100 * float(v) for v in losses[2]], [float(v) for v in losses[3]],
            [[float(x) for x in row] for row in losses[4]]]))
        if logfile_path:
            self.logger.info('Logs written to {}'.format(
                os.path.abspath(os.path.expanduser(logfile_path))))
        for h in list(self.logger.handlers):
            h.flush()
        self.close_log_file()
        notes = 'Proximal map completed: {}\n\n'.format(datetime.datetime.now())
        recon_dict = self.get_recon_dict(recon_params, notes=notes)
        return self._out(recon, output_sharded), recon_dict

    # ── model description ───────────────────────────────────────────────────
    def get_recon_dict(self, recon_params=None, notes=None, save_log=True, save_model=True,
                       str_format=False):
        d = {'recon_params': "# Recon params not saved." if recon_params is None
             else recon_params}
        buf = getattr(self, 'log_buffer', None)
        d['recon_log'] = buf.getvalue() if (buf is not None and save_log) \
            else "# Log info not saved."
        d['notes'] = '# No notes saved' if notes is None else notes
        d['model_params'] = ({k: v.val for k, v in self.params.items()} if save_model
                             else '# Model not saved')
        if str_format:
            d = {k: str(v) for k, v in d.items()}
        return d

    def scale_recon_shape(self, row_scale=1.0, col_scale=1.0, slice_scale=1.0):
        r, c, s = self.get_params('recon_shape')
        nr, nc, ns = int(r * row_scale), int(c * col_scale), int(s * slice_scale)
        self.set_params(recon_shape=(nr, nc, ns))
        return nr - r, nc - c, ns - s

    def reshape_recon(self, recon):
        return recon.reshape(self.get_params('recon_shape'))
