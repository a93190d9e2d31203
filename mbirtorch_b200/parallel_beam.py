"""ParallelBeamModel and recon_simple_parallel.

Constructor, parameters, recon geometry and psf radius follow the reference
(parallel_beam.py:134-232, 672-722); projection runs in the sm_100a kernels
(detector row r is recon slice r).
"""

import math

import numpy as np
import torch

from .kernels import make_geometry
from .tomography_model import TomographyModel


class ParallelBeamModel(TomographyModel):
    """Parallel-beam geometry.

    Args:
        sinogram_shape (tuple): (views, rows, channels).
        angles (array): one projection angle (radians) per view.
        view_batch_size, compile_mode: accepted for compatibility; no effect.
    """

    rows_track_slices = True

    def __init__(self, sinogram_shape, angles, view_batch_size=None, compile_mode='auto'):
        angles = np.asarray(angles, dtype=np.float32)
        super().__init__(sinogram_shape, view_batch_size=view_batch_size,
                         compile_mode=compile_mode, geometry_type='parallel',
                         view_params_name='angles', angles=angles)

    def get_magnification(self):
        return 1.0

    def get_psf_radius(self):
        """Channel taps either side of the centre (parallel_beam.py:172-180)."""
        ddc, dv, vra = self.get_params(['delta_det_channel', 'delta_voxel', 'voxel_row_aspect'])
        return int(np.ceil(np.ceil(max(dv, vra * dv) / ddc) / 2))

    def auto_set_recon_geometry(self, no_compile=False, no_warning=False):
        ddr, ddc, vra = self.get_params(['delta_det_row', 'delta_det_channel',
                                         'voxel_row_aspect'])
        mag = self.get_magnification()
        dv = ddc / mag
        dvr = vra * dv
        rows, chans = self.get_params('sinogram_shape')[1:3]
        recon_shape = (int(np.ceil(chans * ddc / (dvr * mag))),
                       int(np.ceil(chans * ddc / (dv * mag))),
                       int(np.round(rows * ((ddr / dv) / mag))))
        self.set_params(no_compile=no_compile, no_warning=no_warning, recon_shape=recon_shape,
                        delta_voxel=dv)

    def verify_valid_params(self):
        super().verify_valid_params()
        shape, angles, vra, vsa = self.get_params(['sinogram_shape', 'angles',
                                                   'voxel_row_aspect', 'voxel_slice_aspect'])
        if vra <= 0:
            raise ValueError(f'Voxel row aspect ratio must be positive. \nGot {vra} for '
                             'voxel_row_aspect.')
        if vsa != 1.0:
            raise ValueError('Setting voxel slice aspect ratio is not supported for parallel '
                             f'beam model. \nGot {vsa}.')
        if np.asarray(angles).shape[0] != shape[0]:
            raise ValueError('Number of view dependent parameter vectors must equal the number '
                             'of views.')
        recon_shape = self.get_params('recon_shape')
        if recon_shape[2] != shape[1]:
            raise ValueError('Number of recon slices must match number of sinogram rows. \n'
                             f'Got {recon_shape} for recon_shape and {shape} for '
                             'sinogram_shape')

    def _geometry(self):
        ddc, off, dv, vra = self.get_params(['delta_det_channel', 'det_channel_offset',
                                             'delta_voxel', 'voxel_row_aspect'])
        V, R, C = self.get_params('sinogram_shape')
        rs = self.get_params('recon_shape')
        return make_geometry('parallel', V, R, C, rs[0], rs[1], rs[2], self.get_psf_radius(),
                             delta_det_channel=ddc, det_channel_offset=off, delta_voxel=dv,
                             delta_voxel_row=vra * dv, source_detector_dist=math.inf)

    def _view_params_array(self):
        return np.asarray(self.get_params('angles'), dtype=np.float32)

    # ── direct recon ────────────────────────────────────────────────────────
    def fbp_filter(self, sinogram, filter_name="ramp", output_sharded=False):
        dv, vra = self.get_params(['delta_voxel', 'voxel_row_aspect'])
        return self._apply_direct_recon_filter(sinogram, filter_name,
                                               filter_scale=1.0 / (dv * (vra * dv)),
                                               output_sharded=output_sharded)

    def recon_fbp(self, sinogram, filter_name="ramp", output_sharded=False):
        """Filtered back projection with the adjoint back projector
        (parallel_beam.py:321-368)."""
        filtered = self.fbp_filter(sinogram, filter_name=filter_name, output_sharded=True)
        return self.back_project(filtered, output_sharded=output_sharded)

    def recon_direct(self, sinogram, filter_name="ramp", output_sharded=False):
        return self.recon_fbp(sinogram, filter_name=filter_name, output_sharded=output_sharded)

    def direct_filter(self, sinogram, filter_name="ramp", output_sharded=False):
        return self.fbp_filter(sinogram, filter_name=filter_name, output_sharded=output_sharded)


def recon_simple_parallel(sinogram, angles, weights=None, sharpness=1.0, max_iterations=15):
    """One-call parallel-beam reconstruction (parallel_beam.py:672-722)."""
    if torch.is_tensor(angles):
        angles = angles.detach().cpu().numpy()
    model = ParallelBeamModel(tuple(sinogram.shape), angles)
    model.set_params(sharpness=sharpness)
    return model.recon(sinogram, weights=weights, max_iterations=max_iterations)
