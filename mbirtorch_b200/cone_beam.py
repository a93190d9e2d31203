"""ConeBeamModel (flat and curved detectors, circular and helical scans) and
recon_simple_cone.

Constructor, parameters, recon geometry, psf radii, FDK and the DC-damping
slice profile follow the reference (cone_beam.py:319-796, 1134-1190);
projection and the VCD update (with DC damping) run in the sm_100a kernels.
"""

import warnings

import numpy as np
import torch

from .kernels import make_geometry
from .tomography_model import TomographyModel
from .vcd_utils import get_support_radius

_DC_DAMPING_DEFAULT = (0.25, 100.0, 0.7, 0.5)


class ConeBeamModel(TomographyModel):
    """Cone-beam geometry.

    Args:
        sinogram_shape (tuple): (views, rows, channels).
        angles (array): projection angles in radians.
        source_detector_dist (float): source-to-detector distance (ALU).
        source_iso_dist (float): source-to-rotation-axis distance.
        helical_z_shifts (array, optional): per-view z shift (helical).
        use_curved_detector (bool): cylindrical detector of radius SDD.
        view_batch_size, compile_mode: accepted for compatibility; no effect.
    """

    _dc_damping = _DC_DAMPING_DEFAULT

    def __init__(self, sinogram_shape, angles, source_detector_dist, source_iso_dist,
                 helical_z_shifts=None, use_curved_detector=False, view_batch_size=None,
                 compile_mode='auto'):
        angles = np.asarray(angles, dtype=np.float32).flatten()
        if helical_z_shifts is None:
            helical_z_shifts = np.zeros_like(angles)
        else:
            helical_z_shifts = np.asarray(helical_z_shifts, dtype=np.float32).flatten()
        if helical_z_shifts.shape != angles.shape:
            raise ValueError("Incompatible view dependent vector lengths: all view-dependent "
                             "vectors must have the same length.")
        super().__init__(sinogram_shape, view_batch_size=view_batch_size,
                         compile_mode=compile_mode, geometry_type='cone',
                         view_params_name='view_params_array',
                         view_params_array=np.stack([angles, helical_z_shifts], axis=1),
                         source_detector_dist=source_detector_dist,
                         source_iso_dist=source_iso_dist, recon_slice_offset=0.0,
                         axial_pad_fraction=0.0, use_curved_detector=use_curved_detector)

    def get_magnification(self):
        sdd, sid = self.get_params(['source_detector_dist', 'source_iso_dist'])
        if np.isinf(sdd):
            return 1
        return sdd / sid

    def get_psf_radii(self):
        """(psf_radius, bp_psf_radius) of cone_beam.py:530-566."""
        (ddr, ddc, sdd, recon_shape, dv, vra, vsa) = self.get_params(
            ['delta_det_row', 'delta_det_channel', 'source_detector_dist', 'recon_shape',
             'delta_voxel', 'voxel_row_aspect', 'voxel_slice_aspect'])
        mag = self.get_magnification()
        dvr, dvs = vra * dv, vsa * dv
        d_det = min(ddr, ddc)
        if np.isinf(sdd):
            mmax = mmin = 1
        else:
            sid = sdd / mag
            half = max(0.5 * recon_shape[1] * dv, 0.5 * recon_shape[0] * dvr)
            mmax = sdd / (sid - half)
            mmin = sdd / (sid + half)
        psf = int(np.ceil(np.ceil(max(dv, dvr, dvs) * mmax / d_det) / 2))
        bp = int(np.ceil(np.ceil(d_det / (mmin * min(dv, dvr, dvs))) / 2))
        return psf, bp

    def get_psf_radius(self):
        return self.get_psf_radii()[0]

    @staticmethod
    def detector_mn_to_uv(m, n, delta_det_channel, delta_det_row, det_channel_offset,
                          det_row_offset, num_det_rows, num_det_channels):
        v = (m - (num_det_rows - 1) / 2.0) * delta_det_row - det_row_offset
        u = (n - (num_det_channels - 1) / 2.0) * delta_det_channel - det_channel_offset
        return u, v

    def auto_set_recon_geometry(self, no_compile=False, no_warning=False):
        """Recon shape from the detector field of view, helical travel and
        axial padding (cone_beam.py:582-658)."""
        ddr, ddc = self.get_params(['delta_det_row', 'delta_det_channel'])
        vra, vsa = self.get_params(['voxel_row_aspect', 'voxel_slice_aspect'])
        mag = self.get_magnification()
        dv = ddc / mag
        dvr, dvs = vra * dv, vsa * dv
        rows, chans = self.get_params('sinogram_shape')[1:3]
        nr = int(np.round(chans * ((ddc / dvr) / mag)))
        nc = int(np.round(chans * ((ddc / dv) / mag)))
        zs = np.asarray(self.get_params('view_params_array'))[:, 1]
        z_min, z_max = float(np.min(zs)), float(np.max(zs))
        H_iso = rows * (ddr / mag)
        ns = max(1, int(np.ceil((H_iso + (z_max - z_min)) / dvs)))
        rso = 0.5 * (z_min + z_max)
        sdd, dro, dco, use_ror = self.get_params(['source_detector_dist', 'det_row_offset',
                                                  'det_channel_offset', 'use_ror_mask'])
        support = get_support_radius((nr, nc), dvr, dv, use_ror_mask=use_ror)
        _, v_lo = self.detector_mn_to_uv(-0.5, 0.0, ddc, ddr, dco, dro, rows, chans)
        _, v_hi = self.detector_mn_to_uv(rows - 0.5, 0.0, ddc, ddr, dco, dro, rows, chans)
        v_bot, v_top = max(float(v_lo), float(v_hi)), min(float(v_lo), float(v_hi))
        z_per_v = 1.0 / float(mag)
        if not np.isinf(sdd):
            z_per_v += support / float(sdd)
        ex_bot = max(0.0, v_bot * z_per_v - float(H_iso) / 2)
        ex_top = max(0.0, -v_top * z_per_v - float(H_iso) / 2)
        apf = self.get_params('axial_pad_fraction')
        if isinstance(apf, (tuple, list)):
            if len(apf) != 2:
                raise ValueError('axial_pad_fraction must be a float or a (top_fraction, '
                                 f'bottom_fraction) pair; got {apf!r}.')
            f_top, f_bot = (float(f) for f in apf)
        else:
            f_top = f_bot = float(apf)
        if f_top < 0 or f_bot < 0:
            raise ValueError(f'axial_pad_fraction must be >= 0; got {apf!r}.')
        n_top = int(np.ceil(f_top * ex_top / dvs))
        n_bot = int(np.ceil(f_bot * ex_bot / dvs))
        ns += n_top + n_bot
        rso += 0.5 * (n_bot - n_top) * float(dvs)
        self.set_params(no_compile=no_compile, no_warning=no_warning,
                        recon_shape=(nr, nc, ns), delta_voxel=dv, recon_slice_offset=rso)

    def verify_valid_params(self):
        super().verify_valid_params()
        shape, vpa = self.get_params(['sinogram_shape', 'view_params_array'])
        vra, vsa = self.get_params(['voxel_row_aspect', 'voxel_slice_aspect'])
        if vpa is None:
            raise ValueError("view_params_array was not set.")
        if tuple(np.shape(vpa)) != (shape[0], 2):
            raise ValueError('Number of view dependent parameter vectors must equal the number '
                             'of views.')
        if vra <= 0 or vsa <= 0:
            raise ValueError('Voxel aspect ratios must be positive.')
        sdd, ddr, dro = self.get_params(['source_detector_dist', 'delta_det_row',
                                         'det_row_offset'])
        if ddr * shape[1] / 2 + abs(dro) > sdd:
            warnings.warn('Cone angle is more than 45 degrees.  This will likely produce '
                          'recon artifacts.')

    def _geometry(self):
        (ddr, ddc, dro, dco, sdd, dv, vra, vsa, rso, curved) = self.get_params(
            ['delta_det_row', 'delta_det_channel', 'det_row_offset', 'det_channel_offset',
             'source_detector_dist', 'delta_voxel', 'voxel_row_aspect', 'voxel_slice_aspect',
             'recon_slice_offset', 'use_curved_detector'])
        V, R, C = self.get_params('sinogram_shape')
        rs = self.get_params('recon_shape')
        psf, bp = self.get_psf_radii()
        return make_geometry('cone', V, R, C, rs[0], rs[1], rs[2], psf, bp, curved, ddc, ddr,
                             dco, dro, dv, vra * dv, vsa * dv, rso, self.get_magnification(), sdd)

    def _view_params_array(self):
        return np.asarray(self.get_params('view_params_array'), dtype=np.float32)

    def _dc_damping_profile(self):
        """Per-slice damping s_k (cone_beam.py:424-477), or None if off."""
        cfg = self._dc_damping
        if cfg is None:
            return None
        a, b, p, c = cfg
        rs = self.get_params('recon_shape')
        dv, vsa, oz = self.get_params(['delta_voxel', 'voxel_slice_aspect',
                                       'recon_slice_offset'])
        R = self.get_params('source_iso_dist')
        zs = np.asarray(self.get_params('view_params_array'))[:, 1]
        nz = rs[2]
        L = rs[0] * dv
        dz = vsa * dv
        z = (np.arange(nz) - (nz - 1) / 2.0) * dz + oz

        def profile(t):
            return (c * t ** p + a * b ** p) / (t ** p + b ** p)

        if zs.max() - zs.min() == 0:
            s = profile(L * np.abs(z - zs[0]) / (R * dz))
        else:
            s = profile(L * np.abs(z[:, None] - zs[None, :]) / (R * dz)).mean(axis=1)
        return s.astype(np.float32)

    # ── direct recon (FDK) ──────────────────────────────────────────────────
    def fdk_filter(self, sinogram, filter_name="ramp", output_sharded=False):
        """Row filter with the FDK cosine pre-weight and scale (cone_beam.py:661-695)."""
        _, rows, chans = (int(x) for x in self.get_params('sinogram_shape'))
        sdd = self.get_params('source_detector_dist')
        dv, ddr, ddc, vra, vsa = self.get_params(['delta_voxel', 'delta_det_row',
                                                  'delta_det_channel', 'voxel_row_aspect',
                                                  'voxel_slice_aspect'])
        dro, dco = self.get_params(['det_row_offset', 'det_channel_offset'])
        vol = dv * (vra * dv) * (vsa * dv)
        M = self.get_magnification()
        m, n = np.meshgrid(np.arange(rows), np.arange(chans), indexing='ij')
        u, v = self.detector_mn_to_uv(m, n, ddc, ddr, dco, dro, rows, chans)
        wmap = sdd / np.sqrt(sdd ** 2 + u ** 2 + v ** 2)
        wt = torch.as_tensor(wmap.astype(np.float32), device=self.torch_device)
        return self._apply_direct_recon_filter(sinogram, filter_name,
                                               filter_scale=ddr / (vol * M),
                                               output_sharded=output_sharded, row_weight=wt)

    def _helical_z_weight_row(self):
        V, rows, _ = self.get_params('sinogram_shape')
        zs = np.asarray(self.get_params('view_params_array'))[:, 1]
        dv, vsa, rs, rso, ddr = self.get_params(['delta_voxel', 'voxel_slice_aspect',
                                                 'recon_shape', 'recon_slice_offset',
                                                 'delta_det_row'])
        M = self.get_magnification()
        ns = rs[2]
        z_k = vsa * dv * (np.arange(ns) - (ns - 1) / 2.0) + rso
        half = 0.5 * rows * ddr / M
        cov = np.sum(np.abs(z_k[:, None] - zs[None, :]) <= half, axis=1)
        return np.where(cov > 0, V / np.maximum(cov, 1), 0.0)

    def helical_fdk_z_weight(self, recon, sinogram=None):
        w = torch.as_tensor(self._helical_z_weight_row().astype(np.float32),
                            device=recon.device)
        return recon * w[None, None, :]

    def recon_fdk(self, sinogram, filter_name="ramp", output_sharded=False):
        """FDK with the exact adjoint as back projection (cone_beam.py:753-796)."""
        filtered = self.fdk_filter(sinogram, filter_name=filter_name, output_sharded=True)
        recon = self.back_project(filtered, output_sharded=True)
        zs = np.asarray(self.get_params('view_params_array'))[:, 1]
        if float(np.max(zs) - np.min(zs)) > 0:
            recon = self.helical_fdk_z_weight(recon)
        return self._out(recon, output_sharded)

    def recon_direct(self, sinogram, filter_name="ramp", output_sharded=False):
        return self.recon_fdk(sinogram, filter_name=filter_name, output_sharded=output_sharded)

    def direct_filter(self, sinogram, filter_name="ramp", output_sharded=False):
        return self.fdk_filter(sinogram, filter_name=filter_name, output_sharded=output_sharded)


def recon_simple_cone(sinogram, angles, source_detector_dist, source_iso_dist, weights=None,
                      sharpness=1.0, max_iterations=15):
    """One-call cone-beam reconstruction (cone_beam.py:1134-1190)."""
    if torch.is_tensor(angles):
        angles = angles.detach().cpu().numpy()
    model = ConeBeamModel(tuple(sinogram.shape), angles, source_detector_dist=source_detector_dist,
                          source_iso_dist=source_iso_dist)
    model.set_params(sharpness=sharpness)
    return model.recon(sinogram, weights=weights, max_iterations=max_iterations)
