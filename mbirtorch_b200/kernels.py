"""Projector entry points over the sm_100a C ABI.

Two layers:

* :class:`DeviceProjector` -- a model's projector pair bound to its geometry
  and its view parameters resident on the device.  Whole view ranges go to
  the kernels in one launch: the kernels materialize no per-view transient,
  so the reference's view batching (projectors.py:304-516, a memory knob
  for its torch bodies) is not needed.

* The four BODY functions with the reference's exact body signatures
  (parallel_beam.py:56-94, cone_beam.py:161-299), so they drop into a
  ``_view_batch_bodies()`` seam (parallel_beam.py:234-276,
  cone_beam.py:354-395) unchanged: same argument names and meaning, a fresh
  output tensor, ``coeff_power`` 1 or 2, slice bands for cone.  They carry
  the reference's ``_mbirtorch_no_compile`` marker.
"""

import math

import torch

from . import _lib
from ._lib import (MBIR_CONE, MBIR_LAYOUT_VCR, MBIR_LAYOUT_VRC, MBIR_PARALLEL, Geometry,
                   as_f32_contig, as_i64_contig, ptr, require_cuda, stream_of)


def make_geometry(kind, num_views, num_det_rows, num_det_channels, num_recon_rows,
                  num_recon_cols, num_slices, psf_radius, bp_psf_radius=1,
                  use_curved_detector=False, delta_det_channel=1.0, delta_det_row=1.0,
                  det_channel_offset=0.0, det_row_offset=0.0, delta_voxel=1.0,
                  delta_voxel_row=1.0, delta_voxel_slice=1.0, recon_slice_offset=0.0,
                  magnification=1.0, source_detector_dist=math.inf):
    if psf_radius > _lib.MAX_TAP_RADIUS or bp_psf_radius > _lib.MAX_TAP_RADIUS:
        raise ValueError(
            f"tap radius above {_lib.MAX_TAP_RADIUS} is not supported (psf_radius="
            f"{psf_radius}, bp_psf_radius={bp_psf_radius}): the kernels unroll at most "
            f"{_lib.MAX_TAP_RADIUS} taps a side, where the reference's torch bodies "
            "(horizontal_fan.py:74-154) take any radius.  The radius is "
            "ceil(ceil(voxel pitch x magnification / detector pitch) / 2): voxels wider than "
            f"{2 * _lib.MAX_TAP_RADIUS} detector cells exceed it; use finer voxels or a "
            "coarser detector binning")
    return Geometry(MBIR_CONE if kind == 'cone' else MBIR_PARALLEL, int(num_views),
                    int(num_det_rows), int(num_det_channels), int(num_recon_rows),
                    int(num_recon_cols), int(num_slices), int(psf_radius), int(bp_psf_radius),
                    int(bool(use_curved_detector)), float(delta_det_channel),
                    float(delta_det_row), float(det_channel_offset), float(det_row_offset),
                    float(delta_voxel), float(delta_voxel_row), float(delta_voxel_slice),
                    float(recon_slice_offset), float(magnification), float(source_detector_dist))


def _view_params_2col(view_params, device):
    """(V,) angles or (V, 2) [angle, z_shift] -> contiguous (V, 2) f32."""
    vp = torch.as_tensor(view_params, dtype=torch.float32, device=device)
    if vp.dim() == 1:
        vp = torch.stack([vp, torch.zeros_like(vp)], dim=1)
    return vp.reshape(-1, 2).contiguous()


BINNED_BYTES_PER_PIXEL_VIEW = 52  # a binned forward's record + list entry


class DeviceProjector:
    """Forward/back projection of one geometry on one CUDA device.

    Whole-cylinder forward projections go through the channel-sorted bins
    (``mbir_forward_project_binned``) wherever those kernels apply (psf
    radius 1, up to 1024 detector rows): the records of a chunk of views
    are formed and sorted once, and each (view, channel block) CTA walks
    only the pixels that reach it, where the scanning forward tests every
    pixel in every block.  The workspace (up to about 1 GiB of records, from
    torch's caching allocator) is the one transient.
    """

    binned_forward = {MBIR_PARALLEL: True, MBIR_CONE: True}

    def __init__(self, geom, view_params, device):
        self.geom = geom
        self.device = torch.device(device)
        self.view_params = _view_params_2col(view_params, self.device)
        if self.view_params.shape[0] != geom.num_views:
            raise ValueError("view parameter count does not match the geometry's views")

    def _binned_workspace(self, device, view_count, num_pixels):
        """The binned forward's workspace, or None where it does not apply."""
        if not self.binned_forward.get(self.geom.geometry, False) or num_pixels <= 0:
            return None
        nbytes = int(_lib.query(device, 'mbir_forward_project_binned_workspace_size', self.geom,
                                view_count, num_pixels))
        if nbytes <= 0:
            return None
        return torch.empty(nbytes, dtype=torch.uint8, device=device)

    def _forward_binned(self, values, by_pixel, idx, view_start, vc, out, layout, ws):
        _lib.call(values.device, 'mbir_forward_project_binned', self.geom,
                  ptr(self.view_params), view_start, vc, ptr(values), by_pixel, ptr(idx),
                  idx.shape[0], ptr(out), layout, ptr(ws), ws.numel(), stream_of(values.device))

    @property
    def sino_shape(self):
        g = self.geom
        return (g.num_views, g.num_det_rows, g.num_det_channels)

    def forward(self, values, pixel_indices, slice_start=0, layout=MBIR_LAYOUT_VRC,
                view_start=0, view_count=None, out=None):
        """(P, L) cylinders -> (Vc, R, C) [VRC] or (Vc, C, R) [VCR] f32."""
        g = self.geom
        values = as_f32_contig(values)
        idx = as_i64_contig(pixel_indices)
        require_cuda(values, idx)
        vc = g.num_views - view_start if view_count is None else int(view_count)
        L = values.shape[1]
        shape = ((vc, g.num_det_rows, g.num_det_channels) if layout == MBIR_LAYOUT_VRC
                 else (vc, g.num_det_channels, g.num_det_rows))
        if out is None:
            out = torch.empty(shape, dtype=torch.float32, device=values.device)
        ws = (self._binned_workspace(values.device, vc, idx.shape[0])
              if slice_start == 0 and L == g.num_slices else None)
        if ws is not None:
            self._forward_binned(values, 0, idx, view_start, vc, out, layout, ws)
            return out
        _lib.call(values.device, 'mbir_forward_project', g, ptr(self.view_params), view_start,
                  vc, ptr(values), idx.shape[0], L, slice_start, ptr(idx), ptr(out), layout,
                  stream_of(values.device))
        return out

    def forward_volume(self, flat_volume, pixel_indices, layout=MBIR_LAYOUT_VRC, out=None):
        """Whole cylinders read at rows ``pixel_indices`` of a flat (N*N, S)
        volume (no gathered copy) -> (V, R, C) [VRC] or (V, C, R) [VCR]."""
        g = self.geom
        flat = as_f32_contig(flat_volume)
        idx = as_i64_contig(pixel_indices)
        require_cuda(flat, idx)
        if flat.shape[-1] != g.num_slices or flat.shape[0] != g.num_recon_rows * g.num_recon_cols:
            raise ValueError(f"flat volume must be ({g.num_recon_rows * g.num_recon_cols}, "
                             f"{g.num_slices}); got {tuple(flat.shape)}")
        shape = ((g.num_views, g.num_det_rows, g.num_det_channels) if layout == MBIR_LAYOUT_VRC
                 else (g.num_views, g.num_det_channels, g.num_det_rows))
        if out is None:
            out = torch.empty(shape, dtype=torch.float32, device=flat.device)
        ws = self._binned_workspace(flat.device, g.num_views, idx.shape[0])
        if ws is not None:
            self._forward_binned(flat, 1, idx, 0, g.num_views, out, layout, ws)
            return out
        _lib.call(flat.device, 'mbir_forward_project_volume', g, ptr(self.view_params), 0,
                  g.num_views, ptr(flat), ptr(idx), idx.shape[0], ptr(out), layout,
                  stream_of(flat.device))
        return out

    def back(self, sino, pixel_indices, coeff_power=1, slice_start=0, band_slices=None,
             layout=MBIR_LAYOUT_VRC, view_start=0):
        """Sinogram (Vc, ...) f32 -> (P, band) cylinders summed over views."""
        g = self.geom
        sino = as_f32_contig(sino)
        idx = as_i64_contig(pixel_indices)
        require_cuda(sino, idx)
        vc = sino.shape[0]
        band = g.num_slices - slice_start if band_slices is None else int(band_slices)
        out = torch.empty((idx.shape[0], band), dtype=torch.float32, device=sino.device)
        nbytes = _lib.query(sino.device, 'mbir_back_project_workspace_size', g, vc,
                            idx.shape[0], band)
        ws = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=sino.device)
        _lib.call(sino.device, 'mbir_back_project', g, ptr(self.view_params), view_start, vc,
                  ptr(sino), layout, ptr(idx), idx.shape[0], int(coeff_power), int(slice_start),
                  band, ptr(out), ptr(ws), ws.numel(), stream_of(sino.device))
        return out


# ── the reference body signatures ─────────────────────────────────────────
def _parallel_geom(num_views, num_rows_det, num_rows, num_cols, num_channels,
                   delta_det_channel, det_channel_offset, delta_voxel, delta_voxel_row,
                   psf_radius):
    return make_geometry('parallel', num_views, num_rows_det, num_channels, num_rows, num_cols,
                         num_rows_det, psf_radius, delta_det_channel=delta_det_channel,
                         det_channel_offset=det_channel_offset, delta_voxel=delta_voxel,
                         delta_voxel_row=delta_voxel_row)


def parallel_forward_view_batch(values, pixel_indices, view_params_batch, num_rows, num_cols,
                                num_channels, delta_det_channel, det_channel_offset,
                                delta_voxel, delta_voxel_row, psf_radius, slice_start=0,
                                plan=None):
    """Parallel forward for one view batch (parallel_beam.py:56-73):
    (P, L) cylinders -> (Vb, L, C)."""
    if slice_start != 0:
        raise ValueError("parallel beam projects whole cylinders (slice_start must be 0)")
    vb = int(view_params_batch.shape[0])
    g = _parallel_geom(vb, values.shape[1], num_rows, num_cols, num_channels, delta_det_channel,
                       det_channel_offset, delta_voxel, delta_voxel_row, psf_radius)
    return DeviceProjector(g, view_params_batch, values.device).forward(values, pixel_indices)


def parallel_back_view_batch(sino_batch, pixel_indices, view_params_batch, num_rows, num_cols,
                             num_channels, delta_det_channel, det_channel_offset, delta_voxel,
                             delta_voxel_row, psf_radius, coeff_power=1, slice_start=0,
                             band_slices=None, plan=None):
    """Parallel back for one view batch (parallel_beam.py:76-94):
    (Vb, L, C) -> (P, L) summed over the batch's views."""
    if slice_start != 0 or band_slices is not None:
        raise ValueError("parallel beam back-projects whole cylinders")
    vb = int(view_params_batch.shape[0])
    g = _parallel_geom(vb, sino_batch.shape[1], num_rows, num_cols, num_channels,
                       delta_det_channel, det_channel_offset, delta_voxel, delta_voxel_row,
                       psf_radius)
    return DeviceProjector(g, view_params_batch, sino_batch.device).back(
        sino_batch, pixel_indices, coeff_power=coeff_power)


def _cone_geom(vb, num_rows_r, num_channels, num_recon_rows, num_recon_cols, num_slices,
               delta_voxel, delta_voxel_row, delta_voxel_slice, delta_det_channel,
               delta_det_row, det_channel_offset, det_row_offset, recon_slice_offset,
               magnification, source_detector_dist, use_curved_detector, psf_radius,
               bp_psf_radius):
    return make_geometry('cone', vb, num_rows_r, num_channels, num_recon_rows, num_recon_cols,
                         num_slices, psf_radius, bp_psf_radius, use_curved_detector,
                         delta_det_channel, delta_det_row, det_channel_offset, det_row_offset,
                         delta_voxel, delta_voxel_row, delta_voxel_slice, recon_slice_offset,
                         magnification, source_detector_dist)


def cone_forward_view_batch(values, pixel_indices, view_params_batch, num_rows_r, num_channels,
                            num_recon_rows, num_recon_cols, num_slices, delta_voxel,
                            delta_voxel_row, delta_voxel_slice, delta_det_channel, delta_det_row,
                            det_channel_offset, det_row_offset, recon_slice_offset,
                            magnification, source_detector_dist, use_curved_detector, psf_radius,
                            bp_psf_radius, slice_start=0, plan=None):
    """Cone forward for one view batch (cone_beam.py:161-234): a (P, L) slice
    band starting at global slice ``slice_start`` -> (Vb, R, C) partial."""
    vb = int(view_params_batch.shape[0])
    g = _cone_geom(vb, num_rows_r, num_channels, num_recon_rows, num_recon_cols, num_slices,
                   delta_voxel, delta_voxel_row, delta_voxel_slice, delta_det_channel,
                   delta_det_row, det_channel_offset, det_row_offset, recon_slice_offset,
                   magnification, source_detector_dist, use_curved_detector, psf_radius,
                   bp_psf_radius)
    return DeviceProjector(g, view_params_batch, values.device).forward(
        values, pixel_indices, slice_start=slice_start)


def cone_back_view_batch(sino_batch, pixel_indices, view_params_batch, num_rows_r, num_channels,
                         num_recon_rows, num_recon_cols, num_slices, delta_voxel,
                         delta_voxel_row, delta_voxel_slice, delta_det_channel, delta_det_row,
                         det_channel_offset, det_row_offset, recon_slice_offset, magnification,
                         source_detector_dist, use_curved_detector, psf_radius, bp_psf_radius,
                         coeff_power=1, slice_start=0, band_slices=None, plan=None):
    """Cone back for one view batch (cone_beam.py:237-299): (Vb, R, C) ->
    (P, band) summed over the batch's views."""
    vb = int(view_params_batch.shape[0])
    g = _cone_geom(vb, num_rows_r, num_channels, num_recon_rows, num_recon_cols, num_slices,
                   delta_voxel, delta_voxel_row, delta_voxel_slice, delta_det_channel,
                   delta_det_row, det_channel_offset, det_row_offset, recon_slice_offset,
                   magnification, source_detector_dist, use_curved_detector, psf_radius,
                   bp_psf_radius)
    return DeviceProjector(g, view_params_batch, sino_batch.device).back(
        sino_batch, pixel_indices, coeff_power=coeff_power, slice_start=slice_start,
        band_slices=band_slices)


for _f in (parallel_forward_view_batch, parallel_back_view_batch, cone_forward_view_batch,
           cone_back_view_batch):
    _f._mbirtorch_no_compile = True
    # (bytes per view, nominal view chunk): the scanning kernels hold no
    # per-view transient, so a whole view range is one batch
    # (projectors.py:475-516).
    _f._view_batch_cost = lambda num_pixels, band_cols, args: (1, 1 << 30)
# The whole-cylinder forward bins its views: one record (48 bytes) and one
# list entry (4 bytes) per (view, pixel).
for _f in (parallel_forward_view_batch, cone_forward_view_batch):
    _f._view_batch_cost = (
        lambda num_pixels, band_cols, args: (BINNED_BYTES_PER_PIXEL_VIEW * max(1, int(num_pixels)),
                                             1 << 30))
del _f
