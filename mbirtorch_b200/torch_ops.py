"""Dispatcher registration of the four projector bodies (namespace ``mbir_b200``).

``import mbirtorch_b200.torch_ops`` registers

* ``torch.ops.mbir_b200.parallel_fwd`` / ``parallel_back`` -- the bodies of
  parallel_beam.py:56-94 (triton_parallel.py:250-257, 598-604 for the
  wrapper signatures);
* ``torch.ops.mbir_b200.cone_fwd`` / ``cone_back`` -- the bodies of
  cone_beam.py:161-299 (triton_cone.py:333-343, 640-650).

Arguments are the reference bodies' own, without the ``plan`` cache argument.
Each op returns a fresh tensor, as the bodies do.  The CUDA implementation is
the C ABI (through :mod:`mbirtorch_b200.kernels`, which makes the tensors'
device current for every call).  The fake (meta) implementations give the
output shapes, so graph tracers can treat the ops as opaque.  The C ABI
itself takes no torch types; this module is the torch-facing registration
only.
"""

from typing import Optional

import torch

from . import kernels

_NS = "mbir_b200"


@torch.library.custom_op(f"{_NS}::parallel_fwd", mutates_args=(), device_types="cuda")
def parallel_fwd(values: torch.Tensor, pixel_indices: torch.Tensor,
                 view_params: torch.Tensor, num_rows: int, num_cols: int, num_channels: int,
                 delta_det_channel: float, det_channel_offset: float, delta_voxel: float,
                 delta_voxel_row: float, psf_radius: int) -> torch.Tensor:
    """(P, L) cylinders -> (Vb, L, C) sinogram block."""
    return kernels.parallel_forward_view_batch(
        values, pixel_indices, view_params, num_rows, num_cols, num_channels,
        delta_det_channel, det_channel_offset, delta_voxel, delta_voxel_row, psf_radius)


@parallel_fwd.register_fake
def _(values, pixel_indices, view_params, num_rows, num_cols, num_channels,
      delta_det_channel, det_channel_offset, delta_voxel, delta_voxel_row, psf_radius):
    return values.new_empty((view_params.shape[0], values.shape[1], num_channels))


@torch.library.custom_op(f"{_NS}::parallel_back", mutates_args=(), device_types="cuda")
def parallel_back(sino: torch.Tensor, pixel_indices: torch.Tensor, view_params: torch.Tensor,
                  num_rows: int, num_cols: int, num_channels: int, delta_det_channel: float,
                  det_channel_offset: float, delta_voxel: float, delta_voxel_row: float,
                  psf_radius: int, coeff_power: int = 1) -> torch.Tensor:
    """(Vb, L, C) sinogram block -> (P, L), summed over the block's views."""
    return kernels.parallel_back_view_batch(
        sino, pixel_indices, view_params, num_rows, num_cols, num_channels, delta_det_channel,
        det_channel_offset, delta_voxel, delta_voxel_row, psf_radius, coeff_power=coeff_power)


@parallel_back.register_fake
def _(sino, pixel_indices, view_params, num_rows, num_cols, num_channels, delta_det_channel,
      det_channel_offset, delta_voxel, delta_voxel_row, psf_radius, coeff_power=1):
    return sino.new_empty((pixel_indices.shape[0], sino.shape[1]))


@torch.library.custom_op(f"{_NS}::cone_fwd", mutates_args=(), device_types="cuda")
def cone_fwd(values: torch.Tensor, pixel_indices: torch.Tensor, view_params: torch.Tensor,
             num_rows_r: int, num_channels: int, num_recon_rows: int, num_recon_cols: int,
             num_slices: int, delta_voxel: float, delta_voxel_row: float,
             delta_voxel_slice: float, delta_det_channel: float, delta_det_row: float,
             det_channel_offset: float, det_row_offset: float, recon_slice_offset: float,
             magnification: float, source_detector_dist: float, use_curved_detector: bool,
             psf_radius: int, bp_psf_radius: int, slice_start: int = 0) -> torch.Tensor:
    """(P, L) slice band starting at ``slice_start`` -> (Vb, R, C) partial."""
    return kernels.cone_forward_view_batch(
        values, pixel_indices, view_params, num_rows_r, num_channels, num_recon_rows,
        num_recon_cols, num_slices, delta_voxel, delta_voxel_row, delta_voxel_slice,
        delta_det_channel, delta_det_row, det_channel_offset, det_row_offset,
        recon_slice_offset, magnification, source_detector_dist, use_curved_detector,
        psf_radius, bp_psf_radius, slice_start=slice_start)


@cone_fwd.register_fake
def _(values, pixel_indices, view_params, num_rows_r, num_channels, num_recon_rows,
      num_recon_cols, num_slices, delta_voxel, delta_voxel_row, delta_voxel_slice,
      delta_det_channel, delta_det_row, det_channel_offset, det_row_offset, recon_slice_offset,
      magnification, source_detector_dist, use_curved_detector, psf_radius, bp_psf_radius,
      slice_start=0):
    return values.new_empty((view_params.shape[0], num_rows_r, num_channels))


@torch.library.custom_op(f"{_NS}::cone_back", mutates_args=(), device_types="cuda")
def cone_back(sino: torch.Tensor, pixel_indices: torch.Tensor, view_params: torch.Tensor,
              num_rows_r: int, num_channels: int, num_recon_rows: int, num_recon_cols: int,
              num_slices: int, delta_voxel: float, delta_voxel_row: float,
              delta_voxel_slice: float, delta_det_channel: float, delta_det_row: float,
              det_channel_offset: float, det_row_offset: float, recon_slice_offset: float,
              magnification: float, source_detector_dist: float, use_curved_detector: bool,
              psf_radius: int, bp_psf_radius: int, coeff_power: int = 1, slice_start: int = 0,
              band_slices: Optional[int] = None) -> torch.Tensor:
    """(Vb, R, C) -> (P, band) cylinders of slices [slice_start, slice_start + band)."""
    return kernels.cone_back_view_batch(
        sino, pixel_indices, view_params, num_rows_r, num_channels, num_recon_rows,
        num_recon_cols, num_slices, delta_voxel, delta_voxel_row, delta_voxel_slice,
        delta_det_channel, delta_det_row, det_channel_offset, det_row_offset,
        recon_slice_offset, magnification, source_detector_dist, use_curved_detector,
        psf_radius, bp_psf_radius, coeff_power=coeff_power, slice_start=slice_start,
        band_slices=band_slices)


@cone_back.register_fake
def _(sino, pixel_indices, view_params, num_rows_r, num_channels, num_recon_rows,
      num_recon_cols, num_slices, delta_voxel, delta_voxel_row, delta_voxel_slice,
      delta_det_channel, delta_det_row, det_channel_offset, det_row_offset, recon_slice_offset,
      magnification, source_detector_dist, use_curved_detector, psf_radius, bp_psf_radius,
      coeff_power=1, slice_start=0, band_slices=None):
    band = num_slices - slice_start if band_slices is None else band_slices
    return sino.new_empty((pixel_indices.shape[0], band))
