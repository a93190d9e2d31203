"""Device-resident VCD state and the subset/partition drivers.

The reference keeps its error sinogram as an FP32 (V, R, C) tensor and runs
each subset update as ~13 separate sinogram sweeps of torch ops
(tomography_model.py:2508-2657).  Here the whole update is the fused launch
chain of ``mbir_vcd_subset_update`` (csrc/vcd.cuh), and the loop state
lives on the device in the resident form:

* :class:`ResidentSinogram` -- a sinogram-shaped array in the channel-major
  (V, C, R) layout and a storage precision (float32, bfloat16 or float16)
  with a per-view scale; arithmetic is FP32, reductions FP64.
* :class:`VcdEngine` -- one reconstruction's constants (geometry,
  regularization, Hessian diagonal, weights, DC-damping profile) plus the
  workspace, exposing the subset update (the reference's
  ``create_vcd_subset_updater`` callable) and the partition pass (its
  ``vcd_partition_iterator``).
"""

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import (STORAGE_CODES, STORAGE_DTYPES, VcdParams, host_int32, ptr, require_cuda,
                   stream_of)


def storage_code(storage_dtype):
    if isinstance(storage_dtype, torch.dtype):
        storage_dtype = str(storage_dtype).replace('torch.', '')
    name = {'fp32': 'float32', 'f32': 'float32', 'bf16': 'bfloat16',
            'fp16': 'float16', 'f16': 'float16', 'half': 'float16'}.get(storage_dtype,
                                                                         storage_dtype)
    if name not in STORAGE_CODES:
        raise ValueError(f"storage dtype must be float32, bfloat16 or float16; got "
                         f"{storage_dtype!r}")
    return STORAGE_CODES[name]


class ResidentSinogram:
    """A (V, R, C) sinogram held on the device as (V, C, R) in a storage
    precision with a per-view scale (stored = value / scale[v])."""

    def __init__(self, data, scale, rows, storage):
        self.data = data
        self.scale = scale
        self.rows = rows
        self.storage = storage

    @classmethod
    def from_vrc(cls, sino, storage=_lib.MBIR_F32):
        sino = _lib.as_f32_contig(sino)
        require_cuda(sino)
        V, R, C = sino.shape
        data = torch.empty((V, C, R), dtype=STORAGE_DTYPES[storage], device=sino.device)
        scale = torch.empty(V, dtype=torch.float32, device=sino.device)
        _lib.call(sino.device, 'mbir_sino_convert', 0, V, R, C, ptr(sino), ptr(data), storage,
                  ptr(scale), 1, stream_of(sino.device))
        return cls(data, scale, R, storage)

    @property
    def shape(self):
        V, C, R = self.data.shape
        return (V, R, C)

    @property
    def device(self):
        return self.data.device

    def to_vrc(self):
        V, C, R = self.data.shape
        out = torch.empty((V, R, C), dtype=torch.float32, device=self.data.device)
        _lib.call(self.data.device, 'mbir_sino_convert', 1, V, R, C, ptr(self.data), ptr(out),
                  self.storage, ptr(self.scale), 0, stream_of(self.data.device))
        return out

    def nbytes(self):
        return self.data.numel() * self.data.element_size() + self.scale.numel() * 4


def make_vcd_params(fm_constant, sigma_x, p, q, T, b, max_alpha, positivity, storage,
                    prox_constant=0.0, prox_input_ptr=None):
    """``mbir_vcd_params``; a proximal-map prior is given by the device
    pointer of its (N*N, S) float32 mean and 1 / sigma_prox^2."""
    prm = VcdParams()
    prm.fm_constant = float(fm_constant)
    prm.sigma_x = float(sigma_x)
    prm.p, prm.q, prm.T = float(p), float(q), float(T)
    for j in range(6):
        prm.b[j] = float(b[j])
    prm.max_alpha = float(max_alpha)
    prm.positivity = int(bool(positivity))
    prm.storage = int(storage)
    prm.prox_constant = float(prox_constant)
    prm.reserved = 0
    prm.prox_input = prox_input_ptr
    return prm


class VcdEngine:
    """Constants and workspace of one reconstruction on one device."""

    def __init__(self, geom, view_params, params, fm_hessian_flat, weights=None,
                 dc_profile=None, max_subset_pixels=1):
        self.geom = geom
        self.view_params = view_params
        self.params = params
        self.H = _lib.as_f32_contig(fm_hessian_flat)
        self.weights = weights
        self.dc = None if dc_profile is None else _lib.as_f32_contig(dc_profile)
        self.device = require_cuda(self.H, view_params, self.dc)
        self.num_slices = geom.num_slices
        self.accum = torch.zeros(2 + self.num_slices, dtype=torch.float64, device=self.device)
        self.alpha_buf = torch.zeros(1, dtype=torch.float32, device=self.device)
        self._ws = None
        self._ws_pixels = 0
        self.reserve(max_subset_pixels)

    def reserve(self, max_subset_pixels):
        if max_subset_pixels <= self._ws_pixels:
            return
        n = _lib.query(self.device, 'mbir_vcd_workspace_size', self.geom,
                       int(max_subset_pixels), self.params)
        self._ws = torch.empty(int(n), dtype=torch.uint8, device=self.device)
        self._ws_pixels = int(max_subset_pixels)

    def workspace_bytes(self):
        return 0 if self._ws is None else self._ws.numel()

    def _common(self, err):
        if err.storage != self.params.storage:
            raise ValueError("error sinogram storage does not match the engine's")
        w = self.weights
        return (ptr(err.data), ptr(err.scale), None if w is None else ptr(w.data),
                None if w is None else ptr(w.scale))

    def subset_update(self, flat_recon, err, pixel_indices):
        """One subset update in place; returns (ell1, alpha, delta_sumsq)
        as device tensors (FP64 ell1 and sums, FP32 alpha)."""
        idx = _lib.as_i64_contig(pixel_indices)
        require_cuda(flat_recon, idx)
        self.reserve(idx.shape[0])
        acc = torch.zeros(2 + self.num_slices, dtype=torch.float64, device=self.device)
        e, es, w, wsc = self._common(err)
        _lib.call(self.device, 'mbir_vcd_subset_update', self.geom, ptr(self.view_params),
                  self.params, ptr(flat_recon), e, es, w, wsc, ptr(self.H), ptr(self.dc),
                  ptr(idx), idx.shape[0], ptr(acc), ptr(self.alpha_buf), ptr(self._ws),
                  self._ws.numel(), stream_of(self.device))
        return acc[0], self.alpha_buf[0].clone(), acc[2:]

    def partition_pass(self, flat_recon, err, partition, order, accum=None):
        """All subsets of ``partition`` (K, n) in the host ``order``; adds
        ell1, alpha and per-slice sums of squares into ``accum``."""
        part = _lib.as_i64_contig(partition)
        require_cuda(flat_recon, part)
        K, n = part.shape
        self.reserve(n)
        accum = self.accum if accum is None else accum
        order_np, order_p = host_int32(order)
        e, es, w, wsc = self._common(err)
        _lib.call(self.device, 'mbir_vcd_partition_pass', self.geom, ptr(self.view_params),
                  self.params, ptr(flat_recon), e, es, w, wsc, ptr(self.H), ptr(self.dc),
                  ptr(part), K, n, order_p, ptr(accum), ptr(self._ws), self._ws.numel(),
                  stream_of(self.device))
        del order_np
        return accum


def partition_pass_batched(engines, flats, errs, partitions, orders, accums=None):
    """One VCD iteration of several reconstructions that share a geometry,
    each kernel of the subset step launched once for all of them
    (``mbir_vcd_partition_pass_batched``): job j updates the subsets of
    ``partitions[j]`` (all (K, n)) in ``orders[j]``, exactly as its own
    :meth:`VcdEngine.partition_pass` would."""
    n = len(engines)
    if not 1 <= n <= _lib.MAX_BATCH:
        raise ValueError(f'a batch holds 1 to {_lib.MAX_BATCH} jobs, got {n}')
    e0 = engines[0]
    parts = [_lib.as_i64_contig(p) for p in partitions]
    K, npix = parts[0].shape
    for p in parts:
        if tuple(p.shape) != (K, npix):
            raise ValueError('every job of a batch needs partitions of the same shape')
    require_cuda(*flats, *parts)
    for e in engines:
        e.reserve(npix)
    accums = [e.accum for e in engines] if accums is None else list(accums)
    c = ctypes

    keep = []   # the host arrays must outlive the call

    def arr(vals):
        a = (c.c_void_p * n)(*[None if v is None else v.data_ptr() for v in vals])
        keep.append(a)
        return c.cast(a, c.c_void_p)

    params_arr = (VcdParams * n)(*[e.params for e in engines])
    params = c.cast(params_arr, c.c_void_p)
    order = np.ascontiguousarray(np.stack([np.asarray(o) for o in orders]).astype(np.int32))
    ws_bytes = min(e.workspace_bytes() for e in engines)
    _lib.call(e0.device, 'mbir_vcd_partition_pass_batched', n, e0.geom, ptr(e0.view_params),
              params, arr(flats), arr([r.data for r in errs]), arr([r.scale for r in errs]),
              arr([None if e.weights is None else e.weights.data for e in engines]),
              arr([None if e.weights is None else e.weights.scale for e in engines]),
              arr([e.H for e in engines]), ptr(e0.dc), arr(parts), K, npix,
              order.ctypes.data_as(c.c_void_p), arr(accums), arr([e._ws for e in engines]),
              ws_bytes, stream_of(e0.device))
    return accums


def _refresh(engine, flat_recon, err, pixel_indices, y_vcr):
    idx = _lib.as_i64_contig(pixel_indices)
    require_cuda(flat_recon, idx, y_vcr)
    g = engine.geom
    nbytes = int(_lib.query(engine.device, 'mbir_forward_project_binned_workspace_size', g,
                            g.num_views, idx.shape[0]))
    # the bins' workspace (torch's caching allocator); none: the scanning forward
    ws = torch.empty(nbytes, dtype=torch.uint8, device=engine.device) if nbytes > 0 else None
    _lib.call(engine.device, 'mbir_vcd_refresh_error', g, ptr(engine.view_params),
              ptr(flat_recon), ptr(idx), idx.shape[0], ptr(y_vcr), ptr(err.data),
              ptr(err.scale), err.storage, ptr(ws), 0 if ws is None else ws.numel(),
              stream_of(engine.device))


VcdEngine.refresh_error = _refresh
VcdEngine.refresh_error.__doc__ = (
    "Re-form err = y - A x from the FP32 measured sinogram ``y_vcr`` (V, C, R).")


def iteration_stats(err, weights, flat_recon):
    """FP64 [sum w e^2, sum w, sum e^2, sum |x|] as a device tensor."""
    V, C, R = err.data.shape
    out = torch.empty(4, dtype=torch.float64, device=err.device)
    ws = torch.empty(int(_lib.query(err.device, 'mbir_iteration_stats_workspace_size')),
                     dtype=torch.uint8, device=err.device)
    _lib.call(err.device, 'mbir_iteration_stats', V, R, C, ptr(err.data), ptr(err.scale),
              None if weights is None else ptr(weights.data),
              None if weights is None else ptr(weights.scale), err.storage, ptr(flat_recon),
              flat_recon.numel(), ptr(out), ptr(ws), ws.numel(), stream_of(err.device))
    return out


def error_init(y, ax, weights, scale_to_data):
    """(error = y - alpha Ax, alpha) with the reference's optimal scale
    (tomography_model.py:1666-1712); FP64 reductions on the device."""
    y = _lib.as_f32_contig(y)
    ax = _lib.as_f32_contig(ax)
    w = None if weights is None else _lib.as_f32_contig(weights)
    require_cuda(y, ax, w)
    err = torch.empty_like(y)
    alpha = torch.empty(1, dtype=torch.float64, device=y.device)
    ws = torch.empty(int(_lib.query(y.device, 'mbir_error_init_workspace_size', y.numel())),
                     dtype=torch.uint8, device=y.device)
    _lib.call(y.device, 'mbir_error_init', y.numel(), ptr(y), ptr(ax), ptr(w),
              int(bool(scale_to_data)), ptr(err), ptr(alpha), ptr(ws), ws.numel(),
              stream_of(y.device))
    return err, alpha


def order_array(n_subsets, rng=None):
    """The per-iteration subset order: one draw from numpy's global RNG,
    exactly as the reference (tomography_model.py:2684-2686), or from
    ``rng`` (a RandomState) with the same call."""
    return (np.random if rng is None else rng).permutation(n_subsets).astype(np.int32)
