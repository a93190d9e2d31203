"""ctypes binding of ``libmbir_b200.so`` (the C ABI of include/mbir_b200.h).

The library is the only compute path: there is no CPU or eager fallback.
Loading fails loudly when the built library is missing, and every compute
entry point checks that its tensors live on a CUDA device.  Torch is used
for device memory and streams only: tensors are passed to the ABI as raw
device pointers on the current stream of their device.
"""

import ctypes
import os
import threading

import numpy as np
import torch

from . import _build

MBIR_OK = 0
MBIR_ERR_INVALID, MBIR_ERR_CUDA, MBIR_ERR_WORKSPACE = 1, 2, 3
MBIR_PARALLEL, MBIR_CONE = 0, 1
MBIR_LAYOUT_VRC, MBIR_LAYOUT_VCR = 0, 1
MBIR_F32, MBIR_BF16, MBIR_F16 = 0, 1, 2
MAX_TAP_RADIUS = 3
MAX_BATCH = 16

STORAGE_CODES = {'float32': MBIR_F32, 'bfloat16': MBIR_BF16, 'float16': MBIR_F16}
STORAGE_DTYPES = {MBIR_F32: torch.float32, MBIR_BF16: torch.bfloat16, MBIR_F16: torch.float16}


class MbirError(RuntimeError):
    """A failed call into the sm_100a library (message from mbir_last_error)."""


class Geometry(ctypes.Structure):
    """mirror of ``mbir_geometry``."""
    _fields_ = [
        ("geometry", ctypes.c_int32),
        ("num_views", ctypes.c_int32),
        ("num_det_rows", ctypes.c_int32),
        ("num_det_channels", ctypes.c_int32),
        ("num_recon_rows", ctypes.c_int32),
        ("num_recon_cols", ctypes.c_int32),
        ("num_slices", ctypes.c_int32),
        ("psf_radius", ctypes.c_int32),
        ("bp_psf_radius", ctypes.c_int32),
        ("use_curved_detector", ctypes.c_int32),
        ("delta_det_channel", ctypes.c_float),
        ("delta_det_row", ctypes.c_float),
        ("det_channel_offset", ctypes.c_float),
        ("det_row_offset", ctypes.c_float),
        ("delta_voxel", ctypes.c_float),
        ("delta_voxel_row", ctypes.c_float),
        ("delta_voxel_slice", ctypes.c_float),
        ("recon_slice_offset", ctypes.c_float),
        ("magnification", ctypes.c_float),
        ("source_detector_dist", ctypes.c_float),
    ]


class VcdParams(ctypes.Structure):
    """mirror of ``mbir_vcd_params``."""
    _fields_ = [
        ("fm_constant", ctypes.c_float),
        ("sigma_x", ctypes.c_float),
        ("p", ctypes.c_float),
        ("q", ctypes.c_float),
        ("T", ctypes.c_float),
        ("b", ctypes.c_float * 6),
        ("max_alpha", ctypes.c_float),
        ("positivity", ctypes.c_int32),
        ("storage", ctypes.c_int32),
        ("prox_constant", ctypes.c_float),
        ("reserved", ctypes.c_int32),
        ("prox_input", ctypes.c_void_p),
    ]


# Exported symbols and their ctypes signatures.  The CPU test suite checks
# that the built library exports every one of them.
_c = ctypes
_vp = _c.c_void_p
_i32, _i64, _sz = _c.c_int32, _c.c_int64, _c.c_size_t
_GP, _PP = _c.POINTER(Geometry), _c.POINTER(VcdParams)
SIGNATURES = {
    "mbir_abi_version": (_i32, []),
    "mbir_last_error": (_c.c_char_p, []),
    "mbir_launch_count": (_c.c_ulonglong, []),
    "mbir_timing_enable": (_i32, [_i32]),
    "mbir_timing_collect": (_i32, [_c.c_char_p, _i32, _vp, _vp, _i32]),
    "mbir_forward_project": (_i32, [_GP, _vp, _i32, _i32, _vp, _i64, _i32, _i32, _vp, _vp,
                                    _i32, _vp]),
    "mbir_forward_project_volume": (_i32, [_GP, _vp, _i32, _i32, _vp, _vp, _i64, _vp, _i32,
                                           _vp]),
    "mbir_forward_project_binned": (_i32, [_GP, _vp, _i32, _i32, _vp, _i32, _vp, _i64, _vp,
                                           _i32, _vp, _sz, _vp]),
    "mbir_forward_project_binned_workspace_size": (_sz, [_GP, _i32, _i64]),
    "mbir_vcd_refresh_error": (_i32, [_GP, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _i32, _vp, _sz,
                                      _vp]),
    "mbir_back_project_workspace_size": (_sz, [_GP, _i32, _i64, _i32]),
    "mbir_back_project": (_i32, [_GP, _vp, _i32, _i32, _vp, _i32, _vp, _i64, _i32, _i32, _i32,
                                 _vp, _vp, _sz, _vp]),
    "mbir_back_project_noalloc": (_i32, [_GP, _vp, _i32, _i32, _vp, _i32, _vp, _i64, _i32,
                                         _i32, _i32, _vp, _vp]),
    "mbir_sino_convert": (_i32, [_i32, _i32, _i32, _i32, _vp, _vp, _i32, _vp, _i32, _vp]),
    "mbir_error_init": (_i32, [_i64, _vp, _vp, _vp, _i32, _vp, _vp, _vp, _sz, _vp]),
    "mbir_error_init_workspace_size": (_sz, [_i64]),
    "mbir_vcd_workspace_size": (_sz, [_GP, _i64, _PP]),
    "mbir_vcd_subset_update": (_i32, [_GP, _vp, _PP, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                      _i64, _vp, _vp, _vp, _sz, _vp]),
    "mbir_vcd_partition_pass": (_i32, [_GP, _vp, _PP, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                       _i32, _i64, _vp, _vp, _vp, _sz, _vp]),
    "mbir_vcd_partition_pass_batched": (_i32, [_i32, _GP, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                               _vp, _vp, _vp, _i32, _i64, _vp, _vp, _vp, _sz,
                                               _vp]),
    "mbir_iteration_stats": (_i32, [_i32, _i32, _i32, _vp, _vp, _vp, _vp, _i32, _vp, _i64,
                                    _vp, _vp, _sz, _vp]),
    "mbir_iteration_stats_workspace_size": (_sz, []),
    "mbir_denoise_workspace_size": (_sz, [_i32, _i64]),
    "mbir_denoise_pass": (_i32, [_i32, _i32, _i32, _PP, _vp, _vp, _vp, _i32, _i64, _vp, _vp,
                                 _sz, _vp]),
}

_lib = None
_lock = threading.Lock()


def library_path():
    return _build.LIB_PATH


def load(build_if_missing=True):
    """Load (and, when the toolchain is present and the library is missing
    or stale, build) libmbir_b200.so."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIB_PATH
        if build_if_missing and not _build.up_to_date():
            try:
                _build.build()
            except Exception as exc:  # no toolchain: use what is there
                if not os.path.exists(path):
                    raise MbirError(
                        f"{path} is missing and could not be built ({exc}); "
                        "run python -m mbirtorch_b200._build") from exc
        if not os.path.exists(path):
            raise MbirError(f"{path} is missing; run python -m mbirtorch_b200._build")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(rc):
    if rc != MBIR_OK:
        raise MbirError(load().mbir_last_error().decode(errors="replace"))


def call(device, name, *args):
    """Call the ABI function ``name`` with ``device`` current and raise on a
    nonzero return.  The C side launches on the CURRENT device, so every
    call is bracketed by the device of the tensors it is given, whatever
    device the calling thread has current (the reference brackets its
    launches the same way, triton_cone.py:433-445)."""
    fn = getattr(load(), name)
    with torch.cuda.device(device):
        check(fn(*args))


def query(device, name, *args):
    """A size query (``*_workspace_size``) answered for ``device``: launch
    shapes, and so workspace sizes, follow that device's SM count.  Without
    a CUDA device the library answers for a B200."""
    fn = getattr(load(), name)
    device = None if device is None else torch.device(device)
    if device is None or device.type != 'cuda' or not torch.cuda.is_available():
        return fn(*args)
    with torch.cuda.device(device):
        return fn(*args)


def launch_count():
    return int(load().mbir_launch_count())


_timing_on = False


def timing_enable(on=True):
    """Turn the library's per-launch CUDA-event timing on or off; returns
    the previous setting."""
    global _timing_on
    _timing_on = bool(on)
    return bool(load().mbir_timing_enable(int(_timing_on)))


def timing_enabled():
    return _timing_on


def timing_collect(max_entries=64):
    """{kernel name: (total ms, launches)} since the last collect."""
    lib = load()
    names = ctypes.create_string_buffer(8192)
    ms = (ctypes.c_double * max_entries)()
    cnt = (ctypes.c_int64 * max_entries)()
    n = lib.mbir_timing_collect(names, len(names), ctypes.cast(ms, ctypes.c_void_p),
                                ctypes.cast(cnt, ctypes.c_void_p), max_entries)
    keys = names.value.decode().split('\n')[:n]
    return {k: (ms[i], cnt[i]) for i, k in enumerate(keys)}


def require_cuda(*tensors):
    """Every tensor must be a CUDA tensor on one device; returns that device."""
    dev = None
    for t in tensors:
        if t is None:
            continue
        if not t.is_cuda:
            raise RuntimeError(
                "mbirtorch_b200 computes on CUDA only (sm_100a kernels); got a tensor on "
                f"{t.device}.  There is no CPU fallback.")
        if dev is None:
            dev = t.device
        elif t.device != dev:
            raise RuntimeError(f"tensors on different devices: {dev} and {t.device}")
    return dev


def ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_of(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def as_f32_contig(t):
    t = t.to(torch.float32)
    return t if t.is_contiguous() else t.contiguous()


def as_i64_contig(t):
    t = t.to(torch.int64)
    return t if t.is_contiguous() else t.contiguous()


def host_int32(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
    return a, a.ctypes.data_as(ctypes.c_void_p)
