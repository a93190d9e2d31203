"""ctypes wrappers for the C oracle projectors (TEST INFRASTRUCTURE ONLY).

All arrays are converted to contiguous float64 before the call; results are
float64 numpy arrays in the reference bodies' layouts:

  * values    (P, L)      voxel cylinders
  * sinogram  (V, R, C)   views x detector rows x channels
  * back out  (P, L)

The per-function docstrings cite the reference body each one restates.
"""

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "oracle_proj.c")
_BUILD_DIR = os.path.join(_HERE, "_build")
_LIB_PATH = os.path.join(_BUILD_DIR, "liboracle.so")
_lib = None


def library_path():
    return _LIB_PATH


def build(force=False):
    """Compile oracle_proj.c with gcc (-O2 -fopenmp) into _build/liboracle.so."""
    if (not force and os.path.exists(_LIB_PATH)
            and os.path.getmtime(_LIB_PATH) >= os.path.getmtime(_SRC)):
        return _LIB_PATH
    os.makedirs(_BUILD_DIR, exist_ok=True)
    tmp = _LIB_PATH + ".tmp%d" % os.getpid()
    cmd = ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c11",
           "-o", tmp, _SRC, "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, _LIB_PATH)
    return _LIB_PATH


class _CGeom(ctypes.Structure):
    _fields_ = [
        ("num_views", ctypes.c_int32),
        ("num_det_rows", ctypes.c_int32),
        ("num_det_channels", ctypes.c_int32),
        ("num_recon_rows", ctypes.c_int32),
        ("num_recon_cols", ctypes.c_int32),
        ("num_slices", ctypes.c_int32),
        ("delta_det_channel", ctypes.c_double),
        ("delta_det_row", ctypes.c_double),
        ("det_channel_offset", ctypes.c_double),
        ("det_row_offset", ctypes.c_double),
        ("delta_voxel", ctypes.c_double),
        ("delta_voxel_row", ctypes.c_double),
        ("delta_voxel_slice", ctypes.c_double),
        ("recon_slice_offset", ctypes.c_double),
        ("magnification", ctypes.c_double),
        ("source_detector_dist", ctypes.c_double),
        ("use_curved_detector", ctypes.c_int32),
        ("psf_radius", ctypes.c_int32),
        ("bp_psf_radius", ctypes.c_int32),
    ]


@dataclass
class OracleGeometry:
    """Geometry scalars of one model, in the reference's parameter names.

    Parallel beam uses the channel/voxel fields and ``psf_radius`` only
    (``num_slices`` == detector rows); cone beam uses all of them.
    """
    num_det_rows: int
    num_det_channels: int
    num_recon_rows: int
    num_recon_cols: int
    num_slices: int
    delta_det_channel: float = 1.0
    delta_det_row: float = 1.0
    det_channel_offset: float = 0.0
    det_row_offset: float = 0.0
    delta_voxel: float = 1.0
    delta_voxel_row: float = 1.0
    delta_voxel_slice: float = 1.0
    recon_slice_offset: float = 0.0
    magnification: float = 1.0
    source_detector_dist: float = float("inf")
    use_curved_detector: bool = False
    psf_radius: int = 1
    bp_psf_radius: int = 1

    def _c(self, num_views):
        return _CGeom(int(num_views), int(self.num_det_rows),
                      int(self.num_det_channels), int(self.num_recon_rows),
                      int(self.num_recon_cols), int(self.num_slices),
                      float(self.delta_det_channel), float(self.delta_det_row),
                      float(self.det_channel_offset), float(self.det_row_offset),
                      float(self.delta_voxel), float(self.delta_voxel_row),
                      float(self.delta_voxel_slice),
                      float(self.recon_slice_offset), float(self.magnification),
                      float(self.source_detector_dist),
                      int(bool(self.use_curved_detector)),
                      int(self.psf_radius), int(self.bp_psf_radius))


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        d, i64 = P(ctypes.c_double), P(ctypes.c_int64)
        g = P(_CGeom)
        lib.oracle_parallel_forward.argtypes = [g, d, d, ctypes.c_int32, i64,
                                                ctypes.c_int64, d]
        lib.oracle_parallel_back.argtypes = [g, d, d, ctypes.c_int32, i64,
                                             ctypes.c_int64, ctypes.c_int32, d]
        lib.oracle_cone_forward.argtypes = [g, d, d, ctypes.c_int32,
                                            ctypes.c_int32, i64, ctypes.c_int64, d]
        lib.oracle_cone_back.argtypes = [g, d, d, ctypes.c_int32, ctypes.c_int32,
                                         ctypes.c_int32, i64, ctypes.c_int64, d]
        for name in ("oracle_parallel_forward", "oracle_parallel_back",
                     "oracle_cone_forward", "oracle_cone_back"):
            getattr(lib, name).restype = None
        _lib = lib
    return _lib


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _i64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


def parallel_forward(geom, angles, values, pixel_indices):
    """Restates ``_parallel_forward_view_batch`` (parallel_beam.py:56-73):
    (P, L) cylinders -> (V, L, C) sinogram block."""
    angles, values, idx = _f64(angles), _f64(values), _i64(pixel_indices)
    V, (P, L) = angles.shape[0], values.shape
    out = np.empty((V, L, geom.num_det_channels), dtype=np.float64)
    cg = geom._c(V)
    _load().oracle_parallel_forward(ctypes.byref(cg), _dp(angles), _dp(values),
                                    L, _ip(idx), P, _dp(out))
    return out


def parallel_back(geom, angles, sino, pixel_indices, coeff_power=1):
    """Restates ``_parallel_back_view_batch`` (parallel_beam.py:76-94):
    (V, L, C) sinogram -> (P, L) cylinders summed over the views."""
    angles, sino, idx = _f64(angles), _f64(sino), _i64(pixel_indices)
    V, L = angles.shape[0], sino.shape[1]
    P = idx.shape[0]
    out = np.empty((P, L), dtype=np.float64)
    cg = geom._c(V)
    _load().oracle_parallel_back(ctypes.byref(cg), _dp(angles), _dp(sino), L,
                                 _ip(idx), P, int(coeff_power), _dp(out))
    return out


def cone_forward(geom, view_params, values, pixel_indices, slice_start=0):
    """Restates ``_cone_forward_view_batch`` (cone_beam.py:161-234):
    (P, L) band of cylinders -> (V, R, C) partial sinogram."""
    vp, values, idx = _f64(view_params), _f64(values), _i64(pixel_indices)
    vp = vp.reshape(-1, 2)
    V, (P, L) = vp.shape[0], values.shape
    out = np.empty((V, geom.num_det_rows, geom.num_det_channels), np.float64)
    cg = geom._c(V)
    _load().oracle_cone_forward(ctypes.byref(cg), _dp(vp), _dp(values), L,
                                int(slice_start), _ip(idx), P, _dp(out))
    return out


def cone_back(geom, view_params, sino, pixel_indices, coeff_power=1,
              slice_start=0, band_slices=None):
    """Restates ``_cone_back_view_batch`` (cone_beam.py:237-299):
    (V, R, C) sinogram -> (P, band) cylinders summed over the views."""
    vp, sino, idx = _f64(view_params), _f64(sino), _i64(pixel_indices)
    vp = vp.reshape(-1, 2)
    V, P = vp.shape[0], idx.shape[0]
    band = geom.num_slices if band_slices is None else int(band_slices)
    out = np.empty((P, band), dtype=np.float64)
    cg = geom._c(V)
    _load().oracle_cone_back(ctypes.byref(cg), _dp(vp), _dp(sino),
                             int(coeff_power), int(slice_start), band, _ip(idx),
                             P, _dp(out))
    return out
