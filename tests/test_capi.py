"""The C ABI library: it loads, exports every symbol include/mbir_b200.h
declares, and rejects invalid arguments on the host with a message (no
kernel is launched by these checks, so they run without a GPU)."""

import ctypes
import math
import os
import re

import pytest

from conftest import ROOT
from mbirtorch_b200 import _lib
from mbirtorch_b200.kernels import make_geometry

HEADER = os.path.join(ROOT, "include", "mbir_b200.h")


def _declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mbir_[a-z0-9_]+)\s*\(", text)))


def test_library_builds_and_loads():
    lib = _lib.load()
    assert lib.mbir_abi_version() == 10100
    assert os.path.exists(_lib.library_path())


def test_every_declared_symbol_is_exported_and_bound():
    lib = _lib.load()
    declared = _declared_functions()
    assert len(declared) >= 14
    for name in declared:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name


def test_struct_layouts_match_header():
    assert ctypes.sizeof(_lib.Geometry) == 10 * 4 + 10 * 4
    assert ctypes.sizeof(_lib.VcdParams) == 12 * 4 + 2 * 4 + 2 * 4 + 8


def _geom(**kw):
    base = dict(kind='cone', num_views=8, num_det_rows=4, num_det_channels=6,
                num_recon_rows=5, num_recon_cols=5, num_slices=4, psf_radius=1,
                bp_psf_radius=1, delta_voxel=1.0, delta_voxel_row=1.0, delta_voxel_slice=1.0,
                magnification=2.0, source_detector_dist=20.0)
    base.update(kw)
    return make_geometry(**base)


def _fwd(lib, g, **kw):
    args = dict(view_start=0, view_count=g.num_views, band=g.num_slices, slice_start=0,
                layout=0, values=1, idx=1, out=1, vp=1)
    args.update(kw)
    nz = ctypes.c_void_p(16) if args['values'] else None
    return lib.mbir_forward_project(g, ctypes.c_void_p(16) if args['vp'] else None,
                                    args['view_start'], args['view_count'], nz, 3,
                                    args['band'], args['slice_start'],
                                    ctypes.c_void_p(16) if args['idx'] else None,
                                    ctypes.c_void_p(16) if args['out'] else None,
                                    args['layout'], None)


@pytest.mark.parametrize("bad,match", [
    (dict(view_count=9), "view range"),
    (dict(band=5), "slice band"),
    (dict(layout=7), "layout"),
    (dict(values=0), "NULL"),
])
def test_forward_rejects_bad_arguments(bad, match):
    lib = _lib.load()
    rc = _fwd(lib, _geom(), **bad)
    assert rc == 1
    assert re.search(match, lib.mbir_last_error().decode())


def test_geometry_validation():
    lib = _lib.load()
    g = _geom()
    g.psf_radius = 4   # past the unrolled maximum: the C side must refuse it
    assert _fwd(lib, g) == 1
    assert "tap radii" in lib.mbir_last_error().decode()
    assert _fwd(lib, _geom(kind='parallel', num_det_rows=3)) == 1
    assert "num_det_rows == num_slices" in lib.mbir_last_error().decode()
    assert _fwd(lib, _geom(magnification=0.0)) == 1
    with pytest.raises(ValueError):
        make_geometry('cone', 1, 1, 1, 1, 1, 1, psf_radius=5)


def test_back_and_vcd_validation():
    lib = _lib.load()
    g = _geom()
    p = ctypes.c_void_p(16)
    rc = lib.mbir_back_project(g, p, 0, 8, p, 0, p, 3, 3, 0, 4, p, None, 0, None)
    assert rc == 1 and "coeff_power" in lib.mbir_last_error().decode()
    rc = lib.mbir_back_project(g, p, 0, 8, p, 0, p, 3, 1, 0, 4, p, None, 0, None)
    assert rc == 3 and "workspace" in lib.mbir_last_error().decode()
    prm = _lib.VcdParams()
    prm.storage = 9
    rc = lib.mbir_vcd_subset_update(g, p, prm, p, p, p, None, None, p, None, p, 3, p, None,
                                    None, 0, None)
    assert rc == 1 and "storage" in lib.mbir_last_error().decode()
    order = (ctypes.c_int32 * 2)(0, 5)
    rc = lib.mbir_vcd_partition_pass(g, p, prm, p, p, p, None, None, p, None, p, 2, 3,
                                     ctypes.cast(order, ctypes.c_void_p), p, None, 0, None)
    assert rc == 1 and "order" in lib.mbir_last_error().decode()


def test_workspace_sizes_are_positive_and_monotone():
    lib = _lib.load()
    g = _geom(num_views=64, num_det_rows=32, num_det_channels=48, num_recon_rows=32,
              num_recon_cols=32, num_slices=32)
    prm = _lib.VcdParams()
    prm.storage = 0
    a = lib.mbir_vcd_workspace_size(g, 10, prm)
    b = lib.mbir_vcd_workspace_size(g, 100, prm)
    assert 0 < a <= b
    prm.storage = 1
    assert lib.mbir_vcd_workspace_size(g, 100, prm) < b
    assert lib.mbir_back_project_workspace_size(g, 64, 10, 32) > 0
    assert lib.mbir_iteration_stats_workspace_size() > 0
    assert not math.isnan(float(lib.mbir_error_init_workspace_size(100)))
