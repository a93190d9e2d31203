"""The torch-facing boundary on the CPU: every library call runs with its
tensors' device current, the dispatcher ops are registered with correct
shapes, the availability probe answers without raising, and the C side
refuses shapes its launches cannot express."""

import ast
import contextlib
import ctypes
import glob
import os
import re

import pytest
import torch

from conftest import ROOT
from mbirtorch_b200 import _lib, availability
from mbirtorch_b200.kernels import make_geometry


class _FakeLib:
    """Records the device that is current when each ABI function runs."""

    def __init__(self, state):
        self.state = state
        self.seen = []

    def __getattr__(self, name):
        def fn(*args):
            self.seen.append((name, self.state['current']))
            return 0
        return fn


def test_call_makes_the_tensor_device_current(monkeypatch):
    state = {'current': torch.device('cuda', 0)}

    @contextlib.contextmanager
    def fake_device(dev):
        prev = state['current']
        state['current'] = torch.device(dev)
        try:
            yield
        finally:
            state['current'] = prev

    fake = _FakeLib(state)
    monkeypatch.setattr(_lib, 'load', lambda build_if_missing=True: fake)
    monkeypatch.setattr(torch.cuda, 'device', fake_device)
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: True)
    _lib.call(torch.device('cuda', 1), 'mbir_forward_project', 1, 2)
    _lib.query(torch.device('cuda', 3), 'mbir_vcd_workspace_size', 1)
    assert fake.seen == [('mbir_forward_project', torch.device('cuda', 1)),
                         ('mbir_vcd_workspace_size', torch.device('cuda', 3))]
    assert state['current'] == torch.device('cuda', 0)   # restored afterwards


def test_call_raises_with_the_library_message(monkeypatch):
    class Failing:
        def mbir_forward_project(self, *a):
            return 1

        def mbir_last_error(self):
            return b"view range [0, 9) outside [0, 8)"

    monkeypatch.setattr(_lib, 'load', lambda build_if_missing=True: Failing())
    monkeypatch.setattr(torch.cuda, 'device', lambda d: contextlib.nullcontext())
    with pytest.raises(_lib.MbirError, match="view range"):
        _lib.call(torch.device('cuda', 0), 'mbir_forward_project')


def test_no_library_call_bypasses_the_device_guard():
    """Outside _lib.py, ABI functions are reached only by name through
    _lib.call / _lib.query (which bracket the device)."""
    offenders = []
    for path in glob.glob(os.path.join(ROOT, 'mbirtorch_b200', '*.py')):
        if os.path.basename(path) == '_lib.py':
            continue
        tree = ast.parse(open(path).read())
        for node in ast.walk(tree):
            if isinstance(node, ast.Attribute) and node.attr.startswith('mbir_'):
                offenders.append(f"{os.path.basename(path)}:{node.lineno} .{node.attr}")
    assert offenders == []


def test_torch_ops_are_registered_with_shape_functions():
    from torch._subclasses.fake_tensor import FakeTensorMode
    import mbirtorch_b200.torch_ops  # noqa: F401
    ops = torch.ops.mbir_b200
    with FakeTensorMode():
        idx = torch.empty(10, dtype=torch.int64)
        vp = torch.empty(6)
        assert ops.parallel_fwd(torch.empty(10, 4), idx, vp, 4, 4, 7, 1.0, 0.0, 1.0, 1.0,
                                1).shape == (6, 4, 7)
        assert ops.parallel_back(torch.empty(6, 4, 7), idx, vp, 4, 4, 7, 1.0, 0.0, 1.0, 1.0,
                                 1, 2).shape == (10, 4)
        vp2 = torch.empty(6, 2)
        cone = (5, 7, 4, 4, 8, 1., 1., 1., 1., 1., 0., 0., 0., 2., 40., False, 1, 1)
        assert ops.cone_fwd(torch.empty(10, 3), idx, vp2, *cone,
                            slice_start=2).shape == (6, 5, 7)
        assert ops.cone_back(torch.empty(6, 5, 7), idx, vp2, *cone, slice_start=2,
                             band_slices=3).shape == (10, 3)
        assert ops.cone_back(torch.empty(6, 5, 7), idx, vp2, *cone,
                             slice_start=2).shape == (10, 6)


def test_availability_answers_without_raising():
    ok, reason = availability.kernels_available()
    assert isinstance(ok, bool) and isinstance(reason, str) and reason
    if not torch.cuda.is_available():
        assert not ok and 'CUDA' in reason
        assert availability.projectors_usable('cuda:0') == (ok, reason)
        with pytest.raises(RuntimeError, match='unusable'):
            availability.require_usable('cuda:0')


def test_availability_kill_switch(monkeypatch):
    monkeypatch.setenv(availability.DISABLE_ENV_VAR, '1')
    assert availability._probe() == (False, f'disabled by {availability.DISABLE_ENV_VAR}=1')


def _geom(**kw):
    base = dict(kind='cone', num_views=8, num_det_rows=4, num_det_channels=6,
                num_recon_rows=5, num_recon_cols=5, num_slices=4, psf_radius=1,
                bp_psf_radius=1, magnification=2.0, source_detector_dist=20.0)
    base.update(kw)
    return make_geometry(**base)


def test_views_beyond_the_grid_limit_are_refused():
    lib = _lib.load()
    p = ctypes.c_void_p(16)
    g = _geom(num_views=70000)
    rc = lib.mbir_forward_project(g, p, 0, 8, p, 3, 4, 0, p, p, 0, None)
    assert rc == 1 and 'at most 65535 views' in lib.mbir_last_error().decode()
    rc = lib.mbir_sino_convert(0, 70000, 4, 4, p, p, 0, p, 1, None)
    assert rc == 1 and 'views' in lib.mbir_last_error().decode()


def test_noalloc_validates_arguments_before_its_scratch_limit():
    lib = _lib.load()
    p = ctypes.c_void_p(16)
    g = _geom(num_det_rows=-4)
    rc = lib.mbir_back_project_noalloc(g, p, 0, 8, p, 0, p, 3, 1, 0, 4, p, None)
    assert rc == 1 and 'positive' in lib.mbir_last_error().decode()
    g = _geom()
    rc = lib.mbir_back_project_noalloc(g, p, 0, 9, p, 0, p, 3, 1, 0, 4, p, None)
    assert rc == 1 and 'view range' in lib.mbir_last_error().decode()
    g = _geom(num_views=200, num_det_rows=256, num_det_channels=256)
    rc = lib.mbir_back_project_noalloc(g, p, 0, 200, p, 0, p, 3, 1, 0, 4, p, None)
    assert rc == 3 and 'static scratch' in lib.mbir_last_error().decode()


def test_dc_sum_chunks_run_along_grid_x():
    """The DC-sum launch puts the pixel chunks on grid x (limit 2^31 - 1), so
    a subset of every pixel of a 2048 x 2048 volume (131,072 chunks, above
    the 65,535 grid-y limit) is launchable."""
    src = open(os.path.join(ROOT, 'mbirtorch_b200', 'csrc', 'capi.cu')).read()
    m = re.search(r"dim3 gs\(([^,]+),[^;]*;\s*tpre\(st\);\s*launchb<DcSumsB>\(gs", src)
    assert m and m.group(1).strip() == 'w.dc_chunks'
    kern = open(os.path.join(ROOT, 'mbirtorch_b200', 'csrc', 'vcd.cuh')).read()
    assert 'const int chunk = blockIdx.x;' in kern
    assert (2048 * 2048 + 31) // 32 > 65535
