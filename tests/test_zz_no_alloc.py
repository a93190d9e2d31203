"""mbir_back_project_noalloc: back projection for callers that cannot
allocate device memory.

Some applications own the GPU's memory through another allocator (a
framework's caching pool, a pipeline with a fixed memory budget); they cannot
hand the library a fresh workspace, and a cudaMalloc of the library's own
would bypass that owner.  The no-allocation entry point keeps its scratch in
a static device array instead.  This test calls it through the C ABI and
checks it against mbir_back_project with a caller-provided workspace, on two
calls in a row (the second reuses the static scratch the first one left
behind), for both sinogram layouts and both geometries.  It lives in a file
of its own that pytest collects last.
"""

import ctypes

import numpy as np
import pytest
import torch

import mbirtorch_b200 as mb
from conftest import rel_l2
from mbirtorch_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-6   # same kernels, possibly a different number of view chunks


def _models():
    cone = mb.ConeBeamModel((48, 20, 28), np.linspace(0, 2 * np.pi, 48, endpoint=False),
                            source_detector_dist=200.0, source_iso_dist=100.0)
    par = mb.ParallelBeamModel((36, 12, 30), np.linspace(0, np.pi, 36, endpoint=False))
    for m in (cone, par):
        m.set_params(no_warning=True, verbose=0)
    return cone, par


def _noalloc(m, sino, idx, layout, cp=1):
    lib = _lib.load()
    g = m.projector.geom
    out = torch.empty((idx.shape[0], g.num_slices), dtype=torch.float32, device=sino.device)
    rc = lib.mbir_back_project_noalloc(
        g, ctypes.c_void_p(m.projector.view_params.data_ptr()), 0, g.num_views,
        ctypes.c_void_p(sino.data_ptr()), layout, ctypes.c_void_p(idx.data_ptr()),
        idx.shape[0], cp, 0, g.num_slices, ctypes.c_void_p(out.data_ptr()),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.mbir_last_error().decode()
    return out


@pytest.mark.parametrize("which", [0, 1])
def test_noalloc_matches_workspace_version_twice(which):
    m = _models()[which]
    rs = m.get_params('recon_shape')
    full = torch.as_tensor(mb.gen_full_indices(rs), dtype=torch.int64, device='cuda')
    gen = torch.Generator(device='cuda').manual_seed(7)
    for call in range(2):
        sino = torch.randn(*m.get_params('sinogram_shape'), device='cuda', generator=gen)
        idx = full if call == 0 else full[::5].contiguous()
        for layout in (_lib.MBIR_LAYOUT_VRC, _lib.MBIR_LAYOUT_VCR):
            s_in = sino if layout == _lib.MBIR_LAYOUT_VRC else sino.transpose(1, 2).contiguous()
            for cp in (1, 2):
                got = _noalloc(m, s_in, idx, layout, cp)
                ref = m.projector.back(s_in, idx, coeff_power=cp, layout=layout)
                torch.cuda.synchronize()
                assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= TOL, (call, layout, cp)


def test_noalloc_rejects_oversized_input():
    """A (views, rows, channels) input above the 32 MiB static scratch is
    refused on the host, before any launch."""
    m = mb.ConeBeamModel((300, 128, 256), np.linspace(0, 2 * np.pi, 300, endpoint=False),
                         source_detector_dist=2000.0, source_iso_dist=1000.0)
    m.set_params(no_warning=True, verbose=0)
    lib = _lib.load()
    g = m.projector.geom
    p = ctypes.c_void_p(m.projector.view_params.data_ptr())
    rc = lib.mbir_back_project_noalloc(g, p, 0, g.num_views, p, _lib.MBIR_LAYOUT_VRC, p, 1, 1,
                                       0, g.num_slices, p, None)
    assert rc == 3
    assert "static scratch" in lib.mbir_last_error().decode()
