"""sm_100a projector parity (GPU).

Bars (the reference's own kernel-vs-body gate, triton tests): relative L2
<= 1e-5 for FP32 projections, coeff_power 1 and 2, against both the
reference's torch-body outputs (golden fixtures) and the FP64 oracle; the
adjoint identity <Ax, y> = <x, A^T y> to 1e-5; bitwise determinism.
"""

import math

import numpy as np
import pytest
import torch

import mbirtorch_b200 as mb
from _cases import (PROJECTOR_NAMES, build_model, is_cone, load_projector_case, oracle_back,
                    oracle_forward)
from conftest import rel_l2
from mbirtorch_b200 import _lib, kernels

pytestmark = pytest.mark.gpu
TOL = 1e-5

DEV = 'cuda'


def _t(a, dtype=torch.float32):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device=DEV)


@pytest.mark.parametrize("name", PROJECTOR_NAMES)
@pytest.mark.parametrize("tag", ["full", "subset"])
def test_projectors_match_reference_and_oracle(name, tag):
    d = load_projector_case(name)
    m = build_model(d)
    idx = d[f'{tag}_indices']
    fwd = m.sparse_forward_project(_t(d[f'{tag}_values']), _t(idx, torch.int64)).cpu().numpy()
    assert rel_l2(fwd, d[f'{tag}_fwd']) <= TOL
    assert rel_l2(fwd, oracle_forward(d, d[f'{tag}_values'], idx)) <= TOL
    for cp in (1, 2):
        back = m.sparse_back_project(_t(d[f'{tag}_sino']), _t(idx, torch.int64),
                                     coeff_power=cp).cpu().numpy()
        assert rel_l2(back, d[f'{tag}_back{cp}']) <= TOL, cp
        assert rel_l2(back, oracle_back(d, d[f'{tag}_sino'], idx, cp)) <= TOL, cp


@pytest.mark.parametrize("name", PROJECTOR_NAMES)
def test_body_seam_functions_match_reference(name):
    """The four body functions take the reference bodies' exact arguments."""
    d = load_projector_case(name)
    m = build_model(d)
    g = m._geometry()
    idx = _t(d['subset_indices'], torch.int64)
    vals, sino = _t(d['subset_values']), _t(d['subset_sino'])
    if is_cone(d):
        args = dict(num_rows_r=g.num_det_rows, num_channels=g.num_det_channels,
                    num_recon_rows=g.num_recon_rows, num_recon_cols=g.num_recon_cols,
                    num_slices=g.num_slices, delta_voxel=g.delta_voxel,
                    delta_voxel_row=g.delta_voxel_row, delta_voxel_slice=g.delta_voxel_slice,
                    delta_det_channel=g.delta_det_channel, delta_det_row=g.delta_det_row,
                    det_channel_offset=g.det_channel_offset, det_row_offset=g.det_row_offset,
                    recon_slice_offset=g.recon_slice_offset, magnification=g.magnification,
                    source_detector_dist=g.source_detector_dist,
                    use_curved_detector=bool(g.use_curved_detector), psf_radius=g.psf_radius,
                    bp_psf_radius=g.bp_psf_radius)
        vp = _t(d['view_params'])
        fwd = kernels.cone_forward_view_batch(vals, idx, vp, **args)
        back = kernels.cone_back_view_batch(sino, idx, vp, coeff_power=2, **args)
    else:
        args = dict(num_rows=g.num_recon_rows, num_cols=g.num_recon_cols,
                    num_channels=g.num_det_channels, delta_det_channel=g.delta_det_channel,
                    det_channel_offset=g.det_channel_offset, delta_voxel=g.delta_voxel,
                    delta_voxel_row=g.delta_voxel_row, psf_radius=g.psf_radius)
        vp = _t(d['view_params'])
        fwd = kernels.parallel_forward_view_batch(vals, idx, vp, **args)
        back = kernels.parallel_back_view_batch(sino, idx, vp, coeff_power=2, **args)
    assert rel_l2(fwd.cpu().numpy(), d['subset_fwd']) <= TOL
    assert rel_l2(back.cpu().numpy(), d['subset_back2']) <= TOL


@pytest.mark.parametrize("name", PROJECTOR_NAMES)
def test_adjoint_identity(name):
    """<Ax, y> == <x, A^T y>: relative 1e-5 on positive inputs (the
    reference's test_adjoint.py:15-34 uses uniform [0, 1) values), and for
    signed inputs normalised by ||Ax|| ||y|| (the signed inner product
    cancels, so its own magnitude is no scale)."""
    d = load_projector_case(name)
    m = build_model(d)
    idx = _t(d['full_indices'], torch.int64)
    for x, y, signed in ((_t(np.abs(d['full_values'])), _t(np.abs(d['full_sino'])), False),
                         (_t(d['full_values']), _t(d['full_sino']), True)):
        ax = m.sparse_forward_project(x, idx).double()
        aty = m.sparse_back_project(y, idx).double()
        lhs = float((ax * y.double()).sum())
        rhs = float((x.double() * aty).sum())
        if signed:
            assert abs(lhs - rhs) / float(ax.norm() * y.double().norm()) <= 1e-6
        else:
            assert abs(lhs - rhs) / max(abs(lhs), abs(rhs)) <= TOL


def _cone_model(views=90, rows=40, chans=56, curved=False, helical=False, sdd=300.0, sid=150.0):
    ang = np.linspace(0, (4 if helical else 2) * np.pi, views, endpoint=False)
    zs = np.linspace(-4.0, 4.0, views) if helical else None
    m = mb.ConeBeamModel((views, rows, chans), ang, sdd, sid, helical_z_shifts=zs,
                         use_curved_detector=curved)
    m.set_params(no_warning=True, verbose=0)
    return m


def _oracle_geom(m):
    from oracle import OracleGeometry
    g = m._geometry()
    return OracleGeometry(
        num_det_rows=g.num_det_rows, num_det_channels=g.num_det_channels,
        num_recon_rows=g.num_recon_rows, num_recon_cols=g.num_recon_cols,
        num_slices=g.num_slices, delta_det_channel=g.delta_det_channel,
        delta_det_row=g.delta_det_row, det_channel_offset=g.det_channel_offset,
        det_row_offset=g.det_row_offset, delta_voxel=g.delta_voxel,
        delta_voxel_row=g.delta_voxel_row, delta_voxel_slice=g.delta_voxel_slice,
        recon_slice_offset=g.recon_slice_offset, magnification=g.magnification,
        source_detector_dist=g.source_detector_dist,
        use_curved_detector=bool(g.use_curved_detector), psf_radius=g.psf_radius,
        bp_psf_radius=g.bp_psf_radius)


@pytest.mark.parametrize("kind", ["flat", "curved", "helical"])
def test_medium_cone_vs_oracle(kind):
    """A case large enough for multi-round pixel lists and view chunking."""
    import oracle
    m = _cone_model(curved=kind == 'curved', helical=kind == 'helical')
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(3)
    idx = mb.gen_full_indices(rs).astype(np.int64)
    x = rng.standard_normal((idx.size, rs[2])).astype(np.float32)
    y = rng.standard_normal(m.get_params('sinogram_shape')).astype(np.float32)
    g = _oracle_geom(m)
    vp = m._view_params_array().astype(np.float64)
    f = m.sparse_forward_project(_t(x), _t(idx, torch.int64)).cpu().numpy()
    assert rel_l2(f, oracle.cone_forward(g, vp, x, idx)) <= TOL
    sub = np.sort(rng.choice(idx, size=37, replace=False))
    b = m.sparse_back_project(_t(y), _t(sub, torch.int64)).cpu().numpy()
    assert rel_l2(b, oracle.cone_back(g, vp, y, sub)) <= TOL


def test_medium_parallel_vs_oracle_with_view_tail():
    import oracle
    m = mb.ParallelBeamModel((141, 37, 90), np.linspace(0, np.pi, 141, endpoint=False))
    m.set_params(no_warning=True, verbose=0)
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(4)
    idx = mb.gen_full_indices(rs).astype(np.int64)
    x = rng.standard_normal((idx.size, rs[2])).astype(np.float32)
    y = rng.standard_normal(m.get_params('sinogram_shape')).astype(np.float32)
    g = _oracle_geom(m)
    vp = m._view_params_array().astype(np.float64)
    f = m.sparse_forward_project(_t(x), _t(idx, torch.int64)).cpu().numpy()
    assert rel_l2(f, oracle.parallel_forward(g, vp, x, idx)) <= TOL
    for n in (1, 31, 255, 257):
        sub = np.sort(rng.choice(idx, size=n, replace=False))
        b = m.sparse_back_project(_t(y), _t(sub, torch.int64), coeff_power=2).cpu().numpy()
        assert rel_l2(b, oracle.parallel_back(g, vp, y, sub, 2)) <= TOL, n


@pytest.mark.parametrize("rows", [16, 32, 64, 128])
def test_parallel_back_four_slices_per_lane_team_widths(rows):
    """Rows a multiple of 4 take the back projector with four consecutive
    slices per lane, in teams of 4, 8, 16 and 32 lanes (16, 32, 64 and 128
    rows): full and subset back projections, coefficient power 1 and 2,
    against the FP64 oracle."""
    import oracle
    m = mb.ParallelBeamModel((37, rows, 48), np.linspace(0, np.pi, 37, endpoint=False))
    m.set_params(no_warning=True, verbose=0)
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(rows)
    idx = mb.gen_full_indices(rs).astype(np.int64)
    y = rng.standard_normal(m.get_params('sinogram_shape')).astype(np.float32)
    g = _oracle_geom(m)
    vp = m._view_params_array().astype(np.float64)
    for cp in (1, 2):
        b = m.sparse_back_project(_t(y), _t(idx, torch.int64), coeff_power=cp).cpu().numpy()
        assert rel_l2(b, oracle.parallel_back(g, vp, y, idx, cp)) <= TOL, cp
    sub = np.sort(rng.choice(idx, size=33, replace=False))
    b = m.sparse_back_project(_t(y), _t(sub, torch.int64)).cpu().numpy()
    assert rel_l2(b, oracle.parallel_back(g, vp, y, sub, 1)) <= TOL


def test_cone_slice_band_and_layouts():
    """Banded cone calls sum to the unbanded projection; VCR == VRC^T."""
    m = _cone_model(views=30, rows=24, chans=32)
    rs = m.get_params('recon_shape')
    idx = _t(mb.gen_full_indices(rs), torch.int64)
    x = torch.randn(idx.shape[0], rs[2], device=DEV)
    full = m.projector.forward(x, idx)
    s0 = rs[2] // 3
    banded = m.projector.forward(x[:, :s0].contiguous(), idx, slice_start=0) + \
        m.projector.forward(x[:, s0:].contiguous(), idx, slice_start=s0)
    assert rel_l2(banded.cpu().numpy(), full.cpu().numpy()) <= TOL
    vcr = m.projector.forward(x, idx, layout=_lib.MBIR_LAYOUT_VCR)
    assert torch.equal(vcr.transpose(1, 2), full)
    y = torch.randn(*full.shape, device=DEV)
    b_full = m.projector.back(y, idx)
    b_band = m.projector.back(y, idx, slice_start=s0, band_slices=rs[2] - s0)
    assert rel_l2(b_band.cpu().numpy(), b_full[:, s0:].cpu().numpy()) <= TOL
    b_vcr = m.projector.back(y.transpose(1, 2).contiguous(), idx, layout=_lib.MBIR_LAYOUT_VCR)
    assert torch.equal(b_vcr, b_full)


def test_deterministic_repeat():
    m = _cone_model(views=60, rows=30, chans=40)
    rs = m.get_params('recon_shape')
    idx = _t(mb.gen_full_indices(rs), torch.int64)
    x = torch.randn(idx.shape[0], rs[2], device=DEV)
    y = torch.randn(*m.get_params('sinogram_shape'), device=DEV)
    f1, f2 = m.projector.forward(x, idx), m.projector.forward(x, idx)
    b1, b2 = m.projector.back(y, idx[:50]), m.projector.back(y, idx[:50])
    assert torch.equal(f1, f2) and torch.equal(b1, b2)


def test_full_volume_api_roundtrip():
    """forward_project / back_project on volumes: ROR masking and numpy out."""
    m = mb.ParallelBeamModel((48, 8, 40), np.linspace(0, np.pi, 48, endpoint=False))
    m.set_params(no_warning=True, verbose=0)
    rs = m.get_params('recon_shape')
    vol = np.random.default_rng(0).random(rs).astype(np.float32)
    s = m.forward_project(vol)
    assert isinstance(s, np.ndarray) and s.shape == tuple(m.get_params('sinogram_shape'))
    b = m.back_project(s)
    mask = mb.get_2d_ror_mask(rs)
    assert np.all(b[~mask] == 0)
    y = np.random.default_rng(1).random(s.shape).astype(np.float32)
    lhs = float(np.sum(s.astype(np.float64) * y))
    rhs = float(np.sum(vol[mask].astype(np.float64) * m.back_project(y)[mask]))
    assert abs(lhs - rhs) / abs(lhs) <= TOL


def test_empty_and_single_pixel():
    m = _cone_model(views=12, rows=10, chans=14)
    rs = m.get_params('recon_shape')
    empty = torch.zeros(0, dtype=torch.int64, device=DEV)
    out = m.projector.forward(torch.zeros(0, rs[2], device=DEV), empty)
    assert out.shape[0] == 12 and float(out.abs().sum()) == 0.0
    assert m.projector.back(torch.randn(12, 10, 14, device=DEV), empty).shape == (0, rs[2])
    one = _t([int(mb.gen_full_indices(rs)[len(mb.gen_full_indices(rs)) // 2])], torch.int64)
    f = m.projector.forward(torch.ones(1, rs[2], device=DEV), one)
    assert float(f.sum()) > 0 and math.isfinite(float(f.sum()))


def _direct_forward(m, x, idx, entry, layout=_lib.MBIR_LAYOUT_VRC, view_start=0,
                    view_count=None, ws_bytes=None, by_pixel=0):
    """One call of the scanning ('scan') or binned ('binned') forward entry
    point on whole cylinders, into an output pre-filled with NaN (every cell
    must be written)."""
    from mbirtorch_b200._lib import ptr, stream_of
    g = m._geometry()
    p = m.projector
    vc = g.num_views - view_start if view_count is None else view_count
    shape = ((vc, g.num_det_rows, g.num_det_channels) if layout == _lib.MBIR_LAYOUT_VRC
             else (vc, g.num_det_channels, g.num_det_rows))
    out = torch.full(shape, float('nan'), device=DEV)
    if entry == 'scan':
        _lib.call(x.device, 'mbir_forward_project', g, ptr(p.view_params), view_start, vc,
                  ptr(x), idx.shape[0], g.num_slices, 0, ptr(idx), ptr(out), layout,
                  stream_of(x.device))
    else:
        need = int(_lib.query(x.device, 'mbir_forward_project_binned_workspace_size', g, vc,
                              idx.shape[0]))
        assert need > 0
        ws = torch.empty(need if ws_bytes is None else ws_bytes, dtype=torch.uint8, device=DEV)
        _lib.call(x.device, 'mbir_forward_project_binned', g, ptr(p.view_params), view_start,
                  vc, ptr(x), by_pixel, ptr(idx), idx.shape[0], ptr(out), layout, ptr(ws),
                  ws.numel(), stream_of(x.device))
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("case", ["parallel37", "parallel128", "cone_flat", "cone_helical"])
def test_binned_full_forward_matches_oracle_and_scanning(case):
    """The binned whole-cylinder forward (mbir_forward_project_binned) against
    the FP64 oracle (1e-5) and the scanning forward (same operator, another
    summation order: 1e-6), in both layouts, over view ranges, with a
    workspace of one view's bins (one chunk per view), from a gathered array
    and from the flat volume; a sparse subset leaves tiles no pixel reaches,
    which must come out zero (the output starts as NaN)."""
    import oracle
    rng = np.random.default_rng(11)
    if case.startswith('parallel'):
        rows = 37 if case == 'parallel37' else 128
        m = mb.ParallelBeamModel((61, rows, 90), np.linspace(0, np.pi, 61, endpoint=False))
        m.set_params(no_warning=True, verbose=0)
    else:
        m = _cone_model(views=45, helical=case == 'cone_helical')
    rs = m.get_params('recon_shape')
    idx_np = mb.gen_full_indices(rs).astype(np.int64)
    idx = _t(idx_np, torch.int64)
    x_np = rng.standard_normal((idx_np.size, rs[2])).astype(np.float32)
    x = _t(x_np)
    g = _oracle_geom(m)
    vp = m._view_params_array().astype(np.float64)
    ref = (oracle.parallel_forward(g, vp, x_np, idx_np) if case.startswith('parallel')
           else oracle.cone_forward(g, vp, x_np, idx_np))
    scan = _direct_forward(m, x, idx, 'scan')
    binned = _direct_forward(m, x, idx, 'binned')
    assert not torch.isnan(binned).any()
    assert rel_l2(binned.cpu().numpy(), ref) <= TOL
    assert rel_l2(binned.cpu().numpy(), scan.cpu().numpy()) <= 1e-6
    # channel-major layout, a view range, one view per chunk
    one = int(_lib.query(x.device, 'mbir_forward_project_binned_workspace_size', m._geometry(),
                         1, idx.shape[0]))
    part = _direct_forward(m, x, idx, 'binned', layout=_lib.MBIR_LAYOUT_VCR, view_start=7,
                           view_count=20, ws_bytes=one)
    assert torch.equal(part.transpose(1, 2), binned[7:27])
    # cylinders read from the flat volume
    flat = torch.zeros(rs[0] * rs[1], rs[2], device=DEV)
    flat[idx] = x
    by_pix = _direct_forward(m, flat, idx, 'binned', by_pixel=1)
    assert torch.equal(by_pix, binned)
    # a sparse subset: most tiles receive no pixel
    sub = _t(np.sort(rng.choice(idx_np, size=5, replace=False)), torch.int64)
    xs = torch.randn(5, rs[2], device=DEV)
    sb = _direct_forward(m, xs, sub, 'binned')
    ss = _direct_forward(m, xs, sub, 'scan')
    assert not torch.isnan(sb).any()
    assert rel_l2(sb.cpu().numpy(), ss.cpu().numpy()) <= 1e-6
    assert torch.equal(sb == 0, ss == 0) and int((sb == 0).sum()) > sb.numel() // 2


def test_binned_full_forward_refusals():
    """Refused on the host: a workspace too small for one view's bins, an
    unaligned workspace, and a geometry the binned kernels do not cover."""
    import ctypes
    from mbirtorch_b200._lib import ptr, stream_of
    m = mb.ParallelBeamModel((20, 8, 40), np.linspace(0, np.pi, 20, endpoint=False))
    m.set_params(no_warning=True, verbose=0)
    rs = m.get_params('recon_shape')
    idx = _t(mb.gen_full_indices(rs), torch.int64)
    x = torch.randn(idx.shape[0], rs[2], device=DEV)
    g = m._geometry()
    out = torch.empty(20, 8, 40, device=DEV)
    ws = torch.empty(4096, dtype=torch.uint8, device=DEV)
    lib = _lib.load()
    for base, nbytes in ((ptr(ws), 1024), (ctypes.c_void_p(ws.data_ptr() + 16), 4000)):
        rc = lib.mbir_forward_project_binned(g, ptr(m.projector.view_params), 0, 20, ptr(x), 0,
                                             ptr(idx), idx.shape[0], ptr(out), 0, base, nbytes,
                                             stream_of(x.device))
        assert rc == _lib.MBIR_ERR_WORKSPACE
    g2 = kernels.make_geometry('parallel', 20, 8, 40, rs[0], rs[1], rs[2], 2)
    assert lib.mbir_forward_project_binned_workspace_size(g2, 20, idx.shape[0]) == 0
    rc = lib.mbir_forward_project_binned(g2, ptr(m.projector.view_params), 0, 20, ptr(x), 0,
                                         ptr(idx), idx.shape[0], ptr(out), 0, ptr(ws), 4096,
                                         stream_of(x.device))
    assert rc == _lib.MBIR_ERR_INVALID
