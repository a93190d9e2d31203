"""VCD reconstruction parity on the GPU.

* Seeded recon() against the reference's own seeded recon (golden traces):
  relative L2 <= 1e-4 on the volume after the fixed iteration count, and
  the fm_rmse / alpha traces to 1e-4 (the reconstruction parity bar).
* The same against the FP64 oracle.
* Mixed-precision storage (bfloat16, float16) against the FP64 oracle at
  relative L2 <= 1e-3.
* Bitwise reproducibility and the subset-updater / partition seams.
"""

import numpy as np
import pytest
import torch

import mbirtorch_b200 as mb
from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

GRANULARITY = [1, 2, 4, 8, 16, 32, 64, 128, 128, 128, 128]
SEQUENCE = [2, 4, 6] + [7, 8, 9, 10] * 25


def _model(name, d):
    V = d['sino'].shape[0]
    if name.startswith('recon_parallel'):
        m = mb.ParallelBeamModel(d['sino'].shape, np.linspace(0, np.pi, V, endpoint=False))
    else:
        zs = d['z_shifts'] if name == 'recon_cone_helical' else None
        ang = np.linspace(0, (4 if name == 'recon_cone_helical' else 2) * np.pi, V,
                          endpoint=False)
        m = mb.ConeBeamModel(d['sino'].shape, ang, 64.0, 32.0, helical_z_shifts=zs)
    m.set_params(no_warning=True, verbose=0)
    if name == 'recon_parallel_weighted':
        m.set_params(no_warning=True, positivity_flag=True)
    return m


def _run(name, storage='float32'):
    d = load_golden(f'{name}.npz')
    m = _model(name, d)
    m.set_storage_precision(storage)
    np.random.seed(int(d['seed']))
    w = d['weights'] if 'weights' in d.files else None
    rec, rd = m.recon(d['sino'], weights=w, max_iterations=int(d['max_iterations']),
                      stop_threshold_change_pct=0, logfile_path=None, print_logs=False)
    return d, m, rec, rd


def _oracle(name, m, d):
    from oracle import OracleGeometry, vcd
    g = m._geometry()
    og = OracleGeometry(
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
    kind = 'cone' if name.startswith('recon_cone') else 'parallel'
    prob = vcd.Problem(kind, og, m._view_params_array(), m.get_params('recon_shape'),
                       source_iso_dist=32.0)
    np.random.seed(int(d['seed']))
    parts = [vcd.pixel_partition(prob.recon_shape, n) for n in GRANULARITY]
    seq = vcd.partition_sequence(SEQUENCE, int(d['max_iterations']))
    w = d['weights'] if 'weights' in d.files else None
    dc = vcd.dc_damping_profile(prob) if kind == 'cone' else None
    return vcd.recon(prob, d['sino'], d['reg'][0], d['reg'][1], parts, seq, weights=w,
                     dc_profile=dc, positivity=w is not None)


NAMES = ["recon_parallel", "recon_parallel_weighted", "recon_cone", "recon_cone_helical"]


@pytest.mark.parametrize("name", NAMES)
def test_recon_matches_reference_and_oracle(name):
    d, m, rec, rd = _run(name)
    rp = rd['recon_params']
    np.testing.assert_allclose(rp['regularization_params']['sigma_y'], d['reg'][0], rtol=1e-6)
    assert rel_l2(rec, d['recon']) <= 1e-4
    np.testing.assert_allclose(rp['fm_rmse'], d['fm_rmse'], rtol=1e-4)
    np.testing.assert_allclose(rp['alpha_values'], d['alpha'], rtol=1e-4)
    orec, _ = _oracle(name, m, d)
    assert rel_l2(rec, orec) <= 1e-4
    assert rp['num_iterations'] == int(d['max_iterations'])
    assert len(rp['delta_norm_per_slice']) == int(d['max_iterations'])


# Both 16-bit storages are held to the north-star bar against the FP64
# oracle.  bfloat16 runs finish their last iterations with the error
# sinogram re-formed in float16 (the same two bytes a cell), which removes
# the quantization noise bfloat16's 8-bit significand leaves in the volume.
MP_TOL = {"float16": 1e-3, "bfloat16": 1e-3}


@pytest.mark.parametrize("storage", ["bfloat16", "float16"])
@pytest.mark.parametrize("name", ["recon_parallel", "recon_cone", "recon_parallel_weighted"])
def test_mixed_precision_vs_fp64_oracle(name, storage):
    d, m, rec, _ = _run(name, storage)
    orec, _ = _oracle(name, m, d)
    assert rel_l2(rec, orec) <= MP_TOL[storage]


def test_recon_is_bitwise_reproducible():
    _, _, r1, d1 = _run("recon_cone")
    _, _, r2, d2 = _run("recon_cone")
    assert np.array_equal(r1, r2)
    assert d1['recon_params']['fm_rmse'] == d2['recon_params']['fm_rmse']


def test_subset_updater_seam_matches_oracle_step():
    """create_vcd_subset_updater on a (V, R, C) tensor: one subset step
    against the FP64 oracle's SubsetUpdater from the same state."""
    from oracle import vcd as ovcd
    d = load_golden('recon_cone.npz')
    m = _model('recon_cone', d)
    m.auto_set_regularization_params(d['sino'])
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(5)
    x0 = (0.1 * rng.random(rs)).astype(np.float32)
    e0 = d['sino'] - m.forward_project(x0)
    H = m.compute_hessian_diagonal()
    upd = m.create_vcd_subset_updater(H, weights=1)
    idx = np.sort(rng.choice(mb.gen_full_indices(rs), size=20, replace=False)).astype(np.int64)
    flat = torch.as_tensor(x0.reshape(-1, rs[2]), device='cuda').clone()
    err = torch.as_tensor(e0, device='cuda').clone()
    flat, err, ell1, alpha, sumsq = upd(flat, err, torch.as_tensor(idx, device='cuda'))
    prob = _oracle_problem(m)
    sy, sx = m.get_params(['sigma_y', 'sigma_x'])
    ou = ovcd.SubsetUpdater(prob, H.reshape(-1, rs[2]), None, sy, sx,
                            dc_profile=ovcd.dc_damping_profile(prob))
    oflat = x0.reshape(-1, rs[2]).astype(np.float64)
    oerr = e0.astype(np.float64)
    oell1, oalpha, osumsq = ou(oflat, oerr, idx)
    assert abs(float(alpha) - oalpha) / oalpha <= 1e-4
    assert rel_l2(flat.cpu().numpy(), oflat) <= 1e-5
    assert rel_l2(err.cpu().numpy(), oerr) <= 1e-5
    assert abs(float(ell1) - oell1) / oell1 <= 1e-4
    assert rel_l2(sumsq.cpu().numpy(), osumsq) <= 1e-4


def _oracle_problem(m):
    from oracle import OracleGeometry, vcd
    g = m._geometry()
    og = OracleGeometry(
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
    kind = 'cone' if g.geometry == 1 else 'parallel'
    return vcd.Problem(kind, og, m._view_params_array(), m.get_params('recon_shape'),
                       source_iso_dist=m.get_params('source_iso_dist') if kind == 'cone'
                       else None)


def test_checkpoint_resume_matches_continuous_run():
    """_vcd_recon's init_error_sinogram / fm_hessian resume path: 2 + 1
    iterations equal 3 (same partition order)."""
    d = load_golden('recon_parallel.npz')
    m = _model('recon_parallel', d)
    m.auto_set_regularization_params(d['sino'])
    rs = m.get_params('recon_shape')
    parts = [mb.gen_pixel_partition(rs, n) for n in (4, 16, 64)]
    np.random.seed(1)
    full, _ = m._vcd_recon(d['sino'], parts, np.array([0, 1, 2]), 0)
    np.random.seed(1)
    r1, _, ck = m._vcd_recon(d['sino'], parts, np.array([0, 1]), 0, return_checkpoint=True)
    r2, _ = m._vcd_recon(d['sino'], parts, np.array([2]), 0, init_recon=r1,
                         init_error_sinogram=ck['error_sinogram'], fm_hessian=ck['fm_hessian'])
    assert rel_l2(r2.cpu().numpy(), full.cpu().numpy()) <= 1e-6


def test_recon_simple_parallel_equals_model_path():
    d = load_golden('recon_parallel.npz')
    np.random.seed(3)
    r1, _ = mb.recon_simple_parallel(d['sino'], np.linspace(0, np.pi, d['sino'].shape[0],
                                                            endpoint=False), max_iterations=2)
    np.random.seed(3)
    m = mb.ParallelBeamModel(d['sino'].shape, np.linspace(0, np.pi, d['sino'].shape[0],
                                                          endpoint=False))
    r2, _ = m.recon(d['sino'], max_iterations=2)
    assert rel_l2(r1, r2) <= 1e-6


def test_cone_subset_step_binned_view_chunks_weights_positivity():
    """A whole-image cone subset (65536 pixels x 40 views) splits the binned
    forward into view chunks; weighted, with positivity: one step against
    the FP64 oracle."""
    from oracle import vcd as ovcd
    V = 40
    m = mb.ConeBeamModel((V, 8, 320), np.linspace(0, 2 * np.pi, V, endpoint=False),
                         2048.0, 1024.0)
    m.set_params(no_warning=True, verbose=0, delta_det_channel=2.0, delta_det_row=2.0)
    m.auto_set_recon_geometry(no_warning=True)
    m.set_params(no_warning=True, recon_shape=(256, 256, 4), positivity_flag=True)
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(11)
    x_true = rng.random(rs).astype(np.float32)
    sino = m.forward_project(x_true)
    w = (0.5 + rng.random(sino.shape)).astype(np.float32)
    m.auto_set_regularization_params(sino, weights=w)
    x0 = (0.05 * rng.standard_normal(rs)).astype(np.float32)
    e0 = sino - m.forward_project(x0)
    H = m.compute_hessian_diagonal(weights=w)
    upd = m.create_vcd_subset_updater(H, weights=torch.as_tensor(w, device='cuda'))
    idx = np.arange(rs[0] * rs[1], dtype=np.int64)
    flat = torch.as_tensor(x0.reshape(-1, rs[2]), device='cuda').clone()
    err = torch.as_tensor(e0, device='cuda').clone()
    flat, err, ell1, alpha, sumsq = upd(flat, err, torch.as_tensor(idx, device='cuda'))
    prob = _oracle_problem(m)
    sy, sx = m.get_params(['sigma_y', 'sigma_x'])
    ou = ovcd.SubsetUpdater(prob, H.reshape(-1, rs[2]), w, sy, sx, positivity=True,
                            dc_profile=ovcd.dc_damping_profile(prob))
    oflat = x0.reshape(-1, rs[2]).astype(np.float64)
    oerr = e0.astype(np.float64)
    _, oalpha, _ = ou(oflat, oerr, idx)
    assert abs(float(alpha) - oalpha) / oalpha <= 1e-4
    assert rel_l2(flat.cpu().numpy(), oflat) <= 1e-5
    assert rel_l2(err.cpu().numpy(), oerr) <= 1e-5


def test_sixteen_bit_view_scales_are_powers_of_two():
    from mbirtorch_b200.vcd_engine import ResidentSinogram
    rng = np.random.default_rng(2)
    s = torch.as_tensor((rng.standard_normal((7, 5, 6)) * 10 ** rng.uniform(-3, 3, (7, 1, 1)))
                        .astype(np.float32), device='cuda')
    s[3] = 0
    vmax = s.abs().amax(dim=(1, 2)).cpu().numpy()
    # float16: max |e_v| / scale in (128, 256]; bfloat16 keeps f32's exponent
    # range and a unit scale.
    r = ResidentSinogram.from_vrc(s, 2)
    sc = r.scale.cpu().numpy().astype(np.float64)
    assert np.array_equal(np.exp2(np.round(np.log2(sc))), sc)
    assert np.all(vmax / sc <= 256) and np.all((vmax == 0) | (vmax / sc > 128))
    assert rel_l2(r.to_vrc().cpu().numpy(), s.cpu().numpy()) <= 1e-3
    r = ResidentSinogram.from_vrc(s, 1)
    assert np.all(r.scale.cpu().numpy() == 1)
    assert rel_l2(r.to_vrc().cpu().numpy(), s.cpu().numpy()) <= 4e-3


@pytest.mark.parametrize("name", ["prox_parallel", "prox_cone"])
def test_prox_map_matches_reference_and_oracle(name):
    """prox_map (proximal-map prior) against the reference's seeded run and
    the FP64 oracle."""
    from oracle import vcd as ovcd
    d = load_golden(f'{name}.npz')
    V = d['sino'].shape[0]
    if name == 'prox_parallel':
        m = mb.ParallelBeamModel(d['sino'].shape, np.linspace(0, np.pi, V, endpoint=False))
        sigma_prox = None
    else:
        m = mb.ConeBeamModel(d['sino'].shape, np.linspace(0, 2 * np.pi, V, endpoint=False),
                             64.0, 32.0)
        sigma_prox = float(d['sigma_prox'])
    m.set_params(no_warning=True, verbose=0)
    np.random.seed(int(d['seed']))
    rec, rd = m.prox_map(d['prox_input'], d['sino'], sigma_prox=sigma_prox,
                         max_iterations=int(d['max_iterations']), stop_threshold_change_pct=0,
                         logfile_path=None, print_logs=False)
    rp = rd['recon_params']
    assert rel_l2(rec, d['recon']) <= 1e-4
    np.testing.assert_allclose(rp['fm_rmse'], d['fm_rmse'], rtol=1e-4)
    np.testing.assert_allclose(rp['alpha_values'], d['alpha'], rtol=1e-4)
    np.testing.assert_allclose(rp['regularization_params']['sigma_prox'], d['reg'][2],
                               rtol=1e-6)
    prob = _oracle_problem(m)
    np.random.seed(int(d['seed']))
    parts = [ovcd.pixel_partition(prob.recon_shape, n) for n in GRANULARITY]
    seq = ovcd.partition_sequence(SEQUENCE, int(d['max_iterations']))
    dc = ovcd.dc_damping_profile(prob) if name == 'prox_cone' else None
    orec, _ = ovcd.recon(prob, d['sino'], d['reg'][0], d['reg'][1], parts, seq, dc_profile=dc,
                         prox_input=d['prox_input'], sigma_prox=float(d['reg'][2]))
    assert rel_l2(rec, orec) <= 1e-4
    # a second call reusing the first call's partitions and regularization
    rec2, _ = m.prox_map(rec, d['sino'], sigma_prox=sigma_prox, do_initialization=False,
                         max_iterations=1, logfile_path=None, print_logs=False)
    assert np.isfinite(rec2).all() and rec2.shape == rec.shape
    with pytest.raises(ValueError, match='prox_input'):
        m.prox_map(d['prox_input'][:, :, :2], d['sino'], max_iterations=1, logfile_path=None,
                   print_logs=False)


def test_cone_partition_pass_truncated_detector_ragged_channels():
    """A partition pass (each step bins the next subset in its tail) on a
    cone geometry whose detector (37 channels: a ragged last channel block)
    sees only the middle of the object: pixels centred off the detector,
    and on its edge channels -1 and C, against the FP64 oracle applying the
    same subsets in the same order."""
    from oracle import vcd as ovcd
    from mbirtorch_b200.vcd_engine import ResidentSinogram
    from mbirtorch_b200 import _lib
    V, R, C = 24, 8, 37
    m = mb.ConeBeamModel((V, R, C), np.linspace(0, 2 * np.pi, V, endpoint=False), 512.0, 256.0)
    m.set_params(no_warning=True, verbose=0, delta_det_channel=2.0, delta_det_row=2.0)
    m.auto_set_recon_geometry(no_warning=True)
    m.set_params(no_warning=True, recon_shape=(48, 48, 4))
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(17)
    x_true = rng.random(rs).astype(np.float32)
    sino = m.forward_project(x_true)
    m.auto_set_regularization_params(sino)
    x0 = (0.05 * rng.standard_normal(rs)).astype(np.float32)
    e0 = sino - m.forward_project(x0)
    H = m.compute_hessian_diagonal()
    upd = m.create_vcd_subset_updater(H, weights=1)
    np.random.seed(4)
    part = mb.gen_pixel_partition(rs, 8)
    order = np.random.permutation(8).astype(np.int32)
    flat = torch.as_tensor(x0.reshape(-1, rs[2]), device='cuda').clone()
    err = ResidentSinogram.from_vrc(torch.as_tensor(e0, device='cuda'), _lib.MBIR_F32)
    acc = torch.zeros(2 + rs[2], dtype=torch.float64, device='cuda')
    upd.engine.partition_pass(flat, err, torch.as_tensor(part, device='cuda'), order, acc)
    prob = _oracle_problem(m)
    sy, sx = m.get_params(['sigma_y', 'sigma_x'])
    ou = ovcd.SubsetUpdater(prob, H.reshape(-1, rs[2]), None, sy, sx,
                            dc_profile=ovcd.dc_damping_profile(prob))
    oflat = x0.reshape(-1, rs[2]).astype(np.float64)
    oerr = e0.astype(np.float64)
    alpha_sum = 0.0
    for k in order:
        _, oalpha, _ = ou(oflat, oerr, part[k].astype(np.int64))
        alpha_sum += oalpha
    assert abs(float(acc[1]) - alpha_sum) / alpha_sum <= 1e-4
    assert rel_l2(flat.cpu().numpy(), oflat) <= 2e-5
    assert rel_l2(err.to_vrc().cpu().numpy(), oerr) <= 2e-5


def test_cone_subset_step_wide_detector_scanning_forward():
    """6000 channels: too many centre-channel keys for the binning's shared
    memory, so the subset step takes the scanning forward and the separate
    update kernels.  One step against the FP64 oracle.  Channel coordinates
    near 3000 resolve to 2.4e-4 of a channel in FP32, so the tap weights
    carry ~1e-4 relative error at this width (the same object on a
    384-channel detector agrees to 1.5e-6 / 4.9e-6); the bounds follow that
    resolution."""
    from oracle import vcd as ovcd
    V, R, C = 4, 4, 6000
    m = mb.ConeBeamModel((V, R, C), np.linspace(0, np.pi, V, endpoint=False), 2048.0, 1024.0)
    m.set_params(no_warning=True, verbose=0, delta_det_channel=0.02, delta_det_row=0.02)
    m.auto_set_recon_geometry(no_warning=True)
    m.set_params(no_warning=True, recon_shape=(32, 32, 2))
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(23)
    x_true = rng.random(rs).astype(np.float32)
    sino = m.forward_project(x_true)
    m.auto_set_regularization_params(sino)
    x0 = (0.05 * rng.standard_normal(rs)).astype(np.float32)
    e0 = sino - m.forward_project(x0)
    H = m.compute_hessian_diagonal()
    upd = m.create_vcd_subset_updater(H, weights=1)
    idx = np.sort(rng.choice(mb.gen_full_indices(rs), size=100, replace=False)).astype(np.int64)
    flat = torch.as_tensor(x0.reshape(-1, rs[2]), device='cuda').clone()
    err = torch.as_tensor(e0, device='cuda').clone()
    flat, err, ell1, alpha, sumsq = upd(flat, err, torch.as_tensor(idx, device='cuda'))
    prob = _oracle_problem(m)
    sy, sx = m.get_params(['sigma_y', 'sigma_x'])
    ou = ovcd.SubsetUpdater(prob, H.reshape(-1, rs[2]), None, sy, sx,
                            dc_profile=ovcd.dc_damping_profile(prob))
    oflat = x0.reshape(-1, rs[2]).astype(np.float64)
    oerr = e0.astype(np.float64)
    _, oalpha, _ = ou(oflat, oerr, idx)
    assert abs(float(alpha) - oalpha) / oalpha <= 1e-4
    assert rel_l2(flat.cpu().numpy(), oflat) <= 1e-4
    assert rel_l2(err.cpu().numpy(), oerr) <= 2e-4


def test_parallel_partition_pass_ragged_channels_many_rows():
    """Parallel beam takes the binned subset forward too.  A partition pass
    on a 37-channel detector (a ragged last channel block) that sees only
    the middle of the object, with 300 slices (more detector rows than one
    warp multiple of 256 threads), weighted, against the FP64 oracle
    applying the same subsets in the same order."""
    from oracle import vcd as ovcd
    from mbirtorch_b200.vcd_engine import ResidentSinogram
    from mbirtorch_b200 import _lib
    V, R, C = 20, 300, 37
    m = mb.ParallelBeamModel((V, R, C), np.linspace(0, np.pi, V, endpoint=False))
    m.set_params(no_warning=True, verbose=0, recon_shape=(48, 48, R))
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(19)
    x_true = rng.random(rs).astype(np.float32)
    sino = m.forward_project(x_true)
    w = (0.5 + rng.random(sino.shape)).astype(np.float32)
    m.auto_set_regularization_params(sino, weights=w)
    x0 = (0.05 * rng.standard_normal(rs)).astype(np.float32)
    e0 = sino - m.forward_project(x0)
    H = m.compute_hessian_diagonal(weights=w)
    upd = m.create_vcd_subset_updater(H, weights=torch.as_tensor(w, device='cuda'))
    np.random.seed(5)
    part = mb.gen_pixel_partition(rs, 8)
    order = np.random.permutation(8).astype(np.int32)
    flat = torch.as_tensor(x0.reshape(-1, rs[2]), device='cuda').clone()
    err = ResidentSinogram.from_vrc(torch.as_tensor(e0, device='cuda'), _lib.MBIR_F32)
    acc = torch.zeros(2 + rs[2], dtype=torch.float64, device='cuda')
    upd.engine.partition_pass(flat, err, torch.as_tensor(part, device='cuda'), order, acc)
    prob = _oracle_problem(m)
    sy, sx = m.get_params(['sigma_y', 'sigma_x'])
    ou = ovcd.SubsetUpdater(prob, H.reshape(-1, rs[2]), w, sy, sx)
    oflat = x0.reshape(-1, rs[2]).astype(np.float64)
    oerr = e0.astype(np.float64)
    alpha_sum = 0.0
    for k in order:
        _, oalpha, _ = ou(oflat, oerr, part[k].astype(np.int64))
        alpha_sum += oalpha
    assert abs(float(acc[1]) - alpha_sum) / alpha_sum <= 1e-4
    assert rel_l2(flat.cpu().numpy(), oflat) <= 2e-5
    assert rel_l2(err.to_vrc().cpu().numpy(), oerr) <= 2e-5


@pytest.mark.parametrize("rows", [4, 128])
def test_parallel_subset_step_binned_view_chunks_positivity(rows):
    """A whole-image parallel subset (65536 pixels x 40 views) splits the
    binned forward into view chunks; weighted, with positivity (the
    re-projection goes through the bins too): one step against the FP64
    oracle.  128 rows take the four-rows-per-thread forward, whose 16-bit
    epilogue is checked too (float16 storage against the FP32 step)."""
    from oracle import vcd as ovcd
    from mbirtorch_b200.vcd_engine import ResidentSinogram
    from mbirtorch_b200 import _lib
    V = 40
    m = mb.ParallelBeamModel((V, rows, 320), np.linspace(0, np.pi, V, endpoint=False))
    m.set_params(no_warning=True, verbose=0, recon_shape=(256, 256, rows),
                 positivity_flag=True)
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(13)
    x_true = rng.random(rs).astype(np.float32)
    sino = m.forward_project(x_true)
    w = (0.5 + rng.random(sino.shape)).astype(np.float32)
    m.auto_set_regularization_params(sino, weights=w)
    x0 = (0.05 * rng.standard_normal(rs)).astype(np.float32)
    e0 = sino - m.forward_project(x0)
    H = m.compute_hessian_diagonal(weights=w)
    upd = m.create_vcd_subset_updater(H, weights=torch.as_tensor(w, device='cuda'))
    idx = np.arange(rs[0] * rs[1], dtype=np.int64)
    flat = torch.as_tensor(x0.reshape(-1, rs[2]), device='cuda').clone()
    err = torch.as_tensor(e0, device='cuda').clone()
    flat, err, ell1, alpha, sumsq = upd(flat, err, torch.as_tensor(idx, device='cuda'))
    prob = _oracle_problem(m)
    sy, sx = m.get_params(['sigma_y', 'sigma_x'])
    ou = ovcd.SubsetUpdater(prob, H.reshape(-1, rs[2]), w, sy, sx, positivity=True)
    oflat = x0.reshape(-1, rs[2]).astype(np.float64)
    oerr = e0.astype(np.float64)
    _, oalpha, _ = ou(oflat, oerr, idx)
    assert abs(float(alpha) - oalpha) / oalpha <= 1e-4
    assert rel_l2(flat.cpu().numpy(), oflat) <= 1e-5
    assert rel_l2(err.cpu().numpy(), oerr) <= 1e-5
    if rows == 128:
        w16 = ResidentSinogram.from_vrc(torch.as_tensor(w, device='cuda'), _lib.MBIR_F16)
        Hd = torch.as_tensor(np.ascontiguousarray(np.asarray(H).reshape(-1, rs[2])),
                             device='cuda')
        eng = m._make_engine(Hd, w16, _lib.MBIR_F16, max_subset_pixels=idx.size)
        f16 = torch.as_tensor(x0.reshape(-1, rs[2]), device='cuda').clone()
        e16 = ResidentSinogram.from_vrc(torch.as_tensor(e0, device='cuda'), _lib.MBIR_F16)
        # storing e in float16 alone (before any step) costs this much
        q0 = rel_l2(e16.to_vrc().cpu().numpy(), e0)
        _, a16, _ = eng.subset_update(f16, e16, torch.as_tensor(idx, device='cuda'))
        assert abs(float(a16) - float(alpha)) / float(alpha) <= 1e-3
        assert rel_l2(f16.cpu().numpy(), flat.cpu().numpy()) <= 1e-3
        # the step's error, in units of |e0| (the step shrinks e, so relative
        # to the new e it reads larger): the rounding of e0, of A delta and
        # of the new e, each at most the storage rounding q0
        e_new = err.cpu().numpy().astype(np.float64)
        gap = np.linalg.norm(e16.to_vrc().cpu().numpy() - e_new) / np.linalg.norm(e0)
        assert gap <= 3 * q0


def test_curved_cone_partition_pass_weighted_positivity():
    """A curved-detector cone partition pass (the geometry of the large
    mixed-precision configuration), weighted, with positivity and DC
    damping, against the FP64 oracle applying the same subsets in the same
    order."""
    from oracle import vcd as ovcd
    from mbirtorch_b200.vcd_engine import ResidentSinogram
    from mbirtorch_b200 import _lib
    V, R, C = 30, 12, 40
    m = mb.ConeBeamModel((V, R, C), np.linspace(0, 2 * np.pi, V, endpoint=False), 256.0, 128.0,
                         use_curved_detector=True)
    m.set_params(no_warning=True, verbose=0, delta_det_channel=2.0, delta_det_row=2.0,
                 positivity_flag=True)
    m.auto_set_recon_geometry(no_warning=True)
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(29)
    x_true = rng.random(rs).astype(np.float32)
    sino = m.forward_project(x_true)
    w = (0.5 + rng.random(sino.shape)).astype(np.float32)
    m.auto_set_regularization_params(sino, weights=w)
    x0 = (0.05 * rng.standard_normal(rs)).astype(np.float32)
    e0 = sino - m.forward_project(x0)
    H = m.compute_hessian_diagonal(weights=w)
    w_res = ResidentSinogram.from_vrc(torch.as_tensor(w, device='cuda'), _lib.MBIR_F32)
    upd = m.create_vcd_subset_updater(H, weights=w_res)
    np.random.seed(6)
    part = mb.gen_pixel_partition(rs, 8)
    order = np.random.permutation(8).astype(np.int32)
    flat = torch.as_tensor(x0.reshape(-1, rs[2]), device='cuda').clone()
    err = ResidentSinogram.from_vrc(torch.as_tensor(e0, device='cuda'), _lib.MBIR_F32)
    acc = torch.zeros(2 + rs[2], dtype=torch.float64, device='cuda')
    upd.engine.partition_pass(flat, err, torch.as_tensor(part, device='cuda'), order, acc)
    prob = _oracle_problem(m)
    sy, sx = m.get_params(['sigma_y', 'sigma_x'])
    ou = ovcd.SubsetUpdater(prob, H.reshape(-1, rs[2]), w, sy, sx, positivity=True,
                            dc_profile=ovcd.dc_damping_profile(prob))
    oflat = x0.reshape(-1, rs[2]).astype(np.float64)
    oerr = e0.astype(np.float64)
    alpha_sum = 0.0
    for k in order:
        _, oalpha, _ = ou(oflat, oerr, part[k].astype(np.int64))
        alpha_sum += oalpha
    assert abs(float(acc[1]) - alpha_sum) / alpha_sum <= 1e-4
    assert rel_l2(flat.cpu().numpy(), oflat) <= 2e-5
    assert rel_l2(err.to_vrc().cpu().numpy(), oerr) <= 2e-5


@pytest.mark.parametrize("kind", ["parallel", "cone"])
@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_error_refresh_binned_equals_scanning(kind, storage):
    """The error refresh e = (y - A x) / scale through the channel-sorted bins
    (a workspace given) against the scanning forward (none given): the same
    operator summed in another order.  e is a small difference of large
    terms (y and A x), so the differences are measured against ||y||: FP32
    rounding of A x (1e-6) in FP32 storage, one 16-bit rounding step of e in
    float16."""
    from mbirtorch_b200 import _lib
    from mbirtorch_b200._lib import ptr, stream_of
    from mbirtorch_b200.vcd_engine import ResidentSinogram
    dev = torch.device('cuda', 0)
    if kind == 'parallel':
        m = mb.ParallelBeamModel((50, 128, 70), np.linspace(0, np.pi, 50, endpoint=False))
        m.set_params(no_warning=True, verbose=0)
    else:
        m = mb.ConeBeamModel((40, 24, 56), np.linspace(0, 2 * np.pi, 40, endpoint=False),
                             300.0, 150.0)
        m.set_params(no_warning=True, verbose=0)
    rs = m.get_params('recon_shape')
    g = m._geometry()
    idx = torch.as_tensor(mb.gen_full_indices(rs).astype(np.int64), device=dev)
    flat = torch.rand(rs[0] * rs[1], rs[2], device=dev)
    y = m.projector.forward_volume(flat, idx) + 0.1 * torch.randn(
        *m.get_params('sinogram_shape'), device=dev)
    y_vcr = y.transpose(1, 2).contiguous()
    code = {'float32': _lib.MBIR_F32, 'float16': _lib.MBIR_F16}[storage]
    outs = []
    for binned in (False, True):
        err = ResidentSinogram.from_vrc(y, code)
        ws = None
        if binned:
            nb = int(_lib.query(dev, 'mbir_forward_project_binned_workspace_size', g,
                                g.num_views, idx.shape[0]))
            ws = torch.empty(nb, dtype=torch.uint8, device=dev)
        _lib.call(dev, 'mbir_vcd_refresh_error', g, ptr(m.projector.view_params), ptr(flat),
                  ptr(idx), idx.shape[0], ptr(y_vcr), ptr(err.data), ptr(err.scale), code,
                  ptr(ws), 0 if ws is None else ws.numel(), stream_of(dev))
        outs.append(err.data.float() * err.scale.view(-1, 1, 1))
    torch.cuda.synchronize()
    ynorm = float(y.norm())
    d = float((outs[0] - outs[1]).norm()) / ynorm
    assert d <= (1e-6 if storage == 'float32' else 1e-3 * float(outs[0].norm()) / ynorm), d
    ref = (y - m.projector.forward_volume(flat, idx)).transpose(1, 2)
    d_ref = float((outs[1] - ref).norm()) / ynorm
    assert d_ref <= (1e-6 if storage == 'float32' else 1e-3 * float(ref.norm()) / ynorm), d_ref


@pytest.mark.parametrize("slices,subset", [(8, None), (7, 300)])
def test_large_subset_step_vs_oracle(slices, subset):
    """Subset steps against the FP64 oracle's SubsetUpdater from the same
    state: a subset of every ROR pixel (above 16 384 pixels: its records are
    binned with 1024 threads per view, as in the first pass of a large
    recon), and a 7-slice volume (cylinders that are not a multiple of 4
    slices: the forward stages them synchronously)."""
    from oracle import vcd as ovcd
    m = mb.ConeBeamModel((40, 20, 330), np.linspace(0, 2 * np.pi, 40, endpoint=False),
                         300.0, 150.0)
    m.set_params(no_warning=True, verbose=0, recon_shape=(160, 160, slices))
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(9)
    x_true = rng.random(rs).astype(np.float32)
    sino = m.forward_project(x_true)
    m.auto_set_regularization_params(sino)
    x0 = (0.1 * rng.random(rs)).astype(np.float32)
    e0 = sino - m.forward_project(x0)
    H = m.compute_hessian_diagonal()
    upd = m.create_vcd_subset_updater(H, weights=1)
    idx = mb.gen_full_indices(rs).astype(np.int64)
    assert idx.size >= 16384
    if subset is not None:
        idx = np.sort(rng.choice(idx, size=subset, replace=False)).astype(np.int64)
    flat = torch.as_tensor(x0.reshape(-1, rs[2]), device='cuda').clone()
    err = torch.as_tensor(e0, device='cuda').clone()
    flat, err, ell1, alpha, sumsq = upd(flat, err, torch.as_tensor(idx, device='cuda'))
    prob = _oracle_problem(m)
    sy, sx = m.get_params(['sigma_y', 'sigma_x'])
    ou = ovcd.SubsetUpdater(prob, np.asarray(H).reshape(-1, rs[2]), None, sy, sx,
                            dc_profile=ovcd.dc_damping_profile(prob))
    oflat = x0.reshape(-1, rs[2]).astype(np.float64)
    oerr = e0.astype(np.float64)
    oell1, oalpha, osumsq = ou(oflat, oerr, idx)
    assert abs(float(alpha) - oalpha) / oalpha <= 1e-4
    assert rel_l2(flat.cpu().numpy(), oflat) <= 1e-5
    assert rel_l2(err.cpu().numpy(), oerr) <= 1e-5


@pytest.mark.parametrize("rows", [256, 300])
def test_long_band_back_projection_and_step_vs_oracle(rows):
    """Cone bands of more than 128 slices (8 slices per lane) on detectors of
    256 rows (column batches 8 rows deep per lane) and 300 rows (6 rows deep,
    the depth that covers 257..384 rows in fewer row slots): the sparse back
    projection and a VCD subset step against the FP64 oracle."""
    import oracle
    from oracle import vcd as ovcd
    m = mb.ConeBeamModel((12, rows, 40), np.linspace(0, 2 * np.pi, 12, endpoint=False),
                         300.0, 150.0)
    m.set_params(no_warning=True, verbose=0, recon_shape=(24, 24, 200))
    rs = m.get_params('recon_shape')
    g = m._geometry()
    assert g.num_det_rows == rows and rs[2] == 200
    rng = np.random.default_rng(21)
    idx = mb.gen_full_indices(rs).astype(np.int64)
    y = rng.standard_normal(m.get_params('sinogram_shape')).astype(np.float32)
    sub = np.sort(rng.choice(idx, size=40, replace=False))
    b = m.sparse_back_project(torch.as_tensor(y, device='cuda'),
                              torch.as_tensor(sub, device='cuda')).cpu().numpy()
    prob = _oracle_problem(m)
    vp = m._view_params_array().astype(np.float64)
    assert rel_l2(b, oracle.cone_back(prob.geom, vp, y, sub)) <= 1e-5

    x_true = rng.random(rs).astype(np.float32)
    sino = m.forward_project(x_true)
    m.auto_set_regularization_params(sino)
    x0 = (0.1 * rng.random(rs)).astype(np.float32)
    e0 = sino - m.forward_project(x0)
    H = m.compute_hessian_diagonal()
    upd = m.create_vcd_subset_updater(H, weights=1)
    flat = torch.as_tensor(x0.reshape(-1, rs[2]), device='cuda').clone()
    err = torch.as_tensor(e0, device='cuda').clone()
    flat, err, ell1, alpha, sumsq = upd(flat, err, torch.as_tensor(sub, device='cuda'))
    sy, sx = m.get_params(['sigma_y', 'sigma_x'])
    ou = ovcd.SubsetUpdater(prob, np.asarray(H).reshape(-1, rs[2]), None, sy, sx,
                            dc_profile=ovcd.dc_damping_profile(prob))
    oflat = x0.reshape(-1, rs[2]).astype(np.float64)
    oerr = e0.astype(np.float64)
    oell1, oalpha, osumsq = ou(oflat, oerr, sub)
    assert abs(float(alpha) - oalpha) / oalpha <= 1e-4
    assert rel_l2(flat.cpu().numpy(), oflat) <= 1e-5
    assert rel_l2(err.cpu().numpy(), oerr) <= 1e-5
