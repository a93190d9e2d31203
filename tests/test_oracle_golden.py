"""Pin the FP64 CPU oracle against the reference's own outputs.

Every fixture under tests/golden/ was produced by the reference (mbirtorch
0.0.2) itself -- its torch bodies, qGGMRF, partitions, direct recon and
seeded VCD recon -- by tests/golden/make_golden.py.  The oracle must match
each one; the sm_100a kernels are then checked against the oracle.

Tolerances: the reference runs in FP32 and the oracle in FP64, so the
residual is FP32 rounding (~1e-6 relative L2).  Projectors are held to 1e-5
(the reference's own kernel-vs-body bar), reconstructions to 1e-4.
"""

import numpy as np
import pytest

from _cases import (PROJECTOR_NAMES, load_projector_case, oracle_back,
                    oracle_forward)
from conftest import load_golden, rel_l2

import oracle
from oracle import OracleGeometry, vcd
from oracle import qggmrf as oq

GRANULARITY = [1, 2, 4, 8, 16, 32, 64, 128, 128, 128, 128]
SEQUENCE = [2, 4, 6] + [7, 8, 9, 10] * 25


@pytest.fixture(scope="module", autouse=True)
def _built():
    oracle.build()


@pytest.mark.parametrize("name", PROJECTOR_NAMES)
@pytest.mark.parametrize("tag", ["full", "subset"])
def test_projectors_match_reference(name, tag):
    d = load_projector_case(name)
    idx = d[f'{tag}_indices']
    fwd = oracle_forward(d, d[f'{tag}_values'], idx)
    assert fwd.shape == d[f'{tag}_fwd'].shape
    assert rel_l2(fwd, d[f'{tag}_fwd']) < 1e-5
    for cp in (1, 2):
        back = oracle_back(d, d[f'{tag}_sino'], idx, cp)
        assert rel_l2(back, d[f'{tag}_back{cp}']) < 1e-5


@pytest.mark.parametrize("name", PROJECTOR_NAMES)
def test_oracle_adjoint_identity(name):
    """<A x, y> == <x, A^T y> in FP64 (the reference gate is 1e-4 in FP32)."""
    d = load_projector_case(name)
    idx = d['full_indices']
    x, y = d['full_values'], d['full_sino']
    lhs = float(np.sum(oracle_forward(d, x, idx) * y))
    rhs = float(np.sum(x * oracle_back(d, y, idx)))
    assert abs(lhs - rhs) / max(abs(lhs), abs(rhs)) < 1e-12


@pytest.mark.parametrize("tag", ["default", "aniso", "p15"])
def test_qggmrf_matches_reference(tag):
    d = load_golden('qggmrf.npz')
    pr = d[f'{tag}_params']
    b = oq.b_from_nbr_wts(list(pr[:3]))
    g, h = oq.gradient_and_hessian(d['flat'], d['recon_shape'], d['indices'], b, *pr[3:])
    assert rel_l2(g, d[f'{tag}_grad']) < 1e-5
    assert rel_l2(h, d[f'{tag}_hess']) < 1e-5


@pytest.mark.parametrize("tag,seed", [("a", 3), ("b", 5)])
def test_partitions_match_reference(tag, seed):
    d = load_golden('partitions.npz')
    np.random.seed(seed)
    for i, n in enumerate(d[f'{tag}_gran']):
        p = vcd.pixel_partition(tuple(d[f'{tag}_shape']), int(n))
        np.testing.assert_array_equal(p, d[f'{tag}_part{i}'])
    # The RNG is left exactly where the reference leaves it.
    np.testing.assert_array_equal(np.random.randint(0, 2 ** 30, size=4), d[f'{tag}_after'])


def test_partition_sequence_and_mask():
    d = load_golden('partitions.npz')
    np.testing.assert_array_equal(vcd.partition_sequence(SEQUENCE, 120), d['seq'])
    np.testing.assert_array_equal(vcd.partition_sequence([0, 1, 2], 2), d['seq_short'])
    np.testing.assert_array_equal(vcd.ror_mask((18, 13)), d['mask_18x13'])


def _parallel_problem(sino, angles):
    V, R, C = sino.shape
    g = OracleGeometry(num_det_rows=R, num_det_channels=C, num_recon_rows=C,
                       num_recon_cols=C, num_slices=R)
    return vcd.Problem('parallel', g, np.asarray(angles, np.float32), (C, C, R))


def _cone_problem(d, tag, sino, angles, z_shifts, curved=False):
    V, R, C = sino.shape
    rs = tuple(int(v) for v in d[f'{tag}_recon_shape'])
    psf, bp = d[f'{tag}_psf']
    g = OracleGeometry(num_det_rows=R, num_det_channels=C, num_recon_rows=rs[0],
                       num_recon_cols=rs[1], num_slices=rs[2], delta_voxel=0.5,
                       delta_voxel_row=0.5, delta_voxel_slice=0.5,
                       recon_slice_offset=float(d[f'{tag}_rso']), magnification=2.0,
                       source_detector_dist=64.0, use_curved_detector=curved,
                       psf_radius=int(psf), bp_psf_radius=int(bp))
    vp = np.stack([np.asarray(angles, np.float32), np.asarray(z_shifts, np.float32)], 1)
    return vcd.Problem('cone', g, vp, rs, source_iso_dist=32.0)


def _cone_views(tag, V):
    if tag == 'helical':
        return (np.linspace(0, 4 * np.pi, V, endpoint=False),
                np.linspace(-2.0, 2.0, V))
    return np.linspace(0, 2 * np.pi, V, endpoint=False), np.zeros(V)


def test_direct_recon_parallel_matches_reference():
    d = load_golden('direct.npz')
    sino = d['par_sino']
    prob = _parallel_problem(sino, np.linspace(0, np.pi, sino.shape[0], endpoint=False))
    assert rel_l2(vcd.direct_recon(prob, sino), d['par_fbp']) < 1e-5


@pytest.mark.parametrize("tag", ["cone", "curved", "helical"])
def test_direct_recon_cone_and_damping_match_reference(tag):
    d = load_golden('direct.npz')
    sino = d[f'{tag}_sino']
    ang, zs = _cone_views(tag, sino.shape[0])
    prob = _cone_problem(d, tag, sino, ang, zs, curved=(tag == 'curved'))
    assert rel_l2(vcd.direct_recon(prob, sino), d[f'{tag}_fdk']) < 1e-5
    np.testing.assert_allclose(vcd.dc_damping_profile(prob), d[f'{tag}_dc'], rtol=0, atol=0)


@pytest.mark.parametrize("name", ["recon_parallel", "recon_parallel_weighted"])
def test_parallel_recon_matches_reference(name):
    d = load_golden(f'{name}.npz')
    sino = d['sino']
    prob = _parallel_problem(sino, d['angles'])
    np.random.seed(int(d['seed']))
    parts = [vcd.pixel_partition(prob.recon_shape, n) for n in GRANULARITY]
    seq = vcd.partition_sequence(SEQUENCE, int(d['max_iterations']))
    w = d['weights'] if 'weights' in d.files else None
    rec, st = vcd.recon(prob, sino, d['reg'][0], d['reg'][1], parts, seq, weights=w,
                        positivity=w is not None)
    assert rel_l2(rec, d['recon']) < 1e-4
    np.testing.assert_allclose(st['fm_rmse'], d['fm_rmse'], rtol=1e-4)
    np.testing.assert_allclose(st['alpha'], d['alpha'], rtol=1e-4)


@pytest.mark.parametrize("name,tag", [("recon_cone", "cone"),
                                      ("recon_cone_helical", "helical")])
def test_cone_recon_matches_reference(name, tag):
    d = load_golden(f'{name}.npz')
    dd = load_golden('direct.npz')
    sino = d['sino']
    prob = _cone_problem(dd, tag, sino, d['angles'], d['z_shifts'])
    np.random.seed(int(d['seed']))
    parts = [vcd.pixel_partition(prob.recon_shape, n) for n in GRANULARITY]
    seq = vcd.partition_sequence(SEQUENCE, int(d['max_iterations']))
    rec, st = vcd.recon(prob, sino, d['reg'][0], d['reg'][1], parts, seq,
                        dc_profile=vcd.dc_damping_profile(prob))
    assert rel_l2(rec, d['recon']) < 1e-4
    np.testing.assert_allclose(st['fm_rmse'], d['fm_rmse'], rtol=1e-4)
    np.testing.assert_allclose(st['alpha'], d['alpha'], rtol=1e-4)


@pytest.mark.parametrize("name", ["prox_parallel", "prox_cone"])
def test_prox_map_matches_reference(name):
    """prox_map's proximal-map prior: the reference's seeded run (automatic
    sigma_prox for parallel, a given one for cone) against the oracle."""
    d = load_golden(f'{name}.npz')
    sino = d['sino']
    if name == 'prox_parallel':
        prob, dc = _parallel_problem(sino, d['angles']), None
    else:
        prob = _cone_problem(load_golden('direct.npz'), 'cone', sino, d['angles'], d['z_shifts'])
        dc = vcd.dc_damping_profile(prob)
    np.random.seed(int(d['seed']))
    parts = [vcd.pixel_partition(prob.recon_shape, n) for n in GRANULARITY]
    seq = vcd.partition_sequence(SEQUENCE, int(d['max_iterations']))
    rec, st = vcd.recon(prob, sino, d['reg'][0], d['reg'][1], parts, seq, dc_profile=dc,
                        prox_input=d['prox_input'], sigma_prox=float(d['reg'][2]))
    assert rel_l2(rec, d['recon']) < 1e-4
    np.testing.assert_allclose(st['fm_rmse'], d['fm_rmse'], rtol=1e-4)
    np.testing.assert_allclose(st['alpha'], d['alpha'], rtol=1e-4)


@pytest.mark.parametrize("tag", ["given", "auto"])
def test_denoiser_matches_reference(tag):
    """QGGMRFDenoiser.denoise: the reference's seeded sweep against the
    oracle, with the regularization scalars the reference used."""
    from oracle import denoise as oden
    d = load_golden('denoise.npz')
    noisy = d['noisy']
    np.random.seed(13)
    part = vcd.pixel_partition(noisy.shape, 16, use_ror_mask=False)
    sigma_y, sigma_x = d[f'{tag}_reg'][:2]
    out, alphas, nmaes = oden.denoise(noisy, sigma_y, sigma_x, part, 4)
    assert rel_l2(out, d[f'{tag}_out']) < 1e-5
    np.testing.assert_allclose(alphas, d[f'{tag}_alpha'], rtol=1e-4)
    np.testing.assert_allclose(100 * nmaes, d[f'{tag}_nmae_pct'], rtol=1e-4)
