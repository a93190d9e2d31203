"""Cross-job batching of the VCD subset step (GPU).

Reconstructions that share a geometry step their subsets together: every
kernel of the subset step is launched once for all of them, with the job on
grid z (mbir_vcd_partition_pass_batched).  Each job's subsets, orders,
regularization and data are its own, and the batched pass must give every
job exactly what its own partition pass gives: bit for bit, for cone and
parallel beam, weighted with positivity, and in the 16-bit storages.  The
server batches same-geometry jobs and serves the same results as without
batching.
"""

import numpy as np
import pytest
import torch

import mbirtorch_b200 as mb
from mbirtorch_b200 import _lib
from mbirtorch_b200.serving import ReconServer
from mbirtorch_b200.vcd_engine import ResidentSinogram, partition_pass_batched

pytestmark = pytest.mark.gpu

DEV = torch.device('cuda', 0)
CODES = {'float32': _lib.MBIR_F32, 'bfloat16': _lib.MBIR_BF16, 'float16': _lib.MBIR_F16}


def _model(kind, positivity):
    if kind == 'parallel':
        m = mb.ParallelBeamModel((36, 8, 40), np.linspace(0, np.pi, 36, endpoint=False))
        m.set_params(no_warning=True, verbose=0, recon_shape=(40, 40, 8))
    else:
        m = mb.ConeBeamModel((30, 12, 40), np.linspace(0, 2 * np.pi, 30, endpoint=False),
                             256.0, 128.0)
        m.set_params(no_warning=True, verbose=0, delta_det_channel=2.0, delta_det_row=2.0)
        m.auto_set_recon_geometry(no_warning=True)
    m.set_params(no_warning=True, positivity_flag=positivity)
    return m


def _job(kind, storage, weighted, positivity, seed):
    """One job's model, engine, state and partition (8 subsets) with its
    own data and regularization."""
    m = _model(kind, positivity)
    rs = m.get_params('recon_shape')
    rng = np.random.default_rng(seed)
    x_true = rng.random(rs).astype(np.float32)
    sino = m.forward_project(x_true)
    w = (0.5 + rng.random(sino.shape)).astype(np.float32) if weighted else None
    m.auto_set_regularization_params(sino, weights=w)
    x0 = (0.05 * rng.standard_normal(rs)).astype(np.float32)
    e0 = sino - m.forward_project(x0)
    H = m.compute_hessian_diagonal(weights=w)
    code = CODES[storage]
    w_res = None if w is None else ResidentSinogram.from_vrc(torch.as_tensor(w, device=DEV), code)
    Hd = torch.as_tensor(np.ascontiguousarray(np.asarray(H).reshape(-1, rs[2])), device=DEV)
    rs_np = np.random.RandomState(seed)
    part = mb.gen_pixel_partition(rs, 8, rng=rs_np)
    order = rs_np.permutation(8).astype(np.int32)
    eng = m._make_engine(Hd, w_res, code, max_subset_pixels=part.shape[1])

    def state():
        flat = torch.as_tensor(x0.reshape(-1, rs[2]), device=DEV).clone()
        err = ResidentSinogram.from_vrc(torch.as_tensor(e0, device=DEV), code)
        acc = torch.zeros(2 + rs[2], dtype=torch.float64, device=DEV)
        return flat, err, acc

    return eng, torch.as_tensor(part, device=DEV), order, state


@pytest.mark.parametrize("kind,storage,weighted,positivity", [
    ("cone", "float32", False, False),
    ("cone", "float32", True, True),
    ("cone", "float16", False, False),
    ("parallel", "float32", True, True),
    ("parallel", "bfloat16", False, False),
])
def test_batched_pass_equals_each_jobs_own_pass(kind, storage, weighted, positivity):
    jobs = [_job(kind, storage, weighted, positivity, 60 + j) for j in range(3)]
    single = []
    for eng, part, order, state in jobs:
        flat, err, acc = state()
        eng.partition_pass(flat, err, part, order, acc)
        single.append((flat, err, acc))
    states = [state() for _, _, _, state in jobs]
    launches = _lib.launch_count()
    partition_pass_batched([j[0] for j in jobs], [s[0] for s in states],
                           [s[1] for s in states], [j[1] for j in jobs], [j[2] for j in jobs],
                           [s[2] for s in states])
    torch.cuda.synchronize()
    batched_launches = _lib.launch_count() - launches
    for (f1, e1, a1), (f2, e2, a2) in zip(single, states):
        assert torch.equal(f1, f2)
        assert torch.equal(e1.data, e2.data) and torch.equal(e1.scale, e2.scale)
        assert torch.equal(a1, a2)
    # one launch per kernel of each subset step for all three jobs
    eng, part, order, state = jobs[0]
    flat, err, acc = state()
    torch.cuda.synchronize()
    launches = _lib.launch_count()
    eng.partition_pass(flat, err, part, order, acc)
    torch.cuda.synchronize()
    assert batched_launches == _lib.launch_count() - launches


def test_server_batches_same_geometry_jobs_with_the_same_results():
    """Four jobs of one cone geometry (own data and seeds) served with and
    without batching: bitwise the same results; batched iterations ran."""
    def make():
        m = mb.ConeBeamModel((30, 12, 40), np.linspace(0, 2 * np.pi, 30, endpoint=False),
                             256.0, 128.0)
        m.set_params(no_warning=True, verbose=0, delta_det_channel=2.0, delta_det_row=2.0)
        m.auto_set_recon_geometry(no_warning=True)
        return m

    sinos = []
    for j in range(4):
        m = make()
        rng = np.random.default_rng(80 + j)
        sinos.append(m.forward_project(rng.random(m.get_params('recon_shape'))
                                       .astype(np.float32)))
    out = {}
    for batching in (False, True):
        srv = ReconServer(storage_dtype='float16', max_active=4, batching=batching)
        reqs = [srv.submit(make(), s, max_iterations=6, seed=90 + j)
                for j, s in enumerate(sinos)]
        srv.run_until_idle(timeout_s=300)
        assert srv.stats()['failed'] == 0
        out[batching] = (reqs, srv.batched_iterations)
    assert out[False][1] == 0 and out[True][1] > 0
    for a, b in zip(out[False][0], out[True][0]):
        assert np.array_equal(a.recon, b.recon)
        assert a.recon_params['fm_rmse'] == b.recon_params['fm_rmse']
