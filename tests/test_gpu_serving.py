"""Continuous-batching server (GPU).

* Each job's result is bitwise the same served alone and served in a mix of
  concurrent jobs of different geometry and size -- and the same as
  model.recon() with np.random seeded like the job.
* Admission respects the memory ledger; a failing request frees its slot
  and the others complete.
* Latency statistics are reported.
"""

import numpy as np
import pytest
import torch

import mbirtorch_b200 as mb
from mbirtorch_b200.serving import ReconServer

pytestmark = pytest.mark.gpu


def _phantom(rs, seed):
    rng = np.random.default_rng(seed)
    g0 = np.linspace(-1, 1, rs[1])
    g1 = np.linspace(-1, 1, rs[0])
    z = np.linspace(-1, 1, rs[2])
    X, Y = np.meshgrid(g0, g1)
    vol = np.zeros(rs, np.float32)
    for _ in range(4):
        c, a = rng.uniform(-0.4, 0.4, 3), rng.uniform(0.1, 0.4, 3)
        inside = ((X - c[0]) / a[0]) ** 2 + ((Y - c[1]) / a[1]) ** 2
        vol += rng.uniform(0.2, 1.0) * ((inside[:, :, None] + ((z - c[2]) / a[2]) ** 2) <= 1)
    return vol


def _jobs():
    """(model factory, sinogram) for a small mix: parallel, cone, helical."""
    out = []
    specs = [('parallel', (48, 8, 40)), ('cone', (40, 12, 24)), ('helical', (60, 10, 20)),
             ('parallel', (36, 4, 30)), ('cone', (32, 16, 28))]
    for i, (kind, shape) in enumerate(specs):
        V = shape[0]
        if kind == 'parallel':
            def make(V=V, shape=shape):
                return mb.ParallelBeamModel(shape, np.linspace(0, np.pi, V, endpoint=False))
        elif kind == 'cone':
            def make(V=V, shape=shape):
                return mb.ConeBeamModel(shape, np.linspace(0, 2 * np.pi, V, endpoint=False),
                                        source_detector_dist=4.0 * shape[2],
                                        source_iso_dist=2.0 * shape[2])
        else:
            def make(V=V, shape=shape):
                return mb.ConeBeamModel(shape, np.linspace(0, 4 * np.pi, V, endpoint=False),
                                        source_detector_dist=4.0 * shape[2],
                                        source_iso_dist=2.0 * shape[2],
                                        helical_z_shifts=np.linspace(-2, 2, V))
        m = make()
        m.set_params(no_warning=True, verbose=0)
        sino = m.forward_project(_phantom(m.get_params('recon_shape'), i))
        sino = sino + np.random.default_rng(100 + i).normal(0, 0.01 * sino.max(), sino.shape)
        out.append((make, sino.astype(np.float32)))
    return out


def _serve(jobs, idxs, storage, max_active=8, budget=None, iterations=3, cuda_graphs=True):
    srv = ReconServer(storage_dtype=storage, max_active=max_active, memory_budget_bytes=budget,
                      cuda_graphs=cuda_graphs)
    reqs = []
    for i in idxs:
        make, sino = jobs[i]
        m = make()
        m.set_params(no_warning=True, verbose=0)
        reqs.append(srv.submit(m, sino, max_iterations=iterations, seed=1000 + i))
    srv.run_until_idle(timeout_s=300)
    return srv, reqs


@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_results_same_alone_and_in_mix(storage):
    jobs = _jobs()
    _, mix = _serve(jobs, range(len(jobs)), storage, max_active=5)
    for i in range(len(jobs)):
        _, alone = _serve(jobs, [i], storage)
        assert alone[0].error is None and mix[i].error is None
        assert np.array_equal(alone[0].recon, mix[i].recon), i
        assert alone[0].recon_params['fm_rmse'] == mix[i].recon_params['fm_rmse']


@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_graph_replay_equals_direct_launch(storage):
    """Seven iterations use the 128-subset partitions four times: the server
    captures that pass shape once per job and replays it.  Every served
    result equals the one served with direct launches, bit for bit."""
    jobs = _jobs()
    _, direct = _serve(jobs, range(len(jobs)), storage, max_active=5, iterations=7,
                       cuda_graphs=False)
    _, graphed = _serve(jobs, range(len(jobs)), storage, max_active=5, iterations=7)
    for d, g in zip(direct, graphed):
        assert d.error is None and g.error is None
        assert d.graph_replays == 0 and g.graph_replays == 4
        assert np.array_equal(d.recon, g.recon)
        assert d.recon_params['fm_rmse'] == g.recon_params['fm_rmse']
        assert d.recon_params['alpha_values'] == g.recon_params['alpha_values']


def test_server_equals_model_recon_with_same_seed():
    jobs = _jobs()
    _, reqs = _serve(jobs, [1], 'float32')
    make, sino = jobs[1]
    m = make()
    m.set_params(no_warning=True, verbose=0)
    np.random.seed(1001)
    rec, _ = m.recon(sino, max_iterations=3, stop_threshold_change_pct=0.0, logfile_path=None,
                     print_logs=False)
    assert np.array_equal(rec, reqs[0].recon)


def test_admission_respects_ledger_and_failures_are_isolated():
    jobs = _jobs()
    # A budget one byte short of all jobs resident at once: some admissions
    # must wait for a finished job's release.
    srv = ReconServer(storage_dtype='float16', max_active=8, memory_budget_bytes=1)
    charges = [srv.job_charge(make(), False, 2) for make, _ in jobs]
    budget = sum(res for _, res in charges) - 1
    assert max(peak for peak, _ in charges) <= budget
    srv = ReconServer(storage_dtype='float16', max_active=8, memory_budget_bytes=budget)
    reqs = []
    for i, (make, sino) in enumerate(jobs):
        m = make()
        m.set_params(no_warning=True, verbose=0)
        reqs.append(srv.submit(m, sino, max_iterations=2, seed=i))
    bad = make()
    bad.set_params(no_warning=True, verbose=0)
    reqs.append(srv.submit(bad, np.zeros((3, 3, 3), np.float32), max_iterations=2))
    srv.run_until_idle(timeout_s=300)
    assert srv.ledger.high_water <= srv.ledger.budget
    assert srv.max_concurrent < len(jobs) and srv.deferred > 0
    assert all(r.error is None for r in reqs[:-1])
    assert isinstance(reqs[-1].error, ValueError)
    st = srv.stats()
    assert st['completed'] == len(jobs) and st['failed'] == 1
    assert st['p99_latency_s'] >= st['p50_latency_s'] > 0
    assert srv.ledger.used == 0


def test_poisson_schedule_overlaps_jobs():
    jobs = _jobs()
    rng = np.random.default_rng(0)
    t = np.cumsum(rng.exponential(0.01, size=len(jobs)))
    sched = []
    for i, (make, sino) in enumerate(jobs):
        m = make()
        m.set_params(no_warning=True, verbose=0)
        sched.append((float(t[i]), dict(model=m, sinogram=sino, max_iterations=4, seed=i)))
    srv = ReconServer(storage_dtype='float16', max_active=4)
    done = srv.serve_schedule(sched, timeout_s=300)
    assert len(done) == len(jobs) and all(r.error is None for r in done)
    assert srv.max_concurrent >= 2
    torch.cuda.synchronize()


@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_preempt_checkpoint_resume_equals_uninterrupted(storage, tmp_path):
    """A cone job preempted after two of three iterations, its resident state
    written to disk and resumed in another server, ends bitwise where the
    uninterrupted job ends."""
    jobs = _jobs()
    make, sino = jobs[1]
    _, alone = _serve(jobs, [1], storage)
    srv = ReconServer(storage_dtype=storage, max_active=2)
    m = make()
    m.set_params(no_warning=True, verbose=0)
    r = srv.submit(m, sino, max_iterations=3, seed=1001)
    while r._run is None or r._run.done < 1:
        srv.step()
    state = srv.preempt(r)   # collects the iteration in flight: two done
    assert int(state['done']) == 2 and not bool(state['finished'])
    assert r.preempted and srv.ledger.used == 0 and not srv.active
    np.savez(tmp_path / 'job.npz', **state)
    with np.load(tmp_path / 'job.npz') as f:
        loaded = {k: f[k] for k in f.files}
    srv2 = ReconServer(storage_dtype=storage, max_active=2)
    m2 = make()
    m2.set_params(no_warning=True, verbose=0)
    r2 = srv2.resume(m2, loaded)
    srv2.run_until_idle(timeout_s=300)
    assert r2.error is None
    assert np.array_equal(r2.recon, alone[0].recon)
    assert r2.recon_params['fm_rmse'] == alone[0].recon_params['fm_rmse']


def test_served_bfloat16_results_against_fp64_oracle():
    """Served with bfloat16 storage (admission by the ledger, jobs resident
    together): a parallel, a cone and a two-turn helical cone job, 128^2 x 16
    with Poisson data and 10 iterations, each within 1e-3 of the FP64
    oracle's seeded reconstruction of the same data and partitions."""
    from oracle import vcd as ovcd
    from _cases import oracle_problem
    N, S, V = 128, 16, 180
    C = int(1.5 * N)

    def make(kind):
        if kind == 'parallel':
            m = mb.ParallelBeamModel((V, S, C), np.linspace(0, np.pi, V, endpoint=False))
        else:
            if kind == 'helical':
                ang = (2 * np.pi / (V // 2)) * np.arange(V)
                zs = np.linspace(-S, S, V)
            else:
                ang, zs = np.linspace(0, 2 * np.pi, V, endpoint=False), None
            m = mb.ConeBeamModel((V, S, C), ang, source_detector_dist=4.0 * N,
                                 source_iso_dist=2.0 * N, helical_z_shifts=zs)
            m.set_params(no_warning=True, delta_det_channel=2.0, delta_det_row=2.0)
            m.auto_set_recon_geometry(no_warning=True)
        m.set_params(no_warning=True, verbose=0, recon_shape=(N, N, S))
        return m

    jobs = []
    for i, kind in enumerate(['parallel', 'cone', 'helical']):
        m = make(kind)
        clean = m.forward_project(_phantom((N, N, S), 30 + i))
        mu = 3.0 / float(clean.max())
        counts = np.random.default_rng(40 + i).poisson(1e4 * np.exp(-mu * clean))
        jobs.append((kind, (-np.log(np.maximum(counts, 1) / 1e4) / mu).astype(np.float32)))
    srv = ReconServer(storage_dtype='bfloat16', max_active=3)
    reqs = [srv.submit(make(kind), sino, max_iterations=10, seed=50 + i)
            for i, (kind, sino) in enumerate(jobs)]
    srv.run_until_idle(timeout_s=600)
    assert srv.stats()['failed'] == 0
    for i, ((kind, sino), r) in enumerate(zip(jobs, reqs)):
        m = make(kind)
        reg = m.auto_set_regularization_params(sino)
        prob = oracle_problem(m)
        # the server draws a job's partitions and orders from RandomState(seed)
        rng = np.random.RandomState(50 + i)
        state = np.random.get_state()
        np.random.set_state(rng.get_state())
        try:
            parts = [ovcd.pixel_partition(prob.recon_shape, n)
                     for n in m.get_params('granularity')]
            seq = ovcd.partition_sequence(m.get_params('partition_sequence'), 10)
            dc = ovcd.dc_damping_profile(prob) if kind != 'parallel' else None
            orec, _ = ovcd.recon(prob, sino, reg['sigma_y'], reg['sigma_x'], parts, seq,
                                 dc_profile=dc)
        finally:
            np.random.set_state(state)
        err = float(np.linalg.norm(r.recon - orec) / np.linalg.norm(orec))
        assert err <= 1e-3, (kind, err)
