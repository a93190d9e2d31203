"""Serving-layer host logic without a GPU: the memory ledger and its
closed-form per-job charge."""

import numpy as np

import mbirtorch_b200 as mb
from mbirtorch_b200.serving import MemoryLedger


def _cone(shape):
    return mb.ConeBeamModel(shape, np.linspace(0, 2 * np.pi, shape[0], endpoint=False),
                            source_detector_dist=4.0 * shape[2], source_iso_dist=2.0 * shape[2])


def test_ledger_admits_within_budget_and_releases():
    led = MemoryLedger(1000)
    assert led.fits(600)
    led.take(600)
    assert not led.fits(500) and led.fits(400)
    led.release(600)
    assert led.used == 0 and led.fits(1000)


def test_job_charge_grows_with_size_and_shrinks_with_precision():
    small, big = _cone((40, 12, 24)), _cone((80, 24, 48))
    ps, rs = MemoryLedger.job_bytes(small, 'float32', False, 64)
    pb, rb = MemoryLedger.job_bytes(big, 'float32', False, 64)
    assert pb > ps and rb > rs and ps >= rs
    _, r16 = MemoryLedger.job_bytes(big, 'float16', False, 64)
    _, rw = MemoryLedger.job_bytes(big, 'float16', True, 64)
    V, R, C = big.get_params('sinogram_shape')
    # 16-bit storage keeps an FP32 copy of the measurements for the refresh
    # but halves the error and delta sinograms; weights add one array.
    assert rw - r16 == 2 * V * R * C
    assert r16 > 0


def test_job_charge_matches_drawn_partitions():
    from mbirtorch_b200 import vcd_utils
    from mbirtorch_b200.serving import ReconServer
    m = _cone((40, 12, 24))
    srv = ReconServer(device='cuda:0', memory_budget_bytes=1 << 30, storage_dtype='float16')
    rs, gran, ror = m.get_params(['recon_shape', 'granularity', 'use_ror_mask'])
    rng = np.random.RandomState(5)
    parts = [vcd_utils.gen_pixel_partition(rs, n, use_ror_mask=ror, rng=rng) for n in gran]
    for iters in (1, 3, 20):
        seq = vcd_utils.gen_partition_sequence(m.get_params('partition_sequence'), iters)
        max_ps = max(int(parts[int(i)].shape[1]) for i in seq)
        assert srv.job_charge(m, False, iters) == \
            MemoryLedger.job_bytes(m, 'float16', False, max_ps)


def test_admission_policy_shortest_first_with_wait_bound(monkeypatch):
    """'shortest' admits the waiting request with the least estimated work
    (pixels x slices x views x iterations); a request waiting past max_wait_s
    goes first; 'fifo' keeps arrival order."""
    import time
    from mbirtorch_b200.serving import ReconServer
    now = time.perf_counter()
    big, mid, small = _cone((80, 24, 48)), _cone((40, 12, 24)), _cone((20, 6, 12))
    srv = ReconServer(device='cuda:0', memory_budget_bytes=1 << 30, storage_dtype='float16',
                      admission='shortest', max_wait_s=5.0)
    reqs = [srv.submit(m, None, max_iterations=10, arrival=now) for m in (big, mid, small)]
    assert reqs[2].work < reqs[1].work < reqs[0].work
    assert srv._next_waiting() == 2
    srv.waiting[0].arrival = now - 10.0      # the oldest has waited past the bound
    assert srv._next_waiting() == 0
    fifo = ReconServer(device='cuda:0', memory_budget_bytes=1 << 30, storage_dtype='float16',
                       admission='fifo')
    for m in (big, small):
        fifo.submit(m, None, max_iterations=10, arrival=now)
    assert fifo._next_waiting() == 0
    rs = small.get_params('recon_shape')
    n_pix = int(mb.get_2d_ror_mask(rs).sum())
    assert reqs[2].work == n_pix * rs[2] * 20 * 10
