"""Continuous-batching reconstruction server.

Requests -- reconstructions of mixed geometry and size -- arrive over time.
The server admits a request as soon as a slot and device memory allow it
(a byte ledger, not a queue alone), keeps every admitted job's volume, error
sinogram and VCD state resident on the device, and advances all admitted
jobs concurrently: each job owns a CUDA stream, and the scheduler enqueues
a job's next VCD iteration as soon as its previous one has finished, so the
iterations of different jobs overlap on the GPU.  A finished job releases
its memory and slot, which admits the next waiting request.

Each job draws its partitions and subset orders from its own seeded
RandomState (in the reference's call order), and every kernel is
deterministic, so a job's result is bitwise the same whether it runs alone
or in a mix.  Latency is measured from arrival to result on the host clock;
:meth:`ReconServer.stats` reports p50/p99 and recons/s.

The device memory ledger follows the closed-form design of the reference's
memory model (_memory_ledger.py:1-38): a job is charged its peak bytes
during preparation (sinogram-sized FP32 transients of the direct-recon init)
and its resident bytes afterwards.
"""

import math
import time

import numpy as np
import torch

from . import _lib, vcd_utils
from .vcd_engine import make_vcd_params, storage_code
from .vcd_run import VcdRun


_STREAMS = {}


def _free_streams(device):
    """The process-wide free list of server streams on ``device``."""
    key = torch.device(device).index
    if key is None:
        key = torch.cuda.current_device()
    return _STREAMS.setdefault(key, [])


class MemoryLedger:
    """Admission by device bytes: ``fits`` / ``take`` / ``release``."""

    def __init__(self, budget_bytes):
        self.budget = int(budget_bytes)
        self.used = 0
        self.high_water = 0

    def fits(self, nbytes):
        return self.used + int(nbytes) <= self.budget

    def take(self, nbytes):
        self.used += int(nbytes)
        self.high_water = max(self.high_water, self.used)

    def release(self, nbytes):
        self.used -= int(nbytes)

    @staticmethod
    def job_bytes(model, storage_dtype, weighted, max_subset_pixels):
        """(peak during preparation, resident afterwards) in bytes."""
        V, R, C = model.get_params('sinogram_shape')
        nr, nc, ns = model.get_params('recon_shape')
        n_sino, n_vol = V * R * C, nr * nc * ns
        code = storage_code(storage_dtype)
        s = 4 if code == _lib.MBIR_F32 else 2
        prm = make_vcd_params(1.0, 1.0, 2.0, 1.2, 1.0, [1 / 6] * 6, 1.5, False, code)
        ws = int(_lib.query(getattr(model, 'torch_device', None), 'mbir_vcd_workspace_size',
                            model._geometry(), int(max_subset_pixels), prm))
        y = 4 * n_sino if code != _lib.MBIR_F32 else 0
        # the binned whole-volume forward's workspace (initialisation, and
        # every error refresh of a 16-bit job; torch's caching allocator
        # keeps it)
        rs, ror = model.get_params(['recon_shape', 'use_ror_mask'])
        n_pix = int(vcd_utils.get_2d_ror_mask(rs, use_ror_mask=ror).sum()) \
            if ror is not False else rs[0] * rs[1]
        bins = int(_lib.query(getattr(model, 'torch_device', None),
                              'mbir_forward_project_binned_workspace_size', model._geometry(),
                              V, n_pix))
        resident = y + (2 if weighted else 1) * s * n_sino + ws + 8 * n_vol + (bins if y else 0)
        init = 4 * 4 * n_sino + 3 * 4 * n_vol + y + (4 * n_sino if weighted else 0) + bins
        return max(init, resident), resident


class Request:
    """One reconstruction request and, once served, its result."""

    def __init__(self, rid, model, sinogram, weights, max_iterations, stop_threshold_change_pct,
                 seed, arrival):
        self.id = rid
        self.model = model
        self.sinogram = sinogram
        self.weights = weights
        self.max_iterations = int(max_iterations)
        self.stop_pct = float(stop_threshold_change_pct)
        self.seed = int(seed)
        self.arrival = arrival
        self.admitted = None
        self.finished = None
        self.recon = None
        self.recon_params = None
        self.error = None
        self._run = None
        self._stream = None
        self._charge = 0
        self._out = None
        self._out_event = None
        self._state = None       # a preempted run's state, to resume from
        self.preempted = False   # taken off the device by ReconServer.preempt
        self.graph_replays = 0   # partition passes replayed from a captured graph

    def done(self):
        return self.finished is not None

    @property
    def latency(self):
        return None if self.finished is None else self.finished - self.arrival

    def result(self):
        if self.error is not None:
            raise self.error
        return self.recon


class ReconServer:
    """Serve reconstructions with continuous batching on one GPU.

    Args:
        device: CUDA device (default: the current one).
        memory_budget_bytes: ledger budget (default: 80% of the free memory).
        max_active: most jobs resident at once.
        storage_dtype: resident precision of the error sinogram, weights and
            delta sinogram ('float16' by default; see TomographyModel).
        cuda_graphs: replay each job's recurring partition passes as captured
            CUDA graphs (default True; see :class:`VcdRun`).  Results are
            bitwise the same either way; the graphs take the per-kernel
            launch work off the scheduler thread.
        batching: step the iterations of resident jobs that share a geometry
            (and storage, options and partition shape) together, each kernel
            of their subset steps launched once for all of them
            (:func:`vcd_run.enqueue_batched_iteration`, up to 16 jobs).  A job
            that becomes ready while a same-geometry partner is still running
            waits up to ``batch_hold_s`` for it, so that partners fall into
            step.  Results are bitwise the same batched or not.  Off by
            default: on one B200, eight same-geometry jobs served on their own
            streams (with CUDA graph replay) ran 1.06x (small parallel scans)
            to 1.21x (256^2 x 64 cone scans) faster than batched, because
            independent streams overlap one job's HBM-bound sinogram update
            with another's compute-bound projection, where lockstep batching
            runs every job in the same phase at once.
        admission: 'fifo' (the default) admits waiting requests in arrival
            order; 'shortest' admits the one with the least estimated work
            first (voxel-views per iteration times iterations), except that a
            request waiting longer than ``max_wait_s`` goes first, in arrival
            order (the wait bound caps how long a large job can be passed
            over).
    """

    def __init__(self, device=None, memory_budget_bytes=None, max_active=8,
                 storage_dtype='float16', cuda_graphs=True, admission='fifo',
                 max_wait_s=20.0, batching=False, batch_hold_s=0.05):
        self.device = torch.device('cuda', torch.cuda.current_device()) if device is None \
            else torch.device(device)
        if memory_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            memory_budget_bytes = int(0.8 * free)
        self.ledger = MemoryLedger(memory_budget_bytes)
        self.max_active = int(max_active)
        if admission not in ('fifo', 'shortest'):
            raise ValueError(f"admission must be 'fifo' or 'shortest', got {admission!r}")
        self.admission = admission
        self.max_wait_s = float(max_wait_s)
        self.batching = bool(batching)
        self.batch_hold_s = float(batch_hold_s)
        self._batch_stream = None
        self.batched_iterations = 0   # job-iterations run inside a batch
        self.storage_dtype = storage_dtype
        self.cuda_graphs = bool(cuda_graphs)
        storage_code(storage_dtype)
        self.waiting = []
        self.active = []
        self.completed = []
        self._next_id = 0
        self.max_concurrent = 0
        self.deferred = 0   # admissions put off because the ledger was full
        # Streams are reused from job to job, and from server to server in
        # one process: the caching allocator keeps its freed blocks per
        # stream, so fresh streams would grow the pool (cudaMalloc calls)
        # instead of reusing it.  A stream is out of the shared free list
        # while a job holds it.
        self._streams = _free_streams(self.device)
        self.t0 = None

    # ── requests ───────────────────────────────────────────────────────────
    def submit(self, model, sinogram, weights=None, max_iterations=10,
               stop_threshold_change_pct=0.0, seed=0, arrival=None):
        """Queue a reconstruction; returns its :class:`Request`."""
        now = time.perf_counter()
        if self.t0 is None:
            self.t0 = now
        r = Request(self._next_id, model, sinogram, weights, max_iterations,
                    stop_threshold_change_pct, seed, now if arrival is None else arrival)
        r.work = self.estimated_work(model, max_iterations)
        self._next_id += 1
        self.waiting.append(r)
        return r

    # ── scheduling ─────────────────────────────────────────────────────────
    def job_charge(self, model, weighted, max_iterations):
        """(peak, resident) ledger bytes of a job on ``model``.  Subsets are
        equal sized, ceil(ROR pixels / subsets), so the largest one in the
        partition sequence is known before any partition is drawn."""
        rs, gran, ror = model.get_params(['recon_shape', 'granularity', 'use_ror_mask'])
        n_pix = int(vcd_utils.get_2d_ror_mask(rs, use_ror_mask=ror).sum()) \
            if ror is not False else rs[0] * rs[1]
        seq = vcd_utils.gen_partition_sequence(model.get_params('partition_sequence'),
                                               max_iterations)
        max_ps = max((-(-n_pix // min(int(gran[int(i)]), n_pix)) for i in seq), default=1)
        return MemoryLedger.job_bytes(model, self.storage_dtype, weighted, max_ps)

    @staticmethod
    def estimated_work(model, max_iterations):
        """Voxel-views a request projects: ROR pixels x slices x views per
        projector pass, times its iterations."""
        V = model.get_params('sinogram_shape')[0]
        rs, ror = model.get_params(['recon_shape', 'use_ror_mask'])
        n_pix = int(vcd_utils.get_2d_ror_mask(rs, use_ror_mask=ror).sum()) \
            if ror is not False else rs[0] * rs[1]
        return float(n_pix) * rs[2] * V * max(1, int(max_iterations))

    def _next_waiting(self):
        """Index in ``waiting`` of the request to admit next."""
        if self.admission == 'fifo' or len(self.waiting) == 1:
            return 0
        now = time.perf_counter()
        if now - self.waiting[0].arrival > self.max_wait_s:
            return 0   # the oldest has waited past the bound
        return min(range(len(self.waiting)), key=lambda k: (self.waiting[k].work, k))

    def _admit_state(self, r):
        m = r.model
        m.configure_devices(devices=[self.device])
        m.setup_logger(logfile_path=None, print_logs=False)
        state = r._state
        m.storage_dtype = {_lib.MBIR_F32: 'float32', _lib.MBIR_BF16: 'bfloat16',
                           _lib.MBIR_F16: 'float16'}[int(state['storage'])]
        seq = np.asarray(state['seq'])
        parts = [state[f'partition_{k}'] for k in range(int(state['num_partitions']))]
        max_ps = max((int(parts[int(i)].shape[1]) for i in seq), default=1)
        _, resident = MemoryLedger.job_bytes(m, m.storage_dtype, 'w' in state, max_ps)
        if not self.ledger.fits(resident):
            if self.active:
                self.deferred += 1
                return False
            raise MemoryError(f'request {r.id} needs {resident} bytes; the ledger budget is '
                              f'{self.ledger.budget}')
        r._stream = self._streams.pop() if self._streams else torch.cuda.Stream(self.device)
        with torch.cuda.device(self.device):
            r._run = VcdRun.from_state(m, state, stream=r._stream,
                                       cuda_graphs=self.cuda_graphs)
        r._state = None
        self.ledger.take(resident)
        r._charge = resident
        r.admitted = time.perf_counter()
        if r._run.finished:
            self._finish(r)
        else:
            r._run.enqueue_iteration()
        return True

    def _admit(self, r):
        if getattr(r, '_state', None) is not None:
            return self._admit_state(r)
        m = r.model
        peak, resident = self.job_charge(m, r.weights is not None, r.max_iterations)
        if not self.ledger.fits(peak):
            if self.active:
                self.deferred += 1
                return False
            raise MemoryError(f'request {r.id} needs {peak} bytes; the ledger budget is '
                              f'{self.ledger.budget}')
        m.storage_dtype = self.storage_dtype
        m.configure_devices(devices=[self.device])
        m.setup_logger(logfile_path=None, print_logs=False)
        rng = np.random.RandomState(r.seed)
        rs, gran, ror = m.get_params(['recon_shape', 'granularity', 'use_ror_mask'])
        parts = [vcd_utils.gen_pixel_partition(rs, n, use_ror_mask=ror, rng=rng) for n in gran]
        seq = vcd_utils.gen_partition_sequence(m.get_params('partition_sequence'),
                                               r.max_iterations)
        m.auto_set_regularization_params(r.sinogram, weights=r.weights)
        r._stream = self._streams.pop() if self._streams else torch.cuda.Stream(self.device)
        r._run = VcdRun(m, r.sinogram, parts, seq, r.stop_pct, weights=r.weights, rng=rng,
                        stream=r._stream, cuda_graphs=self.cuda_graphs)
        self.ledger.take(peak)
        r._charge = peak
        r.admitted = time.perf_counter()
        with torch.cuda.device(self.device):
            r._run.prepare()
        self.ledger.release(peak - resident)
        r._charge = resident
        if not r._run.finished:
            r._run.enqueue_iteration()
        return True

    def _finish(self, r):
        run = r._run
        r.graph_replays += run.graph_replays
        with torch.cuda.stream(r._stream):
            r._out = torch.empty(run.flat.shape, dtype=torch.float32, pin_memory=True)
            r._out.copy_(run.flat, non_blocking=True)
            r._out_event = torch.cuda.Event()
            r._out_event.record(r._stream)
        fm, _, nmae, alphas, dnorm = run.losses()
        r.recon_params = {'num_iterations': run.done, 'fm_rmse': [float(v) for v in fm],
                          'stop_threshold_change_pct': [100 * float(v) for v in nmae],
                          'alpha_values': [float(v) for v in alphas]}

    # ── preemption ─────────────────────────────────────────────────────────
    def preempt(self, request):
        """Take an admitted request off the device between iterations: its
        resident state comes back as a host dict (:meth:`VcdRun.state_dict`)
        and its memory and slot are freed.  :meth:`resume` continues it,
        here or in another server, to the same result it would have reached
        uninterrupted."""
        if request not in self.active or request._run is None or request._out_event is not None:
            raise ValueError(f'request {request.id} is not running')
        run = request._run
        if run._event is not None:
            if run.collect():
                pass  # finished now; the checkpoint still carries its state
        state = run.state_dict()
        state['request_max_iterations'] = np.array(request.max_iterations)
        self.active.remove(request)
        self._streams.append(request._stream)
        request._stream = None
        request._run = None
        self.ledger.release(request._charge)
        request._charge = 0
        request.preempted = True
        return state

    def resume(self, model, state, arrival=None):
        """Queue a preempted request (its model and its :meth:`preempt`
        state) to continue; returns the new :class:`Request`."""
        r = self.submit(model, None, max_iterations=int(state['request_max_iterations']),
                        arrival=arrival)
        r._state = state
        return r

    def _enqueue_ready(self, ready):
        """Enqueue the next iteration of each ready job: same-key jobs as one
        batch; a job whose same-geometry partner is still running waits for
        it (up to batch_hold_s)."""
        from .vcd_run import enqueue_batched_iteration
        now = time.perf_counter()
        groups = {}
        for r in ready:
            key = r._run.batch_key() if self.batching else None
            groups.setdefault(key if key is not None else ('solo', r.id), []).append(r)
        # jobs with an iteration in flight, by the batch key of the iteration
        # they will take next
        running = {}
        if self.batching:
            for r in self.active:
                run = r._run
                if run is not None and run._event is not None and r._out_event is None and \
                        run.done + 1 < len(run.seq):
                    nxt = tuple(run.parts_dev[int(run.seq[run.done + 1])].shape)
                    running.setdefault((run.batch_key_geometry(), nxt), []).append(r)
        for key, rs in groups.items():
            if self.batching and key[0] != 'solo':
                partners = running.get((key[0], key[2]), [])
                if partners and len(rs) < 16 and \
                        now - min(r._ready_since for r in rs) < self.batch_hold_s:
                    continue   # a partner is finishing its iteration: wait for it
            for k in range(0, len(rs), 16):
                chunk = rs[k:k + 16]
                if len(chunk) == 1:
                    chunk[0]._run.enqueue_iteration()
                else:
                    if self._batch_stream is None:
                        self._batch_stream = torch.cuda.Stream(self.device)
                    with torch.cuda.device(self.device):
                        enqueue_batched_iteration([r._run for r in chunk], self._batch_stream)
                    self.batched_iterations += len(chunk)
                for r in chunk:
                    r._ready_since = None

    def step(self):
        """One scheduler pass; returns True if it did anything."""
        busy = False
        ready = []
        # advance the admitted jobs
        for r in list(self.active):
            if r._out_event is not None:
                if r._out_event.query():
                    rs = r._run.recon_shape
                    r.recon = r._out.numpy().reshape(rs)
                    r.finished = time.perf_counter()
                    r._run = None
                    self._streams.append(r._stream)
                    r._stream = None
                    self.ledger.release(r._charge)
                    r._charge = 0
                    self.active.remove(r)
                    self.completed.append(r)
                    busy = True
                continue
            if r._run.ready():
                if r._run.collect():
                    self._finish(r)
                else:
                    r._ready_since = time.perf_counter()
                    ready.append(r)
                busy = True
        # jobs held for a same-geometry partner from an earlier pass
        ready += [r for r in self.active if r._run is not None and r._out_event is None
                  and getattr(r, '_ready_since', None) is not None and r not in ready]
        if ready:
            self._enqueue_ready(ready)
        # admit waiting requests (in the admission policy's order) while
        # slots and memory allow
        while self.waiting and len(self.active) < self.max_active:
            k = self._next_waiting()
            r = self.waiting[k]
            try:
                if not self._admit(r):
                    break
            except Exception as exc:  # a failing job frees its slot, others go on
                r.error = exc
                r.finished = time.perf_counter()
                r._run = None
                if r._stream is not None:
                    self._streams.append(r._stream)
                    r._stream = None
                if r._charge:
                    self.ledger.release(r._charge)
                    r._charge = 0
                self.waiting.pop(k)
                self.completed.append(r)
                busy = True
                continue
            self.waiting.pop(k)
            self.active.append(r)
            busy = True
        self.max_concurrent = max(self.max_concurrent, len(self.active))
        return busy

    def run_until_idle(self, poll_s=2e-4, timeout_s=None):
        t_end = None if timeout_s is None else time.perf_counter() + timeout_s
        while self.waiting or self.active:
            if not self.step():
                time.sleep(poll_s)
            if t_end is not None and time.perf_counter() > t_end:
                raise TimeoutError('server did not drain in time')

    def serve_schedule(self, schedule, poll_s=2e-4, timeout_s=None):
        """Submit requests at their arrival offsets (seconds from now) while
        serving: ``schedule`` is a list of (offset_s, submit_kwargs)."""
        start = time.perf_counter()
        if self.t0 is None:
            self.t0 = start
        pending = sorted(schedule, key=lambda s: s[0])
        t_end = None if timeout_s is None else start + timeout_s
        i = 0
        while i < len(pending) or self.waiting or self.active:
            now = time.perf_counter()
            while i < len(pending) and start + pending[i][0] <= now:
                kw = dict(pending[i][1])
                kw.setdefault('arrival', start + pending[i][0])
                self.submit(**kw)
                i += 1
            if not self.step():
                time.sleep(poll_s)
            if t_end is not None and time.perf_counter() > t_end:
                raise TimeoutError('server did not drain in time')
        return self.completed

    # ── metrics ────────────────────────────────────────────────────────────
    def stats(self):
        ok = [r for r in self.completed if r.error is None]
        lat = np.array([r.latency for r in ok]) if ok else np.zeros(0)
        span = (max(r.finished for r in ok) - min(r.arrival for r in ok)) if ok else 0.0
        return {
            'completed': len(ok), 'failed': len(self.completed) - len(ok),
            'recons_per_s': (len(ok) / span) if span > 0 else math.nan,
            'p50_latency_s': float(np.percentile(lat, 50)) if ok else math.nan,
            'p99_latency_s': float(np.percentile(lat, 99)) if ok else math.nan,
            'max_concurrent': self.max_concurrent, 'span_s': span,
            'batched_iterations': self.batched_iterations,
        }
