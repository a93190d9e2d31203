"""One reconstruction's device state, split into steps.

This is the body of the reference's ``_vcd_recon`` (tomography_model.py:
2699-3013) restructured so that the same code serves a single blocking
``recon()`` and a server that interleaves many reconstructions:

* :meth:`VcdRun.prepare` -- host prep done by the caller (partitions, the
  partition sequence and the regularization), then, on the run's CUDA
  stream: the sinogram upload, the direct-recon init, the optimally scaled
  initial error state, the Hessian diagonal and the resident VCD state.
  No host synchronization.
* :meth:`VcdRun.enqueue_iteration` -- one VCD iteration (one partition pass
  in an order drawn from the run's RNG), the optional 16-bit refresh and the
  statistics, with an asynchronous copy of the statistics to pinned host
  memory and an event.
* :meth:`VcdRun.ready` / :meth:`VcdRun.collect` -- poll the event, then turn
  the statistics into the reference's per-iteration traces and the stopping
  decision.

Every run owns its stream, its RNG and its buffers, and the kernels are
deterministic, so a run's result does not depend on what else is running.

With ``cuda_graphs=True`` (the server's default) a partition pass whose
shape -- (subsets, pixels per subset) -- recurs later in the run is
captured once as a CUDA graph and replayed.  The graph walks the subsets of
a run-owned "ordered partition" buffer in row order; before each replay one
small gather writes the iteration's subsets into that buffer in the drawn
order (``ordered[k] = partition[order[k]]``).  The graph therefore depends
only on the shape, not on the partition or the order, and the kernels see
exactly the pixel lists the direct launch path gives them: the results are
bitwise the same.  A 128-subset pass is ~640 kernel launches; replaying it
costs the host one graph launch, which is what lets many small jobs keep
the device busy from one scheduler thread.
"""

import math

import numpy as np
import torch

from . import _lib
from ._lib import STORAGE_DTYPES
from .vcd_engine import ResidentSinogram, error_init, iteration_stats, order_array, storage_code


class VcdRun:

    def __init__(self, model, sinogram, partitions, partition_sequence,
                 stop_threshold_change_pct, weights=None, init_recon=None,
                 init_error_sinogram=None, fm_hessian=None, rng=None, first_iteration=0,
                 stream=None, prox_input=None, cuda_graphs=False):
        model.verify_valid_params()
        model._require_cuda()
        self.model = model
        self.recon_shape = tuple(model.get_params('recon_shape'))
        self.sinogram_shape = tuple(model.get_params('sinogram_shape'))
        if init_error_sinogram is None and tuple(sinogram.shape) != self.sinogram_shape:
            raise ValueError('sinogram does not have the shape in sinogram_shape. \n'
                             f'Expected {self.sinogram_shape}, got {tuple(sinogram.shape)}.')
        if init_error_sinogram is not None and init_recon is None:
            raise ValueError('init_error_sinogram requires init_recon (the pair must be a '
                             'consistent resume state; see the docstring).')
        self.sinogram = sinogram
        self.weights = weights
        self.init_recon = init_recon
        self.init_error_sinogram = init_error_sinogram
        self.fm_hessian = fm_hessian
        self.prox_input = prox_input
        self.partitions = partitions
        self.seq = np.asarray(partition_sequence)
        self.stop_pct = stop_threshold_change_pct
        self.rng = rng
        self.first_iteration = first_iteration
        self.storage = storage_code(model.storage_dtype)
        self.stream = stream if stream is not None else torch.cuda.current_stream(
            model.torch_device)
        n = len(self.seq)
        self.fm_rmse = np.zeros(n)
        self.pm_loss = np.zeros(n)
        self.nmae = np.zeros(n)
        self.alphas = np.zeros(n)
        self.dnorm = np.zeros((n, self.recon_shape[2]))
        self.done = 0
        self.finished = n == 0
        self._event = None
        self._pending = None
        self.cuda_graphs = bool(cuda_graphs)
        self._graphs = {}
        self._graph_shapes = set()
        self.graph_replays = 0
        self.batched_passes = 0

    # ── device preparation ───────────────────────────────────────────────
    def prepare(self):
        m = self.model
        with torch.cuda.stream(self.stream):
            self._prepare()
        return self

    def _prepare(self):
        m = self.model
        dev = m.torch_device
        log = m.logger
        w_dev = None if self.weights is None else m._sino_device(self.weights)
        self.constant_weights = w_dev is None
        sino = None if self.init_error_sinogram is not None else m._sino_device(self.sinogram)
        refresh = m.error_refresh_interval
        if refresh is None:
            refresh = {_lib.MBIR_F32: 0, _lib.MBIR_F16: 5, _lib.MBIR_BF16: 5}[self.storage]
        self.refresh = refresh
        self.y_vcr = None
        if refresh and sino is not None:
            self.y_vcr = ResidentSinogram.from_vrc(sino, _lib.MBIR_F32).data
        init_recon = self.init_recon
        scale = init_recon is None
        if init_recon is None:
            log.info('Starting direct recon for initial reconstruction')
            init_recon = m.recon_direct(sino, output_sharded=True)
        elif isinstance(init_recon, int):
            init_recon = torch.full(self.recon_shape, float(init_recon), dtype=torch.float32,
                                    device=dev)
        else:
            if tuple(np.shape(init_recon)) != self.recon_shape:
                raise ValueError(f"init_recon does not have the correct shape. Expected "
                                 f"{self.recon_shape}, got {tuple(np.shape(init_recon))}.")
            init_recon = m._recon_device(init_recon)
        if self.init_error_sinogram is not None:
            log.info('Resuming from init_error_sinogram')
            err_vrc = m._sino_device(self.init_error_sinogram)
            x0 = init_recon
        else:
            log.info('Initializing error sinogram')
            fwd = m.forward_project(init_recon, output_sharded=True)
            err_vrc, alpha = error_init(sino, fwd, w_dev, scale)
            del fwd
            # alpha stays on the device: x0 = float32(alpha) * x0, as the
            # reference's python-float scaling (tomography_model.py:1700-1711)
            x0 = init_recon * alpha.to(torch.float32)
        sino = None
        if self.fm_hessian is None:
            log.info('Computing Hessian diagonal')
            hess_idx = None if m.get_params('use_ror_mask') is False \
                else m.full_indices_device()
            self.fm_hessian = m.compute_hessian_diagonal(weights=w_dev, output_sharded=True,
                                                         indices=hess_idx)
        else:
            log.info('Using precomputed Hessian diagonal')
            self.fm_hessian = m._recon_device(self.fm_hessian)
        H = self.fm_hessian.reshape(-1, self.fm_hessian.shape[-1]).contiguous()
        self.flat = x0.reshape(-1, x0.shape[-1]).contiguous().clone()
        self.err = ResidentSinogram.from_vrc(err_vrc, self.storage)
        del err_vrc
        self.w_res = None if w_dev is None else ResidentSinogram.from_vrc(w_dev, self.storage)
        del w_dev
        self.total = float(math.prod(self.sinogram_shape))
        self.parts_dev = [torch.as_tensor(np.ascontiguousarray(p), dtype=torch.int64, device=dev)
                          for p in self.partitions]
        max_ps = max((int(self.partitions[int(i)].shape[1]) for i in self.seq), default=1)
        self.prox_flat = m._prox_flat(self.prox_input)
        self.engine = m._make_engine(H, self.w_res, self.storage, max_subset_pixels=max_ps,
                                     prox_flat=self.prox_flat)
        self.host = torch.empty(2 + self.recon_shape[2] + 4, dtype=torch.float64,
                                pin_memory=True)
        self._set_finish()
        self._graph_setup()
        log.info('Starting VCD iterations')

    # ── the float16 finish of a bfloat16 run ─────────────────────────────
    def _set_finish(self):
        """Iteration at which a bfloat16 run re-forms its error sinogram in
        float16 (None: no switch).  bfloat16's 8-bit significand quantizes
        e to about 2^-9 of its size; the last iterations' updates carry that
        noise into the volume.  Re-forming e = y - A x in float16 (an 11-bit
        significand with power-of-two per-view scales, the same two bytes a
        cell) for the last ``model.bf16_finish_iterations`` iterations
        removes most of it."""
        self.finish_at = None
        k = int(getattr(self.model, 'bf16_finish_iterations', 0) or 0)
        if self.storage == _lib.MBIR_BF16 and self.y_vcr is not None and k > 0:
            self.finish_at = max(self.done, len(self.seq) - k)

    def _finish_in_float16(self):
        m = self.model
        V, R, C = self.sinogram_shape
        dev = m.torch_device
        m.logger.info('Re-forming the error sinogram in float16 for the last {} iterations'
                      .format(len(self.seq) - self.done))
        e32 = ResidentSinogram(torch.empty((V, C, R), dtype=torch.float32, device=dev),
                               torch.ones(V, dtype=torch.float32, device=dev), R, _lib.MBIR_F32)
        self.engine.refresh_error(self.flat, e32, m.full_indices_device(), self.y_vcr)
        e_vrc = e32.to_vrc()
        del e32
        self.err = ResidentSinogram.from_vrc(e_vrc, _lib.MBIR_F16)
        del e_vrc
        if self.w_res is not None:
            self.w_res = ResidentSinogram.from_vrc(self.w_res.to_vrc(), _lib.MBIR_F16)
        self.storage = _lib.MBIR_F16
        H = self.fm_hessian.reshape(-1, self.fm_hessian.shape[-1]).contiguous()
        self.engine = m._make_engine(H, self.w_res, self.storage,
                                     max_subset_pixels=self.engine._ws_pixels,
                                     prox_flat=self.prox_flat)
        self.release_graphs()
        self.finish_at = None

    def _graph_setup(self):
        """Pick the pass shapes worth a graph -- those used at least twice
        in the iterations still to run -- and allocate the buffers their
        replays gather into.  Graphs need a stream of the run's own: the
        legacy default stream cannot be captured."""
        self._graph_shapes = set()
        if not self.cuda_graphs or self.stream == torch.cuda.default_stream(
                self.model.torch_device):
            return
        uses = {}
        for i in self.seq[self.done:]:
            shape = tuple(self.parts_dev[int(i)].shape)
            uses[shape] = uses.get(shape, 0) + 1
        self._graph_shapes = {s for s, u in uses.items() if u >= 2}
        if not self._graph_shapes:
            return
        dev = self.model.torch_device
        k_max = max(s[0] for s in self._graph_shapes)
        self._ordered = torch.empty(max(s[0] * s[1] for s in self._graph_shapes),
                                    dtype=torch.int64, device=dev)
        self._order_dev = torch.empty(k_max, dtype=torch.int64, device=dev)
        self._order_host = torch.empty(k_max, dtype=torch.int64, pin_memory=True)

    def _graph_pass(self, part, order):
        """One partition pass by graph replay (captured on first use of its
        shape).  Called on the run's stream."""
        K, n = part.shape
        oh = self._order_host[:K]
        oh.numpy()[:] = order   # the previous copy from it ended before collect()
        od = self._order_dev[:K]
        od.copy_(oh, non_blocking=True)
        ordered = self._ordered[:K * n].view(K, n)
        torch.index_select(part, 0, od, out=ordered)
        g = self._graphs.get((K, n))
        if g is None:
            self.engine.reserve(n)
            g = torch.cuda.CUDAGraph()
            g.capture_begin(capture_error_mode='thread_local')
            try:
                self.engine.partition_pass(self.flat, self.err, ordered,
                                           np.arange(K, dtype=np.int32))
            except BaseException:
                try:
                    g.capture_end()
                except Exception:
                    pass
                raise
            g.capture_end()
            self._graphs[(K, n)] = g
        g.replay()
        self.graph_replays += 1

    def release_graphs(self):
        """Drop the captured graphs (their device resources go with them)."""
        self._graphs.clear()

    # ── iterations ───────────────────────────────────────────────────────
    def enqueue_iteration(self):
        """Enqueue iteration ``self.done`` on the run's stream (no sync)."""
        if self.finished or self._event is not None:
            raise RuntimeError('no iteration can be enqueued now')
        with torch.cuda.stream(self.stream):
            part, order = self._begin_iteration()
            if tuple(part.shape) in self._graph_shapes and not _lib.timing_enabled():
                self._graph_pass(part, order)
            else:
                self.engine.partition_pass(self.flat, self.err, part, order)
            self._end_iteration(part)

    # The pieces of an iteration, on the current stream (a run's own, or the
    # stream of a batch of runs, enqueue_batched_iteration).
    def _begin_iteration(self):
        i = self.done
        if self.finish_at is not None and i >= self.finish_at:
            self._finish_in_float16()
        part = self.parts_dev[int(self.seq[i])]
        order = order_array(part.shape[0], self.rng)
        self.engine.accum.zero_()
        return part, order

    def _end_iteration(self, part):
        i = self.done
        # (no refresh after the last iteration, whose error sinogram only
        # feeds the statistics, nor right before the float16 finish, which
        # re-forms it anyway)
        if self.y_vcr is not None and (i + 1) % self.refresh == 0 and \
                i + 1 < len(self.seq) and i + 1 != self.finish_at:
            self.engine.refresh_error(self.flat, self.err, self.model.full_indices_device(),
                                      self.y_vcr)
        stats = iteration_stats(self.err, self.w_res, self.flat)
        self.host.copy_(torch.cat([self.engine.accum, stats]), non_blocking=True)
        self._event = torch.cuda.Event()
        self._event.record(torch.cuda.current_stream(self.model.torch_device))
        self._pending = part.shape[0]

    def batch_key_geometry(self):
        """The part of :meth:`batch_key` that does not change from iteration
        to iteration (geometry, view parameters, options, device)."""
        m = self.model
        g = m._geometry()
        return (tuple(getattr(g, f) for f, _ in g._fields_),
                np.asarray(m._view_params_array()).tobytes(),
                bool(m.get_params('positivity_flag')), self.w_res is None,
                self.prox_flat is None, str(m.torch_device))

    def batch_key(self):
        """Runs with equal keys can take their next iteration as one batch
        (:func:`enqueue_batched_iteration`): the same geometry and view
        parameters, storage (after a float16 finish due now), options and
        partition shape.  None when the run cannot be batched."""
        if self.finished or self._event is not None:
            return None
        storage = self.storage
        if self.finish_at is not None and self.done >= self.finish_at:
            storage = _lib.MBIR_F16
        return (self.batch_key_geometry(), storage,
                tuple(self.parts_dev[int(self.seq[self.done])].shape))

    def ready(self):
        return self._event is not None and self._event.query()

    def wait(self):
        if self._event is not None:
            self._event.synchronize()

    def collect(self):
        """Read the finished iteration's statistics; returns True when the
        run is over (iteration count reached or change threshold met)."""
        self.wait()
        i, n_sub = self.done, self._pending
        self._event, self._pending = None, None
        S = self.recon_shape[2]
        h = self.host.numpy()
        acc, st = h[:2 + S], h[2 + S:]
        sigma_y = self.model.get_params('sigma_y')
        avg_w = 1.0 if self.constant_weights else st[1] / self.total
        self.fm_rmse[i] = math.sqrt(st[0] / (avg_w * self.total)) / sigma_y
        self.nmae[i] = acc[0] / st[3] if st[3] else float('nan')
        self.alphas[i] = acc[1] / n_sub
        self.dnorm[i] = np.sqrt(acc[2:])
        log = self.model.logger
        if self.model.get_params('verbose') >= 1:
            n = len(self.seq) + self.first_iteration
            log.info('\nAfter iteration {} of a max of {}: Pct change={:.4f}, Forward loss={:.4f}'
                     .format(i + self.first_iteration, n, 100 * self.nmae[i], self.fm_rmse[i]))
            log.info(f'Relative step size (alpha)={self.alphas[i]:.2f}, '
                     f'Error sino RMSE={math.sqrt(st[2] / self.total):.4f}')
            log.info('Number subsets = {}'.format(n_sub))
        self.done += 1
        if self.nmae[i] < self.stop_pct / 100:
            log.warning('Change threshold stopping condition reached')
            self.finished = True
        if self.done >= len(self.seq):
            self.finished = True
        return self.finished

    def run(self):
        """Blocking: prepare, then iterate to the end."""
        self.prepare()
        while not self.finished:
            self.enqueue_iteration()
            self.collect()
        return self

    # ── results ──────────────────────────────────────────────────────────
    def recon3d(self):
        return self.flat.reshape(self.recon_shape[:2] + (self.flat.shape[-1],))

    def losses(self):
        d = self.done
        return (self.fm_rmse[:d], self.pm_loss[:d], self.nmae[:d], self.alphas[:d],
                self.dnorm[:d])

    def checkpoint(self):
        with torch.cuda.stream(self.stream):
            return {'error_sinogram': self.err.to_vrc(), 'fm_hessian': self.fm_hessian}

    # ── resident-state checkpoint (preemption and restart) ───────────────
    _TRACES = ('fm_rmse', 'pm_loss', 'nmae', 'alphas', 'dnorm')

    def state_dict(self):
        """The run's whole resident state on the host, between iterations:
        the recon, the stored error sinogram (its storage bits and per-view
        scales), weights, the FP32 measurements kept for the 16-bit refresh,
        the Hessian diagonal, the partitions and sequence, the traces so far
        and the position of the run's own RandomState.  A run restored from
        it (:meth:`from_state`) continues exactly as this one would have:
        the same subset orders and bit-identical kernels.  Only runs with
        their own RandomState can be checkpointed (the global numpy
        generator is not theirs to save)."""
        if self._event is not None:
            raise RuntimeError('checkpoint between iterations (collect the pending one first)')
        if not isinstance(self.rng, np.random.RandomState):
            raise RuntimeError('only a run with its own RandomState can be checkpointed')

        def raw(t):  # 16-bit storage travels as its raw bits
            t = t.detach()
            return (t.view(torch.int16) if t.dtype in (torch.float16, torch.bfloat16)
                    else t).cpu().numpy()

        with torch.cuda.stream(self.stream):
            kind, keys, pos, has_gauss, gauss = self.rng.get_state()
            st = {'version': np.array(1), 'storage': np.array(self.storage),
                  'refresh': np.array(self.refresh), 'done': np.array(self.done),
                  'finished': np.array(self.finished), 'seq': np.asarray(self.seq),
                  'stop_pct': np.array(self.stop_pct),
                  'first_iteration': np.array(self.first_iteration),
                  'constant_weights': np.array(self.constant_weights),
                  'recon_shape': np.array(self.recon_shape),
                  'sinogram_shape': np.array(self.sinogram_shape),
                  'flat': raw(self.flat), 'fm_hessian': raw(self.fm_hessian),
                  'err': raw(self.err.data), 'err_scale': raw(self.err.scale),
                  'rng_keys': keys, 'rng_pos': np.array(pos),
                  'rng_gauss': np.array([has_gauss, gauss], dtype=np.float64),
                  'num_partitions': np.array(len(self.partitions)),
                  'reg': np.array([self.model.get_params(k) or 0.0
                                   for k in ('sigma_y', 'sigma_x', 'sigma_prox')],
                                  dtype=np.float64)}
            for k, p in enumerate(self.partitions):
                st[f'partition_{k}'] = np.asarray(p)
            for name in self._TRACES:
                st[name] = getattr(self, name)
            if self.w_res is not None:
                st['w'], st['w_scale'] = raw(self.w_res.data), raw(self.w_res.scale)
            if self.y_vcr is not None:
                st['y_vcr'] = raw(self.y_vcr)
            if self.prox_flat is not None:
                st['prox'] = raw(self.prox_flat)
        return st

    def save_state(self, path):
        """:meth:`state_dict` written to ``path`` (numpy .npz)."""
        np.savez(path, **self.state_dict())

    @classmethod
    def from_state(cls, model, state, stream=None, cuda_graphs=False):
        """A prepared run that continues from ``state`` (a dict from
        :meth:`state_dict` or the path of a :meth:`save_state` file) on
        ``model`` (the same geometry and regularization)."""
        if isinstance(state, (str, bytes)) or hasattr(state, '__fspath__'):
            with np.load(state) as f:
                state = {k: f[k] for k in f.files}
        if int(state['version']) != 1:
            raise ValueError('unknown checkpoint version {}'.format(int(state['version'])))
        if tuple(state['recon_shape']) != tuple(model.get_params('recon_shape')) or \
                tuple(state['sinogram_shape']) != tuple(model.get_params('sinogram_shape')):
            raise ValueError('the checkpoint was taken on another geometry')
        storage = int(state['storage'])
        sy, sx, sp = (float(v) for v in state['reg'])
        model.set_params(no_warning=True, sigma_y=sy, sigma_x=sx, sigma_prox=sp,
                         auto_regularize_flag=False)
        model.storage_dtype = {_lib.MBIR_F32: 'float32', _lib.MBIR_BF16: 'bfloat16',
                               _lib.MBIR_F16: 'float16'}[storage]
        parts = [state[f'partition_{k}'] for k in range(int(state['num_partitions']))]
        rng = np.random.RandomState()
        rng.set_state(('MT19937', state['rng_keys'], int(state['rng_pos']),
                       int(state['rng_gauss'][0]), float(state['rng_gauss'][1])))
        run = cls.__new__(cls)
        run.model = model
        run.recon_shape = tuple(int(v) for v in state['recon_shape'])
        run.sinogram_shape = tuple(int(v) for v in state['sinogram_shape'])
        run.sinogram = run.weights = run.init_recon = run.init_error_sinogram = None
        run.prox_input = None
        run.partitions = parts
        run.seq = np.asarray(state['seq'])
        run.stop_pct = float(state['stop_pct'])
        run.rng = rng
        run.first_iteration = int(state['first_iteration'])
        run.storage = storage
        run.stream = stream if stream is not None else torch.cuda.current_stream(
            model.torch_device)
        for name in cls._TRACES:
            setattr(run, name, np.array(state[name]))
        run.done = int(state['done'])
        run.finished = bool(state['finished'])
        run._event = None
        run._pending = None
        run.cuda_graphs = bool(cuda_graphs)
        run._graphs = {}
        run.graph_replays = 0
        run.batched_passes = 0
        run.refresh = int(state['refresh'])
        run.constant_weights = bool(state['constant_weights'])
        dev = model.torch_device
        sdt = STORAGE_DTYPES[storage]

        def cooked(a, dtype):
            t = torch.as_tensor(a, device=dev)
            return t.view(dtype) if dtype in (torch.float16, torch.bfloat16) else t

        with torch.cuda.stream(run.stream):
            run.flat = cooked(state['flat'], torch.float32).contiguous()
            run.fm_hessian = cooked(state['fm_hessian'], torch.float32)
            V, R, C = run.sinogram_shape
            run.err = ResidentSinogram(cooked(state['err'], sdt).contiguous(),
                                       cooked(state['err_scale'], torch.float32), R, storage)
            run.w_res = None
            if 'w' in state:
                run.w_res = ResidentSinogram(cooked(state['w'], sdt).contiguous(),
                                             cooked(state['w_scale'], torch.float32), R, storage)
            run.y_vcr = cooked(state['y_vcr'], torch.float32) if 'y_vcr' in state else None
            run.prox_flat = cooked(state['prox'], torch.float32) if 'prox' in state else None
            run.total = float(math.prod(run.sinogram_shape))
            run.parts_dev = [torch.as_tensor(np.ascontiguousarray(p), dtype=torch.int64,
                                             device=dev) for p in parts]
            max_ps = max((int(parts[int(i)].shape[1]) for i in run.seq), default=1)
            H = run.fm_hessian.reshape(-1, run.fm_hessian.shape[-1]).contiguous()
            run.engine = model._make_engine(H, run.w_res, storage, max_subset_pixels=max_ps,
                                            prox_flat=run.prox_flat)
            run.host = torch.empty(2 + run.recon_shape[2] + 4, dtype=torch.float64,
                                   pin_memory=True)
            run._set_finish()
            run._graph_setup()
        return run

    def device_bytes(self):
        """Bytes this run holds resident on the device."""
        n = self.flat.numel() * 4 + self.fm_hessian.numel() * 4 + self.err.nbytes()
        n += self.engine.workspace_bytes()
        if self.w_res is not None:
            n += self.w_res.nbytes()
        if self.y_vcr is not None:
            n += self.y_vcr.numel() * 4
        if self._graph_shapes:
            n += (self._ordered.numel() + self._order_dev.numel()) * 8
        return n


def enqueue_batched_iteration(runs, stream):
    """The next iteration of several runs with equal :meth:`VcdRun.batch_key`
    as one batch on ``stream``: each kernel of each subset step is launched
    once for all of them (``mbir_vcd_partition_pass_batched``); every run's
    subsets, orders, statistics and results are its own.  ``stream`` waits
    for the runs' own streams first, and they wait for it afterwards."""
    from .vcd_engine import partition_pass_batched
    if len(runs) == 1:
        runs[0].enqueue_iteration()
        return
    key = runs[0].batch_key()
    if key is None or any(r.batch_key() != key for r in runs[1:]):
        raise ValueError('runs of a batch must share batch_key()')
    with torch.cuda.stream(stream):
        for r in runs:
            stream.wait_stream(r.stream)
        items = [r._begin_iteration() for r in runs]
        partition_pass_batched([r.engine for r in runs], [r.flat for r in runs],
                               [r.err for r in runs], [p for p, _ in items],
                               [o for _, o in items])
        for r, (part, _) in zip(runs, items):
            r._end_iteration(part)
            r.batched_passes += 1
    for r in runs:
        r.stream.wait_stream(stream)
