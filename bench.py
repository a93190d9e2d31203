"""Benchmark: cone-beam MBIR on B200 (one JSON line on stdout).

Headline workload, the largest single-GPU configuration: a 512 x 512 x 256
volume of 10 seeded ellipsoids, 720 views on [0, 2 pi), a curved 320 x 768
detector with 2-unit pixels, source-to-iso 1024, source-to-detector 2048
(magnification 2), Poisson counts at I0 = 1e4 converted back to line
integrals, qGGMRF prior (p = 2, q = 1.2), 20 VCD iterations, FP32 storage.
One STEP is one complete reconstruction (direct-recon init, Hessian, 20
iterations).

  value      recons/s with the sinogram resident in HBM before the timed
             region (model.recon on a CUDA tensor)
  e2e        recons/s through the public API from a pinned host sinogram to a
             host volume (copies inside the timed region)
  roofline   the dominant kernel's algorithmic bytes (one read of each error-
             sinogram cell its subset reaches, counted on the device) over its
             CUDA-event duration, against the measured HBM copy bandwidth
  cpu_baseline  the FP64 C oracle (the reference's algorithm restated, all
             host threads) on one 128-subset VCD step of this workload,
             extrapolated to a whole recon, with the GPU step's parity
             against it; the reference's own eager CPU code (mbirtorch 0.0.2,
             installed under baseline/_ref) timed whole on its small CPU
             configuration beside it

--impl reference times the reference's own CPU code on this workload (rank 0;
other ranks exit): each step one warm 128-subset step over 90 of the 720
views, scaled to the whole scan by a measured full-scan step and to a whole
recon.
Multi-GPU: independent replicas, one per rank (no data exchange).
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
REF_DIR = os.path.join(ROOT, "baseline", "_ref")

SDD, SID = 2048.0, 1024.0
ITERS = 20
I0 = 1e4
# name: (views, detector rows, channels, in-plane N, slices, curved)
CONFIGS = {
    "cone512_curved": (720, 320, 768, 512, 256, True),
    "cone256_flat": (360, 256, 384, 256, 256, False),
}
HEAD = "cone512_curved"
METRIC = "recons/s (cone-beam MBIR 512^2 x 256, 720 views, curved 320 x 768, 20 VCD iterations)"


def workload(name, iters=ITERS, storage="float32"):
    V, R, C, N, S, curved = CONFIGS[name]
    return (f"cone {'curved' if curved else 'flat'} {N}x{N}x{S} volume, {V} views on "
            f"[0, 2pi), {R}x{C} detector (pitch 2), SID 1024, SDD 2048, Poisson I0=1e4, "
            f"qGGMRF p=2 q=1.2, {iters} VCD iterations, {storage} storage")


def config_block(storage="float32", world=1):
    V, R, C, N, S, curved = CONFIGS[HEAD]
    sino_mb = V * R * C * 4 / 1e6
    return {"workload": workload(HEAD, storage=storage), "volume": [N, N, S], "views": V,
            "detector_rows_channels": [R, C], "curved_detector": curved,
            "iterations": ITERS, "storage": storage, "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2 ({sino_mb:.0f} MB f32 sinogram vs 126 MB L2)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mbir", choices=["mbir", "reference"])
    ap.add_argument("--storage", default="float32")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip every extra measurement (headline value and e2e only)")
    ap.add_argument("--only-extra", default=None,
                    help="run only these extras (comma-separated names, e.g. "
                         "triton_reference,mixed_precision) after the headline")
    ap.add_argument("--serving-config5", action="store_true",
                    help="run the serving configuration (200 Poisson arrivals) against "
                         "sequential plain FP32 solves and print its JSON (minutes)")
    ap.add_argument("--profile-case", choices=["recon", "subset", "projectors",
                                               "subset-parallel", "subset-cone64",
                                               "subset-small"], default=None,
                    help="run one untimed pass of the workload for an external profiler "
                         "and exit (no JSON line)")
    return ap.parse_args()


# ── synthetic data ──────────────────────────────────────────────────────────
def phantom_torch(torch, shape, seed, dev):
    """10 seeded ellipsoids on [-1, 1]^3 grids, built on the device: centres
    U[-0.5, 0.5], semi-axes U[0.05, 0.4], in-plane angle U[0, 180) deg,
    density U[0.1, 1]."""
    rng = np.random.default_rng(seed)
    nr, nc, ns = shape
    g1 = torch.linspace(-1, 1, nr, device=dev)
    g0 = torch.linspace(-1, 1, nc, device=dev)
    gz = torch.linspace(-1, 1, ns, device=dev)
    Y, X = torch.meshgrid(g1, g0, indexing="ij")
    vol = torch.zeros(shape, device=dev)
    for _ in range(10):
        c = rng.uniform(-0.5, 0.5, 3)
        a = rng.uniform(0.05, 0.4, 3)
        ang = np.deg2rad(rng.uniform(0, 180))
        dens = float(rng.uniform(0.1, 1.0))
        ca, sa = float(np.cos(ang)), float(np.sin(ang))
        xr = ca * (X - c[0]) + sa * (Y - c[1])
        yr = -sa * (X - c[0]) + ca * (Y - c[1])
        xy = (xr / a[0]) ** 2 + (yr / a[1]) ** 2
        z = ((gz - c[2]) / a[2]) ** 2
        vol += dens * ((xy[:, :, None] + z[None, None, :]) <= 1).float()
    return vol


def cone_model(pkg, name, views=None, **ctor):
    """The configuration's ConeBeamModel in package ``pkg`` (this one or the
    reference); ``views`` keeps every k-th view of the scan."""
    V, R, C, N, S, curved = CONFIGS[name]
    ang = np.linspace(0, 2 * np.pi, V, endpoint=False)
    if views is not None:
        ang = ang[views]
    m = pkg.ConeBeamModel((len(ang), R, C), ang, source_detector_dist=SDD, source_iso_dist=SID,
                          use_curved_detector=curved, **ctor)
    m.set_params(no_warning=True, verbose=0, delta_det_channel=2.0, delta_det_row=2.0)
    m.auto_set_recon_geometry(no_warning=True)
    m.set_params(no_warning=True, recon_shape=(N, N, S))
    return m


def make_data(m, torch, dev, seed):
    """Noisy line integrals on the device: the phantom is scaled so that the
    largest line integral is 3 (transmission >= 5%), counts ~ Poisson(I0
    exp(-Ax)), y = -log(max(counts, 1) / I0), returned in phantom units."""
    vol = phantom_torch(torch, tuple(m.get_params('recon_shape')), seed, dev)
    clean = m.forward_project(vol, output_sharded=True)
    del vol
    mu = 3.0 / float(clean.max())
    gen = torch.Generator(device=dev).manual_seed(seed)
    counts = torch.poisson(I0 * torch.exp(-mu * clean), generator=gen)
    del clean
    y = (-torch.log(torch.clamp(counts, min=1.0) / I0) / mu).to(torch.float32).contiguous()
    return y


def recon(m, sino, iters=ITERS, seed=0, **kw):
    np.random.seed(seed)
    return m.recon(sino, max_iterations=iters, stop_threshold_change_pct=0, logfile_path=None,
                   print_logs=False, **kw)


# ── clocks ──────────────────────────────────────────────────────────────────
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ── the reference's own CPU code (baseline/_ref) ───────────────────────────
def import_reference():
    """mbirtorch 0.0.2 from its install under baseline/_ref (None if absent)."""
    if not os.path.isdir(os.path.join(REF_DIR, "mbirtorch")):
        return None
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    import mbirtorch
    return mbirtorch


# A 20-iteration recon in subset steps: 4 + 16 + 64 + 17 x 128 steps, plus
# the direct recon, the initial error and the Hessian (about three full
# projections = 1.5 x 128 subset steps' projector work).  The larger subsets
# of the first three iterations are counted at the cost of a 128-subset step,
# which under-counts their projector work (in the reference's favour).
SUBSET_STEPS_PER_RECON = 4 + 16 + 64 + 17 * 128 + 1.5 * 128


class ReferenceStep:
    """One 128-subset VCD step of the reference's own eager CPU updater
    (create_vcd_subset_updater, tomography_model.py:2434-2660) on a
    configuration restricted to every ``view_stride``-th view, from a zero
    volume and a seeded stand-in error sinogram (a step's cost does not
    depend on the values; the state is updated in place call after call)."""

    def __init__(self, ref, torch, name, view_stride, seed=0):
        m = cone_model(ref, name, views=slice(None, None, view_stride), compile_mode='off')
        m.configure_devices(devices=['cpu'])
        m.set_params(no_warning=True, sigma_y=1.0, sigma_x=0.1)
        rs = m.get_params('recon_shape')
        self.views = int(m.get_params('sinogram_shape')[0])
        V, R, C = m.get_params('sinogram_shape')
        rng = np.random.default_rng(seed)
        self.err = m._as_shards(torch.as_tensor(rng.random((V, R, C), dtype=np.float32)),
                                m.sino_placement)
        self.flat = m._as_shards(torch.zeros(rs[0] * rs[1], rs[2]), m.recon_placement)
        H = m._as_shards(torch.ones(rs[0] * rs[1], rs[2]), m.recon_placement)
        self.upd = m.create_vcd_subset_updater(H, weights=1)
        np.random.seed(seed)
        self.idx = torch.as_tensor(ref.gen_pixel_partition(rs, 128)[0], dtype=torch.int64)
        self.pixels = int(self.idx.shape[0])

    def seconds(self):
        t = time.perf_counter()
        self.upd(self.flat, self.err, self.idx)
        return time.perf_counter() - t


class ReferenceCpu:
    """The reference's own CPU recon rate on the headline workload, from a
    bounded sample.  Each sample times one warm 128-subset step over 90 of
    the 720 views.  The ratio of a warm 720-view step to a warm 90-view step,
    measured once at the first sample (the reference's cost is not linear in
    the view count: its driver projects in view batches), scales a sample to
    the whole scan, and SUBSET_STEPS_PER_RECON to a whole recon."""

    def __init__(self, torch):
        self.torch = torch
        self.ref = import_reference()
        torch.set_num_threads(os.cpu_count())
        self.V = CONFIGS[HEAD][0]
        self.s90 = None
        self.t_full_cal = self.t90_cal = None

    def available(self):
        return self.ref is not None

    def sample(self):
        if self.s90 is None:
            full = ReferenceStep(self.ref, self.torch, HEAD, 1)
            full.seconds()                 # first call: allocator and thread-pool warm-up
            self.t_full_cal = full.seconds()
            del full
            self.s90 = ReferenceStep(self.ref, self.torch, HEAD, 8)
            self.s90.seconds()
            self.t90_cal = self.s90.seconds()
        t90 = self.s90.seconds()
        ratio = self.t_full_cal / self.t90_cal
        t_full = t90 * ratio
        per_recon = t_full * SUBSET_STEPS_PER_RECON
        return {"value": 1.0 / per_recon, "unit": "recons/s", "cores": os.cpu_count(),
                "cpu_model": cpu_model(), "kind": "reference",
                "sample": (f"mbirtorch 0.0.2's own eager CPU subset updater (torch "
                           f"{self.torch.__version__}, {self.torch.get_num_threads()} threads) "
                           f"on one warm 128-subset step of the headline workload "
                           f"({self.s90.pixels} pixels x 256 slices) over {self.s90.views} "
                           f"views ({t90:.2f} s), scaled by the measured ratio of a warm "
                           f"{self.V}-view step ({self.t_full_cal:.1f} s) to a warm "
                           f"{self.s90.views}-view step ({self.t90_cal:.2f} s) and multiplied by "
                           f"{SUBSET_STEPS_PER_RECON:.0f} subset-step equivalents per recon"),
                "seconds_per_recon_extrapolated": per_recon,
                "subset_step_seconds": t_full,
                "subset_step_seconds_full_scan_measured": self.t_full_cal}


def reference_cpu_recon_cfg1(torch):
    """The reference's own recon_simple_parallel on its CPU configuration
    (128 x 128 x 16 phantom, 180 views, 16 x 192 detector, 10 iterations),
    timed whole: no extrapolation."""
    ref = import_reference()
    if ref is None:
        return {"value": None, "error": "reference not installed under baseline/_ref"}
    torch.set_num_threads(os.cpu_count())
    shape = (180, 16, 192)
    ang = np.linspace(0, np.pi, shape[0], endpoint=False)
    mp = ref.ParallelBeamModel(shape, ang, compile_mode='off')
    mp.set_params(no_warning=True, verbose=0, recon_shape=(128, 128, 16))
    mp.configure_devices(devices=['cpu'])
    vol = phantom_torch(torch, (128, 128, 16), 61, torch.device('cpu')).numpy()
    clean = mp.forward_project(vol)
    rng = np.random.default_rng(62)
    sino = (clean + rng.normal(0, 0.01 * clean.max(), clean.shape)).astype(np.float32)
    m = ref.ParallelBeamModel(shape, ang, compile_mode='off')
    m.configure_devices(devices=['cpu'])
    m.set_params(no_warning=True, verbose=0)
    np.random.seed(63)
    t = time.perf_counter()
    m.recon(sino, max_iterations=10, stop_threshold_change_pct=0, logfile_path=None,
            print_logs=False)
    dt = time.perf_counter() - t
    return {"value": 1.0 / dt, "unit": "recons/s", "seconds": dt, "cores": os.cpu_count(),
            "threads": torch.get_num_threads(), "cpu_model": cpu_model(), "kind": "reference",
            "workload": "recon of a 128x128x16 ellipsoid phantom's parallel sinogram (180 "
                        "views, 16 x 192, 1% Gaussian noise) at the default 192x192x16 grid, "
                        "10 VCD iterations, eager torch on the CPU, timed whole",
            "sino": sino}


# ── the CPU-baseline leg: reference timing, FP64 oracle parity ─────────────
def oracle_problem(m):
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


def subset_parity(m, mb, torch, y, x, seed=1):
    """One GPU subset step from the state (x, e = y - A x) against the FP64
    oracle's step from the same state (one subset of the 128-subset
    partition).  Returns the relative errors and the oracle step's seconds.
    The caller passes a state some way from convergence, so that the update
    itself is large against the FP32 rounding of the volume."""
    import oracle
    from oracle import vcd as ovcd
    oracle.build()
    rs = m.get_params('recon_shape')
    dev = y.device
    e0 = (y - m.forward_project(x, output_sharded=True)).contiguous()
    H = m.compute_hessian_diagonal(output_sharded=True)
    upd = m.create_vcd_subset_updater(H, weights=1)
    rng = np.random.RandomState(seed)
    idx = mb.gen_pixel_partition(rs, 128, rng=rng)[rng.randint(128)].astype(np.int64)
    flat = x.reshape(-1, rs[2]).clone()
    err = e0.clone()
    flat, err, ell1, alpha, _ = upd(flat, err, torch.as_tensor(idx, device=dev))
    prob = oracle_problem(m)
    sy, sx = m.get_params(['sigma_y', 'sigma_x'])
    ou = ovcd.SubsetUpdater(prob, H.reshape(-1, rs[2]).cpu().numpy(), None, sy, sx,
                            dc_profile=ovcd.dc_damping_profile(prob))
    oflat = x.reshape(-1, rs[2]).cpu().numpy().astype(np.float64)
    oerr = e0.cpu().numpy().astype(np.float64)
    x_sub = oflat[idx].copy()
    t = time.perf_counter()
    _, oalpha, _ = ou(oflat, oerr, idx)
    dt = time.perf_counter() - t
    got = flat.cpu().numpy().astype(np.float64)

    def rel(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    return {"state": "0.9 x the timed recon", "pixels": int(idx.size),
            "alpha": float(alpha), "alpha_oracle": float(oalpha),
            "alpha_rel": abs(float(alpha) - oalpha) / abs(oalpha),
            "update_rel_l2": rel(got[idx] - x_sub, oflat[idx] - x_sub),
            "recon_rel_l2": rel(got, oflat),
            "error_sinogram_rel_l2": rel(err.cpu().numpy().astype(np.float64), oerr),
            "oracle_step_s": dt, "oracle_threads": os.cpu_count()}


def cpu_baseline_leg(m, mb, torch, y, rec):
    """The CPU-baseline leg of the headline line: the FP64 oracle (the
    reference's algorithm restated in C with OpenMP, all host threads) on one
    128-subset step of the headline workload from the state the timed recon
    ended in, extrapolated to a whole recon; the GPU step's parity against
    that oracle step; and the reference's own eager CPU code timed whole on
    its small CPU configuration.  (`bench.py --impl reference` times the
    reference's own code on the headline workload.)"""
    out = {}
    try:
        # 0.9 x the timed recon: a state with a sizeable update
        par = subset_parity(m, mb, torch, y, 0.9 * rec)
        per_recon = par["oracle_step_s"] * SUBSET_STEPS_PER_RECON
        out["cpu_baseline"] = {
            "value": 1.0 / per_recon, "unit": "recons/s", "cores": os.cpu_count(),
            "cpu_model": cpu_model(), "kind": "port",
            "sample": (f"one 128-subset VCD step of the headline workload ({par['pixels']} "
                       f"pixels x 256 slices x 720 views, {par['oracle_step_s']:.2f} s) by the "
                       f"FP64 C oracle with OpenMP, multiplied by {SUBSET_STEPS_PER_RECON:.0f} "
                       f"subset-step equivalents per recon"),
            "seconds_per_recon_extrapolated": per_recon}
        out["parity_vs_fp64_oracle"] = par
    except Exception as exc:
        out["cpu_baseline"] = {"value": None, "error": repr(exc)[:300]}
    r1 = reference_cpu_recon_cfg1(torch)
    r1.pop("sino", None)
    out["reference_cpu_recon_small"] = r1
    return out


# ── measured extras ─────────────────────────────────────────────────────────
def subset_touch(m, torch, y, n_subsets=128, samples=4):
    """Mean count of error-sinogram cells a subset step must read (N_touch):
    the cells where A has a nonzero entry for some pixel of the subset,
    counted on the device by forward-projecting ones over whole cylinders
    of `samples` subsets of the `n_subsets`-subset partition."""
    import mbirtorch_b200 as mb
    rs = m.get_params('recon_shape')
    rng = np.random.RandomState(11)
    part = mb.gen_pixel_partition(rs, n_subsets, rng=rng)
    counts = []
    for k in range(samples):
        idx = torch.as_tensor(part[k].astype(np.int64), device=y.device)
        ones = torch.ones(idx.shape[0], rs[2], device=y.device)
        s = m.projector.forward(ones, idx)
        counts.append(int((s != 0).sum()))
    return float(np.mean(counts)), int(part.shape[1])


def kernel_timing(m, torch, y, storage):
    """One recon with the library's per-launch CUDA events: {name: (ms, n)}.
    Timing mode launches each kernel the ordinary way (no programmatic
    dependent launch) so that an event pair brackets one kernel."""
    from mbirtorch_b200 import _lib
    m.set_storage_precision(storage)
    _lib.timing_collect()
    _lib.timing_enable(True)
    recon(m, y, output_sharded=True)
    torch.cuda.synchronize()
    _lib.timing_enable(False)
    return _lib.timing_collect()


def roofline_block(m, torch, y, kt, storage, hbm):
    """The dominant kernel against HBM with the survey's algorithmic bytes:
    b_e per reached error-sinogram cell for the gradient and for the forward
    with line search (one read of e; its A delta store is the design's, and
    counts only in `traffic`), 2 b_e for the tail (read and write e)."""
    b_e = 4 if storage == "float32" else 2
    n_touch, ps = subset_touch(m, torch, y)
    per = {"vcd gradient (back projection)": 1.0, "vcd forward + line search": 1.0,
           "vcd pixel + sinogram update": 2.0}
    total = sum(v[0] for v in kt.values())
    top = max((k for k in kt if k in per), key=lambda k: kt[k][0])
    tms, tcnt = kt[top]
    alg = per[top] * b_e * n_touch
    ach = alg / (tms / tcnt / 1e3) / 1e9
    V, R, C = m.get_params('sinogram_shape')
    # DRAM bytes per launch of the dominant kernel (ncu, dram__bytes_read.sum +
    # dram__bytes_write.sum) on this workload's 128-subset step, FP32 storage.
    traffic = {("vcd forward + line search", "float32"): TRAFFIC_FWD_LS_FP32}
    # The kernel is instruction-issue-bound, not HBM-bound: its warp
    # instructions per launch (ncu smsp__inst_executed.sum) over the same
    # CUDA-event launch time, against one warp instruction per cycle per SM
    # sub-partition at the maximum SM clock.
    issue = None
    winst = {("vcd forward + line search", "float32"): WARP_INST_FWD_LS_FP32}.get((top, storage))
    if winst:
        props = torch.cuda.get_device_properties(torch.cuda.current_device())
        peak_i = props.multi_processor_count * 4 * SM_MAX_MHZ * 1e6
        ach_i = winst / (tms / tcnt / 1e3)
        issue = {"warp_instructions_per_launch": winst, "achieved_warp_inst_per_s": ach_i,
                 "peak_warp_inst_per_s": peak_i, "frac": ach_i / peak_i,
                 "peak_rule": f"{props.multi_processor_count} SMs x 4 sub-partitions x "
                              f"{SM_MAX_MHZ} MHz"}
    return {"kernel": top, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
            "issue": issue,
            "frac": ach / hbm, "traffic": traffic.get((top, storage)),
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch "
                              "(profiles/), 128-subset step of this workload",
            "algorithmic_bytes_per_launch": alg,
            "algorithmic_bytes_rule": f"{per[top]:g} x {b_e} B x N_touch",
            "n_touch_cells": n_touch, "subset_pixels": ps,
            "n_touch_fraction_of_sinogram": n_touch / (V * R * C),
            "avg_launch_ms": tms / tcnt, "launches": tcnt,
            "share_of_kernel_time": tms / total,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}


# DRAM traffic of one forward + line-search launch of the headline workload's
# 128-subset step (ncu dram__bytes_read.sum 555.4 MB + dram__bytes_write.sum
# 455.4 MB, one captured launch): one read of e (439 MB), the A delta store
# (439 MB) and the records and cylinders.
TRAFFIC_FWD_LS_FP32 = 1010784512.0
# Warp instructions of the same launch (ncu smsp__inst_executed.sum), and
# the SM clock the issue peak is taken at (clocks.max.sm of this pool's B200s).
WARP_INST_FWD_LS_FP32 = 1028039755
SM_MAX_MHZ = 1965


def projector_block(m, torch, dev):
    """Full-volume forward and back projection of the model's ROR pixels."""
    S = m.get_params('recon_shape')[2]
    V = m.get_params('sinogram_shape')[0]
    idx = m.full_indices_device()
    vals = torch.rand(idx.shape[0], S, device=dev)
    for _ in range(2):
        s = m.projector.forward(vals, idx)
        m.projector.back(s, idx)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    for _ in range(3):
        s = m.projector.forward(vals, idx)
    ev[1].record()
    for _ in range(3):
        m.projector.back(s, idx)
    ev[2].record()
    torch.cuda.synchronize()
    tf = ev[0].elapsed_time(ev[1]) / 3 / 1e3
    tb = ev[1].elapsed_time(ev[2]) / 3 / 1e3
    vv = idx.shape[0] * S * V
    return {"voxel_views": int(vv), "forward_gvox_views_per_s": vv / tf / 1e9,
            "back_gvox_views_per_s": vv / tb / 1e9, "forward_ms": tf * 1e3,
            "back_ms": tb * 1e3, "pixels_ror": int(idx.shape[0])}


def precision_block(m, torch, y, ref_rec, parity_f32=None):
    """bfloat16 / float16 storage recons of the same data: recons/s (one
    untimed warm-up recon each, then one timed) and relative L2 to the FP32
    recon.  The FP32 path's own distance to the FP64 oracle is bounded per
    step by `parity_vs_fp64_oracle`; the 16-bit paths are held to the FP64
    oracle directly at smaller sizes by the tests."""
    out = {}
    ref = ref_rec.double()
    for st in ("bfloat16", "float16"):
        m.set_storage_precision(st)
        recon(m, y, output_sharded=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r2, _ = recon(m, y, output_sharded=True)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out[st] = {"recons_per_s": 1.0 / dt, "seconds": dt,
                   "rel_l2_vs_f32_recon": float((r2.double() - ref).norm() / ref.norm())}
        del r2
    m.set_storage_precision("float32")
    return out


def cone256_extra(mb, torch, dev):
    """The 256^3 flat-cone configuration (360 views, 256 x 384): recons/s at
    FP32 (three timed recons after a warm-up) and the 16-bit storages."""
    m = cone_model(mb, "cone256_flat")
    y = make_data(m, torch, dev, 0)
    recon(m, y, output_sharded=True)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    for _ in range(3):
        r, rd = recon(m, y, output_sharded=True)
    ev[1].record()
    torch.cuda.synchronize()
    s = ev[0].elapsed_time(ev[1]) / 3 / 1e3
    out = {"workload": workload("cone256_flat"), "recons_per_s": 1.0 / s, "seconds": s,
           "fm_rmse_final": rd["recon_params"]["fm_rmse"][-1]}
    out["mixed_precision"] = precision_block(m, torch, y, r)
    return out


# The HBM-bound VCD case: a parallel-beam subset step touches most of the
# sinogram for few voxel-views (512^2 x 256 volume, 720 views).
PAR_V, PAR_R, PAR_C, PAR_N = 720, 256, 768, 512


def parallel_pass_setup(mb, torch):
    """A parallel 512^2 x 256 model, 720 views, 256 x 768 detector, its VCD
    engine (FP32 storage, unweighted) on a seeded stand-in error sinogram
    (566 MB, above L2; a step's cost does not depend on the values), and one
    128-subset partition with its order."""
    from mbirtorch_b200 import _lib
    from mbirtorch_b200.vcd_engine import ResidentSinogram
    m = mb.ParallelBeamModel((PAR_V, PAR_R, PAR_C), np.linspace(0, np.pi, PAR_V, endpoint=False))
    m.set_params(no_warning=True, verbose=0, recon_shape=(PAR_N, PAR_N, PAR_R))
    dev = torch.device("cuda", 0)
    gen = torch.Generator(device=dev).manual_seed(3)
    y = torch.rand((PAR_V, PAR_R, PAR_C), generator=gen, device=dev)
    m.auto_set_regularization_params(y)
    H = m.compute_hessian_diagonal(output_sharded=True)
    upd = m.create_vcd_subset_updater(H, weights=1)
    rs = m.get_params("recon_shape")
    flat = torch.zeros(rs[0] * rs[1], rs[2], device=dev)
    err = ResidentSinogram.from_vrc(y, _lib.MBIR_F32)
    rng = np.random.RandomState(0)
    part = torch.as_tensor(mb.gen_pixel_partition(rs, 128, rng=rng), device=dev)
    order = rng.permutation(part.shape[0]).astype(np.int32)
    acc = torch.zeros(2 + rs[2], dtype=torch.float64, device=dev)
    return m, upd, flat, err, part, order, acc, y


def parallel_subset_extra(mb, torch, hbm):
    """One 128-subset partition pass of the parallel workload above: the
    pass's CUDA-event time (kernels chained as in a recon), then each
    kernel's CUDA-event average from a second, per-launch timed pass, and
    the forward + line search and the tail against the measured HBM
    bandwidth (algorithmic bytes: one e read over the reached cells, resp.
    an e read and write)."""
    from mbirtorch_b200 import _lib
    m, upd, flat, err, part, order, acc, y = parallel_pass_setup(mb, torch)
    upd.engine.partition_pass(flat, err, part, order, acc)  # warm-up
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record()
    upd.engine.partition_pass(flat, err, part, order, acc)
    ev[1].record()
    torch.cuda.synchronize()
    pass_ms = ev[0].elapsed_time(ev[1])
    _lib.timing_collect()
    _lib.timing_enable(True)
    upd.engine.partition_pass(flat, err, part, order, acc)
    torch.cuda.synchronize()
    _lib.timing_enable(False)
    kt = _lib.timing_collect()
    n_touch, ps = subset_touch(m, torch, y)
    out = {"workload": f"parallel {PAR_N}^2 x {PAR_R} volume, {PAR_V} views, {PAR_R} x {PAR_C} "
                       f"detector, FP32 storage, one 128-subset pass ({ps} pixels per subset)",
           "subset_step_us": 1e3 * pass_ms / part.shape[0], "n_touch_cells": n_touch,
           "n_touch_fraction_of_sinogram": n_touch / (PAR_V * PAR_R * PAR_C),
           "kernels_us": {k: 1e3 * v[0] / v[1] for k, v in kt.items()}}
    for name, nbytes in (("vcd forward + line search", 4 * n_touch),
                         ("vcd gradient (back projection)", 4 * n_touch),
                         ("vcd pixel + sinogram update", 2 * 4 * n_touch)):
        if name in kt:
            t = kt[name][0] / kt[name][1] / 1e3
            out[name] = {"algorithmic_bytes": nbytes, "achieved_gbs": nbytes / t / 1e9,
                         "frac_of_measured_hbm": nbytes / t / 1e9 / hbm}
    vv = ps * PAR_R * PAR_V
    t_f = kt["vcd forward + line search"][0] / kt["vcd forward + line search"][1] / 1e3
    out["forward_gvox_views_per_s"] = vv / t_f / 1e9
    return out


def autograd_extra(mb, torch, steps=3):
    """The differentiable-projector configuration: a batch of 4 volumes of
    128^3 (Gaussian-smoothed N(0, 1) fields, seeded), loss
    sum w (A x - y)^2 with y from a second seeded volume and random
    positive weights, forward + backward through weighted_residual_loss
    (sinogram formed in view chunks of at most 2 GB, A x recomputed in the
    backward), for parallel beam (256 views, 128 x 192) and cone beam (256
    views, 128 x 192, magnification 1.5).  Per step: 3 projector calls per
    volume (A x, A x again in the backward, A^T r)."""
    dev = torch.device("cuda", 0)
    gen = torch.Generator(device=dev).manual_seed(4)

    def field(n):
        x = torch.randn((n, 1, 128, 128, 128), generator=gen, device=dev)
        k = torch.exp(-0.5 * (torch.arange(-4, 5, device=dev, dtype=torch.float32) / 2.0) ** 2)
        k = k / k.sum()
        for dim in range(3):
            shape = [1, 1, 1, 1, 1]
            shape[2 + dim] = 9
            pad = [0, 0, 0, 0, 0, 0]
            pad[2 * (2 - dim)] = pad[2 * (2 - dim) + 1] = 4
            x = torch.nn.functional.conv3d(torch.nn.functional.pad(x, pad, mode="replicate"),
                                           k.view(shape))
        return x[:, 0].contiguous()

    out = {}
    for kind in ("parallel", "cone"):
        if kind == "parallel":
            m = mb.ParallelBeamModel((256, 128, 192), np.linspace(0, np.pi, 256, endpoint=False))
        else:
            m = mb.ConeBeamModel((256, 128, 192), np.linspace(0, 2 * np.pi, 256, endpoint=False),
                                 source_detector_dist=1152.0, source_iso_dist=768.0)
            m.set_params(no_warning=True, delta_det_channel=1.5, delta_det_row=1.5)
            m.auto_set_recon_geometry(no_warning=True)
        m.set_params(no_warning=True, verbose=0, recon_shape=(128, 128, 128))
        x = field(4).requires_grad_(True)
        with torch.no_grad():
            y = mb.forward_project_differentiable(m, field(4))
        w = 0.5 + torch.rand(y.shape, generator=gen, device=dev)
        for _ in range(2):
            loss = mb.weighted_residual_loss(m, x, y, w)
            loss.backward()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        for _ in range(steps):
            x.grad = None
            loss = mb.weighted_residual_loss(m, x, y, w)
            loss.backward()
        ev[1].record()
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1]) / steps
        vv = int(m.full_indices_device().shape[0]) * 128 * 256
        out[kind] = {"ms_per_step": ms, "volumes": 4,
                     "gvox_views_per_s": 3 * 4 * vv / (ms / 1e3) / 1e9,
                     "loss": float(loss.detach())}
    return out


def mix_jobs(mb, torch, n_jobs=16, seed=7):
    """A seeded sample of the serving mix, scaled to run in seconds: 40%
    parallel, 40% cone, 20% helical cone (2 turns); slices in {16, 64},
    in-plane size in {128, 256}, views in {180, 360}, channels 1.5x the
    in-plane size, rows = slices; ellipsoid phantoms with Poisson noise
    at I0 = 1e4 (largest line integral scaled to 3).  Returns
    [(model factory, sinogram, seed)]."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(n_jobs):
        kind = rng.choice(["parallel", "cone", "helical"], p=[0.4, 0.4, 0.2])
        S, N, Vj = int(rng.choice([16, 64])), int(rng.choice([128, 256])), int(rng.choice([180, 360]))
        Cj = int(1.5 * N)

        def make(kind=kind, S=S, N=N, Vj=Vj, Cj=Cj):
            if kind == "parallel":
                mj = mb.ParallelBeamModel((Vj, S, Cj), np.linspace(0, np.pi, Vj, endpoint=False))
            else:
                turns = 2 if kind == "helical" else 1
                ang = np.linspace(0, 2 * np.pi * turns, Vj, endpoint=False)
                zs = np.linspace(-S / 4, S / 4, Vj) if kind == "helical" else None
                mj = mb.ConeBeamModel((Vj, S, Cj), ang, source_detector_dist=4.0 * N,
                                      source_iso_dist=2.0 * N, helical_z_shifts=zs)
                mj.set_params(no_warning=True, delta_det_channel=2.0, delta_det_row=2.0)
                mj.auto_set_recon_geometry(no_warning=True)
            mj.set_params(no_warning=True, verbose=0, recon_shape=(N, N, S))
            return mj

        mj = make()
        rs = mj.get_params("recon_shape")
        g = np.linspace(-1, 1, N, dtype=np.float32)
        X, Y = np.meshgrid(g, g)
        z = np.linspace(-1, 1, S, dtype=np.float32)
        vol = np.zeros(rs, np.float32)
        for _ in range(6):
            c, a = rng.uniform(-0.4, 0.4, 3), rng.uniform(0.1, 0.4, 3)
            inside = ((X - c[0]) / a[0]) ** 2 + ((Y - c[1]) / a[1]) ** 2
            vol += np.float32(rng.uniform(0.2, 1.0)) * (
                (inside[:, :, None] + ((z - c[2]) / a[2]) ** 2) <= 1)
        clean = mj.forward_project(vol)
        mu = 3.0 / max(float(clean.max()), 1e-6)
        counts = rng.poisson(I0 * np.exp(-mu * clean))
        sino = (-np.log(np.maximum(counts, 1) / I0) / mu).astype(np.float32)
        jobs.append((make, sino, 1000 + j))
    return jobs


def serving_mix_extra(mb, torch, n_jobs=16):
    """The north-star comparison on a sample of the serving mix: the plain
    form (each job alone, FP32, one after another through model.recon) vs
    the served form (all jobs submitted at once to a ReconServer with
    float16 storage: resident, admitted against the memory ledger, advancing
    concurrently; recurring partition passes replayed as CUDA graphs, and
    the same with direct launches).  Both with 10 VCD iterations and the
    same per-job seeds, so each served result is compared with its own plain
    result.  Each arm is timed three times (interleaved) and the median run
    is reported, with all samples."""
    from mbirtorch_b200.serving import ReconServer
    jobs = mix_jobs(mb, torch, n_jobs)
    iters = 10

    def plain():
        out = []
        t0 = time.perf_counter()
        for make, sino, seed in jobs:
            mj = make()
            np.random.seed(seed)
            r, _ = mj.recon(sino, max_iterations=iters, stop_threshold_change_pct=0,
                            logfile_path=None, print_logs=False)
            out.append(r)
        return out, time.perf_counter() - t0

    def served(graphs=True):
        srv = ReconServer(storage_dtype="float16", max_active=8, cuda_graphs=graphs)
        t0 = time.perf_counter()
        reqs = [srv.submit(make(), sino, max_iterations=iters, seed=seed, arrival=t0)
                for make, sino, seed in jobs]
        srv.run_until_idle(timeout_s=600)
        return reqs, time.perf_counter() - t0, srv.stats()

    plain()        # warm-up (library load, allocator)
    served()
    t_plains, t_srvs, t_ngs, runs = [], [], [], []
    for _ in range(3):
        ref, tp = plain()
        reqs_ng, tn, _ = served(graphs=False)
        reqs, ts, st = served()
        t_plains.append(tp)
        t_ngs.append(tn)
        t_srvs.append(ts)
        runs.append((ts, st))
    t_plain = float(np.median(t_plains))
    t_srv_ng = float(np.median(t_ngs))
    t_srv, st = sorted(runs, key=lambda r: r[0])[1]
    same = all(np.array_equal(a.recon, b.recon) for a, b in zip(reqs, reqs_ng))
    rel = [float(np.linalg.norm(r.recon.astype(np.float64) - p) / np.linalg.norm(p))
           for r, p in zip(reqs, ref)]
    kinds = {}
    for make, _, _ in jobs:
        k = type(make()).__name__
        kinds[k] = kinds.get(k, 0) + 1
    return {"jobs": n_jobs, "iterations": iters, "models": kinds,
            "plain_f32_recons_per_s": n_jobs / t_plain,
            "served_f16_recons_per_s": n_jobs / t_srv,
            "served_over_plain": t_plain / t_srv,
            "served_f16_direct_launch_recons_per_s": n_jobs / t_srv_ng,
            "samples_recons_per_s": {"plain_f32": [n_jobs / t for t in t_plains],
                                     "served_f16": [n_jobs / t for t in t_srvs],
                                     "served_f16_direct_launch": [n_jobs / t for t in t_ngs]},
            "graph_replays": int(sum(r.graph_replays for r in reqs)),
            "graphs_bitwise_equal_direct": bool(same),
            "served_p50_latency_s": st["p50_latency_s"],
            "served_p99_latency_s": st["p99_latency_s"],
            "max_concurrent": st["max_concurrent"], "failed": st["failed"],
            "max_rel_l2_served_vs_plain_f32": max(rel)}


def serving_batching_extra(mb, torch, jobs=8, iters=10):
    """Cross-job batching on a scanner-protocol workload: `jobs` requests of
    one geometry (own phantoms, noise and seeds) submitted together, served
    with same-geometry batching (each kernel of a subset step launched once
    for all of them) and without it (each job on its own stream), float16
    storage, CUDA graphs on; medians of three interleaved runs per arm.
    Two protocols: a small parallel scan (128^2 x 16, 180 views, 16 x 192)
    and a medium cone scan (256^2 x 64, 360 views, 64 x 384 flat, pitch 2,
    magnification 2)."""
    from mbirtorch_b200.serving import ReconServer
    dev = torch.device("cuda", 0)

    def protocols():
        def par():
            m = mb.ParallelBeamModel((180, 16, 192), np.linspace(0, np.pi, 180, endpoint=False))
            m.set_params(no_warning=True, verbose=0, recon_shape=(128, 128, 16))
            return m

        def cone():
            m = mb.ConeBeamModel((360, 64, 384), np.linspace(0, 2 * np.pi, 360, endpoint=False),
                                 source_detector_dist=1024.0, source_iso_dist=512.0)
            m.set_params(no_warning=True, delta_det_channel=2.0, delta_det_row=2.0)
            m.auto_set_recon_geometry(no_warning=True)
            m.set_params(no_warning=True, verbose=0, recon_shape=(256, 256, 64))
            return m
        return {"parallel 128^2 x 16, 180 views": par, "cone 256^2 x 64, 360 views": cone}

    out = {"jobs": jobs, "iterations": iters, "storage": "float16"}
    for name, make in protocols().items():
        sinos = []
        for j in range(jobs):
            m = make()
            rs = tuple(m.get_params('recon_shape'))
            with torch.no_grad():
                vol = phantom_torch(torch, rs, 500 + j, dev)
                clean = m.forward_project(vol, output_sharded=True)
                mu = 3.0 / float(clean.max())
                gen = torch.Generator(device=dev).manual_seed(600 + j)
                counts = torch.poisson(I0 * torch.exp(-mu * clean), generator=gen)
                sinos.append((-torch.log(torch.clamp(counts, min=1.0) / I0) / mu).cpu().numpy())

        def serve(batching):
            srv = ReconServer(storage_dtype="float16", max_active=jobs, batching=batching)
            t0 = time.perf_counter()
            reqs = [srv.submit(make(), s, max_iterations=iters, seed=700 + j, arrival=t0)
                    for j, s in enumerate(sinos)]
            srv.run_until_idle(timeout_s=600)
            torch.cuda.synchronize()
            return time.perf_counter() - t0, reqs, srv.batched_iterations

        serve(True)
        serve(False)
        t_b, t_n = [], []
        for _ in range(3):
            tb, rb, nb = serve(True)
            tn, rn, _ = serve(False)
            t_b.append(tb)
            t_n.append(tn)
        same = all(np.array_equal(a.recon, b.recon) for a, b in zip(rb, rn))
        out[name] = {"batched_recons_per_s": jobs / float(np.median(t_b)),
                     "per_job_streams_recons_per_s": jobs / float(np.median(t_n)),
                     "batched_over_streams": float(np.median(t_n)) / float(np.median(t_b)),
                     "samples_s": {"batched": t_b, "per_job_streams": t_n},
                     "batched_job_iterations": nb, "results_bitwise_equal": bool(same)}
    return out


# ── serving configuration: 200 requests with Poisson arrivals ──────────────
def config5_jobs(mb, torch, n_jobs=200, rate=5.0, seed=11):
    """The serving configuration: n_jobs requests with Poisson arrivals at
    `rate` per second (seeded exponential gaps); 40% parallel, 40% cone, 20%
    helical cone (pitch 1, 2 turns of 720 views: the source rises two
    detector heights at iso over the scan, the volume centred); slices
    uniform in {16, 64, 128, 256} (= detector rows), in-plane size in {128,
    256, 512}, views in {180, 360, 720} (not helical), channels 1.5x the
    in-plane size; cone magnification 2 with a pitch-2 detector; ellipsoid
    phantoms (largest line integral 3) with Poisson counts at I0 = 1e4.
    Returns [(arrival offset s, kind, model factory, sinogram on the host,
    seed)]."""
    rng = np.random.default_rng(seed)
    dev = torch.device("cuda", 0)
    t = 0.0
    jobs = []
    for j in range(n_jobs):
        t += float(rng.exponential(1.0 / rate))
        kind = str(rng.choice(["parallel", "cone", "helical"], p=[0.4, 0.4, 0.2]))
        S = int(rng.choice([16, 64, 128, 256]))
        N = int(rng.choice([128, 256, 512]))
        Vj = 1440 if kind == "helical" else int(rng.choice([180, 360, 720]))
        Cj = int(1.5 * N)

        def make(kind=kind, S=S, N=N, Vj=Vj, Cj=Cj):
            if kind == "parallel":
                mj = mb.ParallelBeamModel((Vj, S, Cj), np.linspace(0, np.pi, Vj, endpoint=False))
            else:
                sdd, sid = 4.0 * N, 2.0 * N
                if kind == "helical":
                    # 720 views per turn; z rises by pitch x detector height at
                    # iso (S rows of 2 / magnification 2) per turn
                    ang = (2 * np.pi / 720) * np.arange(Vj)
                    z_range = 2 * 1.0 * S
                    zs = np.linspace(-0.5 * z_range, 0.5 * z_range, Vj)
                else:
                    ang, zs = np.linspace(0, 2 * np.pi, Vj, endpoint=False), None
                mj = mb.ConeBeamModel((Vj, S, Cj), ang, source_detector_dist=sdd,
                                      source_iso_dist=sid, helical_z_shifts=zs)
                mj.set_params(no_warning=True, delta_det_channel=2.0, delta_det_row=2.0)
                mj.auto_set_recon_geometry(no_warning=True)
            mj.set_params(no_warning=True, verbose=0, recon_shape=(N, N, S))
            return mj

        mj = make()
        with torch.no_grad():
            vol = phantom_torch(torch, (N, N, S), 1000 + j, dev)
            clean = mj.forward_project(vol, output_sharded=True)
            del vol
            mu = 3.0 / max(float(clean.max()), 1e-6)
            gen = torch.Generator(device=dev).manual_seed(2000 + j)
            counts = torch.poisson(I0 * torch.exp(-mu * clean), generator=gen)
            del clean
            sino = (-torch.log(torch.clamp(counts, min=1.0) / I0) / mu).cpu().numpy()
            del counts
        jobs.append((t, kind, make, sino, 3000 + j))
    return jobs


def serving_config5(mb, torch, n_jobs=200, iters=10,
                    arms=(("bfloat16", "shortest"), ("float32", "shortest"), ("bfloat16", "fifo")),
                    max_active=8):
    """The served form against sequential plain FP32 solves on the same
    requests.  Plain: each job alone through model.recon (FP32), one after
    another in arrival order; its latencies are those of a FIFO single-job
    server fed the same arrivals (start = max(arrival, previous finish),
    from the measured per-job times).  Served: the requests submitted at
    their real arrival times to a ReconServer (bfloat16 storage, admission
    against the memory ledger, up to `max_active` jobs resident), once per
    (storage precision, admission policy) arm.  Each served result is
    compared with its own plain result."""
    from mbirtorch_b200.serving import ReconServer
    t_gen = time.perf_counter()
    jobs = config5_jobs(mb, torch, n_jobs)
    t_gen = time.perf_counter() - t_gen
    torch.cuda.empty_cache()
    # warm-up of both paths on the smallest two jobs
    small = sorted(jobs, key=lambda j: j[3].size)[:2]
    for _, _, make, sino, seed in small:
        np.random.seed(seed)
        make().recon(sino, max_iterations=2, stop_threshold_change_pct=0, logfile_path=None,
                     print_logs=False)
    srv = ReconServer(storage_dtype=arms[0][0], max_active=max_active)
    for _, _, make, sino, seed in small:
        srv.submit(make(), sino, max_iterations=2, seed=seed)
    srv.run_until_idle(timeout_s=600)
    # plain FP32, sequential
    plain, durations = [], []
    for _, _, make, sino, seed in jobs:
        t0 = time.perf_counter()
        np.random.seed(seed)
        r, _ = make().recon(sino, max_iterations=iters, stop_threshold_change_pct=0,
                            logfile_path=None, print_logs=False)
        durations.append(time.perf_counter() - t0)
        plain.append(r)
    finish, lat = 0.0, []
    for (arr, _, _, _, _), d in zip(jobs, durations):
        finish = max(arr, finish) + d
        lat.append(finish - arr)
    plain_span = finish - jobs[0][0]
    torch.cuda.empty_cache()
    out = {"requests": n_jobs, "arrival_rate_per_s": 5.0, "iterations": iters,
           "max_active": max_active, "arrivals_span_s": jobs[-1][0] - jobs[0][0],
           "data_generation_s": t_gen,
           "plain_f32": {"recons_per_s": n_jobs / plain_span,
                         "busy_recons_per_s": n_jobs / sum(durations),
                         "p50_latency_s": float(np.percentile(lat, 50)),
                         "p99_latency_s": float(np.percentile(lat, 99)),
                         "span_s": plain_span}}
    kinds = {}
    for _, kind, _, _, _ in jobs:
        kinds[kind] = kinds.get(kind, 0) + 1
    out["kinds"] = kinds
    # served, at the real arrival times, once per storage precision
    for storage, admission in arms:
        srv = ReconServer(storage_dtype=storage, max_active=max_active, admission=admission)
        schedule = [(arr, dict(model=make(), sinogram=sino, max_iterations=iters, seed=seed))
                    for arr, _, make, sino, seed in jobs]
        done = srv.serve_schedule(schedule, timeout_s=3600)
        st = srv.stats()
        by_id = {r.id: r for r in done}
        rel = [float(np.linalg.norm(by_id[k].recon.astype(np.float64) - p) / np.linalg.norm(p))
               for k, p in enumerate(plain)]
        out[f"served_{storage}_{admission}"] = {
            "recons_per_s": st["recons_per_s"], "p50_latency_s": st["p50_latency_s"],
            "p99_latency_s": st["p99_latency_s"], "span_s": st["span_s"],
            "max_concurrent": st["max_concurrent"], "failed": st["failed"],
            "deferred_admissions": srv.deferred,
            "ledger_high_water_gb": srv.ledger.high_water / 1e9,
            "over_plain_recons_per_s": st["recons_per_s"] / (n_jobs / plain_span),
            "rel_l2_vs_plain_f32": {"max": max(rel), "median": float(np.median(rel))}}
        del srv, done
        torch.cuda.empty_cache()
    return out


# ── the reference's own GPU kernels on this GPU ────────────────────────────
def _time_cuda(torch, fn, reps=3):
    fn()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    for _ in range(reps):
        fn()
    ev[1].record()
    torch.cuda.synchronize()
    return ev[0].elapsed_time(ev[1]) / reps


def triton_reference_extra(mb, torch):
    """The reference's own GPU path (mbirtorch 0.0.2 from baseline/_ref: its
    Triton projector bodies selected by _view_batch_bodies after its own
    availability self-checks, its view-batch driver, its subset updater) on
    this GPU, against this package on identical device-resident inputs:
    full-volume sparse_forward_project / sparse_back_project and one VCD
    subset step of a 128-subset partition, for the 256^3 flat-cone and the
    headline curved-cone configurations, plus the parallel 512^2 x 256 /
    720-view case.  Times are CUDA-event milliseconds after a warm-up call
    (Triton compiles on first use)."""
    ref = import_reference()
    if ref is None:
        return {"unavailable": "reference not installed under baseline/_ref"}
    from mbirtorch import kernel_availability as ka
    dev = torch.device("cuda", 0)
    out = {"reference": f"mbirtorch {ref.__version__} (baseline/_ref), compile_mode='off'",
           "triton_probe": list(ka.triton_available())}
    cases = [("cone256_flat", None), ("cone512_curved", None), ("parallel512_720v", None)]
    for name, _ in cases:
        res = {}
        try:
            if name == "parallel512_720v":
                ang = np.linspace(0, np.pi, PAR_V, endpoint=False)
                rm = ref.ParallelBeamModel((PAR_V, PAR_R, PAR_C), ang, compile_mode='off')
                mm = mb.ParallelBeamModel((PAR_V, PAR_R, PAR_C), ang)
                for x in (rm, mm):
                    x.set_params(no_warning=True, verbose=0, recon_shape=(PAR_N, PAR_N, PAR_R))
            else:
                rm = cone_model(ref, name, compile_mode='off')
                mm = cone_model(mb, name)
            rm.configure_devices(devices=['cuda:0'])
            bodies = rm._view_batch_bodies()
            res["reference_bodies"] = [b.__name__ for b in bodies]
            rs = mm.get_params('recon_shape')
            V, R, C = mm.get_params('sinogram_shape')
            idx = torch.as_tensor(mb.gen_full_indices(rs).astype(np.int64), device=dev)
            gen = torch.Generator(device=dev).manual_seed(5)
            vals = torch.rand(idx.shape[0], rs[2], generator=gen, device=dev)
            sino = torch.rand((V, R, C), generator=gen, device=dev)
            vv = int(idx.shape[0]) * rs[2] * V
            for who, model in (("reference", rm), ("mbirtorch_b200", mm)):
                tf = _time_cuda(torch, lambda: model.sparse_forward_project(vals, idx))
                tb = _time_cuda(torch, lambda: model.sparse_back_project(sino, idx))
                res[who] = {"forward_ms": tf, "back_ms": tb,
                            "forward_gvox_views_per_s": vv / tf / 1e6,
                            "back_gvox_views_per_s": vv / tb / 1e6}
            f_r = rm.sparse_forward_project(vals, idx)
            f_m = mm.sparse_forward_project(vals, idx)
            b_r = rm.sparse_back_project(sino, idx)
            b_m = mm.sparse_back_project(sino, idx)
            res["forward_rel_l2_mine_vs_reference"] = float((f_m - f_r).norm() / f_r.norm())
            res["back_rel_l2_mine_vs_reference"] = float((b_m - b_r).norm() / b_r.norm())
            del f_r, f_m, b_r, b_m
            # one VCD subset step (128-subset partition) from a zero volume
            rng = np.random.RandomState(0)
            sub = torch.as_tensor(mb.gen_pixel_partition(rs, 128, rng=rng)[0].astype(np.int64),
                                  device=dev)
            H = torch.ones(rs[0] * rs[1], rs[2], device=dev)
            for x in (rm, mm):
                x.set_params(no_warning=True, sigma_y=1.0, sigma_x=0.1)
            r_upd = rm.create_vcd_subset_updater(rm._as_shards(H, rm.recon_placement), weights=1)
            r_flat = rm._as_shards(torch.zeros_like(H), rm.recon_placement)
            r_err = rm._as_shards(sino.clone(), rm.sino_placement)
            m_upd = mm.create_vcd_subset_updater(H, weights=1)
            from mbirtorch_b200 import _lib
            from mbirtorch_b200.vcd_engine import ResidentSinogram
            m_flat = torch.zeros_like(H)
            m_err = ResidentSinogram.from_vrc(sino, _lib.MBIR_F32)
            t_r = _time_cuda(torch, lambda: r_upd(r_flat, r_err, sub))
            t_m = _time_cuda(torch, lambda: m_upd.engine.subset_update(m_flat, m_err, sub))
            res["subset_step"] = {"pixels": int(sub.shape[0]), "reference_ms": t_r,
                                  "mbirtorch_b200_ms": t_m}
            res["ratio_forward"] = res["reference"]["forward_ms"] / res["mbirtorch_b200"]["forward_ms"]
            res["ratio_back"] = res["reference"]["back_ms"] / res["mbirtorch_b200"]["back_ms"]
            res["ratio_subset_step"] = t_r / t_m
            del r_err, m_err, sino, vals
        except Exception as exc:
            res["error"] = repr(exc)[:400]
        torch.cuda.empty_cache()
        out[name] = res
    return out


def reference_gpu_recon_extra(mb, torch, names=("cone256_flat", HEAD)):
    """Whole reconstructions by the reference's own GPU path (mbirtorch 0.0.2
    from baseline/_ref on this GPU: its Triton projector bodies, its eager
    torch VCD updater and loop, compile_mode='off') against this package on
    the same numpy sinogram with the same seed (so the same partitions):
    seconds per recon through each package's `recon` (host sinogram in, host
    volume out), and the relative L2 between the two volumes."""
    ref = import_reference()
    if ref is None:
        return {"unavailable": "reference not installed under baseline/_ref"}
    dev = torch.device("cuda", 0)
    out = {"reference": f"mbirtorch {ref.__version__} (baseline/_ref), compile_mode='off'"}
    for name in names:
        res = {}
        try:
            mm = cone_model(mb, name)
            rm = cone_model(ref, name, compile_mode='off')
            rm.configure_devices(devices=['cuda:0'])
            y = make_data(mm, torch, dev, 5).cpu().numpy()
            for who, model in (("mbirtorch_b200", mm), ("reference", rm)):
                recon(model, y, iters=2)  # warm-up (Triton compiles on first use)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                r, rd = recon(model, y)
                torch.cuda.synchronize()
                res[who] = {"seconds": time.perf_counter() - t0,
                            "fm_rmse_final": float(rd["recon_params"]["fm_rmse"][-1])}
                res[who + "_volume"] = np.asarray(r, dtype=np.float64)
            a, b = res.pop("mbirtorch_b200_volume"), res.pop("reference_volume")
            res["rel_l2_mine_vs_reference"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
            res["ratio"] = res["reference"]["seconds"] / res["mbirtorch_b200"]["seconds"]
            res["workload"] = workload(name)
        except Exception as exc:
            res = {"error": repr(exc)[:400]}
        torch.cuda.empty_cache()
        out[name] = res
    return out


# ── main ────────────────────────────────────────────────────────────────────
def main():
    args = parse()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return main_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    import mbirtorch_b200 as mb
    from mbirtorch_b200 import _lib
    from mbirtorch_b200.replicas import max_over_ranks, replica_rate

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    if args.profile_case:
        return profile_case(args.profile_case, mb, torch, dev, args.storage)
    if args.serving_config5:
        print(json.dumps({"serving_config5": serving_config5(mb, torch)}), flush=True)
        return
    m = cone_model(mb, HEAD)
    m.set_storage_precision(args.storage)
    y = make_data(m, torch, dev, 5)
    y_pinned = y.cpu().pin_memory()

    for _ in range(args.warmup):
        rec, rd = recon(m, y, output_sharded=True)
    barrier()
    # ── value: device-resident sinogram ──
    launches0 = _lib.launch_count()
    with Clocks(local) as clk:
        barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(args.steps):
            rec, rd = recon(m, y, output_sharded=True)
        t1.record()
        barrier()
    launches = _lib.launch_count() - launches0
    ms = max_over_ranks(t0.elapsed_time(t1), dev)
    ms_per_step = ms / args.steps
    value = replica_rate(args.steps, ms / 1e3, world)
    clocks = clk.summary()
    rec_ref = rec.detach().clone()

    # ── e2e: pinned host sinogram in, host volume out, through model.recon ──
    k_e2e = min(args.steps, 3)
    barrier()
    t0e = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(k_e2e):
        rec_np, _ = recon(m, y_pinned)
    e1.record()
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), dev)
    e2e = {"value": replica_rate(k_e2e, ms_e2e / 1e3, world), "unit": "recons/s",
           "steps": k_e2e, "h2d_bytes_per_step": int(y_pinned.numel() * 4),
           "d2h_bytes_per_step": int(rec_np.nbytes), "wall_s": time.perf_counter() - t0e}

    out = {"metric": METRIC, "value": value, "unit": "recons/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": {"float32": "f32", "bfloat16": "bf16 storage, f32 math",
                     "float16": "f16 storage, f32 math"}.get(args.storage, args.storage),
           "data": "synthetic (seeded ellipsoid phantom, Poisson noise)",
           "config": config_block(args.storage, world),
           "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
           "fm_rmse_final": rd["recon_params"]["fm_rmse"][-1]}

    if rank == 0 and not args.no_extras:
        out.update(extras(args, m, mb, torch, dev, y, rec_ref, full=world == 1))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


EXTRAS = ("roofline", "cpu_baseline", "projectors", "mixed_precision", "cone256_flat",
          "parallel_subset", "serving_mix", "serving_batching", "autograd", "triton_reference",
          "reference_gpu_recon")


def extras(args, m, mb, torch, dev, y, rec_ref, full=True):
    res = {}
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    want = set(EXTRAS) if args.only_extra is None else set(args.only_extra.split(","))

    def run(name, fn):
        if name not in want:
            return
        try:
            res[name] = fn()
        except Exception as exc:  # reported, never fatal to the headline line
            res[name] = {"error": repr(exc)[:400]}

    if "roofline" in want:
        kt = kernel_timing(m, torch, y, args.storage)
        total = sum(v[0] for v in kt.values())
        res["roofline"] = roofline_block(m, torch, y, kt, args.storage, hbm)
        res["kernel_time_share"] = {
            "mode": "timing mode: per-launch CUDA events, no programmatic dependent launch "
                    "(so kernels do not overlap their neighbours' tails, and the sum exceeds "
                    "ms_per_step)",
            "kernels": {k: {"ms": v[0], "launches": v[1], "share": v[0] / total}
                        for k, v in sorted(kt.items(), key=lambda kv: -kv[1][0])}}
    if not full:
        return res
    if "cpu_baseline" in want:
        res.update(cpu_baseline_leg(m, mb, torch, y, rec_ref))
    run("projectors", lambda: projector_block(m, torch, dev))
    run("mixed_precision", lambda: precision_block(m, torch, y, rec_ref))
    m.set_storage_precision(args.storage)
    run("cone256_flat", lambda: cone256_extra(mb, torch, dev))
    run("parallel_subset", lambda: parallel_subset_extra(mb, torch, hbm))
    run("serving_mix", lambda: serving_mix_extra(mb, torch))
    run("serving_batching", lambda: serving_batching_extra(mb, torch))
    run("autograd", lambda: autograd_extra(mb, torch))
    run("triton_reference", lambda: triton_reference_extra(mb, torch))
    run("reference_gpu_recon", lambda: reference_gpu_recon_extra(mb, torch))
    return res


def profile_case(case, mb, torch, dev, storage="float32"):
    """One pass for a profiler (no JSON line).  'recon' is one whole headline
    reconstruction; 'subset' is three VCD subset steps of its 128-subset
    partition from a zero volume; 'subset-small' the same on the 256^3
    flat-cone configuration; 'projectors' one full-volume forward and back
    projection; 'subset-parallel' one partition pass of the parallel
    512^2 x 256 workload; 'subset-cone64' one of a 64-slice serving-mix
    cone job, with per-kernel averages printed."""
    from mbirtorch_b200.vcd_engine import ResidentSinogram, storage_code
    if case == "subset-parallel":
        _, upd, flat, err, part, order, acc, _ = parallel_pass_setup(mb, torch)
        upd.engine.partition_pass(flat, err, part, order, acc)
        torch.cuda.synchronize()
        return
    if case == "subset-cone64":
        return cone64_pass(mb, torch)
    m = cone_model(mb, "cone256_flat" if case == "subset-small" else HEAD)
    m.set_storage_precision(storage)
    y = make_data(m, torch, dev, 5)
    if case == "recon":
        recon(m, y, output_sharded=True)
    elif case in ("subset", "subset-small"):
        m.auto_set_regularization_params(y)
        H = m.compute_hessian_diagonal(output_sharded=True)
        upd = m.create_vcd_subset_updater(H, weights=1)
        rs = m.get_params('recon_shape')
        flat = torch.zeros(rs[0] * rs[1], rs[2], device=dev)
        err = ResidentSinogram.from_vrc(y, storage_code(m.storage_dtype))
        rng = np.random.RandomState(0)
        parts = torch.as_tensor(mb.gen_pixel_partition(rs, 128, rng=rng), device=dev)
        for i in range(3):
            upd.engine.subset_update(flat, err, parts[i])
    else:
        idx = m.full_indices_device()
        vals = torch.rand(idx.shape[0], m.get_params('recon_shape')[2], device=dev)
        s = m.projector.forward(vals, idx)
        m.projector.back(s, idx)
    torch.cuda.synchronize()


def cone64_pass(mb, torch):
    """One 128-subset partition pass of the serving mix's largest cone jobs
    (256^2 x 64 volume, 360 views, 64 x 384 flat detector of pitch 2, SID
    512, SDD 1024; FP32 storage on a seeded stand-in error sinogram), then
    a second pass with per-launch CUDA events, whose per-kernel averages
    are printed (one line each)."""
    from mbirtorch_b200 import _lib
    from mbirtorch_b200.vcd_engine import ResidentSinogram
    dev = torch.device("cuda", 0)
    Vc, Sc, Cc, Nc = 360, 64, 384, 256
    m = mb.ConeBeamModel((Vc, Sc, Cc), np.linspace(0, 2 * np.pi, Vc, endpoint=False),
                         source_detector_dist=4.0 * Nc, source_iso_dist=2.0 * Nc)
    m.set_params(no_warning=True, delta_det_channel=2.0, delta_det_row=2.0)
    m.auto_set_recon_geometry(no_warning=True)
    m.set_params(no_warning=True, verbose=0, recon_shape=(Nc, Nc, Sc))
    y = torch.rand((Vc, Sc, Cc), generator=torch.Generator(device=dev).manual_seed(1),
                   device=dev)
    m.auto_set_regularization_params(y)
    H = m.compute_hessian_diagonal(output_sharded=True)
    upd = m.create_vcd_subset_updater(H, weights=1)
    rs = m.get_params("recon_shape")
    flat = torch.zeros(rs[0] * rs[1], rs[2], device=dev)
    err = ResidentSinogram.from_vrc(y, _lib.MBIR_F32)
    rng = np.random.RandomState(0)
    part = torch.as_tensor(mb.gen_pixel_partition(rs, 128, rng=rng), device=dev)
    order = rng.permutation(part.shape[0]).astype(np.int32)
    acc = torch.zeros(2 + rs[2], dtype=torch.float64, device=dev)
    upd.engine.partition_pass(flat, err, part, order, acc)
    torch.cuda.synchronize()
    _lib.timing_collect()
    _lib.timing_enable(True)
    upd.engine.partition_pass(flat, err, part, order, acc)
    torch.cuda.synchronize()
    _lib.timing_enable(False)
    for k, v in sorted(_lib.timing_collect().items(), key=lambda kv: -kv[1][0]):
        print(f"{k}: {1e3 * v[0] / v[1]:.1f} us x {v[1]}")


def main_reference(args, rank, world):
    """The reference's own CPU implementation on the host cores, rank 0 only:
    each step is one bounded sample (ReferenceCpu), reported as the
    extrapolated whole-recon rate on the headline workload; its
    recon_simple_parallel on its CPU configuration is timed whole beside it."""
    if rank != 0:
        return
    import torch
    rc = ReferenceCpu(torch)
    if not rc.available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "mbirtorch 0.0.2 is not installed under baseline/_ref"}),
              flush=True)
        return
    vals = []
    for i in range(args.warmup + args.steps):
        # the first sample also takes the 180-view step that fits the
        # per-view slope; every later one is a single 90-view step
        cb = rc.sample()
        if i >= args.warmup:
            vals.append(cb["value"])
    v = float(np.mean(vals))
    cb["value"] = v
    small = reference_cpu_recon_cfg1(torch)
    small.pop("sino", None)
    out = {"metric": METRIC, "value": v, "unit": "recons/s", "n_gpus": 0, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "impl": "reference",
           "data": "synthetic (seeded stand-in error sinogram; a step's cost does not depend "
                   "on the values)",
           "config": config_block("float32", world),
           "cpu_baseline": cb, "reference_cpu_recon_small": small,
           "e2e": {"value": v, "unit": "recons/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
