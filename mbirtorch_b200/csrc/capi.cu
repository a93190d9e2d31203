// C ABI of the sm_100a MBIR hot path (declared in include/mbir_b200.h).
//
// Host-side responsibilities: argument validation (before any launch),
// launch-shape selection, workspace carving and the per-subset launch chain.
// Nothing here allocates device memory.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "batch.cuh"

using namespace mbir;

namespace {

thread_local std::string g_last_error;
std::atomic<unsigned long long> g_launches{0};

// Optional per-kernel timing: when enabled, every launch is bracketed by a
// pair of CUDA events recorded on its own stream; mbir_timing_collect sums
// the elapsed times per kernel name.  Off by default (no events recorded).
struct TimedLaunch {
  const char *name;
  cudaEvent_t a, b;
};
std::atomic<int> g_timing{0};
std::mutex g_timing_mu;
std::vector<TimedLaunch> g_timed;
thread_local cudaEvent_t t_pending = nullptr;
thread_local cudaStream_t t_stream = nullptr;

struct BatchRecorder;
thread_local BatchRecorder *t_batch = nullptr;  // see launchb

void tpre(cudaStream_t st) {
  t_stream = st;
  if (!g_timing.load(std::memory_order_relaxed) || t_batch) return;
  cudaEventCreate(&t_pending);
  cudaEventRecord(t_pending, st);
}

void tpost(const char *name) {
  if (!t_pending) return;
  cudaEvent_t b;
  cudaEventCreate(&b);
  cudaEventRecord(b, t_stream);
  std::lock_guard<std::mutex> lk(g_timing_mu);
  g_timed.push_back({name, t_pending, b});
  t_pending = nullptr;
}

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define MBIR_CHECK_LAUNCH(what)                                                     \
  do {                                                                              \
    if (!t_batch) g_launches.fetch_add(1, std::memory_order_relaxed);               \
    tpost(what);                                                                    \
    cudaError_t _e = cudaGetLastError();                                            \
    if (_e != cudaSuccess)                                                          \
      return fail(MBIR_ERR_CUDA, "%s: launch failed: %s", what, cudaGetErrorString(_e)); \
  } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Attributes of the current device, cached per device.  Launch shapes and
// workspace sizes follow the SM count; shared-memory requests are checked
// against the opt-in limit before a launch.  Without a device to query (a
// workspace-size query on a host without a GPU) the B200 values stand in.
constexpr int kMaxDevices = 64;
struct DevAttrs {
  int sms = 148;
  int smem_optin = 227 * 1024;
};
std::atomic<int> g_attr_sms[kMaxDevices];
std::atomic<int> g_attr_smem[kMaxDevices];

DevAttrs device_attrs() {
  DevAttrs a;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return a;
  }
  int sms = g_attr_sms[dev].load(std::memory_order_relaxed);
  int smem = g_attr_smem[dev].load(std::memory_order_relaxed);
  if (sms <= 0 || smem <= 0) {
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
            cudaSuccess ||
        sms <= 0 || smem <= 0) {
      cudaGetLastError();
      return a;
    }
    g_attr_sms[dev].store(sms, std::memory_order_relaxed);
    g_attr_smem[dev].store(smem, std::memory_order_relaxed);
  }
  a.sms = sms;
  a.smem_optin = smem;
  return a;
}

inline int device_sms() { return device_attrs().sms; }

// Opt a kernel into `smem` bytes of dynamic shared memory (above the 48 KB
// default), refusing requests beyond the device's per-block limit.
template <typename K>
int request_smem(K *k, size_t smem, const char *what) {
  if (smem <= 48 * 1024) return MBIR_OK;
  const int limit = device_attrs().smem_optin;
  if (smem > (size_t)limit)
    return fail(MBIR_ERR_INVALID, "%s: needs %zu bytes of shared memory per block, above the "
                "device's %d", what, smem, limit);
  const cudaError_t e =
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess)
    return fail(MBIR_ERR_CUDA, "%s: shared memory request of %zu bytes refused: %s", what, smem,
                cudaGetErrorString(e));
  return MBIR_OK;
}

// Programmatic dependent launch inside a VCD step or denoise pass: while a
// PdlScope is open on this thread, launch() lets each kernel begin as the
// stream's previous kernel winds down (the kernels open with
// MBIR_PDL_ENTRY, which waits for that kernel's writes).  Per-launch timing
// keeps ordinary launches so that each event pair brackets one kernel.
thread_local bool t_pdl = false;
struct PdlScope {
  bool prev;
  PdlScope() : prev(t_pdl) { t_pdl = true; }
  ~PdlScope() { t_pdl = prev; }
};

// Launch errors surface through cudaGetLastError (MBIR_CHECK_LAUNCH).
template <typename... KArgs, typename... Args>
void launch(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
            Args... args) {
  if (!t_pdl || g_timing.load(std::memory_order_relaxed)) {
    k<<<grid, block, smem, st>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  (void)cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}

// ── cross-job batching (batch.cuh) ─────────────────────────────────────────
// While a BatchRecorder is installed on this thread, launchb<B>(...) records
// the launch's arguments for the recorder's current job instead of
// launching; BatchRecorder::replay then issues each recorded launch once,
// for every job, as batched_kernel<B, ...> with the job on grid z.
struct BatchRecorder {
  struct Launch {
    int (*replay)(const Launch &, int jobs, cudaStream_t);
    dim3 grid, block;
    size_t smem;
    const char *what;
    size_t blob;                 // bytes of one job's argument pack
    std::vector<char> args;      // the jobs' packs, one after another
  };
  std::vector<Launch> launches;
  int job = 0;
  size_t cursor = 0;
  bool mismatch = false;

  void begin_job(int j) {
    job = j;
    cursor = 0;
  }
  void record(int (*replay)(const Launch &, int, cudaStream_t), dim3 grid, dim3 block,
              size_t smem, const char *what, const void *pack, size_t bytes) {
    if (job == 0) {
      Launch l{replay, grid, block, smem, what, bytes, {}};
      l.args.resize(bytes * kMaxBatch);
      launches.push_back(std::move(l));
    }
    if (cursor >= launches.size()) {
      mismatch = true;
      return;
    }
    Launch &l = launches[cursor++];
    if (l.replay != replay || l.blob != bytes || l.smem != smem || l.grid.x != grid.x ||
        l.grid.y != grid.y || l.block.x != block.x || l.block.y != block.y) {
      mismatch = true;
      return;
    }
    memcpy(l.args.data() + (size_t)job * bytes, pack, bytes);
  }
};
template <typename B, typename... K>
int replay_batched(const BatchRecorder::Launch &l, int jobs, cudaStream_t st);

template <typename B, typename... KArgs, typename... Args>
void launchb_k(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
               const char *what, Args... args) {
  if (!t_batch) {
    launch(k, grid, block, smem, st, args...);
    return;
  }
  const ArgPack<KArgs...> pack = make_pack(static_cast<KArgs>(args)...);
  t_batch->record(&replay_batched<B, KArgs...>, grid, block, smem, what, &pack, sizeof(pack));
}

// A launch of the subset step's kernel B (batch.cuh) that a BatchRecorder
// can take over.
template <typename B, typename... Args>
void launchb(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const char *what,
             Args... args) {
  launchb_k<B>(B::kernel(), grid, block, smem, st, what, args...);
}

template <typename B, typename... K>
int replay_batched(const BatchRecorder::Launch &l, int jobs, cudaStream_t st) {
  BatchTable<K...> t;
  for (int j = 0; j < jobs; ++j) memcpy(&t.job[j], l.args.data() + (size_t)j * l.blob, l.blob);
  auto k = batched_kernel<B, K...>;
  {
    const int rc_smem = request_smem(k, l.smem, l.what);
    if (rc_smem) return rc_smem;
  }
  dim3 grid = l.grid;
  grid.z = (unsigned)jobs;
  tpre(st);
  launch(k, grid, l.block, l.smem, st, t);
  MBIR_CHECK_LAUNCH(l.what);
  return MBIR_OK;
}

inline int next_pow2(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

inline size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

// Sequential carving of a workspace buffer.
struct Carver {
  char *base;
  size_t used = 0;
  explicit Carver(void *b) : base(static_cast<char *>(b)) {}
  template <typename T> T *take(size_t count) {
    T *p = reinterpret_cast<T *>(base ? base + used : nullptr);
    used += align_up(count * sizeof(T));
    return p;
  }
};

// Views index grid y (forward projections) and grid z (layout changes).
constexpr int kMaxViews = 65535;

int validate_geometry(const mbir_geometry *g) {
  if (!g) return fail(MBIR_ERR_INVALID, "geometry is NULL");
  if (g->geometry != MBIR_PARALLEL && g->geometry != MBIR_CONE)
    return fail(MBIR_ERR_INVALID, "geometry must be MBIR_PARALLEL or MBIR_CONE, got %d", g->geometry);
  if (g->num_views <= 0 || g->num_det_rows <= 0 || g->num_det_channels <= 0 ||
      g->num_recon_rows <= 0 || g->num_recon_cols <= 0 || g->num_slices <= 0)
    return fail(MBIR_ERR_INVALID, "geometry sizes must be positive");
  if (g->num_views > kMaxViews)
    return fail(MBIR_ERR_INVALID, "at most %d views per geometry (got %d): split the scan into "
                "several geometries of consecutive views", kMaxViews, g->num_views);
  if ((long long)g->num_recon_rows * g->num_recon_cols >= (1LL << 31))
    return fail(MBIR_ERR_INVALID, "recon grid too large for 32-bit pixel indices");
  if (g->psf_radius < 0 || g->psf_radius > MBIR_MAX_TAP_RADIUS || g->bp_psf_radius < 0 ||
      g->bp_psf_radius > MBIR_MAX_TAP_RADIUS)
    return fail(MBIR_ERR_INVALID,
                "tap radii must lie in [0, %d] (psf %d, bp %d): the kernels unroll at most "
                "%d taps a side, where the reference's torch bodies take any radius.  A psf "
                "radius ceil(ceil(voxel pitch x magnification / detector pitch) / 2) above %d "
                "means voxels wider than %d detector cells; use finer voxels or a coarser "
                "detector binning", MBIR_MAX_TAP_RADIUS, g->psf_radius, g->bp_psf_radius,
                MBIR_MAX_TAP_RADIUS, MBIR_MAX_TAP_RADIUS, 2 * MBIR_MAX_TAP_RADIUS);
  if (!(g->delta_det_channel > 0.f) || !(g->delta_voxel > 0.f) || !(g->delta_voxel_row > 0.f))
    return fail(MBIR_ERR_INVALID, "detector and voxel pitches must be positive");
  if (g->geometry == MBIR_PARALLEL && g->num_det_rows != g->num_slices)
    return fail(MBIR_ERR_INVALID, "parallel beam needs num_det_rows == num_slices (%d vs %d)",
                g->num_det_rows, g->num_slices);
  if (g->geometry == MBIR_CONE) {
    if (!(g->delta_det_row > 0.f) || !(g->delta_voxel_slice > 0.f) || !(g->magnification > 0.f))
      return fail(MBIR_ERR_INVALID, "cone pitches and magnification must be positive");
    if (!(g->source_detector_dist > 0.f))
      return fail(MBIR_ERR_INVALID, "source_detector_dist must be positive");
    if (g->num_det_rows > 4096)
      return fail(MBIR_ERR_INVALID, "cone beam supports at most 4096 detector rows");
  }
  return MBIR_OK;
}

// ── back projection launch shape ───────────────────────────────────────────
struct BackShape {
  int T, SPL, slice_chunks, blocks_x, nchunks, vpc;
  size_t smem;
};

// l2_views: also split the views so that one chunk's FP32 sinogram slab
// stays within about 32 MB of L2.  CTAs are dispatched chunk by chunk, so
// the warps in flight then share a window of views, and the cells that
// several subset pixels read come from L2 instead of being re-read from
// HBM (a VCD subset reads each reached cell once per pixel whose taps
// reach it).
BackShape back_shape(const mbir_geometry *g, int view_count, long long P, int band,
                     size_t partial_budget_bytes, bool l2_views = false) {
  BackShape s;
  if (g->geometry == MBIR_CONE) {
    s.T = 32;
    s.SPL = band <= 32 ? 1 : (band <= 64 ? 2 : (band <= 128 ? 4 : 8));
    s.smem = (size_t)(kThreads / 32) * (g->num_det_rows + 2 * kPad) * sizeof(float) +
             (size_t)(kThreads / 32) * 32 * sizeof(ConeRec);
  } else {
    if (band <= 8) { s.T = 8; s.SPL = 1; }
    else if (band <= 16) { s.T = 4; s.SPL = 4; }
    else if (band <= 32) { s.T = 8; s.SPL = 4; }
    else if (band <= 64) { s.T = 16; s.SPL = 4; }
    else { s.T = 32; s.SPL = 4; }
    s.smem = 0;
  }
  s.slice_chunks = (band + s.T * s.SPL - 1) / (s.T * s.SPL);
  const long long teams = P * s.slice_chunks;
  const int teams_per_block = kThreads / s.T;
  s.blocks_x = (int)((teams + teams_per_block - 1) / teams_per_block);
  // Enough warps for ~2 full waves of the device's SMs; split views otherwise.
  const long long warps = (teams * s.T + 31) / 32;
  const long long target = (long long)device_sms() * 64;
  long long nch = warps >= target ? 1 : (target + warps - 1) / warps;
  nch = std::min<long long>(nch, std::max(1, view_count / 4));
  if (l2_views) {
    const size_t slab = (size_t)g->num_det_rows * g->num_det_channels * sizeof(float);
    const long long vpc_l2 = std::max<long long>(4, (long long)(((size_t)32 << 20) / slab));
    nch = std::max<long long>(nch, (view_count + vpc_l2 - 1) / vpc_l2);
  }
  nch = std::min<long long>(nch, 64);
  const size_t per_chunk = (size_t)P * band * sizeof(float);
  if (nch > 1 && per_chunk > 0) {
    long long fit = (long long)(partial_budget_bytes / per_chunk);
    if (fit < nch) nch = std::max(1LL, fit);
  }
  s.nchunks = (int)std::max(1LL, nch);
  s.vpc = (view_count + s.nchunks - 1) / s.nchunks;
  s.nchunks = (view_count + s.vpc - 1) / s.vpc;
  return s;
}

size_t back_partial_bytes(const BackShape &s, long long P, int band) {
  return s.nchunks > 1 ? align_up((size_t)s.nchunks * P * band * sizeof(float)) : 0;
}

// Rows per lane of the cone back projector's column batches for bands of
// more than 64 slices: 6 where 192-row batches cover a column of the
// detector's R rows in fewer row slots than 256-row ones (R in 257..384, for
// instance), else 8.  Measured: a 320-row detector's VCD gradient 677 ->
// 642 us per step with 6; a 256-row detector's 97.8 us with 8 against 103.5
// with 6.  Every h row is summed the same way at either depth.
int back_long_batch(int R) {
  const long long s6 = 192LL * ((R + 191) / 192), s8 = 256LL * ((R + 255) / 256);
  return s6 < s8 ? 6 : 8;
}

template <int CP, int SPL, int NT, typename RD, int HBL = 8>
int launch_back_t(const Geo &geo, const mbir_geometry *g, const float *vp, int v_start,
                  int v_count, const BackShape &s, const RD &rd, const int64_t *pix, long long P,
                  int slice_start, int band, float *dst, cudaStream_t st, const char *what,
                  const ConeFwdRec *recs) {
  dim3 grid(s.blocks_x, s.nchunks);
  if (g->geometry == MBIR_CONE) {
    auto k = back_cone_kernel<CP, SPL, NT, RD, HBL>;
    const int rc = request_smem(k, s.smem, what);
    if (rc) return rc;
    tpre(st);
    launchb<BackConeB<CP, SPL, NT, RD, HBL>>(grid, kThreads, s.smem, st, what, geo, vp, v_start,
                                             v_count, s.vpc, rd, pix, (int)P, slice_start, band,
                                             s.slice_chunks, dst, recs);
  } else if (NT == 3 && SPL == 4 && band % 4 == 0 && rd.aligned16() && is_aligned16(dst)) {
    // four consecutive slices per lane: the same teams, one 16-byte load per tap
    tpre(st);
#define MBIR_BACK4(TV)                                                                       \
  launchb<BackParallel4B<CP, TV, RD>>(grid, kThreads, 0, st, what, geo, vp, v_start, v_count, \
                                      s.vpc, rd, pix, (int)P, band, s.slice_chunks, dst)
    if (s.T == 32) MBIR_BACK4(32);
    else if (s.T == 16) MBIR_BACK4(16);
    else if (s.T == 8) MBIR_BACK4(8);
    else MBIR_BACK4(4);
#undef MBIR_BACK4
  } else {
    tpre(st);
    launchb<BackParallelB<CP, SPL, NT, RD>>(grid, kThreads, 0, st, what, geo, vp, v_start,
                                            v_count, s.vpc, rd, pix, (int)P, band, s.T,
                                            s.slice_chunks, dst);
  }
  MBIR_CHECK_LAUNCH(what);
  return MBIR_OK;
}

template <int CP, int NT, typename RD>
int launch_back_spl(const Geo &geo, const mbir_geometry *g, const float *vp, int v_start,
                    int v_count, const BackShape &s, const RD &rd, const int64_t *pix,
                    long long P, int slice_start, int band, float *dst, cudaStream_t st,
                    const char *what, const ConeFwdRec *recs) {
#define MBIR_BACK(SPLV) \
  launch_back_t<CP, SPLV, NT>(geo, g, vp, v_start, v_count, s, rd, pix, P, slice_start, band, dst, st, what, recs)
  if (g->geometry == MBIR_CONE) {
    switch (s.SPL) {
      case 1: return MBIR_BACK(1);
      case 2: return MBIR_BACK(2);
      case 4: return MBIR_BACK(4);
      default:
        if constexpr (NT == 3) {
          if (back_long_batch(g->num_det_rows) == 6)
            return launch_back_t<CP, 8, NT, RD, 6>(geo, g, vp, v_start, v_count, s, rd, pix, P,
                                                   slice_start, band, dst, st, what, recs);
        }
        return MBIR_BACK(8);
    }
  }
  return s.SPL == 1 ? MBIR_BACK(1) : MBIR_BACK(4);
#undef MBIR_BACK
}

template <int CP, typename RD>
int launch_back_nt(const Geo &geo, const mbir_geometry *g, const float *vp, int v_start,
                   int v_count, const BackShape &s, const RD &rd, const int64_t *pix,
                   long long P, int slice_start, int band, float *dst, cudaStream_t st,
                   const char *what, const ConeFwdRec *recs) {
  if (g->psf_radius == 1)
    return launch_back_spl<CP, 3>(geo, g, vp, v_start, v_count, s, rd, pix, P, slice_start, band, dst, st, what, recs);
  return launch_back_spl<CP, 0>(geo, g, vp, v_start, v_count, s, rd, pix, P, slice_start, band, dst, st, what, nullptr);
}

// Back projection with a given reader into `out` (or chunk partials in
// `partials` followed by the fixed-order reduction).  `recs` (cone, psf
// radius 1, coefficient power 1 only): the subset's per-(view, slot)
// records from cone_bin_kernel for views [v_start, v_start + v_count),
// loaded instead of re-formed.
template <typename RD>
int run_back(const mbir_geometry *g, const float *vp, int v_start, int v_count, const RD &rd,
             const int64_t *pix, long long P, int cp, int slice_start, int band, float *out,
             const BackShape &s, float *partials, cudaStream_t st, bool reduce_into_out,
             const char *what = "back projection", const ConeFwdRec *recs = nullptr) {
  const Geo geo = make_geo(*g);
  float *dst = s.nchunks > 1 ? partials : out;
  int rc = cp == 2 ? launch_back_nt<2>(geo, g, vp, v_start, v_count, s, rd, pix, P, slice_start, band, dst, st, what, nullptr)
                   : launch_back_nt<1>(geo, g, vp, v_start, v_count, s, rd, pix, P, slice_start, band, dst, st, what, recs);
  if (rc) return rc;
  if (s.nchunks > 1 && reduce_into_out) {
    const size_t n = (size_t)P * band;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)device_sms() * 16);
    tpre(st);
    launch(reduce_chunks_kernel, blocks, 256, 0, st, (const float *)partials, s.nchunks, n, out);
    MBIR_CHECK_LAUNCH("chunk reduction");
  }
  return MBIR_OK;
}

// ── forward projection launch shape ────────────────────────────────────────
FwdShape fwd_shape(const mbir_geometry *g, int band) {
  FwdShape fs;
  fs.rows = g->geometry == MBIR_CONE ? g->num_det_rows : band;
  fs.TG = std::min(kThreads, next_pow2(std::max(fs.rows, 1)));
  fs.RPT = (fs.rows + fs.TG - 1) / fs.TG;
  const int G = kThreads / fs.TG;
  const int RS = fs.TG * fs.RPT + 1;
  int cb = (int)(32 * 1024 / (sizeof(float) * (size_t)G * RS));
  cb = std::max(8, std::min(cb, 128));
  fs.CB = std::min(cb, g->num_det_channels);
  return fs;
}

template <bool CONE, int NT, typename EPI>
int launch_forward(const mbir_geometry *g, const float *vp, int v_start, int v_count,
                   const float *values, long long P, int band, int slice_start, const int64_t *pix,
                   const FwdShape &fs, const EPI &epi, cudaStream_t st, const char *what,
                   int by_pixel) {
  const Geo geo = make_geo(*g);
  const size_t smem = fs.smem_bytes();
  auto k = forward_kernel<CONE, NT, EPI>;
  {
    const int rc_smem = request_smem(k, smem, "forward");
    if (rc_smem) return rc_smem;
  }
  dim3 grid((g->num_det_channels + fs.CB - 1) / fs.CB, v_count);
  tpre(st);
  launch(k, grid, kThreads, smem, st, geo, vp, v_start, values, (int)P, band, slice_start, pix, fs,
         by_pixel, epi);
  MBIR_CHECK_LAUNCH(what);
  return MBIR_OK;
}

// The register-tiled cone forward covers psf radius 1 and up to 1024
// detector rows (one thread per row); other shapes use forward_kernel.
bool use_cone_rt(const mbir_geometry *g) {
  return g->geometry == MBIR_CONE && g->psf_radius == 1 && g->bp_psf_radius <= 3 &&
         g->num_det_rows <= 1024;
}

int cone_rt_threads(const mbir_geometry *g) { return (g->num_det_rows + 31) / 32 * 32; }

size_t cone_rt_smem(const mbir_geometry *g, int band) {
  const int nthr = cone_rt_threads(g);
  return sizeof(ConeFwdRec) * (size_t)fwd_cap(nthr) +
         sizeof(float) * ((size_t)kFwdEB * (band + 2 * kFwdVPad) + (size_t)(kFwdCB + 4) * nthr);
}

// The binned cone forward with asynchronous staging in batches of eb
// pixels: two stage buffers and smaller record rounds.
size_t cone_binned_async_smem(const mbir_geometry *g, int band, int eb) {
  const int nthr = cone_rt_threads(g);
  return sizeof(ConeFwdRec) * (size_t)fwd_cap_async(nthr) +
         sizeof(float) * ((size_t)2 * eb * (band + 2 * kFwdVPad) + (size_t)(kFwdCB + 4) * nthr);
}

template <typename EPI>
int launch_cone_rt(const mbir_geometry *g, const float *vp, int v_start, int v_count,
                   const float *values, long long P, int band, int slice_start,
                   const int64_t *pix, const EPI &epi, cudaStream_t st, const char *what,
                   int by_pixel) {
  const Geo geo = make_geo(*g);
  const size_t smem = cone_rt_smem(g, band);
  auto k = forward_cone_rt_kernel<EPI>;
  {
    const int rc_smem = request_smem(k, smem, "forward");
    if (rc_smem) return rc_smem;
  }
  dim3 grid((g->num_det_channels + kFwdCB - 1) / kFwdCB, v_count);
  tpre(st);
  launch(k, grid, cone_rt_threads(g), smem, st, geo, vp, v_start, values, (int)P, band,
         slice_start, pix, by_pixel, epi);
  MBIR_CHECK_LAUNCH(what);
  return MBIR_OK;
}

// ── binned cone forward (a subset projected by several launches) ───────────
constexpr size_t kBinBytes = (size_t)128 << 20;  // record + list bytes per view chunk

int fwd_nblk(const mbir_geometry *g) { return (g->num_det_channels + kFwdCB - 1) / kFwdCB; }

// Views per binning chunk for a subset of P pixels.
int bin_views(const mbir_geometry *g, long long P) {
  const size_t per_view = (size_t)P * (sizeof(ConeFwdRec) + sizeof(int)) +
                          (size_t)(fwd_nkeys(g->num_det_channels) + 1) * sizeof(int);
  return (int)std::max<size_t>(1, std::min<size_t>(g->num_views, kBinBytes / per_view));
}

struct FwdBins {
  ConeFwdRec *recs;
  int *list, *offs;
  unsigned char *touched;  // (V, nblk): the tile received a pixel (all views)
  int views;               // views per chunk
};

size_t bin_smem(const mbir_geometry *g, int nthr = kThreads) {
  return sizeof(int) * (size_t)fwd_nkeys(g->num_det_channels) * (1 + nthr / 32);
}

// The binned forward where the row-tiled one applies and the binning's
// per-key counters fit in shared memory (up to about 5,700 channels); wider
// detectors project each subset with the scanning forward.
bool use_cone_binned(const mbir_geometry *g) {
  return use_cone_rt(g) && bin_smem(g) <= (size_t)200 * 1024;
}

// Parallel beam at psf radius 1 with up to 1024 detector rows (one thread
// per row) projects a VCD subset through the same bins.
bool use_par_binned(const mbir_geometry *g) {
  return g->geometry != MBIR_CONE && g->psf_radius == 1 && g->num_det_rows <= 1024 &&
         bin_smem(g) <= (size_t)200 * 1024;
}

bool use_binned(const mbir_geometry *g) { return use_cone_binned(g) || use_par_binned(g); }

// by_pixel: the records name the cylinder's row of `values` as pix[p] (a
// flat volume) instead of the subset slot p.  wide: whole-volume bins, with
// kBinWideThreads threads per view where their counters fit shared memory;
// subsets of at least kBinWidePixels pixels take them too, outside a batch
// recording (the batched binning runs the 256-thread body).
constexpr long long kBinWidePixels = 16384;

int launch_bin(const mbir_geometry *g, const float *vp, int v_start, int v_count,
               const int64_t *pix, long long P, const FwdBins &b, cudaStream_t st,
               int by_pixel = 0, bool wide = false) {
  const Geo geo = make_geo(*g);
  const char *what = wide ? "forward binning" : "vcd forward binning";
  wide = wide || (P >= kBinWidePixels && t_batch == nullptr);
  if (wide && bin_smem(g, kBinWideThreads) <= (size_t)device_attrs().smem_optin) {
    const size_t smem_w = bin_smem(g, kBinWideThreads);
    const int rc_smem = request_smem(cone_bin_wide_kernel, smem_w, what);
    if (rc_smem) return rc_smem;
    tpre(st);
    launch(cone_bin_wide_kernel, v_count, kBinWideThreads, smem_w, st, geo, vp, v_start, pix,
           (int)P, by_pixel, b.recs, b.list, b.offs);
    MBIR_CHECK_LAUNCH(what);
    return MBIR_OK;
  }
  const size_t smem = bin_smem(g);
  {
    const int rc_smem = request_smem(cone_bin_kernel, smem, "forward binning");
    if (rc_smem) return rc_smem;
  }
  tpre(st);
  launchb<ConeBinB>(v_count, kThreads, smem, st, what, geo, vp, v_start, pix,
                    (int)P, by_pixel, b.recs, b.list, b.offs);
  MBIR_CHECK_LAUNCH(what);
  return MBIR_OK;
}

// Launch of the binned cone forward with staging variant AEB (see
// forward_cone_binned_kernel_body).
template <typename EPI, int AEB>
int launch_binned_as(const Geo &geo, const dim3 &grid, int nthr, size_t smem, int v_start,
                     const float *values, long long P, int band, const FwdBins &b,
                     const EPI &epi, cudaStream_t st, const char *what) {
  const int rc_smem = request_smem(forward_cone_binned_kernel<EPI, AEB>, smem, "forward");
  if (rc_smem) return rc_smem;
  tpre(st);
  launchb<FwdConeBinnedB<EPI, AEB>>(grid, nthr, smem, st, what, geo, v_start, values, (int)P,
                                    band, 0, (const ConeFwdRec *)b.recs, (const int *)b.list,
                                    (const int *)b.offs, b.touched, epi);
  MBIR_CHECK_LAUNCH(what);
  return MBIR_OK;
}

// CTAs per SM of a variant (0 when the query fails or it does not fit).
template <typename EPI, int AEB>
int binned_occupancy(int nthr, size_t smem) {
  if (smem > (size_t)device_attrs().smem_optin) return 0;
  if (request_smem(forward_cone_binned_kernel<EPI, AEB>, smem, "forward")) return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, forward_cone_binned_kernel<EPI, AEB>,
                                                    nthr, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

template <typename EPI>
int launch_binned(const mbir_geometry *g, int v_start, int v_count, const float *values,
                  long long P, int band, const FwdBins &b, const EPI &epi, cudaStream_t st,
                  const char *what) {
  const Geo geo = make_geo(*g);
  const dim3 grid = EPI::kViewFastest ? dim3(v_count, fwd_nblk(g)) : dim3(fwd_nblk(g), v_count);
  const int nthr = cone_rt_threads(g);
  const size_t smem_s = cone_rt_smem(g, band);
  const size_t smem_16 = cone_binned_async_smem(g, band, kFwdEB);
  const size_t smem_8 = cone_binned_async_smem(g, band, kFwdEB / 2);
  // Asynchronous staging copies 16-byte chunks: whole cylinders of a
  // multiple of 4 slices from a 16-byte aligned array.  Its second stage
  // buffer can cost a CTA per SM (the 256-row detector of the 256^3 cone
  // workload runs 4 CTAs per SM synchronously, 3 with two 16-pixel
  // buffers), so it is taken in 16-pixel batches where that keeps the
  // synchronous staging's CTAs per SM, else in 8-pixel batches where those
  // keep them, else not.  The choice for the last (device, threads, band)
  // is kept per thread and epilogue.
  int variant = 0;
  if (band >= 4 && band % 4 == 0 && (reinterpret_cast<uintptr_t>(values) & 15) == 0) {
    static thread_local int last_dev = -1, last_nthr = -1, last_band = -1, last_variant = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != last_dev || nthr != last_nthr || band != last_band) {
      const int n_s = binned_occupancy<EPI, 0>(nthr, smem_s);
      const int n_16 = binned_occupancy<EPI, kFwdEB>(nthr, smem_16);
      const int n_8 = binned_occupancy<EPI, kFwdEB / 2>(nthr, smem_8);
      last_variant = (n_16 > 0 && n_16 >= n_s) ? kFwdEB : (n_8 > 0 && n_8 >= n_s) ? kFwdEB / 2 : 0;
      last_dev = dev;
      last_nthr = nthr;
      last_band = band;
    }
    variant = last_variant;
  }
  if (variant == kFwdEB)
    return launch_binned_as<EPI, kFwdEB>(geo, grid, nthr, smem_16, v_start, values, P, band, b,
                                         epi, st, what);
  if (variant == kFwdEB / 2)
    return launch_binned_as<EPI, kFwdEB / 2>(geo, grid, nthr, smem_8, v_start, values, P, band,
                                             b, epi, st, what);
  return launch_binned_as<EPI, 0>(geo, grid, nthr, smem_s, v_start, values, P, band, b, epi, st,
                                  what);
}

template <typename EPI>
int launch_par_binned(const mbir_geometry *g, int v_start, int v_count, const float *values,
                      long long P, int band, const FwdBins &b, const EPI &epi, cudaStream_t st,
                      const char *what) {
  if (band != g->num_det_rows)
    return fail(MBIR_ERR_INVALID, "%s: the binned parallel forward projects whole cylinders "
                "(band %d, detector rows %d)", what, band, g->num_det_rows);
  const Geo geo = make_geo(*g);
  if (band % 4 == 0 && band >= 128 && (reinterpret_cast<uintptr_t>(values) & 15) == 0) {
    // four rows per thread (one 16-byte load of a cylinder's four rows)
    const int nthr4 = (band / 4 + 31) / 32 * 32;
    const size_t smem4 = par_binned4_smem(nthr4);
    auto k4 = forward_parallel_binned4_kernel<EPI>;
    {
      const int rc_smem = request_smem(k4, smem4, "forward");
      if (rc_smem) return rc_smem;
    }
    const dim3 grid =
        EPI::kViewFastest ? dim3(v_count, fwd_nblk(g)) : dim3(fwd_nblk(g), v_count);
    tpre(st);
    launchb<FwdParBinned4B<EPI>>(grid, nthr4, smem4, st, what, geo, v_start, values, (int)P,
                                 band, (const ConeFwdRec *)b.recs, (const int *)b.list,
                                 (const int *)b.offs, b.touched, epi);
    MBIR_CHECK_LAUNCH(what);
    return MBIR_OK;
  }
  const int nthr = cone_rt_threads(g);
  const size_t smem = par_binned_smem(nthr);
  auto k = forward_parallel_binned_kernel<EPI>;
  {
    const int rc_smem = request_smem(k, smem, "forward");
    if (rc_smem) return rc_smem;
  }
  const dim3 grid = EPI::kViewFastest ? dim3(v_count, fwd_nblk(g)) : dim3(fwd_nblk(g), v_count);
  tpre(st);
  launchb<FwdParBinnedB<EPI>>(grid, nthr, smem, st, what, geo, v_start, values, (int)P, band,
                              (const ConeFwdRec *)b.recs, (const int *)b.list,
                              (const int *)b.offs, b.touched, epi);
  MBIR_CHECK_LAUNCH(what);
  return MBIR_OK;
}

// Forward of a (P, band) subset array over all views through the bins: per
// view chunk, bin (when `bin`) and project.  With a single chunk the bins
// outlive the call, so a later projection of the same subset passes
// bin = false.
template <typename EPI>
int run_forward_binned(const mbir_geometry *g, const float *vp, const float *values,
                       long long P, int band, const int64_t *pix, const FwdBins &b, bool bin,
                       const EPI &epi, cudaStream_t st, const char *what) {
  const int V = g->num_views;
  for (int v0 = 0; v0 < V; v0 += b.views) {
    const int nv = std::min(b.views, V - v0);
    int rc;
    if (bin || b.views < V) {
      rc = launch_bin(g, vp, v0, nv, pix, P, b, st);
      if (rc) return rc;
    }
    rc = g->geometry == MBIR_CONE ? launch_binned(g, v0, nv, values, P, band, b, epi, st, what)
                                  : launch_par_binned(g, v0, nv, values, P, band, b, epi, st, what);
    if (rc) return rc;
  }
  return MBIR_OK;
}

template <typename EPI>
int run_forward(const mbir_geometry *g, const float *vp, int v_start, int v_count,
                const float *values, long long P, int band, int slice_start, const int64_t *pix,
                const EPI &epi, cudaStream_t st, const char *what = "forward projection",
                int by_pixel = 0) {
  if (use_cone_rt(g))
    return launch_cone_rt(g, vp, v_start, v_count, values, P, band, slice_start, pix, epi, st,
                          what, by_pixel);
  const FwdShape fs = fwd_shape(g, band);
#define MBIR_FWD(CONEV, NTV) \
  launch_forward<CONEV, NTV>(g, vp, v_start, v_count, values, P, band, slice_start, pix, fs, epi, st, what, by_pixel)
  const bool r1 = g->psf_radius == 1;
  if (g->geometry == MBIR_CONE) return r1 ? MBIR_FWD(true, 3) : MBIR_FWD(true, 0);
  return r1 ? MBIR_FWD(false, 3) : MBIR_FWD(false, 0);
#undef MBIR_FWD
}

// ── binned forward of whole cylinders (the projector entry points) ─────────
// The bins of views [v0, v0 + vc) for P pixels, carved from a workspace,
// with `touched` for every view of the geometry (the kernels index it by
// absolute view).
constexpr size_t kFullBinBytes = (size_t)1 << 30;  // default record budget

size_t full_bin_bytes(const mbir_geometry *g, long long P, int vc) {
  return align_up((size_t)vc * P * sizeof(ConeFwdRec)) + align_up((size_t)vc * P * sizeof(int)) +
         align_up((size_t)vc * (fwd_nkeys(g->num_det_channels) + 1) * sizeof(int)) +
         align_up((size_t)g->num_views * fwd_nblk(g));
}

// Views per chunk that `bytes` of workspace hold (0 when not even one).
int full_bin_views(const mbir_geometry *g, long long P, int view_count, size_t bytes) {
  const size_t fixed = align_up((size_t)g->num_views * fwd_nblk(g));
  if (bytes <= fixed) return 0;
  const size_t per_view = (size_t)P * (sizeof(ConeFwdRec) + sizeof(int)) +
                          (size_t)(fwd_nkeys(g->num_det_channels) + 1) * sizeof(int);
  // an upper bound, then down past the alignment padding (at most 768 bytes)
  int vc = (int)std::min<size_t>((size_t)view_count, (bytes - fixed) / per_view);
  while (vc > 0 && full_bin_bytes(g, P, vc) > bytes) --vc;
  return vc;
}

FwdBins carve_full_bins(const mbir_geometry *g, long long P, int vc, void *ws) {
  Carver c(ws);
  FwdBins b;
  b.recs = c.take<ConeFwdRec>((size_t)vc * P);
  b.list = c.take<int>((size_t)vc * P);
  b.offs = c.take<int>((size_t)vc * (fwd_nkeys(g->num_det_channels) + 1));
  b.touched = c.take<unsigned char>((size_t)g->num_views * fwd_nblk(g));
  b.views = vc;
  return b;
}

int fwd_blocks(const mbir_geometry *g, int band, int v_count) {
  if (use_cone_rt(g) || use_par_binned(g))
    return ((g->num_det_channels + kFwdCB - 1) / kFwdCB) * v_count;
  const FwdShape fs = fwd_shape(g, band);
  return ((g->num_det_channels + fs.CB - 1) / fs.CB) * v_count;
}

// ── VCD workspace ─────────────────────────────────────────────────────────
struct VcdWs {
  float *grad_part, *delta, *gbuf, *hinv, *gpbuf, *hpbuf, *alpha;
  unsigned int *counters;  // [0] spare, [1] recon-update CTAs (last-CTA election)
  double *dc_sums, *prior_part, *fwd_part, *sq_part, *l1_part;
  void *ad;
  FwdBins bins;  // binned cone forward (used when `binned`)
  BackShape bs;
  int dc_chunks, prior_blocks, fwd_blocks, upd_chunks, upd_yblocks;
  bool binned;
  size_t bytes;
};

constexpr int kUpdChunk = 16;   // pixels per update tile (two load batches)

size_t storage_size(int storage) { return storage == MBIR_F32 ? 4 : 2; }

VcdWs vcd_layout(const mbir_geometry *g, long long Ps, const mbir_vcd_params *prm, void *base) {
  VcdWs w;
  const int S = g->num_slices, V = g->num_views;
  const size_t PS = (size_t)Ps * S;
  w.bs = back_shape(g, V, Ps, S, (size_t)64 * PS * sizeof(float), true);
  Carver c(base);
  w.grad_part = c.take<float>((size_t)std::max(1, w.bs.nchunks) * PS);
  w.delta = c.take<float>(PS);
  w.gbuf = c.take<float>(PS);
  w.hinv = c.take<float>(PS);
  w.gpbuf = c.take<float>(PS);
  w.hpbuf = c.take<float>(PS);
  w.dc_chunks = (int)((Ps + kDcChunk - 1) / kDcChunk);
  w.dc_sums = c.take<double>((size_t)w.dc_chunks * S * 2);
  w.prior_blocks = (int)((PS + kThreads - 1) / kThreads);
  // (the damped direction writes one pair per (pixel block, slice block))
  const size_t dc_dir_ctas = (size_t)((Ps + kDcDirPixels - 1) / kDcDirPixels) * ((S + 31) / 32);
  w.prior_part = c.take<double>(std::max<size_t>(w.prior_blocks, dc_dir_ctas) * 2);
  w.fwd_blocks = fwd_blocks(g, S, V);
  w.fwd_part = c.take<double>((size_t)w.fwd_blocks * 2);
  w.upd_chunks = (int)((Ps + kUpdChunk - 1) / kUpdChunk);
  w.upd_yblocks = (S + kThreads - 1) / kThreads;
  w.sq_part = c.take<double>((size_t)w.upd_chunks * S);
  w.l1_part = c.take<double>((size_t)w.upd_chunks * w.upd_yblocks);
  w.alpha = c.take<float>(4);
  w.counters = c.take<unsigned int>(2);
  w.ad = c.take<char>((size_t)V * g->num_det_channels * g->num_det_rows * storage_size(prm->storage));
  w.binned = use_binned(g);
  w.bins = FwdBins{nullptr, nullptr, nullptr, nullptr, 0};
  if (w.binned) {
    const int vc = bin_views(g, Ps);
    w.bins.views = vc;
    w.bins.recs = c.take<ConeFwdRec>((size_t)vc * Ps);
    w.bins.list = c.take<int>((size_t)vc * Ps);
    w.bins.offs = c.take<int>((size_t)vc * (fwd_nkeys(g->num_det_channels) + 1));
    w.bins.touched = c.take<unsigned char>((size_t)V * fwd_nblk(g));
  }
  w.bytes = c.used;
  return w;
}

template <typename T>
int vcd_subset_t(const mbir_geometry *g, const float *vp, const mbir_vcd_params *prm,
                 float *flat, T *err, const float *es, const T *wts, const float *wsc,
                 const float *H, const float *dc, const int64_t *pix, long long Ps,
                 double *accum, float *alpha_user, VcdWs &w, cudaStream_t st,
                 const int64_t *next_pix, bool prebinned, bool *binned_next) {
  const int S = g->num_slices, V = g->num_views, C = g->num_det_channels, R = g->num_det_rows;
  const size_t PS = (size_t)Ps * S;
  const VcdScalars sc = make_scalars(*prm);
  const bool DCon = dc != nullptr;
  int rc;
  // 0. the subset's (view, pixel) records, sorted by centre channel; when one
  //    chunk holds every view the gradient reads them too.
  //    A partition pass may have formed them already in the previous step's
  //    tail (`prebinned`).
  const bool shared_bins = w.binned && w.bins.views >= V && g->psf_radius == 1;
  if (shared_bins && !prebinned) {
    rc = launch_bin(g, vp, 0, V, pix, Ps, w.bins, st);
    if (rc) return rc;
  }
  // (the cone gradient reads them; the parallel one forms its taps itself)
  const ConeFwdRec *recs = shared_bins && g->geometry == MBIR_CONE ? w.bins.recs : nullptr;
  // 1. gradient partials of A^T (w e), one slab per view chunk
  if (wts) {
    ReadWeighted<T> rd{err, es, wts, wsc, C, R};
    rc = run_back(g, vp, 0, V, rd, pix, Ps, 1, 0, S, w.grad_part, w.bs, w.grad_part, st, false,
                  "vcd gradient (back projection)", recs);
  } else {
    ReadScaled<T> rd{err, es, C, R};
    rc = run_back(g, vp, 0, V, rd, pix, Ps, 1, 0, S, w.grad_part, w.bs, w.grad_part, st, false,
                  "vcd gradient (back projection)", recs);
  }
  if (rc) return rc;
  // 2. direction (reduces the chunk slabs in order)
  const int nb = w.prior_blocks;
  int nprior = nb;  // prior line-term partials the alpha kernel folds
  if (!DCon) {
    tpre(st);
    launchb<DirectionB<false>>(nb, kThreads, 0, st, "vcd direction", (int)Ps, S, pix,
                               g->num_recon_rows, g->num_recon_cols, w.grad_part, w.bs.nchunks,
                               flat, H, sc, w.delta, nullptr, nullptr, nullptr, nullptr,
                               w.prior_part);
    MBIR_CHECK_LAUNCH("vcd direction");
  } else {
    tpre(st);
    launchb<DirectionB<true>>(nb, kThreads, 0, st, "vcd direction (damped)", (int)Ps, S, pix,
                              g->num_recon_rows, g->num_recon_cols, w.grad_part, w.bs.nchunks,
                              flat, H, sc, nullptr, w.gbuf, w.hinv, w.gpbuf, w.hpbuf, nullptr);
    MBIR_CHECK_LAUNCH("vcd direction (damped)");
    dim3 gs(w.dc_chunks, (S + 31) / 32);
    tpre(st);
    launchb<DcSumsB>(gs, dim3(32, kDcGroups), 0, st, "vcd DC sums", (int)Ps, S, w.gbuf, w.hinv,
                     w.dc_sums);
    MBIR_CHECK_LAUNCH("vcd DC sums");
    const dim3 gd((unsigned)((Ps + kDcDirPixels - 1) / kDcDirPixels), (S + 31) / 32);
    nprior = (int)(gd.x * gd.y);
    tpre(st);
    launchb<DcDirectionB>(gd, dim3(32, 8), 0, st, "vcd DC direction", (int)Ps, S, w.dc_chunks,
                          w.dc_sums, dc, w.gbuf, w.hinv, w.gpbuf, w.hpbuf, w.delta, w.prior_part);
    MBIR_CHECK_LAUNCH("vcd DC direction");
  }
  // 3. forward A delta + line-search partials
  LineSearchEpi<T> epi{err, es, wts, wsc, static_cast<T *>(w.ad), C, R, w.fwd_part, 1, 0.0, 0.0};
  if (w.binned)
    rc = run_forward_binned(g, vp, w.delta, Ps, S, pix, w.bins, !shared_bins, epi, st,
                            "vcd forward + line search");
  else
    rc = run_forward(g, vp, 0, V, w.delta, Ps, S, 0, pix, epi, st, "vcd forward + line search");
  if (rc) return rc;
  // 4. alpha
  tpre(st);
  launchb<AlphaB>(1, kAlphaThreads, 0, st, "vcd alpha", w.prior_part, nprior, w.fwd_part,
                  w.fwd_blocks, sc.fmc, sc.max_alpha, w.alpha, alpha_user);
  MBIR_CHECK_LAUNCH("vcd alpha");
  if (prm->positivity) {
    tpre(st);
    launchb<PositivityB>((unsigned)((PS + 255) / 256), 256, 0, st, "vcd positivity", (int)Ps, S,
                         pix, flat, w.alpha, w.delta);
    MBIR_CHECK_LAUNCH("vcd positivity");
    LineSearchEpi<T> epi2{err, es, wts, wsc, static_cast<T *>(w.ad), C, R, nullptr, 0, 0.0, 0.0};
    if (w.binned)
      rc = run_forward_binned(g, vp, w.delta, Ps, S, pix, w.bins, false, epi2, st,
                              "vcd forward (positivity)");
    else
      rc = run_forward(g, vp, 0, V, w.delta, Ps, S, 0, pix, epi2, st, "vcd forward (positivity)");
    if (rc) return rc;
  }
  // 5. update
  if (w.binned) {
    // Recon update and the sinogram's touched tiles (elsewhere A delta is
    // zero and e is unchanged) in one launch, with the next subset's bins
    // when the pass has one and they fit one chunk.
    const int nblk = fwd_nblk(g);
    const int nbin = (shared_bins && next_pix != nullptr) ? V : 0;
    const TailBins tb{make_geo(*g), vp, next_pix, (int)Ps, w.bins.recs, w.bins.list,
                      w.bins.offs};
    const size_t smem = nbin ? bin_smem(g) : 0;
    auto k = vcd_tail_kernel<T>;
    {
      const int rc_smem = request_smem(k, smem, "VCD update");
      if (rc_smem) return rc_smem;
    }
    // tiles per tile-role CTA: about 4096 cells each
    const int tpc = std::max(1, std::min(nblk, 4096 / (kFwdCB * R)));
    const long long ctas = (long long)nbin + (long long)w.upd_chunks * w.upd_yblocks +
                           (long long)((nblk + tpc - 1) / tpc) * V;
    tpre(st);
    launchb<TailB<T>>((unsigned)ctas, 256, smem, st, "vcd pixel + sinogram update", nbin, tb,
                      (int)Ps, S, kUpdChunk, pix, w.delta, w.alpha, flat, w.sq_part, w.l1_part,
                      w.counters + 1, accum, w.upd_chunks, w.upd_yblocks, C, R, kFwdCB,
                      w.bins.touched, err, static_cast<const T *>(w.ad), nblk, tpc);
    MBIR_CHECK_LAUNCH("vcd pixel + sinogram update");
    if (binned_next) *binned_next = nbin > 0;
    return MBIR_OK;
  }
  dim3 gu(w.upd_chunks, w.upd_yblocks);
  tpre(st);
  launch(vcd_pixel_update_kernel, gu, kThreads, 0, st, (int)Ps, S, kUpdChunk, pix, w.delta,
         w.alpha, flat, w.sq_part, w.l1_part, w.counters + 1, accum);
  MBIR_CHECK_LAUNCH("vcd pixel update");
  const size_t n = (size_t)V * C * R;
  const int blocks = (int)std::min<size_t>((n / 4 + 255) / 256 + 1, (size_t)device_sms() * 32);
  tpre(st);
  launch(vcd_sino_update_kernel<T>, blocks, 256, 0, st, n, w.alpha, err,
         static_cast<const T *>(w.ad));
  MBIR_CHECK_LAUNCH("vcd sinogram update");
  return MBIR_OK;
}

int validate_vcd(const mbir_geometry *g, const mbir_vcd_params *prm, const void *flat,
                 const void *err, const float *es, const void *wts, const float *wsc,
                 const float *H, long long Ps) {
  int rc = validate_geometry(g);
  if (rc) return rc;
  if (!prm) return fail(MBIR_ERR_INVALID, "params is NULL");
  if (prm->storage != MBIR_F32 && prm->storage != MBIR_BF16 && prm->storage != MBIR_F16)
    return fail(MBIR_ERR_INVALID, "unknown storage dtype %d", prm->storage);
  if (!flat || !err || !es || !H) return fail(MBIR_ERR_INVALID, "NULL state pointer");
  if (wts && !wsc) return fail(MBIR_ERR_INVALID, "weights given without their scale");
  if (Ps <= 0) return fail(MBIR_ERR_INVALID, "subset must have at least one pixel");
  if (!(prm->sigma_x > 0.f) || !(prm->fm_constant > 0.f) || !(prm->T > 0.f))
    return fail(MBIR_ERR_INVALID, "sigma_x, T and fm_constant must be positive");
  if (prm->prox_input != nullptr && !(prm->prox_constant > 0.f))
    return fail(MBIR_ERR_INVALID, "prox_constant (1 / sigma_prox^2) must be positive");
  return MBIR_OK;
}

}  // namespace

extern "C" {

int32_t mbir_abi_version(void) { return 10100; }

const char *mbir_last_error(void) { return g_last_error.c_str(); }

unsigned long long mbir_launch_count(void) { return g_launches.load(); }

int32_t mbir_timing_enable(int32_t on) {
  const int prev = g_timing.exchange(on ? 1 : 0);
  return prev;
}

int32_t mbir_timing_collect(char *names, int32_t names_bytes, double *total_ms,
                            int64_t *counts, int32_t max_entries) {
  std::vector<TimedLaunch> timed;
  {
    std::lock_guard<std::mutex> lk(g_timing_mu);
    timed.swap(g_timed);
  }
  std::vector<std::string> keys;
  std::vector<double> ms;
  std::vector<int64_t> cnt;
  for (auto &t : timed) {
    float e = 0.f;
    cudaEventSynchronize(t.b);
    if (cudaEventElapsedTime(&e, t.a, t.b) != cudaSuccess) e = 0.f;
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
    size_t k = 0;
    while (k < keys.size() && keys[k] != t.name) ++k;
    if (k == keys.size()) {
      keys.push_back(t.name);
      ms.push_back(0.0);
      cnt.push_back(0);
    }
    ms[k] += e;
    cnt[k] += 1;
  }
  std::string joined;
  const int n = (int)std::min<size_t>(keys.size(), (size_t)std::max(0, max_entries));
  for (int k = 0; k < n; ++k) {
    if (total_ms) total_ms[k] = ms[k];
    if (counts) counts[k] = cnt[k];
    joined += keys[k];
    joined += '\n';
  }
  if (names && names_bytes > 0) {
    const size_t m = std::min<size_t>(joined.size(), (size_t)names_bytes - 1);
    memcpy(names, joined.data(), m);
    names[m] = 0;
  }
  cudaGetLastError();
  return n;
}

int32_t mbir_forward_project(const mbir_geometry *geom, const float *view_params,
                             int32_t view_start, int32_t view_count, const float *values,
                             int64_t num_pixels, int32_t band_len, int32_t slice_start,
                             const int64_t *pixel_indices, float *sino_out, int32_t out_layout,
                             void *stream) {
  int rc = validate_geometry(geom);
  if (rc) return rc;
  if (view_start < 0 || view_count < 0 || view_start + view_count > geom->num_views)
    return fail(MBIR_ERR_INVALID, "view range [%d, %d) outside [0, %d)", view_start,
                view_start + view_count, geom->num_views);
  if (num_pixels < 0 || num_pixels >= (1LL << 31)) return fail(MBIR_ERR_INVALID, "bad num_pixels");
  if (band_len <= 0 || slice_start < 0 || slice_start + band_len > geom->num_slices)
    return fail(MBIR_ERR_INVALID, "slice band [%d, %d) outside [0, %d)", slice_start,
                slice_start + band_len, geom->num_slices);
  if (geom->geometry == MBIR_PARALLEL && (slice_start != 0 || band_len != geom->num_det_rows))
    return fail(MBIR_ERR_INVALID, "parallel beam projects whole cylinders (band == rows)");
  if (out_layout != MBIR_LAYOUT_VRC && out_layout != MBIR_LAYOUT_VCR)
    return fail(MBIR_ERR_INVALID, "unknown layout %d", out_layout);
  if (!view_params || !sino_out || (num_pixels > 0 && (!values || !pixel_indices)))
    return fail(MBIR_ERR_INVALID, "NULL array argument");
  if (view_count == 0) return MBIR_OK;
  cudaStream_t st = as_stream(stream);
  if (num_pixels == 0) {
    cudaError_t e = cudaMemsetAsync(sino_out, 0,
        (size_t)view_count * geom->num_det_rows * geom->num_det_channels * sizeof(float), st);
    if (e != cudaSuccess) return fail(MBIR_ERR_CUDA, "memset: %s", cudaGetErrorString(e));
    return MBIR_OK;
  }
  StoreSino epi{sino_out, out_layout, geom->num_det_channels, geom->num_det_rows};
  return run_forward(geom, view_params, view_start, view_count, values, num_pixels, band_len,
                     slice_start, pixel_indices, epi, st);
}

int32_t mbir_forward_project_volume(const mbir_geometry *geom, const float *view_params,
                                    int32_t view_start, int32_t view_count,
                                    const float *flat_volume, const int64_t *pixel_indices,
                                    int64_t num_pixels, float *sino_out, int32_t out_layout,
                                    void *stream) {
  int rc = validate_geometry(geom);
  if (rc) return rc;
  if (view_start < 0 || view_count < 0 || view_start + view_count > geom->num_views)
    return fail(MBIR_ERR_INVALID, "view range [%d, %d) outside [0, %d)", view_start,
                view_start + view_count, geom->num_views);
  if (num_pixels < 0 || num_pixels >= (1LL << 31)) return fail(MBIR_ERR_INVALID, "bad num_pixels");
  if (out_layout != MBIR_LAYOUT_VRC && out_layout != MBIR_LAYOUT_VCR)
    return fail(MBIR_ERR_INVALID, "unknown layout %d", out_layout);
  if (!view_params || !sino_out || (num_pixels > 0 && (!flat_volume || !pixel_indices)))
    return fail(MBIR_ERR_INVALID, "NULL array argument");
  if (view_count == 0) return MBIR_OK;
  cudaStream_t st = as_stream(stream);
  if (num_pixels == 0) {
    cudaError_t e = cudaMemsetAsync(sino_out, 0,
        (size_t)view_count * geom->num_det_rows * geom->num_det_channels * sizeof(float), st);
    if (e != cudaSuccess) return fail(MBIR_ERR_CUDA, "memset: %s", cudaGetErrorString(e));
    return MBIR_OK;
  }
  StoreSino epi{sino_out, out_layout, geom->num_det_channels, geom->num_det_rows};
  return run_forward(geom, view_params, view_start, view_count, flat_volume, num_pixels,
                     geom->num_slices, 0, pixel_indices, epi, st, "forward projection", 1);
}

size_t mbir_forward_project_binned_workspace_size(const mbir_geometry *geom, int32_t view_count,
                                                  int64_t num_pixels) {
  if (!geom || view_count <= 0 || num_pixels <= 0 || num_pixels >= (1LL << 31)) return 0;
  if (geom->num_views <= 0 || geom->num_det_channels <= 0 || !use_binned(geom)) return 0;
  const size_t per_view = (size_t)num_pixels * (sizeof(ConeFwdRec) + sizeof(int));
  const int vc = (int)std::max<size_t>(
      1, std::min<size_t>((size_t)view_count, kFullBinBytes / std::max<size_t>(per_view, 1)));
  return full_bin_bytes(geom, num_pixels, vc);
}

int32_t mbir_forward_project_binned(const mbir_geometry *geom, const float *view_params,
                                    int32_t view_start, int32_t view_count, const float *values,
                                    int32_t values_by_pixel, const int64_t *pixel_indices,
                                    int64_t num_pixels, float *sino_out, int32_t out_layout,
                                    void *workspace, size_t workspace_bytes, void *stream) {
  int rc = validate_geometry(geom);
  if (rc) return rc;
  if (!use_binned(geom))
    return fail(MBIR_ERR_INVALID, "the binned forward covers psf radius 1 and up to 1024 "
                "detector rows; use mbir_forward_project");
  if (view_start < 0 || view_count < 0 || view_start + view_count > geom->num_views)
    return fail(MBIR_ERR_INVALID, "view range [%d, %d) outside [0, %d)", view_start,
                view_start + view_count, geom->num_views);
  if (num_pixels < 0 || num_pixels >= (1LL << 31)) return fail(MBIR_ERR_INVALID, "bad num_pixels");
  if (out_layout != MBIR_LAYOUT_VRC && out_layout != MBIR_LAYOUT_VCR)
    return fail(MBIR_ERR_INVALID, "unknown layout %d", out_layout);
  if (values_by_pixel != 0 && values_by_pixel != 1)
    return fail(MBIR_ERR_INVALID, "values_by_pixel must be 0 or 1");
  if (!view_params || !sino_out || (num_pixels > 0 && (!values || !pixel_indices)))
    return fail(MBIR_ERR_INVALID, "NULL array argument");
  if (view_count == 0) return MBIR_OK;
  cudaStream_t st = as_stream(stream);
  if (num_pixels == 0) {
    cudaError_t e = cudaMemsetAsync(sino_out, 0,
        (size_t)view_count * geom->num_det_rows * geom->num_det_channels * sizeof(float), st);
    if (e != cudaSuccess) return fail(MBIR_ERR_CUDA, "memset: %s", cudaGetErrorString(e));
    return MBIR_OK;
  }
  if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
    return fail(MBIR_ERR_WORKSPACE, "the binned forward needs a 256-byte aligned workspace");
  const int vc = full_bin_views(geom, num_pixels, view_count, workspace_bytes);
  if (vc < 1)
    return fail(MBIR_ERR_WORKSPACE, "workspace of %zu bytes holds no view's bins (%zu needed "
                "for one)", workspace_bytes, full_bin_bytes(geom, num_pixels, 1));
  const FwdBins b = carve_full_bins(geom, num_pixels, vc, workspace);
  const int band = geom->num_slices;
  StoreSino epi{sino_out, out_layout, geom->num_det_channels, geom->num_det_rows, view_start};
  for (int v0 = view_start; v0 < view_start + view_count; v0 += vc) {
    const int nv = std::min(vc, view_start + view_count - v0);
    rc = launch_bin(geom, view_params, v0, nv, pixel_indices, num_pixels, b, st, values_by_pixel,
                    true);
    if (rc) return rc;
    rc = geom->geometry == MBIR_CONE
             ? launch_binned(geom, v0, nv, values, num_pixels, band, b, epi, st,
                             "forward projection (binned)")
             : launch_par_binned(geom, v0, nv, values, num_pixels, band, b, epi, st,
                                 "forward projection (binned)");
    if (rc) return rc;
  }
  return MBIR_OK;
}

int32_t mbir_vcd_refresh_error(const mbir_geometry *geom, const float *view_params,
                               const float *flat_recon, const int64_t *pixel_indices,
                               int64_t num_pixels, const float *y_vcr, void *error_sino,
                               const float *err_scale, int32_t storage, void *workspace,
                               size_t workspace_bytes, void *stream) {
  int rc = validate_geometry(geom);
  if (rc) return rc;
  if (!view_params || !flat_recon || !pixel_indices || !y_vcr || !error_sino || !err_scale ||
      num_pixels <= 0)
    return fail(MBIR_ERR_INVALID, "bad refresh arguments");
  if (storage != MBIR_F32 && storage != MBIR_BF16 && storage != MBIR_F16)
    return fail(MBIR_ERR_INVALID, "unknown storage dtype %d", storage);
  cudaStream_t st = as_stream(stream);
  const int C = geom->num_det_channels, R = geom->num_det_rows, V = geom->num_views;
  const int S = geom->num_slices;
  // Through the bins when a workspace holds at least one view's.
  const bool binned = workspace != nullptr &&
                      (reinterpret_cast<uintptr_t>(workspace) & 255) == 0 && use_binned(geom) &&
                      full_bin_views(geom, num_pixels, V, workspace_bytes) >= 1;
  auto run = [&](auto epi) -> int {
    if (!binned)
      return run_forward(geom, view_params, 0, V, flat_recon, num_pixels, S, 0, pixel_indices,
                         epi, st, "vcd error refresh", 1);
    const int vc = full_bin_views(geom, num_pixels, V, workspace_bytes);
    const FwdBins b = carve_full_bins(geom, num_pixels, vc, workspace);
    for (int v0 = 0; v0 < V; v0 += vc) {
      const int nv = std::min(vc, V - v0);
      int r = launch_bin(geom, view_params, v0, nv, pixel_indices, num_pixels, b, st, 1, true);
      if (r) return r;
      r = geom->geometry == MBIR_CONE
              ? launch_binned(geom, v0, nv, flat_recon, num_pixels, S, b, epi, st,
                              "vcd error refresh (binned)")
              : launch_par_binned(geom, v0, nv, flat_recon, num_pixels, S, b, epi, st,
                                  "vcd error refresh (binned)");
      if (r) return r;
    }
    return MBIR_OK;
  };
  switch (storage) {
    case MBIR_F32:
      return run(RefreshEpi<float>{y_vcr, static_cast<float *>(error_sino), err_scale, C, R});
    case MBIR_BF16:
      return run(RefreshEpi<__nv_bfloat16>{y_vcr, static_cast<__nv_bfloat16 *>(error_sino),
                                           err_scale, C, R});
    default:
      return run(RefreshEpi<__half>{y_vcr, static_cast<__half *>(error_sino), err_scale, C, R});
  }
}

size_t mbir_back_project_workspace_size(const mbir_geometry *geom, int32_t view_count,
                                        int64_t num_pixels, int32_t band_len) {
  if (!geom || view_count <= 0 || num_pixels <= 0 || band_len <= 0) return 0;
  const BackShape s = back_shape(geom, view_count, num_pixels, band_len, (size_t)1 << 40);
  const size_t sino = align_up((size_t)view_count * geom->num_det_rows * geom->num_det_channels *
                               sizeof(float));
  return back_partial_bytes(s, num_pixels, band_len) + sino;
}

int32_t mbir_back_project(const mbir_geometry *geom, const float *view_params, int32_t view_start,
                          int32_t view_count, const float *sino, int32_t sino_layout,
                          const int64_t *pixel_indices, int64_t num_pixels, int32_t coeff_power,
                          int32_t slice_start, int32_t band_len, float *out, void *workspace,
                          size_t workspace_bytes, void *stream) {
  int rc = validate_geometry(geom);
  if (rc) return rc;
  if (view_start < 0 || view_count < 0 || view_start + view_count > geom->num_views)
    return fail(MBIR_ERR_INVALID, "view range [%d, %d) outside [0, %d)", view_start,
                view_start + view_count, geom->num_views);
  if (coeff_power != 1 && coeff_power != 2)
    return fail(MBIR_ERR_INVALID, "coeff_power must be 1 or 2, got %d", coeff_power);
  if (band_len <= 0 || slice_start < 0 || slice_start + band_len > geom->num_slices)
    return fail(MBIR_ERR_INVALID, "slice band [%d, %d) outside [0, %d)", slice_start,
                slice_start + band_len, geom->num_slices);
  if (geom->geometry == MBIR_PARALLEL && (slice_start != 0 || band_len != geom->num_det_rows))
    return fail(MBIR_ERR_INVALID, "parallel beam back-projects whole cylinders (band == rows)");
  if (sino_layout != MBIR_LAYOUT_VRC && sino_layout != MBIR_LAYOUT_VCR)
    return fail(MBIR_ERR_INVALID, "unknown layout %d", sino_layout);
  if (num_pixels < 0 || num_pixels >= (1LL << 31)) return fail(MBIR_ERR_INVALID, "bad num_pixels");
  if (!view_params || (num_pixels > 0 && (!sino || !pixel_indices || !out)))
    return fail(MBIR_ERR_INVALID, "NULL array argument");
  cudaStream_t st = as_stream(stream);
  if (num_pixels == 0) return MBIR_OK;
  if (view_count == 0) {
    cudaError_t e = cudaMemsetAsync(out, 0, (size_t)num_pixels * band_len * sizeof(float), st);
    if (e != cudaSuccess) return fail(MBIR_ERR_CUDA, "memset: %s", cudaGetErrorString(e));
    return MBIR_OK;
  }
  const int C = geom->num_det_channels, R = geom->num_det_rows;
  const size_t sino_bytes = align_up((size_t)view_count * R * C * sizeof(float));
  const size_t need_sino = sino_layout == MBIR_LAYOUT_VRC ? sino_bytes : 0;
  if (workspace_bytes < need_sino || (need_sino && !workspace))
    return fail(MBIR_ERR_WORKSPACE, "workspace of %zu bytes < %zu needed for the layout change",
                workspace_bytes, need_sino);
  const size_t partial_budget = workspace ? workspace_bytes - need_sino : 0;
  const BackShape s = back_shape(geom, view_count, num_pixels, band_len, partial_budget);
  char *ws = static_cast<char *>(workspace);
  const float *vcr = sino;
  if (sino_layout == MBIR_LAYOUT_VRC) {
    float *t = reinterpret_cast<float *>(ws);
    dim3 grid((C + 31) / 32, (R + 31) / 32, view_count);
    tpre(st);
    vrc_to_vcr_kernel<float><<<grid, dim3(32, 8), 0, st>>>(R, C, sino, nullptr, t);
    MBIR_CHECK_LAUNCH("layout change");
    vcr = t;
  }
  float *partials = reinterpret_cast<float *>(ws ? ws + need_sino : nullptr);
  ReadF32 rd{vcr, C, R};
  return run_back(geom, view_params, view_start, view_count, rd, pixel_indices, num_pixels,
                  coeff_power, slice_start, band_len, out, s, partials, st, true);
}

int32_t mbir_sino_convert(int32_t direction, int32_t views, int32_t rows, int32_t channels,
                          const void *src, void *dst, int32_t dtype, float *scale,
                          int32_t compute_scale, void *stream) {
  if (views <= 0 || rows <= 0 || channels <= 0) return fail(MBIR_ERR_INVALID, "bad sinogram shape");
  if (views > kMaxViews)
    return fail(MBIR_ERR_INVALID, "at most %d views per sinogram (got %d)", kMaxViews, views);
  if (!src || !dst || !scale) return fail(MBIR_ERR_INVALID, "NULL array argument");
  if (dtype != MBIR_F32 && dtype != MBIR_BF16 && dtype != MBIR_F16)
    return fail(MBIR_ERR_INVALID, "unknown dtype %d", dtype);
  cudaStream_t st = as_stream(stream);
  const int R = rows, C = channels;
  if (direction == 0) {
    if (compute_scale) {
      if (dtype == MBIR_F16) {
        tpre(st);
        view_scale_kernel<<<views, kThreads, 0, st>>>(R * C, static_cast<const float *>(src),
                                                      256.f, scale);
        MBIR_CHECK_LAUNCH("view scale");
      } else {
        tpre(st);
        fill_kernel<<<(views + 255) / 256, 256, 0, st>>>(views, 1.f, scale);
        MBIR_CHECK_LAUNCH("scale fill");
      }
    }
    dim3 grid((C + 31) / 32, (R + 31) / 32, views);
    const float *s = static_cast<const float *>(src);
    tpre(st);
    if (dtype == MBIR_F32)
      vrc_to_vcr_kernel<float><<<grid, dim3(32, 8), 0, st>>>(R, C, s, scale, static_cast<float *>(dst));
    else if (dtype == MBIR_BF16)
      vrc_to_vcr_kernel<__nv_bfloat16><<<grid, dim3(32, 8), 0, st>>>(R, C, s, scale, static_cast<__nv_bfloat16 *>(dst));
    else
      vrc_to_vcr_kernel<__half><<<grid, dim3(32, 8), 0, st>>>(R, C, s, scale, static_cast<__half *>(dst));
    MBIR_CHECK_LAUNCH("sinogram conversion");
  } else if (direction == 1) {
    dim3 grid((R + 31) / 32, (C + 31) / 32, views);
    float *d = static_cast<float *>(dst);
    tpre(st);
    if (dtype == MBIR_F32)
      vcr_to_vrc_kernel<float><<<grid, dim3(32, 8), 0, st>>>(R, C, static_cast<const float *>(src), scale, d);
    else if (dtype == MBIR_BF16)
      vcr_to_vrc_kernel<__nv_bfloat16><<<grid, dim3(32, 8), 0, st>>>(R, C, static_cast<const __nv_bfloat16 *>(src), scale, d);
    else
      vcr_to_vrc_kernel<__half><<<grid, dim3(32, 8), 0, st>>>(R, C, static_cast<const __half *>(src), scale, d);
    MBIR_CHECK_LAUNCH("sinogram conversion");
  } else {
    return fail(MBIR_ERR_INVALID, "direction must be 0 or 1");
  }
  return MBIR_OK;
}

// Partial-sum blocks of the error-init and statistics reductions: a few
// per SM, capped so that the workspace size does not depend on the device.
constexpr int kInitMaxBlocks = 4096;
constexpr int kStatsMaxBlocks = 2048;
int init_blocks() { return std::min(kInitMaxBlocks, device_sms() * 8); }
int stats_blocks() { return std::min(kStatsMaxBlocks, device_sms() * 4); }

size_t mbir_error_init_workspace_size(int64_t count) {
  (void)count;
  return align_up(sizeof(double) * 2 * kInitMaxBlocks) + 256;
}

int32_t mbir_error_init(int64_t count, const float *y, const float *ax, const float *weights,
                        int32_t scale_to_data, float *error_out, double *alpha_out,
                        void *workspace, size_t workspace_bytes, void *stream) {
  if (count <= 0 || !y || !ax || !error_out || !alpha_out)
    return fail(MBIR_ERR_INVALID, "bad error-init arguments");
  if (!workspace || workspace_bytes < mbir_error_init_workspace_size(count))
    return fail(MBIR_ERR_WORKSPACE, "error init needs %zu workspace bytes",
                mbir_error_init_workspace_size(count));
  cudaStream_t st = as_stream(stream);
  const int nb = init_blocks();
  double *part = static_cast<double *>(workspace);
  tpre(st);
  init_dots_kernel<<<nb, kThreads, 0, st>>>((size_t)count, y, ax, weights, part);
  MBIR_CHECK_LAUNCH("init dots");
  tpre(st);
  init_alpha_kernel<<<1, kThreads, 0, st>>>(nb, part, scale_to_data, alpha_out);
  MBIR_CHECK_LAUNCH("init alpha");
  tpre(st);
  init_error_kernel<<<nb, 256, 0, st>>>((size_t)count, y, ax, alpha_out, error_out);
  MBIR_CHECK_LAUNCH("init error");
  return MBIR_OK;
}

size_t mbir_vcd_workspace_size(const mbir_geometry *geom, int64_t max_subset_pixels,
                               const mbir_vcd_params *params) {
  if (!geom || !params || max_subset_pixels <= 0) return 0;
  return vcd_layout(geom, max_subset_pixels, params, nullptr).bytes;
}

namespace {
// One subset update; `fresh` zeroes the workspace's last-CTA counters first
// (the elected CTAs leave them at zero, so a partition pass zeroes them once).
int32_t subset_update(const mbir_geometry *geom, const float *view_params,
                      const mbir_vcd_params *params, float *flat_recon, void *error_sino,
                      const float *err_scale, const void *weights, const float *w_scale,
                      const float *fm_hessian, const float *dc_profile,
                      const int64_t *pixel_indices, int64_t num_pixels, double *accum,
                      float *alpha_out, void *workspace, size_t workspace_bytes, void *stream,
                      bool fresh, const int64_t *next_pix = nullptr, bool prebinned = false,
                      bool *binned_next = nullptr) {
  int rc = validate_vcd(geom, params, flat_recon, error_sino, err_scale, weights, w_scale,
                        fm_hessian, num_pixels);
  if (rc) return rc;
  if (!view_params || !pixel_indices || !accum) return fail(MBIR_ERR_INVALID, "NULL argument");
  VcdWs w = vcd_layout(geom, num_pixels, params, workspace);
  if (!workspace || workspace_bytes < w.bytes)
    return fail(MBIR_ERR_WORKSPACE, "VCD workspace of %zu bytes < %zu needed", workspace_bytes,
                w.bytes);
  cudaStream_t st = as_stream(stream);
  const PdlScope pdl;
  if (fresh) {
    const cudaError_t e = cudaMemsetAsync(w.counters, 0, 2 * sizeof(unsigned int), st);
    if (e != cudaSuccess)
      return fail(MBIR_ERR_CUDA, "VCD counter reset failed: %s", cudaGetErrorString(e));
  }
  switch (params->storage) {
    case MBIR_F32:
      return vcd_subset_t<float>(geom, view_params, params, flat_recon,
                                 static_cast<float *>(error_sino), err_scale,
                                 static_cast<const float *>(weights), w_scale, fm_hessian,
                                 dc_profile, pixel_indices, num_pixels, accum, alpha_out, w, st,
                                 next_pix, prebinned, binned_next);
    case MBIR_BF16:
      return vcd_subset_t<__nv_bfloat16>(geom, view_params, params, flat_recon,
                                         static_cast<__nv_bfloat16 *>(error_sino), err_scale,
                                         static_cast<const __nv_bfloat16 *>(weights), w_scale,
                                         fm_hessian, dc_profile, pixel_indices, num_pixels, accum,
                                         alpha_out, w, st, next_pix, prebinned, binned_next);
    default:
      return vcd_subset_t<__half>(geom, view_params, params, flat_recon,
                                  static_cast<__half *>(error_sino), err_scale,
                                  static_cast<const __half *>(weights), w_scale, fm_hessian,
                                  dc_profile, pixel_indices, num_pixels, accum, alpha_out, w, st,
                                 next_pix, prebinned, binned_next);
  }
}
}  // namespace

int32_t mbir_vcd_subset_update(const mbir_geometry *geom, const float *view_params,
                               const mbir_vcd_params *params, float *flat_recon, void *error_sino,
                               const float *err_scale, const void *weights,
                               const float *w_scale, const float *fm_hessian,
                               const float *dc_profile, const int64_t *pixel_indices,
                               int64_t num_pixels, double *accum, float *alpha_out,
                               void *workspace, size_t workspace_bytes, void *stream) {
  return subset_update(geom, view_params, params, flat_recon, error_sino, err_scale, weights,
                       w_scale, fm_hessian, dc_profile, pixel_indices, num_pixels, accum,
                       alpha_out, workspace, workspace_bytes, stream, true);
}

int32_t mbir_vcd_partition_pass(const mbir_geometry *geom, const float *view_params,
                                const mbir_vcd_params *params, float *flat_recon, void *error_sino,
                                const float *err_scale, const void *weights, const float *w_scale,
                                const float *fm_hessian, const float *dc_profile,
                                const int64_t *partition, int32_t num_subsets,
                                int64_t subset_pixels, const int32_t *order, double *accum,
                                void *workspace, size_t workspace_bytes, void *stream) {
  if (num_subsets <= 0 || !order || !partition)
    return fail(MBIR_ERR_INVALID, "partition pass needs subsets, a partition and an order");
  for (int i = 0; i < num_subsets; ++i)
    if (order[i] < 0 || order[i] >= num_subsets)
      return fail(MBIR_ERR_INVALID, "order[%d] = %d outside [0, %d)", i, order[i], num_subsets);
  // Each step's tail bins the next subset when the bins allow it.
  bool prebinned = false;
  for (int i = 0; i < num_subsets; ++i) {
    const int64_t *next =
        i + 1 < num_subsets ? partition + (size_t)order[i + 1] * subset_pixels : nullptr;
    bool binned_next = false;
    const int rc = subset_update(
        geom, view_params, params, flat_recon, error_sino, err_scale, weights, w_scale,
        fm_hessian, dc_profile, partition + (size_t)order[i] * subset_pixels, subset_pixels, accum,
        nullptr, workspace, workspace_bytes, stream, i == 0, next, prebinned, &binned_next);
    if (rc) return rc;
    prebinned = binned_next;
  }
  return MBIR_OK;
}

int32_t mbir_vcd_partition_pass_batched(
    int32_t num_jobs, const mbir_geometry *geom, const float *view_params,
    const mbir_vcd_params *params, float *const *flat_recon, void *const *error_sino,
    const float *const *err_scale, const void *const *weights, const float *const *w_scale,
    const float *const *fm_hessian, const float *dc_profile, const int64_t *const *partition,
    int32_t num_subsets, int64_t subset_pixels, const int32_t *order, double *const *accum,
    void *const *workspace, size_t workspace_bytes, void *stream) {
  if (num_jobs < 1 || num_jobs > kMaxBatch)
    return fail(MBIR_ERR_INVALID, "a batch holds 1 to %d jobs, got %d", kMaxBatch, num_jobs);
  if (!params || !flat_recon || !error_sino || !err_scale || !weights || !w_scale ||
      !fm_hessian || !partition || !order || !accum || !workspace)
    return fail(MBIR_ERR_INVALID, "batched partition pass: NULL argument array");
  if (num_subsets <= 0 || subset_pixels <= 0)
    return fail(MBIR_ERR_INVALID, "partition pass needs subsets, a partition and an order");
  for (int j = 0; j < num_jobs; ++j) {
    // Every job of a batch takes the same branches of the subset step.
    const mbir_vcd_params &a = params[0], &b = params[j];
    if (b.storage != a.storage || b.positivity != a.positivity ||
        (b.prox_input == nullptr) != (a.prox_input == nullptr) ||
        (weights[j] == nullptr) != (weights[0] == nullptr))
      return fail(MBIR_ERR_INVALID, "job %d of the batch differs from job 0 in storage, "
                  "positivity, prior or weighting", j);
    for (int i = 0; i < num_subsets; ++i) {
      const int o = order[(size_t)j * num_subsets + i];
      if (o < 0 || o >= num_subsets)
        return fail(MBIR_ERR_INVALID, "order[%d][%d] = %d outside [0, %d)", j, i, o,
                    num_subsets);
    }
  }
  const int rc0 = validate_geometry(geom);
  if (rc0) return rc0;
  if (!use_binned(geom)) {
    // The batched chain covers the binned subset step; other shapes step
    // their jobs one after another.
    for (int j = 0; j < num_jobs; ++j) {
      const int rc = mbir_vcd_partition_pass(
          geom, view_params, &params[j], flat_recon[j], error_sino[j], err_scale[j], weights[j],
          w_scale[j], fm_hessian[j], dc_profile, partition[j], num_subsets, subset_pixels,
          order + (size_t)j * num_subsets, accum[j], workspace[j], workspace_bytes, stream);
      if (rc) return rc;
    }
    return MBIR_OK;
  }
  cudaStream_t st = as_stream(stream);
  const PdlScope pdl;
  bool prebinned = false;
  for (int i = 0; i < num_subsets; ++i) {
    BatchRecorder rec;
    bool binned_next = false;
    for (int j = 0; j < num_jobs; ++j) {
      const int32_t *oj = order + (size_t)j * num_subsets;
      const int64_t *pj = partition[j];
      const int64_t *next = i + 1 < num_subsets ? pj + (size_t)oj[i + 1] * subset_pixels : nullptr;
      rec.begin_job(j);
      t_batch = &rec;
      const int rc = subset_update(geom, view_params, &params[j], flat_recon[j], error_sino[j],
                                   err_scale[j], weights[j], w_scale[j], fm_hessian[j],
                                   dc_profile, pj + (size_t)oj[i] * subset_pixels, subset_pixels,
                                   accum[j], nullptr, workspace[j], workspace_bytes, stream, i == 0,
                                   next, prebinned, &binned_next);
      t_batch = nullptr;
      if (rc) return rc;
      if (rec.mismatch || rec.cursor != rec.launches.size())
        return fail(MBIR_ERR_INVALID, "job %d's subset step does not match job 0's launch "
                    "for launch", j);
    }
    for (const BatchRecorder::Launch &l : rec.launches) {
      const int rc = l.replay(l, num_jobs, st);
      if (rc) return rc;
    }
    prebinned = binned_next;
  }
  return MBIR_OK;
}

namespace {
struct DenoiseWs {
  float *delta, *alpha;
  double *prior, *fwd, *l1;
  unsigned int *counter;
  int blocks;
  size_t bytes;
};

DenoiseWs denoise_layout(int S, long long Ps, void *base) {
  DenoiseWs w;
  const size_t n = (size_t)Ps * S;
  w.blocks = (int)((n + kThreads - 1) / kThreads);
  Carver c(base);
  w.delta = c.take<float>(n);
  w.prior = c.take<double>((size_t)w.blocks * 2);
  w.fwd = c.take<double>((size_t)w.blocks * 2);
  w.l1 = c.take<double>((size_t)w.blocks);
  w.alpha = c.take<float>(4);
  w.counter = c.take<unsigned int>(1);
  w.bytes = c.used;
  return w;
}
}  // namespace

size_t mbir_denoise_workspace_size(int32_t num_slices, int64_t subset_pixels) {
  if (num_slices <= 0 || subset_pixels <= 0) return 0;
  return denoise_layout(num_slices, subset_pixels, nullptr).bytes;
}

int32_t mbir_denoise_pass(int32_t num_rows, int32_t num_cols, int32_t num_slices,
                          const mbir_vcd_params *params, float *flat_image, float *flat_error,
                          const int64_t *partition, int32_t num_subsets, int64_t subset_pixels,
                          double *accum, void *workspace, size_t workspace_bytes,
                          void *stream) {
  if (num_rows <= 0 || num_cols <= 0 || num_slices <= 0)
    return fail(MBIR_ERR_INVALID, "image sizes must be positive");
  if (!params || !flat_image || !flat_error || !partition || !accum)
    return fail(MBIR_ERR_INVALID, "NULL argument");
  if (num_subsets <= 0 || subset_pixels <= 0)
    return fail(MBIR_ERR_INVALID, "denoiser pass needs at least one non-empty subset");
  if (!(params->sigma_x > 0.f) || !(params->fm_constant > 0.f) || !(params->T > 0.f))
    return fail(MBIR_ERR_INVALID, "sigma_x, T and fm_constant must be positive");
  const DenoiseWs w = denoise_layout(num_slices, subset_pixels, workspace);
  if (!workspace || workspace_bytes < w.bytes)
    return fail(MBIR_ERR_WORKSPACE, "denoiser workspace of %zu bytes < %zu needed",
                workspace_bytes, w.bytes);
  cudaStream_t st = as_stream(stream);
  const PdlScope pdl;
  cudaError_t e = cudaMemsetAsync(w.counter, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess)
    return fail(MBIR_ERR_CUDA, "denoiser counter reset failed: %s", cudaGetErrorString(e));
  const VcdScalars sc = make_scalars(*params);
  for (int k = 0; k < num_subsets; ++k) {
    const int64_t *pix = partition + (size_t)k * subset_pixels;
    tpre(st);
    launch(denoise_direction_kernel, w.blocks, kThreads, 0, st, (int)subset_pixels, num_slices,
           pix, num_rows, num_cols, flat_image, flat_error, sc, w.delta, w.prior, w.fwd);
    MBIR_CHECK_LAUNCH("denoise direction");
    tpre(st);
    launch(vcd_alpha_kernel, 1, kAlphaThreads, 0, st, w.prior, w.blocks, w.fwd, w.blocks, sc.fmc,
           sc.max_alpha, w.alpha, nullptr);
    MBIR_CHECK_LAUNCH("denoise alpha");
    tpre(st);
    launch(denoise_update_kernel, w.blocks, kThreads, 0, st, (int)subset_pixels, num_slices, pix,
           w.delta, w.alpha, flat_image, flat_error, w.l1, w.counter, accum);
    MBIR_CHECK_LAUNCH("denoise update");
  }
  return MBIR_OK;
}

size_t mbir_iteration_stats_workspace_size(void) {
  return align_up(sizeof(double) * 3 * kStatsMaxBlocks) + align_up(sizeof(double) * kStatsMaxBlocks);
}

int32_t mbir_iteration_stats(int32_t views, int32_t rows, int32_t channels, const void *error_sino,
                             const float *err_scale, const void *weights, const float *w_scale,
                             int32_t storage, const float *flat_recon, int64_t recon_count,
                             double *out, void *workspace, size_t workspace_bytes, void *stream) {
  if (views <= 0 || rows <= 0 || channels <= 0 || !error_sino || !err_scale || !out ||
      (weights && !w_scale) || (recon_count > 0 && !flat_recon))
    return fail(MBIR_ERR_INVALID, "bad statistics arguments");
  if (!workspace || workspace_bytes < mbir_iteration_stats_workspace_size())
    return fail(MBIR_ERR_WORKSPACE, "statistics need %zu workspace bytes",
                mbir_iteration_stats_workspace_size());
  cudaStream_t st = as_stream(stream);
  const int nb = stats_blocks();
  double *sp = static_cast<double *>(workspace);
  double *lp = reinterpret_cast<double *>(static_cast<char *>(workspace) +
                                          align_up(sizeof(double) * 3 * kStatsMaxBlocks));
  const int CR = rows * channels;
  switch (storage) {
    case MBIR_F32:
      tpre(st);
      stats_sino_kernel<float><<<nb, kThreads, 0, st>>>(views, CR, static_cast<const float *>(error_sino),
          err_scale, static_cast<const float *>(weights), w_scale, sp);
      break;
    case MBIR_BF16:
      tpre(st);
      stats_sino_kernel<__nv_bfloat16><<<nb, kThreads, 0, st>>>(views, CR,
          static_cast<const __nv_bfloat16 *>(error_sino), err_scale,
          static_cast<const __nv_bfloat16 *>(weights), w_scale, sp);
      break;
    case MBIR_F16:
      tpre(st);
      stats_sino_kernel<__half><<<nb, kThreads, 0, st>>>(views, CR, static_cast<const __half *>(error_sino),
          err_scale, static_cast<const __half *>(weights), w_scale, sp);
      break;
    default:
      return fail(MBIR_ERR_INVALID, "unknown storage dtype %d", storage);
  }
  MBIR_CHECK_LAUNCH("stats (sinogram)");
  tpre(st);
  stats_l1_kernel<<<nb, kThreads, 0, st>>>((size_t)std::max<int64_t>(recon_count, 0), flat_recon, lp);
  MBIR_CHECK_LAUNCH("stats (recon)");
  tpre(st);
  stats_finish_kernel<<<1, kThreads, 0, st>>>(nb, sp, nb, lp, out);
  MBIR_CHECK_LAUNCH("stats finish");
  return MBIR_OK;
}

}  // extern "C"

// ── back projection without allocation ─────────────────────────────────────
// Some callers cannot allocate device memory: an application whose device
// memory belongs to another allocator (a framework's caching pool, a
// pipeline with a fixed memory budget) has no way to hand this library a
// fresh workspace, and calling cudaMalloc itself would bypass that owner.
// For them mbir_back_project_noalloc keeps its scratch in the file-scope
// array below.  Every GPU that loads this library holds the array until the
// process exits; every call shares it, and each call overwrites what it
// uses, so nothing in it needs clearing, but calls that overlap on the GPU
// race on it.
constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;  // 32 MiB
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[kMaxDevices] = {};

// The scratch array's device address on the current device.  In host code
// the array's name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, once per device, with that device current.
int noalloc_scratch(void **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(MBIR_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(MBIR_ERR_INVALID, "device ordinal %d", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(MBIR_ERR_CUDA, "cudaGetSymbolAddress(static scratch): %s",
                  cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return MBIR_OK;
}
}  // namespace

extern "C" int32_t mbir_back_project_noalloc(const mbir_geometry *geom,
                                             const float *view_params, int32_t view_start,
                                             int32_t view_count, const float *sino,
                                             int32_t sino_layout,
                                             const int64_t *pixel_indices, int64_t num_pixels,
                                             int32_t coeff_power, int32_t slice_start,
                                             int32_t band_len, float *out, void *stream) {
  // Arguments first, so that a bad size reports itself as such and not as a
  // scratch overflow.
  int rc = validate_geometry(geom);
  if (rc) return rc;
  if (view_start < 0 || view_count < 0 || view_start + view_count > geom->num_views)
    return fail(MBIR_ERR_INVALID, "view range [%d, %d) outside [0, %d)", view_start,
                view_start + view_count, geom->num_views);
  if (sino_layout == MBIR_LAYOUT_VRC && view_count > 0) {
    const size_t need = align_up((size_t)view_count * geom->num_det_rows *
                                 geom->num_det_channels * sizeof(float));
    if (need > kNoAllocScratchBytes)
      return fail(MBIR_ERR_WORKSPACE,
                  "a (views, rows, channels) sinogram of %zu bytes exceeds the %zu-byte static "
                  "scratch of mbir_back_project_noalloc; pass the channel-major layout or "
                  "use mbir_back_project with a workspace", need, kNoAllocScratchBytes);
  }
  void *scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  return mbir_back_project(geom, view_params, view_start, view_count, sino, sino_layout,
                           pixel_indices, num_pixels, coeff_power, slice_start, band_len, out,
                           scratch, kNoAllocScratchBytes, stream);
}
