// VCD subset-step kernels for sm_100a.
//
// One subset update (tomography_model.py:2508-2657) runs as a short chain of
// launches on one stream, with no host synchronization:
//   1. gradient      back projection of (w * e) at the subset's cylinders,
//                    view-chunked partials (projectors.cuh)
//   2. direction     chunk reduction + qGGMRF surrogate gradient/Hessian
//                    (qggmrf.py:77-183) + the preconditioned direction
//                    (tomography_model.py:54-57) + prior line-term partials
//   2'. DC damping   (cone) per-slice H^-1-weighted gradient means and the
//                    damped direction (cone_beam.py:48-55)
//   3. forward       A delta with the line-search reductions fused into the
//                    epilogue (sum w e Ad, sum w Ad^2) and Ad stored in the
//                    storage precision
//   4. alpha         one CTA: FP64 reduction of all partials, the clamped
//                    step (tomography_model.py:2612-2617)
//   5. update        recon += alpha delta with per-slice sum of squares and
//                    ell1 (the last CTA folds them into the accumulators),
//                    then e -= alpha Ad
// Every reduction is a fixed-order tree over per-CTA partials, so a subset
// update is bit-reproducible run to run.
#pragma once

#include "projectors.cuh"

namespace mbir {

constexpr float kF32Eps = 1.1920928955078125e-07f;

struct VcdScalars {
  float fmc;        // 1 / sigma_y^2
  float a_min;      // T * sigma_x * eps_f32
  float t_sx;       // T * sigma_x
  float q_minus_p;  // q - p
  float p_minus_2;  // p - 2
  float two_sx_p;   // 2 * sigma_x ** p
  float q_over_p;   // q / p
  float two_b[6];   // 2 * b[j]  (get_2_b_tilde's b_for_delta * 2.0)
  float b[6];
  float max_alpha;
  float prox_c;        // 1 / sigma_prox^2 (proximal-map prior)
  const float *prox;   // proximal-map prior mean, (N*N, S); NULL: qGGMRF prior
};

inline VcdScalars make_scalars(const mbir_vcd_params &p) {
  VcdScalars s;
  s.fmc = p.fm_constant;
  s.a_min = (float)((double)p.T * (double)p.sigma_x * 1.1920928955078125e-07);
  s.t_sx = (float)((double)p.T * (double)p.sigma_x);
  s.q_minus_p = (float)((double)p.q - (double)p.p);
  s.p_minus_2 = (float)((double)p.p - 2.0);
  s.two_sx_p = (float)(2.0 * pow((double)p.sigma_x, (double)p.p));
  s.q_over_p = (float)((double)p.q / (double)p.p);
  for (int j = 0; j < 6; ++j) {
    s.b[j] = p.b[j];
    s.two_b[j] = (float)((double)p.b[j] * 2.0);
  }
  s.max_alpha = p.max_alpha;
  s.prox_c = p.prox_constant;
  s.prox = p.prox_input;
  return s;
}

// b_tilde_by_definition (qggmrf.py:35-57) without the factor b * 2.
__device__ __forceinline__ float b_tilde(float delta, const VcdScalars &s) {
  const float ad = fmaxf(fabsf(delta), s.a_min);
  const float ds = __fdiv_rn(ad, s.t_sx);
  const float dqp = powf(ds, s.q_minus_p);
  // x^0 is exactly 1 for every x, so the default p = 2 skips the call.
  const float dp2 = s.p_minus_2 == 0.f ? 1.f : powf(ad, s.p_minus_2);
  float num = __fdiv_rn(dp2, s.two_sx_p);
  num = __fmul_rn(__fmul_rn(num, dqp), __fadd_rn(s.q_over_p, dqp));
  const float den = __fadd_rn(1.f, dqp);
  return __fdiv_rn(num, __fmul_rn(den, den));
}

// Block-wide sum of two doubles; returns the totals in thread 0.
__device__ __forceinline__ void block_sum2(double &a, double &b) {
  __shared__ double sa[32], sb[32];
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) {
    sa[warp] = a;
    sb[warp] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      ta += sa[w];
      tb += sb[w];
    }
    a = ta;
    b = tb;
  }
}

// qGGMRF surrogate gradient and Hessian of voxel (pixel, l) (qggmrf.py:
// 117-183): the slice term with reflected ends, then the 4 clamped in-plane
// neighbours.
__device__ __forceinline__ void qggmrf_terms(const float *__restrict__ flat, int pixel, int l,
                                             int S, int NR, int NC, const VcdScalars &sc,
                                             float &g_p, float &h_p) {
  const float *cyl = flat + (size_t)pixel * S;
  const float xs = cyl[l];
  const float dp = (l + 1 < S) ? __fsub_rn(cyl[l + 1], xs) : 0.f;  // delta[l+1]
  const float dm = (l > 0) ? __fsub_rn(xs, cyl[l - 1]) : 0.f;      // delta[l]
  const float bt_p = __fmul_rn(2.f, b_tilde(dp, sc));
  const float bt_m = __fmul_rn(2.f, b_tilde(dm, sc));
  g_p = __fadd_rn(__fmul_rn(-sc.b[4], __fmul_rn(bt_p, dp)),
                  __fmul_rn(sc.b[5], __fmul_rn(bt_m, dm)));
  h_p = __fadd_rn(__fmul_rn(sc.b[4], bt_p), __fmul_rn(sc.b[5], bt_m));
  const int row = pixel / NC, col = pixel - (pixel / NC) * NC;
  const int dr[4] = {1, -1, 0, 0}, dc[4] = {0, 0, 1, -1};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int rr = min(max(row + dr[k], 0), NR - 1);
    const int cc = min(max(col + dc[k], 0), NC - 1);
    const float d = __fsub_rn(xs, flat[((size_t)rr * NC + cc) * S + l]);
    const float w = __fmul_rn(sc.two_b[k], b_tilde(d, sc));
    g_p = __fadd_rn(g_p, __fmul_rn(w, d));
    h_p = __fadd_rn(h_p, w);
  }
}

// ── 2. direction ─────────────────────────────────────────────────────────
// Thread per (pixel p, slice l).  DC = 0: writes delta and the prior
// line-term partials.  DC = 1: writes g, 1/h, g_p, h_p for the damping pass.
template <bool DC>
__device__ __forceinline__ void vcd_direction_kernel_body(int P, int S, const int64_t *__restrict__ pix, int NR, int NC,
                     const float *__restrict__ part, int nchunks,
                     const float *__restrict__ flat, const float *__restrict__ H,
                     VcdScalars sc, float *__restrict__ delta, float *__restrict__ gbuf,
                     float *__restrict__ hinv, float *__restrict__ gpbuf,
                     float *__restrict__ hpbuf, double *__restrict__ partials) {
  MBIR_PDL_ENTRY();
  const size_t n = (size_t)P * S;
  const size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x;
  double pl = 0.0, pq = 0.0;
  if (i < n) {
    const int p = (int)(i / S), l = (int)(i - (size_t)p * S);
    float bp = 0.f;
#pragma unroll 8
    for (int c = 0; c < nchunks; ++c) bp += part[(size_t)c * n + i];
    const int pixel = (int)pix[p];
    const float g_f = __fmul_rn(-sc.fmc, bp);
    const float h_f = __fmul_rn(sc.fmc, H[(size_t)pixel * S + l]);
    const float *cyl = flat + (size_t)pixel * S;
    const float xs = cyl[l];
    float g_p, h_p;
    if (sc.prox != nullptr) {
      // Proximal-map prior (qggmrf.py:186-206): gradient (x - v) / sigma^2,
      // Hessian 1 / sigma^2.
      g_p = __fmul_rn(sc.prox_c, __fsub_rn(xs, sc.prox[(size_t)pixel * S + l]));
      h_p = sc.prox_c;
    } else {
      qggmrf_terms(flat, pixel, l, S, NR, NC, sc, g_p, h_p);
    }
    if (!DC) {
      const float dl = -__fdiv_rn(__fadd_rn(g_f, g_p), __fadd_rn(h_f, h_p));
      delta[i] = dl;
      pl = (double)__fmul_rn(g_p, dl);
      pq = (double)__fmul_rn(__fmul_rn(h_p, dl), dl);
    } else {
      gbuf[i] = __fadd_rn(g_f, g_p);
      hinv[i] = __fdiv_rn(1.f, __fadd_rn(h_f, h_p));
      gpbuf[i] = g_p;
      hpbuf[i] = h_p;
    }
  }
  if (!DC) {
    block_sum2(pl, pq);
    if (threadIdx.x == 0) {
      partials[2 * blockIdx.x] = pl;
      partials[2 * blockIdx.x + 1] = pq;
    }
  }
}

template <bool DC>
__global__ void __launch_bounds__(kThreads)

vcd_direction_kernel(int P, int S, const int64_t *__restrict__ pix, int NR, int NC,
                     const float *__restrict__ part, int nchunks,
                     const float *__restrict__ flat, const float *__restrict__ H,
                     VcdScalars sc, float *__restrict__ delta, float *__restrict__ gbuf,
                     float *__restrict__ hinv, float *__restrict__ gpbuf,
                     float *__restrict__ hpbuf, double *__restrict__ partials) {
  vcd_direction_kernel_body<DC>(P, S, pix, NR, NC, part, nchunks, flat, H, sc, delta, gbuf, hinv, gpbuf, hpbuf, partials);
}

// ── 2'. DC damping ───────────────────────────────────────────────────────
// Per-slice sums over pixel chunks: part[chunk][l] = (sum h^-1 g, sum h^-1).
// A CTA of (32 slices, 8 groups) covers one chunk of kDcChunk pixels:
// group y sums the pixels y, y + 8, ... of the chunk with all its loads in
// flight, then the 8 group sums fold in a fixed order.  The pixel chunks run
// along grid x (up to 2^31 - 1 of them), the 32-slice blocks along grid y.
constexpr int kDcGroups = 8;
constexpr int kDcPerGroup = 4;                       // pixels per group
constexpr int kDcChunk = kDcGroups * kDcPerGroup;    // pixels per chunk
static_assert(kDcChunk == 32, "one DC-sum CTA covers 32 pixels");

__device__ __forceinline__ void vcd_dc_sums_kernel_body(int P, int S, const float *__restrict__ gbuf,
                   const float *__restrict__ hinv, double *__restrict__ part) {
  MBIR_PDL_ENTRY();
  __shared__ double s_num[kDcGroups][32], s_den[kDcGroups][32];
  constexpr int U = kDcPerGroup;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int l = blockIdx.y * 32 + tx;
  const int chunk = blockIdx.x;
  const int p0 = chunk * kDcChunk, p1 = min(P, p0 + kDcChunk);
  double num = 0.0, den = 0.0;
  if (l < S) {
    float hv[U], gv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int p = p0 + ty + kDcGroups * u;
      const size_t i = (size_t)p * S + l;
      hv[u] = p < p1 ? hinv[i] : 0.f;
      gv[u] = p < p1 ? gbuf[i] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (p0 + ty + kDcGroups * u < p1) {
        num += (double)__fmul_rn(hv[u], gv[u]);
        den += (double)hv[u];
      }
    }
  }
  s_num[ty][tx] = num;
  s_den[ty][tx] = den;
  __syncthreads();
  if (ty == 0 && l < S) {
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int k = 0; k < kDcGroups; ++k) {
      a += s_num[k][tx];
      b += s_den[k][tx];
    }
    part[((size_t)chunk * S + l) * 2] = a;
    part[((size_t)chunk * S + l) * 2 + 1] = b;
  }
}

__global__ void __launch_bounds__(32 * kDcGroups)

vcd_dc_sums_kernel(int P, int S, const float *__restrict__ gbuf,
                   const float *__restrict__ hinv, double *__restrict__ part) {
  vcd_dc_sums_kernel_body(P, S, gbuf, hinv, part);
}

// delta = -(g - (1 - s_l) * gbar_l) * h^-1, plus the prior line-term partials.
// A CTA of (32 slices, 8 rows) owns slices [32 y, 32 y + 32) of the pixels
// [kDcDirPixels x, kDcDirPixels (x + 1)): it folds its slices' chunk sums
// once (row r takes the chunks r, r + 8, ...; the 8 row sums fold in a fixed
// order), then row r updates the pixels r, r + 8, ... of its block.  The
// CTA's prior partials go to slot y * gridDim.x + x.
constexpr int kDcDirPixels = 64;

__device__ __forceinline__ void vcd_dc_direction_kernel_body(int P, int S, int nchunks, const double *__restrict__ sums,
                        const float *__restrict__ s_prof, const float *__restrict__ gbuf,
                        const float *__restrict__ hinv, const float *__restrict__ gpbuf,
                        const float *__restrict__ hpbuf, float *__restrict__ delta,
                        double *__restrict__ partials) {
  MBIR_PDL_ENTRY();
  __shared__ double s_a[8][32], s_b[8][32];
  __shared__ float s_fac[32];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int l = blockIdx.y * 32 + tx;
  double num = 0.0, den = 0.0;
  if (l < S) {
    for (int c = ty; c < nchunks; c += 8) {
      num += sums[((size_t)c * S + l) * 2];
      den += sums[((size_t)c * S + l) * 2 + 1];
    }
  }
  s_a[ty][tx] = num;
  s_b[ty][tx] = den;
  __syncthreads();
  if (ty == 0) {
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      a += s_a[k][tx];
      b += s_b[k][tx];
    }
    // (1 - s_l) * gbar_l, gbar_l = sum h^-1 g / sum h^-1
    s_fac[tx] = l < S ? __fmul_rn(__fsub_rn(1.f, s_prof[l]), (float)(a / b)) : 0.f;
  }
  __syncthreads();
  double pl = 0.0, pq = 0.0;
  if (l < S) {
    const float damp = s_fac[tx];
    const int p1 = min(P, (int)(blockIdx.x + 1) * kDcDirPixels);
    for (int p = blockIdx.x * kDcDirPixels + ty; p < p1; p += 8) {
      const size_t i = (size_t)p * S + l;
      const float dl = __fmul_rn(-__fsub_rn(gbuf[i], damp), hinv[i]);
      delta[i] = dl;
      const float g_p = gpbuf[i], h_p = hpbuf[i];
      pl += (double)__fmul_rn(g_p, dl);
      pq += (double)__fmul_rn(__fmul_rn(h_p, dl), dl);
    }
  }
  // fixed-order CTA reduction: the 8 rows of each slice lane, then the lanes
  __syncthreads();
  s_a[ty][tx] = pl;
  s_b[ty][tx] = pq;
  __syncthreads();
  if (ty == 0) {
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      a += s_a[k][tx];
      b += s_b[k][tx];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if (tx == 0) {
      const size_t slot = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
      partials[2 * slot] = a;
      partials[2 * slot + 1] = b;
    }
  }
}

__global__ void __launch_bounds__(256)

vcd_dc_direction_kernel(int P, int S, int nchunks, const double *__restrict__ sums,
                        const float *__restrict__ s_prof, const float *__restrict__ gbuf,
                        const float *__restrict__ hinv, const float *__restrict__ gpbuf,
                        const float *__restrict__ hpbuf, float *__restrict__ delta,
                        double *__restrict__ partials) {
  vcd_dc_direction_kernel_body(P, S, nchunks, sums, s_prof, gbuf, hinv, gpbuf, hpbuf, delta, partials);
}

// Grid-wide "last CTA" election: every CTA calls it once after writing its
// partials; it returns true in exactly one CTA (the last to arrive), which
// then sees every other CTA's writes.  The counter counts `total` arrivals
// (possibly over several launches in stream order) and the elected CTA
// resets it to zero.
__device__ __forceinline__ bool last_cta(unsigned int *counter, unsigned int total) {
  __shared__ bool s_last;
  __threadfence();  // this thread's partial writes, before the arrival
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(counter, 1u) == total - 1u;
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last;
}

// ── 3. forward epilogue: line search + Ad store ───────────────────────────
// The per-view scale is a power of two, so Ad / scale is formed exactly as
// Ad * (1 / scale).
template <typename T>
struct LineSearchEpi {
  static constexpr bool kViewFastest = false;  // binned grids: channel blocks on x
  const T *e;
  const float *es;
  const T *w;
  const float *wsc;
  T *ad;
  int C, R;
  double *partials;
  int with_sums;
  double fl, fq;
  float scale, inv_scale, wscale;
  __device__ __forceinline__ bool channel_fastest() const { return false; }
  __device__ __forceinline__ void begin(int v) {
    fl = 0.0;
    fq = 0.0;
    scale = __ldg(es + v);
    inv_scale = 1.f / scale;
    wscale = w != nullptr ? __ldg(wsc + v) : 1.f;
  }
  // Each warp sends the 128-byte lines of its 32 rows x ncb channels of e
  // (and w) toward L2 (lane j: channel j).
  __device__ __forceinline__ void prefetch(int v, int c0, int ncb) {
    if (!with_sums) return;
    const int lane = threadIdx.x & 31, m0 = threadIdx.x - lane;
    if (lane < ncb && m0 < R) {
      const size_t i = ((size_t)v * C + c0 + lane) * R + m0;
      prefetch_l2(e + i);
      if (w != nullptr) prefetch_l2(w + i);
    }
  }
  __device__ __forceinline__ void cell(int v, int c, int m, float val) {
    const size_t i = ((size_t)v * C + c) * R + m;
    const T stored = from_f32<T>(__fmul_rn(val, inv_scale));
    ad[i] = stored;
    if (!with_sums) return;
    const float adv = __fmul_rn(to_f32(stored), scale);
    const float ev = __fmul_rn(to_f32(e[i]), scale);
    if (w != nullptr) {
      const float wv = __fmul_rn(to_f32(w[i]), wscale);
      fl += (double)__fmul_rn(__fmul_rn(wv, ev), adv);
      fq += (double)__fmul_rn(__fmul_rn(adv, adv), wv);
    } else {
      fl += (double)__fmul_rn(ev, adv);
      fq += (double)__fmul_rn(adv, adv);
    }
  }
  // A row's cells at channels c0 .. c0 + ncb - 1 at once: every load of e
  // and w goes out before the first store of Ad, which the compiler could
  // not otherwise move past (the pointers may alias as far as it knows).
  // The row's products are summed in FP32 (at most N terms, in channel
  // order) and added to the FP64 sums once per row.
  template <int N>
  __device__ __forceinline__ void cells(int v, int c0, int ncb, int m, const float (&acc)[N]) {
    const size_t i0 = ((size_t)v * C + c0) * R + m;
    float ev[N], wv[N];
#pragma unroll
    for (int j = 0; j < N; ++j) {
      ev[j] = 0.f;
      wv[j] = 0.f;
      if (with_sums && j < ncb) {
        ev[j] = to_f32(e[i0 + (size_t)j * R]);
        if (w != nullptr) wv[j] = to_f32(w[i0 + (size_t)j * R]);
      }
    }
    float rl = 0.f, rq = 0.f;
#pragma unroll
    for (int j = 0; j < N; ++j) {
      if (j < ncb) {
        const T stored = from_f32<T>(__fmul_rn(acc[j], inv_scale));
        ad[i0 + (size_t)j * R] = stored;
        if (with_sums) {
          const float adv = __fmul_rn(to_f32(stored), scale);
          const float evs = __fmul_rn(ev[j], scale);
          if (w != nullptr) {
            const float wvs = __fmul_rn(wv[j], wscale);
            rl = __fadd_rn(rl, __fmul_rn(__fmul_rn(wvs, evs), adv));
            rq = __fadd_rn(rq, __fmul_rn(__fmul_rn(adv, adv), wvs));
          } else {
            rl = __fadd_rn(rl, __fmul_rn(evs, adv));
            rq = __fadd_rn(rq, __fmul_rn(adv, adv));
          }
        }
      }
    }
    fl += (double)rl;
    fq += (double)rq;
  }
  // Four consecutive rows m0 .. m0 + 3 of channels c0 .. c0 + ncb - 1 (R and
  // m0 multiples of 4, so each channel's four cells are one aligned 16-byte
  // (FP32) or 8-byte (16-bit) access).  Channel j's four sums are acc[j *
  // stride]; four channels' loads go out before their stores.
  __device__ __forceinline__ void cells4(int v, int c0, int ncb, int m0,
                                         const float4 *__restrict__ acc, int stride) {
    const size_t i0 = ((size_t)v * C + c0) * R + m0;
    for (int g0 = 0; g0 < ncb; g0 += 4) {
      float ev[4][4], wv[4][4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int k = 0; k < 4; ++k) ev[j][k] = wv[j][k] = 0.f;
        if (with_sums && g0 + j < ncb) {
          load4(e + i0 + (size_t)(g0 + j) * R, ev[j]);
          if (w != nullptr) load4(w + i0 + (size_t)(g0 + j) * R, wv[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (g0 + j < ncb) {
          const float4 a4 = acc[(g0 + j) * stride];
          const float a[4] = {a4.x, a4.y, a4.z, a4.w};
          T st[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) st[k] = from_f32<T>(__fmul_rn(a[k], inv_scale));
          store4(ad + i0 + (size_t)(g0 + j) * R, st);
          if (with_sums) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const float adv = __fmul_rn(to_f32(st[k]), scale);
              const float evs = __fmul_rn(ev[j][k], scale);
              if (w != nullptr) {
                const float wvs = __fmul_rn(wv[j][k], wscale);
                fl += (double)__fmul_rn(__fmul_rn(wvs, evs), adv);
                fq += (double)__fmul_rn(__fmul_rn(adv, adv), wvs);
              } else {
                fl += (double)__fmul_rn(evs, adv);
                fq += (double)__fmul_rn(adv, adv);
              }
            }
          }
        }
      }
    }
  }
  // A tile that no pixel reaches: A delta is zero there and is not stored
  // (the sinogram update skips untouched tiles).
  __device__ __forceinline__ void empty_tile(int, int, int) {}
  __device__ __forceinline__ void end(int slot) {
    if (!with_sums) return;
    block_sum2(fl, fq);
    if (threadIdx.x == 0) {
      partials[2 * slot] = fl;
      partials[2 * slot + 1] = fq;
    }
  }
};

// Refresh epilogue: e = (y - A x) / scale[v] stored in T, with y the FP32
// measured sinogram in the same (V, C, R) layout.  Re-forming the error
// sinogram from y bounds the drift that in-place 16-bit updates accumulate.
template <typename T>
struct RefreshEpi {
  static constexpr bool kViewFastest = true;  // binned grids: views on x
  const float *y;
  T *e;
  const float *es;
  int C, R;
  float inv_scale;
  __device__ __forceinline__ bool channel_fastest() const { return false; }
  __device__ __forceinline__ void begin(int v) { inv_scale = 1.f / __ldg(es + v); }
  __device__ __forceinline__ void prefetch(int, int, int) {}
  __device__ __forceinline__ void cell(int v, int c, int m, float val) {
    const size_t i = ((size_t)v * C + c) * R + m;
    e[i] = from_f32<T>(__fmul_rn(__fsub_rn(__ldg(y + i), val), inv_scale));
  }
  template <int N>
  __device__ __forceinline__ void cells(int v, int c0, int ncb, int m, const float (&acc)[N]) {
    const size_t i0 = ((size_t)v * C + c0) * R + m;
    float yv[N];
#pragma unroll
    for (int j = 0; j < N; ++j) yv[j] = j < ncb ? __ldg(y + i0 + (size_t)j * R) : 0.f;
#pragma unroll
    for (int j = 0; j < N; ++j)
      if (j < ncb)
        e[i0 + (size_t)j * R] = from_f32<T>(__fmul_rn(__fsub_rn(yv[j], acc[j]), inv_scale));
  }
  // Rows m0 .. m0 + 3 of channels c0 .. c0 + ncb - 1 (channel j's four sums
  // in acc[j * stride]).
  __device__ __forceinline__ void cells4(int v, int c0, int ncb, int m0,
                                         const float4 *__restrict__ acc, int stride) {
    for (int j = 0; j < ncb; ++j) {
      const float4 a = acc[j * stride];
      const float q[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (m0 + k < R) cell(v, c0 + j, m0 + k, q[k]);
    }
  }
  // A tile that no pixel reaches: A x is zero, so e = y / scale there.
  __device__ __forceinline__ void empty_tile(int v, int c0, int ncb) {
    const float inv = 1.f / __ldg(es + v);
    for (int i = threadIdx.x; i < ncb * R; i += blockDim.x) {
      const size_t k = ((size_t)v * C + c0 + i / R) * R + i % R;
      e[k] = from_f32<T>(__fmul_rn(__ldg(y + k), inv));
    }
  }
  __device__ __forceinline__ void end(int) {}
};

// ── 4. alpha ─────────────────────────────────────────────────────────────
// One CTA of kAlphaThreads.  prior: np pairs (pl, pq); fwd: nf pairs (fl, fq).
constexpr int kAlphaThreads = 1024;

__device__ __forceinline__ void vcd_alpha_kernel_body(const double *__restrict__ prior, int np, const double *__restrict__ fwd, int nf,
                 float fmc, float max_alpha, float *__restrict__ alpha_out,
                 float *__restrict__ alpha_user) {
  MBIR_PDL_ENTRY();
  double pl = 0.0, pq = 0.0, fl = 0.0, fq = 0.0;
  const double2 *pr2 = reinterpret_cast<const double2 *>(prior);
  const double2 *fw2 = reinterpret_cast<const double2 *>(fwd);
#pragma unroll 4
  for (int i = threadIdx.x; i < np; i += kAlphaThreads) {
    const double2 v = pr2[i];
    pl += v.x;
    pq += v.y;
  }
#pragma unroll 4
  for (int i = threadIdx.x; i < nf; i += kAlphaThreads) {
    const double2 v = fw2[i];
    fl += v.x;
    fq += v.y;
  }
  block_sum2(pl, pq);
  block_sum2(fl, fq);
  if (threadIdx.x == 0) {
    // tomography_model.py:2612-2617, with the sums in FP64.
    const double num = (double)fmc * fl - pl;
    const double den = (double)fmc * fq + pq + (double)kF32Eps;
    double a = num / den;
    a = fmin(fmax(a, (double)kF32Eps), (double)max_alpha);
    alpha_out[0] = (float)a;
    if (alpha_user) alpha_user[0] = (float)a;
  }
}

__global__ void __launch_bounds__(kAlphaThreads)

vcd_alpha_kernel(const double *__restrict__ prior, int np, const double *__restrict__ fwd, int nf,
                 float fmc, float max_alpha, float *__restrict__ alpha_out,
                 float *__restrict__ alpha_user) {
  vcd_alpha_kernel_body(prior, np, fwd, nf, fmc, max_alpha, alpha_out, alpha_user);
}

// Positivity: delta = max(-x / (alpha + eps), delta) (tomography_model.py:2624-2633).
__device__ __forceinline__ void vcd_positivity_kernel_body(int P, int S, const int64_t *__restrict__ pix,
                                      const float *__restrict__ flat,
                                      const float *__restrict__ alpha, float *__restrict__ delta) {
  MBIR_PDL_ENTRY();
  const size_t n = (size_t)P * S;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = (int)(i / S), l = (int)(i - (size_t)p * S);
  const float pos_c = __fdiv_rn(1.f, __fadd_rn(alpha[0], kF32Eps));
  const float x = flat[(size_t)pix[p] * S + l];
  delta[i] = fmaxf(__fmul_rn(-pos_c, x), delta[i]);
}

__global__ void 
vcd_positivity_kernel(int P, int S, const int64_t *__restrict__ pix,
                                      const float *__restrict__ flat,
                                      const float *__restrict__ alpha, float *__restrict__ delta) {
  vcd_positivity_kernel_body(P, S, pix, flat, alpha, delta);
}

// ── 5. update ────────────────────────────────────────────────────────────
constexpr int kUpdPix = 8;  // pixels per load batch of the recon update

// One CTA (bx, by) of the pixel update over a (gx, gy) grid: x += alpha
// delta at the subset's voxels, the per-slice sums of squares and the l1
// partials; the last CTA to arrive folds them into accum.
__device__ __forceinline__ void pixel_update_cta(int P, int S, int pchunk,
                                                 const int64_t *__restrict__ pix,
                                                 const float *__restrict__ delta,
                                                 const float *__restrict__ alpha,
                                                 float *__restrict__ flat,
                                                 double *__restrict__ sq_part,
                                                 double *__restrict__ l1_part,
                                                 unsigned int *__restrict__ counter,
                                                 double *__restrict__ accum, int bx, int by,
                                                 int gx, int gy) {
  const int l = by * kThreads + threadIdx.x;
  const int chunk = bx;
  const int p0 = chunk * pchunk, p1 = min(P, p0 + pchunk);
  const float a = alpha[0];
  double sq = 0.0, l1 = 0.0;
  if (l < S) {
    // The pixels of a subset are distinct, so all kUpdPix loads of the
    // cylinders' voxels go out before the first store.
    for (int pb = p0; pb < p1; pb += kUpdPix) {
      float ds[kUpdPix], xv[kUpdPix];
      float *xp[kUpdPix];
#pragma unroll
      for (int u = 0; u < kUpdPix; ++u) {
        const int p = min(pb + u, P - 1);
        ds[u] = __fmul_rn(a, delta[(size_t)p * S + l]);
        xp[u] = flat + (size_t)pix[p] * S + l;
        xv[u] = *xp[u];
      }
#pragma unroll
      for (int u = 0; u < kUpdPix; ++u) {
        if (pb + u < p1) {
          *xp[u] = __fadd_rn(xv[u], ds[u]);
          sq += (double)__fmul_rn(ds[u], ds[u]);
          l1 += (double)fabsf(ds[u]);
        }
      }
    }
    sq_part[(size_t)chunk * S + l] = sq;
  }
  double dummy = 0.0;
  block_sum2(l1, dummy);
  if (threadIdx.x == 0) l1_part[(size_t)by * gx + chunk] = l1;
  // The last CTA folds all partials into the accumulators (fixed order):
  // accum[0] += ell1, accum[1] += alpha, accum[2 + l] += sum_p ds^2.
  if (last_cta(counter, gx * gy)) {
    const int nchunks = gx, nl1 = gx * gy;
    for (int ls = threadIdx.x; ls < S; ls += blockDim.x) {
      double s2 = 0.0;
#pragma unroll 8
      for (int c = 0; c < nchunks; ++c) s2 += __ldcg(sq_part + (size_t)c * S + ls);
      accum[2 + ls] += s2;
    }
    double t1 = 0.0, t2 = 0.0;
#pragma unroll 4
    for (int i = threadIdx.x; i < nl1; i += blockDim.x) t1 += __ldcg(l1_part + i);
    block_sum2(t1, t2);
    if (threadIdx.x == 0) {
      accum[0] += t1;
      accum[1] += (double)alpha[0];
      *counter = 0u;
    }
  }
}

// Recon scatter-add over a (pixel chunk, slice block) tile; per-slice sum of
// squares and ell1 partials.
__global__ void __launch_bounds__(kThreads)
vcd_pixel_update_kernel(int P, int S, int pchunk, const int64_t *__restrict__ pix,
                        const float *__restrict__ delta, const float *__restrict__ alpha,
                        float *__restrict__ flat, double *__restrict__ sq_part,
                        double *__restrict__ l1_part, unsigned int *__restrict__ counter,
                        double *__restrict__ accum) {
  MBIR_PDL_ENTRY();
  pixel_update_cta(P, S, pchunk, pix, delta, alpha, flat, sq_part, l1_part, counter, accum,
                   blockIdx.x, blockIdx.y, gridDim.x, gridDim.y);
}

// e -= alpha * Ad over the whole resident sinogram (both share the per-view
// scale, so the update is scale-free in the stored units).
template <typename T>
__global__ void vcd_sino_update_kernel(size_t n, const float *__restrict__ alpha,
                                       T *__restrict__ e, const T *__restrict__ ad) {
  MBIR_PDL_ENTRY();
  const float a = alpha[0];
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float ev = to_f32(e[i]);
    const float dv = to_f32(ad[i]);
    e[i] = from_f32<T>(__fsub_rn(ev, __fmul_rn(a, dv)));
  }
}

template <>
__global__ void vcd_sino_update_kernel<float>(size_t n, const float *__restrict__ alpha,
                                              float *__restrict__ e,
                                              const float *__restrict__ ad) {
  MBIR_PDL_ENTRY();
  const float a = alpha[0];
  const size_t n4 = n / 4;
  float4 *e4 = reinterpret_cast<float4 *>(e);
  const float4 *d4 = reinterpret_cast<const float4 *>(ad);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4;
       i += (size_t)gridDim.x * blockDim.x) {
    float4 ev = e4[i];
    const float4 dv = d4[i];
    ev.x = __fsub_rn(ev.x, __fmul_rn(a, dv.x));
    ev.y = __fsub_rn(ev.y, __fmul_rn(a, dv.y));
    ev.z = __fsub_rn(ev.z, __fmul_rn(a, dv.z));
    ev.w = __fsub_rn(ev.w, __fmul_rn(a, dv.w));
    e4[i] = ev;
  }
  for (size_t i = n4 * 4 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    e[i] = __fsub_rn(e[i], __fmul_rn(a, ad[i]));
}

// Tiles [bg * tpc, bg * tpc + tpc) of view v (channel blocks of CB channels)
// of the touched-tile sinogram update: e -= alpha * Ad over each tile's CB
// consecutive channels (one contiguous run of CB * R cells), skipping the
// tiles the binned forward marked as not reached.  Short detectors give a
// CTA several tiles (tpc > 1) so that it still moves a few thousand cells.
template <typename T>
__device__ __forceinline__ void sino_tile_cta(int C, int R, int CB,
                                              const unsigned char *__restrict__ touched,
                                              const float *__restrict__ alpha, T *__restrict__ e,
                                              const T *__restrict__ ad, int bg, int v, int nblk,
                                              int tpc) {
  const float a = alpha[0];
  const int b_end = min(nblk, (bg + 1) * tpc);
  for (int b = bg * tpc; b < b_end; ++b) {
    if (!touched[(size_t)v * nblk + b]) continue;
    const int c0 = b * CB;
    const int n = min(CB, C - c0) * R;
    const size_t base = ((size_t)v * C + c0) * R;
    T *et = e + base;
    const T *dt = ad + base;
    constexpr int U = 4;
    for (int i0 = threadIdx.x; i0 < n; i0 += 256 * U) {
      float ev[U], dv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int i = i0 + 256 * u;
        ev[u] = i < n ? to_f32(et[i]) : 0.f;
        dv[u] = i < n ? to_f32(dt[i]) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int i = i0 + 256 * u;
        if (i < n) et[i] = from_f32<T>(__fsub_rn(ev[u], __fmul_rn(a, dv[u])));
      }
    }
  }
}

// The bins of the next subset of a partition pass (cone_bin_kernel's
// arguments for view chunk 0).
struct TailBins {
  Geo g;
  const float *vp;
  const int64_t *pix;
  int P;
  ConeFwdRec *recs;
  int *list, *offs;
};

// The work of a binned subset step after alpha, in one launch: CTAs
// [0, nbin) bin the next subset of a partition pass (cone_bin_view, one
// view each; nbin = 0 when there is none), the next ux * uy CTAs update the
// recon (pixel_update_cta) and the rest update the sinogram's touched tiles
// (sino_tile_cta, ceil(nblk / tpc) x V).  The three roles share no buffer, so the
// latency-bound binning and recon update run under the HBM-bound tile
// update.  Dynamic shared memory: the binning's key counters.  Six CTAs
// per SM (at most 40 registers) keep enough of the tile update's loads in
// flight to hold the copy bandwidth.
template <typename T>
__device__ __forceinline__ void vcd_tail_kernel_body(int nbin, TailBins tb, int P, int S, int pchunk, const int64_t *__restrict__ pix,
                const float *__restrict__ delta, const float *__restrict__ alpha,
                float *__restrict__ flat, double *__restrict__ sq_part,
                double *__restrict__ l1_part, unsigned int *__restrict__ counter,
                double *__restrict__ accum, int ux, int uy, int C, int R, int CB,
                const unsigned char *__restrict__ touched, T *__restrict__ e,
                const T *__restrict__ ad, int nblk, int tpc) {
  MBIR_PDL_ENTRY();
  extern __shared__ int tail_sm[];
  int b = blockIdx.x;
  if (b < nbin) {
    cone_bin_view(tb.g, tb.vp, 0, b, tb.pix, tb.P, 0, tb.recs, tb.list, tb.offs, tail_sm);
    return;
  }
  b -= nbin;
  if (b < ux * uy) {
    pixel_update_cta(P, S, pchunk, pix, delta, alpha, flat, sq_part, l1_part, counter, accum,
                     b % ux, b / ux, ux, uy);
    return;
  }
  b -= ux * uy;
  const int ngrp = (nblk + tpc - 1) / tpc;
  sino_tile_cta<T>(C, R, CB, touched, alpha, e, ad, b % ngrp, b / ngrp, nblk, tpc);
}

template <typename T>
__global__ void __launch_bounds__(256, 6)

vcd_tail_kernel(int nbin, TailBins tb, int P, int S, int pchunk, const int64_t *__restrict__ pix,
                const float *__restrict__ delta, const float *__restrict__ alpha,
                float *__restrict__ flat, double *__restrict__ sq_part,
                double *__restrict__ l1_part, unsigned int *__restrict__ counter,
                double *__restrict__ accum, int ux, int uy, int C, int R, int CB,
                const unsigned char *__restrict__ touched, T *__restrict__ e,
                const T *__restrict__ ad, int nblk, int tpc) {
  vcd_tail_kernel_body<T>(nbin, tb, P, S, pchunk, pix, delta, alpha, flat, sq_part, l1_part, counter, accum, ux, uy, C, R, CB, touched, e, ad, nblk, tpc);
}

// ── QGGMRF denoiser (identity forward model; denoising.py:35-83) ──────────
// Direction at the subset's voxels: the qGGMRF prior terms, the forward
// gradient -fmc * e and forward Hessian 1, and the four line-search sums
// per CTA: (sum g_p d, sum h_p d^2) into prior, (sum e d, sum d^2) into fwd.
__global__ void __launch_bounds__(kThreads)
denoise_direction_kernel(int P, int S, const int64_t *__restrict__ pix, int NR, int NC,
                         const float *__restrict__ flat, const float *__restrict__ err,
                         VcdScalars sc, float *__restrict__ delta, double *__restrict__ prior,
                         double *__restrict__ fwd) {
  MBIR_PDL_ENTRY();
  const size_t n = (size_t)P * S;
  const size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x;
  double pl = 0.0, pq = 0.0, fl = 0.0, fq = 0.0;
  if (i < n) {
    const int p = (int)(i / S), l = (int)(i - (size_t)p * S);
    const int pixel = (int)pix[p];
    float g_p, h_p;
    qggmrf_terms(flat, pixel, l, S, NR, NC, sc, g_p, h_p);
    const float e = err[(size_t)pixel * S + l];
    const float g_f = __fmul_rn(-sc.fmc, e);
    const float dl = -__fdiv_rn(__fadd_rn(g_f, g_p), __fadd_rn(1.f, h_p));
    delta[i] = dl;
    pl = (double)__fmul_rn(g_p, dl);
    pq = (double)__fmul_rn(h_p, __fmul_rn(dl, dl));
    fl = (double)__fmul_rn(e, dl);
    fq = (double)__fmul_rn(dl, dl);
  }
  block_sum2(pl, pq);
  block_sum2(fl, fq);
  if (threadIdx.x == 0) {
    prior[2 * blockIdx.x] = pl;
    prior[2 * blockIdx.x + 1] = pq;
    fwd[2 * blockIdx.x] = fl;
    fwd[2 * blockIdx.x + 1] = fq;
  }
}

// image += alpha d and error -= alpha d at the subset's voxels; the last CTA
// folds ell1 and alpha into accum[0], accum[1] (fixed order).
__global__ void __launch_bounds__(kThreads)
denoise_update_kernel(int P, int S, const int64_t *__restrict__ pix,
                      const float *__restrict__ delta, const float *__restrict__ alpha,
                      float *__restrict__ flat, float *__restrict__ err,
                      double *__restrict__ l1_part, unsigned int *__restrict__ counter,
                      double *__restrict__ accum) {
  MBIR_PDL_ENTRY();
  const size_t n = (size_t)P * S;
  const size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x;
  const float a = alpha[0];
  double l1 = 0.0, dummy = 0.0;
  if (i < n) {
    const int p = (int)(i / S), l = (int)(i - (size_t)p * S);
    const size_t v = (size_t)pix[p] * S + l;
    const float ds = __fmul_rn(a, delta[i]);
    flat[v] = __fadd_rn(flat[v], ds);
    err[v] = __fsub_rn(err[v], ds);
    l1 = (double)fabsf(ds);
  }
  block_sum2(l1, dummy);
  if (threadIdx.x == 0) l1_part[blockIdx.x] = l1;
  if (last_cta(counter, gridDim.x)) {
    double t1 = 0.0, t2 = 0.0;
#pragma unroll 4
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) t1 += __ldcg(l1_part + k);
    block_sum2(t1, t2);
    if (threadIdx.x == 0) {
      accum[0] += t1;
      accum[1] += (double)a;
      *counter = 0u;
    }
  }
}

// ── iteration statistics / init / conversion ─────────────────────────────
template <typename T>
__global__ void __launch_bounds__(kThreads)
stats_sino_kernel(int V, int CR, const T *__restrict__ e, const float *__restrict__ es,
                  const T *__restrict__ w, const float *__restrict__ wsc,
                  double *__restrict__ part) {
  double a = 0.0, b = 0.0, c = 0.0;
  const size_t n = (size_t)V * CR;
  for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (size_t)gridDim.x * kThreads) {
    const int v = (int)(i / CR);
    const float ev = __fmul_rn(to_f32(e[i]), es[v]);
    const float e2 = __fmul_rn(ev, ev);
    if (w != nullptr) {
      const float wv = __fmul_rn(to_f32(w[i]), wsc[v]);
      a += (double)__fmul_rn(e2, wv);
      b += (double)wv;
    } else {
      a += (double)e2;
      b += 1.0;
    }
    c += (double)e2;
  }
  double dummy = 0.0;
  block_sum2(a, b);
  block_sum2(c, dummy);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = a;
    part[3 * blockIdx.x + 1] = b;
    part[3 * blockIdx.x + 2] = c;
  }
}

__global__ void __launch_bounds__(kThreads)
stats_l1_kernel(size_t n, const float *__restrict__ x, double *__restrict__ part) {
  double a = 0.0, dummy = 0.0;
  for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (size_t)gridDim.x * kThreads)
    a += (double)fabsf(x[i]);
  block_sum2(a, dummy);
  if (threadIdx.x == 0) part[blockIdx.x] = a;
}

__global__ void __launch_bounds__(kThreads)
stats_finish_kernel(int nsino, const double *__restrict__ sino_part, int nl1,
                    const double *__restrict__ l1_part, double *__restrict__ out) {
  double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
  for (int i = threadIdx.x; i < nsino; i += kThreads) {
    a += sino_part[3 * i];
    b += sino_part[3 * i + 1];
    c += sino_part[3 * i + 2];
  }
  for (int i = threadIdx.x; i < nl1; i += kThreads) d += l1_part[i];
  block_sum2(a, b);
  block_sum2(c, d);
  if (threadIdx.x == 0) {
    out[0] = a;
    out[1] = b;
    out[2] = c;
    out[3] = d;
  }
}

// Error init: dots (sum w f f, sum w f y) per block.
__global__ void __launch_bounds__(kThreads)
init_dots_kernel(size_t n, const float *__restrict__ y, const float *__restrict__ f,
                 const float *__restrict__ w, double *__restrict__ part) {
  double ff = 0.0, fy = 0.0;
  for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (size_t)gridDim.x * kThreads) {
    const float fv = f[i];
    const float wf = w ? __fmul_rn(w[i], fv) : fv;
    ff += (double)__fmul_rn(wf, fv);
    fy += (double)__fmul_rn(wf, y[i]);
  }
  block_sum2(ff, fy);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = ff;
    part[2 * blockIdx.x + 1] = fy;
  }
}

__global__ void __launch_bounds__(kThreads)
init_alpha_kernel(int nb, const double *__restrict__ part, int scale, double *__restrict__ alpha) {
  double ff = 0.0, fy = 0.0;
  for (int i = threadIdx.x; i < nb; i += kThreads) {
    ff += part[2 * i];
    fy += part[2 * i + 1];
  }
  block_sum2(ff, fy);
  if (threadIdx.x == 0) {
    // The reference forms alpha from FP32 sums and takes it to the host as
    // a python float (tomography_model.py:1700-1706).
    alpha[0] = (ff > 0.0 && scale) ? (double)(float)(fy / ff) : 1.0;
  }
}

__global__ void init_error_kernel(size_t n, const float *__restrict__ y,
                                  const float *__restrict__ f, const double *__restrict__ alpha,
                                  float *__restrict__ e) {
  const float a = (float)alpha[0];
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    e[i] = __fsub_rn(y[i], __fmul_rn(a, f[i]));
}

__global__ void fill_kernel(int n, float v, float *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = v;
}

// Per-view max |value| of an f32 VRC sinogram -> power-of-two scale (16-bit
// storage).
__global__ void __launch_bounds__(kThreads)
view_scale_kernel(int RC, const float *__restrict__ src, float target, float *__restrict__ scale) {
  const int v = blockIdx.x;
  float m = 0.f;
  for (int i = threadIdx.x; i < RC; i += kThreads) m = fmaxf(m, fabsf(src[(size_t)v * RC + i]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
  __shared__ float sm[kThreads / 32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < kThreads / 32; ++w) t = fmaxf(t, sm[w]);
    // The smallest power of two s with t / s <= target, so that scaling
    // and unscaling are exact.
    float s = 1.f;
    if (t > 0.f) {
      int ex;
      const float mant = frexpf(t / target, &ex);
      s = ldexpf(1.f, mant == 0.5f ? ex - 1 : ex);
    }
    scale[v] = s;
  }
}

// Tiled transpose per view: f32 (R, C) <-> T (C, R) with scale.
template <typename T>
__global__ void vrc_to_vcr_kernel(int R, int C, const float *__restrict__ src,
                                  const float *__restrict__ scale, T *__restrict__ dst) {
  __shared__ float t[32][33];
  const int v = blockIdx.z;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const float inv = scale ? 1.f / scale[v] : 1.f;
  const float *s = src + (size_t)v * R * C;
  T *d = dst + (size_t)v * R * C;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = r0 + j, c = c0 + threadIdx.x;
    if (r < R && c < C) t[j][threadIdx.x] = s[(size_t)r * C + c];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + j, r = r0 + threadIdx.x;
    if (r < R && c < C) {
      const float val = t[threadIdx.x][j];
      d[(size_t)c * R + r] = from_f32<T>(scale ? __fmul_rn(val, inv) : val);
    }
  }
}

template <typename T>
__global__ void vcr_to_vrc_kernel(int R, int C, const T *__restrict__ src,
                                  const float *__restrict__ scale, float *__restrict__ dst) {
  __shared__ float t[32][33];
  const int v = blockIdx.z;
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  const float sc = scale ? scale[v] : 1.f;
  const T *s = src + (size_t)v * R * C;
  float *d = dst + (size_t)v * R * C;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + j, r = r0 + threadIdx.x;
    if (r < R && c < C) t[j][threadIdx.x] = __fmul_rn(to_f32(s[(size_t)c * R + r]), sc);
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = r0 + j, c = c0 + threadIdx.x;
    if (r < R && c < C) d[(size_t)r * C + c] = t[threadIdx.x][j];
  }
}

}  // namespace mbir
