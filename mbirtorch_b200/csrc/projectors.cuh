// Projector kernels (parallel and cone; forward and back) for sm_100a.
//
// BACK (gather, adjoint).  A TEAM of T lanes owns one pixel's cylinder (a
// chunk of up to T*SPL slices) and walks a contiguous range of views,
// accumulating in registers.  The per-(view, pixel) geometry -- the
// transcendental-heavy part of the chain -- is computed LANE-PARALLEL: each
// lane of the team takes one view of the next T, writes a small record to
// the team's shared-memory table, and the team then consumes the T records
// (broadcast reads).  The sinogram is read in the resident channel-major
// (V, C, R) layout, so every walk along the slice/row axis is unit-stride.
// For cone beam the warp first forms the view's horizontal detector column
// h(m) = sum_tc Wc * sino[v, c + tc, m] for the rows its slices reach (a
// zero-padded shared buffer per warp), then applies the vertical taps per
// slice: the separable form of cone_beam.py:237-299.  View chunks (grid.y)
// write partial sums reduced in a fixed order: deterministic.
//
// FORWARD (scatter, expressed as a gather).  The cylinders are either a
// (P, band) array in pixel-list order or, with by_pixel, the rows pix[p] of
// a flat (N*N, band) volume.  A CTA owns one view and a block
// of CB detector channels over all rows.  It scans the pixel set computing
// only each pixel's centre channel, compacts the pixels whose footprint
// reaches its block (warp ballot, in pixel order), builds full records for
// those only, and accumulates their taps into shared-memory tiles owned
// privately by thread groups; the groups' tiles are summed in group order.
// No atomics anywhere: the forward is bit-reproducible.  The epilogue writes
// the block in either sinogram layout or, for VCD, fuses the line-search
// reductions against the error sinogram.
#pragma once

#include "mbir_common.cuh"

namespace mbir {

constexpr int kThreads = 256;
constexpr int kListCap = 512;  // forward: pixel records per processing round
constexpr int kPad = 8;        // cone back: zero rows either side of the column buffer

// Cache hints (no architectural effect; every address passed is in bounds).
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
__device__ __forceinline__ void prefetch_l1(const void *p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// ── sinogram readers (resident VCR layout) ─────────────────────────────────
// value(v, c, m) = scale(v) * get(base(v, c) + m)
// get4(i, o): the four values at i .. i + 3 as one vector access (i a
// multiple of 4 and aligned16() true); aligned16() is checked on the host.
__host__ __device__ inline bool is_aligned16(const void *p) {
  return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

struct ReadF32 {
  const float *s;
  int C, R;
  __device__ __forceinline__ size_t base(int v, int c) const { return ((size_t)v * C + c) * R; }
  __device__ __forceinline__ float scale(int) const { return 1.f; }
  __device__ __forceinline__ float get(size_t i) const { return __ldg(s + i); }
  __device__ __forceinline__ void get4(size_t i, float (&o)[4]) const { load4(s + i, o); }
  __host__ bool aligned16() const { return is_aligned16(s); }
};

template <typename T>
struct ReadScaled {
  const T *e;
  const float *es;
  int C, R;
  __device__ __forceinline__ size_t base(int v, int c) const { return ((size_t)v * C + c) * R; }
  __device__ __forceinline__ float scale(int v) const { return __ldg(es + v); }
  __device__ __forceinline__ float get(size_t i) const { return to_f32(e[i]); }
  __device__ __forceinline__ void get4(size_t i, float (&o)[4]) const { load4(e + i, o); }
  __host__ bool aligned16() const { return is_aligned16(e); }
};

// weights * error, the gradient's operand (tomography_model.py:2548-2552).
template <typename T>
struct ReadWeighted {
  const T *e;
  const float *es;
  const T *w;
  const float *ws;
  int C, R;
  __device__ __forceinline__ size_t base(int v, int c) const { return ((size_t)v * C + c) * R; }
  __device__ __forceinline__ float scale(int v) const {
    return __fmul_rn(__ldg(ws + v), __ldg(es + v));
  }
  __device__ __forceinline__ float get(size_t i) const {
    return __fmul_rn(to_f32(w[i]), to_f32(e[i]));
  }
  __device__ __forceinline__ void get4(size_t i, float (&o)[4]) const {
    float ev[4], wv[4];
    load4(e + i, ev);
    load4(w + i, wv);
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = __fmul_rn(wv[k], ev[k]);
  }
  __host__ bool aligned16() const { return is_aligned16(e) && is_aligned16(w); }
};

// Tap loops: NT is the compile-time tap count (3 for psf radius 1, the
// common case) or 0 for a run-time count of 2 psf + 1 <= kMaxTaps.
#define MBIR_TAPS(NT) ((NT) ? (NT) : kMaxTaps)
#define MBIR_TAP_ON(NT, t, nt) ((NT) != 0 || (t) < (nt))

// Per-(view, pixel) records the back projectors share across a team.
struct ParRec {
  int ctr;
  float w[kMaxTaps];
};

struct ConeRec {
  int ctr;
  float w[kMaxTaps];
  float m0, w_r, hw1r, lmaxr, a0, a1;
};

// One cone (view, pixel) at psf radius 1, formed once per subset by
// cone_bin_kernel and read by the register-tiled forward (packed for 16-byte
// shared loads) and by the VCD gradient's back projection.
struct __align__(16) ConeFwdRec {
  float4 a;  // m0, w_r, (w_r + 1) / 2, min(w_r, 1)         (vertical fan)
  float4 b;  // 1 / w_r, tap weights at centre - 1, centre, centre + 1
  float4 c;  // a0, a1 (t(k) = a0 + a1 k), centre channel, value row (int bits)
};

// ── back projection: parallel ─────────────────────────────────────────────
template <int CP, int SPL, int NT, typename RD>
__device__ __forceinline__ void back_parallel_kernel_body(Geo g, const float *__restrict__ vp, int v_start, int v_count, int vpc,
                     RD rd, const int64_t *__restrict__ pix, int P, int band, int T,
                     int slice_chunks, float *__restrict__ out) {
  MBIR_PDL_ENTRY();
  __shared__ ParRec tab[kThreads];
  constexpr int MT = MBIR_TAPS(NT);
  const int RT = NT ? (NT - 1) / 2 : g.psf, nt = 2 * RT + 1;
  const int tid = threadIdx.x;
  const int team = tid / T, tl = tid - team * T;
  const int teams_per_block = kThreads / T;
  const long long gteam = (long long)blockIdx.x * teams_per_block + team;
  const int p = (int)(gteam / slice_chunks);
  const int sc = (int)(gteam - (long long)p * slice_chunks);
  const bool active = p < P;
  const int l0 = sc * T * SPL;
  const int chunk = blockIdx.y;
  const int vb = chunk * vpc, ve = min(v_count, vb + vpc);
  ParRec *mytab = tab + team * T;
  float xt = 0.f, yt = 0.f;
  if (active) pixel_xy(g, (int)pix[p], xt, yt);
  float acc[SPL];
#pragma unroll
  for (int j = 0; j < SPL; ++j) acc[j] = 0.f;

  for (int vg = vb; vg < ve; vg += T) {
    const int nv = min(T, ve - vg);
    __syncwarp();
    if (active && tl < nv) {
      const ParView pv = parallel_view(g, vp[2 * (v_start + vg + tl)]);
      const float n_p = parallel_np(g, pv, xt, yt);
      ParRec r;
      r.ctr = (int)fminf(fmaxf(rintf(n_p), -1.0e6f), 1.0e6f);
#pragma unroll
      for (int t = 0; t < MT; ++t) {
        float a = MBIR_TAP_ON(NT, t, nt)
                      ? tap_weight(n_p, r.ctr + t - RT, pv.half_w1, pv.lmax, pv.ws, g.C)
                      : 0.f;
        r.w[t] = CP == 2 ? __fmul_rn(a, a) : a;
      }
      mytab[tl] = r;
    }
    __syncwarp();
    if (!active) continue;
    // Two views per step: both views' taps are loaded before either is
    // accumulated (the accumulation order is unchanged: view by view).
    constexpr int VU = 2;
    for (int i = 0; i < nv; i += VU) {
      float w[VU][MT], scl[VU], col[VU][SPL][MT];
#pragma unroll
      for (int u = 0; u < VU; ++u) {
        const bool on = i + u < nv;
        const int v = vg + (on ? i + u : i);
        const int ctr = mytab[on ? i + u : i].ctr;
        scl[u] = rd.scale(v);
#pragma unroll
        for (int t = 0; t < MT; ++t) {
          w[u][t] = mytab[on ? i + u : i].w[t];
          const size_t base = rd.base(v, min(max(ctr + t - RT, 0), g.C - 1));
#pragma unroll
          for (int j = 0; j < SPL; ++j) {
            const int l = l0 + tl + T * j;
            col[u][j][t] = (on && l < band && MBIR_TAP_ON(NT, t, nt)) ? rd.get(base + l) : 0.f;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < VU; ++u) {
        if (i + u >= nv) break;
#pragma unroll
        for (int j = 0; j < SPL; ++j) {
          const int l = l0 + tl + T * j;
          if (l < band) {
            float s = 0.f;
#pragma unroll
            for (int t = 0; t < MT; ++t)
              if (MBIR_TAP_ON(NT, t, nt)) s = fmaf(w[u][t], col[u][j][t], s);
            acc[j] = fmaf(scl[u], s, acc[j]);
          }
        }
      }
    }
  }
  if (active) {
    float *o = out + (size_t)chunk * P * band + (size_t)p * band;
#pragma unroll
    for (int j = 0; j < SPL; ++j) {
      const int l = l0 + tl + T * j;
      if (l < band) o[l] = acc[j];
    }
  }
}

template <int CP, int SPL, int NT, typename RD>
__global__ void __launch_bounds__(kThreads)

back_parallel_kernel(Geo g, const float *__restrict__ vp, int v_start, int v_count, int vpc,
                     RD rd, const int64_t *__restrict__ pix, int P, int band, int T,
                     int slice_chunks, float *__restrict__ out) {
  back_parallel_kernel_body<CP, SPL, NT, RD>(g, vp, v_start, v_count, vpc, rd, pix, P, band, T, slice_chunks, out);
}

// The parallel back projector at psf radius 1 with four consecutive slices
// per lane (a team of T lanes covers 4 T slices, as SPL = 4 does):
// each tap of a view is one 16-byte load per lane, and two views' taps are
// in flight before either is accumulated.  Each output is the same sequence
// of FMAs as in back_parallel_kernel.  Needs band a multiple of 4 and the
// operands 16-byte aligned (checked on the host).
template <int CP, int T, typename RD>
__device__ __forceinline__ void back_parallel4_kernel_body(Geo g, const float *__restrict__ vp, int v_start, int v_count, int vpc,
                      RD rd, const int64_t *__restrict__ pix, int P, int band, int slice_chunks,
                      float *__restrict__ out) {
  MBIR_PDL_ENTRY();
  __shared__ ParRec tab[kThreads];
  constexpr int MT = 3;
  const int tid = threadIdx.x;
  const int team = tid / T, tl = tid - team * T;
  const int teams_per_block = kThreads / T;
  const long long gteam = (long long)blockIdx.x * teams_per_block + team;
  const int p = (int)(gteam / slice_chunks);
  const int sc = (int)(gteam - (long long)p * slice_chunks);
  const int l = sc * T * 4 + 4 * tl;  // this lane's slices l .. l + 3
  const bool active = p < P;
  const bool mine = active && l < band;
  const int chunk = blockIdx.y;
  const int vb = chunk * vpc, ve = min(v_count, vb + vpc);
  ParRec *mytab = tab + team * T;
  float xt = 0.f, yt = 0.f;
  if (active) pixel_xy(g, (int)pix[p], xt, yt);
  float acc[4] = {0.f, 0.f, 0.f, 0.f};

  for (int vg = vb; vg < ve; vg += T) {
    const int nv = min(T, ve - vg);
    __syncwarp();
    if (active && tl < nv) {
      const ParView pv = parallel_view(g, vp[2 * (v_start + vg + tl)]);
      const float n_p = parallel_np(g, pv, xt, yt);
      ParRec r;
      r.ctr = (int)fminf(fmaxf(rintf(n_p), -1.0e6f), 1.0e6f);
#pragma unroll
      for (int t = 0; t < MT; ++t) {
        const float a = tap_weight(n_p, r.ctr + t - 1, pv.half_w1, pv.lmax, pv.ws, g.C);
        r.w[t] = CP == 2 ? __fmul_rn(a, a) : a;
      }
      mytab[tl] = r;
    }
    __syncwarp();
    if (!mine) continue;
    constexpr int VU = 2;
    for (int i = 0; i < nv; i += VU) {
      float w[VU][MT], scl[VU], col[VU][MT][4];
#pragma unroll
      for (int u = 0; u < VU; ++u) {
        const int iu = i + u < nv ? i + u : i;
        const int v = vg + iu;
        const int ctr = mytab[iu].ctr;
        scl[u] = rd.scale(v);
#pragma unroll
        for (int t = 0; t < MT; ++t) {
          w[u][t] = mytab[iu].w[t];
          rd.get4(rd.base(v, min(max(ctr + t - 1, 0), g.C - 1)) + l, col[u][t]);
        }
      }
#pragma unroll
      for (int u = 0; u < VU; ++u) {
        if (i + u >= nv) break;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          float s = 0.f;
#pragma unroll
          for (int t = 0; t < MT; ++t) s = fmaf(w[u][t], col[u][t][k], s);
          acc[k] = fmaf(scl[u], s, acc[k]);
        }
      }
    }
  }
  if (mine) {
    float *o = out + (size_t)chunk * P * band + (size_t)p * band + l;
    *reinterpret_cast<float4 *>(o) = make_float4(acc[0], acc[1], acc[2], acc[3]);
  }
}

template <int CP, int T, typename RD>
__global__ void __launch_bounds__(kThreads)

back_parallel4_kernel(Geo g, const float *__restrict__ vp, int v_start, int v_count, int vpc,
                      RD rd, const int64_t *__restrict__ pix, int P, int band, int slice_chunks,
                      float *__restrict__ out) {
  back_parallel4_kernel_body<CP, T, RD>(g, vp, v_start, v_count, vpc, rd, pix, P, band, slice_chunks, out);
}

// Trapezoid tap weight min(max(x, 0), lmax) (cone_beam.py:203-226,
// 268-299).  With lmax = 1 -- a projected voxel at least one row pitch tall,
// the common case -- the clamp is one saturating add; the caller picks SAT
// from lmax for a whole view (the values are the same either way).
template <bool SAT>
__device__ __forceinline__ float trap_w(float x, float lmax) {
  return SAT ? __saturatef(x) : fminf(fmaxf(x, 0.f), lmax);
}

// ── back projection: cone ─────────────────────────────────────────────────
// The vertical gather of one view for a lane's SPL slices l, l + 32, ...:
// taps of the detector column h around the slice's projected row, scaled
// by 1 / cos(phi) (coefficient power 1) or 1 + t^2 (power 2).
template <int CP, int SPL, int NT, bool SAT>
__device__ __forceinline__ void back_cone_slices(float (&acc)[SPL], const float *__restrict__ h,
                                                 int l1, int band, int slice_start, float w_r,
                                                 float m0, float hw1r, float lmaxr, float a0,
                                                 float a1, float mlo_clamp, float mhi_clamp,
                                                 int RT, int nt) {
  constexpr int MT = MBIR_TAPS(NT);
  // k = slice_start + l as a float, formed by adding whole numbers below
  // 2^24 to one conversion (exact, the same value as converting each).
  const float kb = (float)(slice_start + l1);
#pragma unroll
  for (int j = 0; j < SPL; ++j) {
    const int l = l1 + 32 * j;
    if (l < band) {
      const float k = kb + (float)(32 * j);
      const float m_p = fminf(fmaxf(fmaf(w_r, k, m0), mlo_clamp), mhi_clamp);
      const float mcf = rintf(m_p);
      const int mc = (int)mcf;
      const float d = m_p - mcf;
      float s = 0.f;
      if (NT == 3) {
        // |d| <= 1/2 (m_p is rounded to mcf; a clamped m_p is whole), so
        // the outer taps' distances |d +- 1| are 1 +- d.
        const float c1 = hw1r - 1.f;
        float am = trap_w<SAT>(c1 - d, lmaxr), a0 = trap_w<SAT>(hw1r - fabsf(d), lmaxr),
              ap = trap_w<SAT>(c1 + d, lmaxr);
        if (CP == 2) {
          am = am * am;
          a0 = a0 * a0;
          ap = ap * ap;
        }
        s = fmaf(ap, h[mc + 1], fmaf(a0, h[mc], am * h[mc - 1]));
      } else {
#pragma unroll
        for (int t = 0; t < MT; ++t) {
          if (MBIR_TAP_ON(NT, t, nt)) {
            float a = trap_w<SAT>(hw1r - fabsf(d - (float)(t - RT)), lmaxr);
            if (CP == 2) a = a * a;
            s = fmaf(a, h[mc + t - RT], s);
          }
        }
      }
      const float tk = fmaf(a1, k, a0);
      const float ic = CP == 2 ? fmaf(tk, tk, 1.f) : inv_cos_from_t(tk);
      acc[j] = fmaf(ic, s, acc[j]);
    }
  }
}

// HB rows mb, mb + 32, ... of a view's detector column into h: the MT
// channel taps weighted and summed, times the view's scale.  Every load of
// the batch is in flight before the first use.  CHECK: rows past m_hi are
// skipped (the batch's last rows may not exist).
template <int HB, int MT, int NT, bool CHECK, typename RD>
__device__ __forceinline__ void column_batch(const RD &rd, const size_t (&base)[MT],
                                             const float (&w)[MT], float scl, int mb, int m_hi,
                                             float *__restrict__ h, int nt) {
  float col[HB][MT];
#pragma unroll
  for (int u = 0; u < HB; ++u) {
    const int m = mb + 32 * u;
#pragma unroll
    for (int t = 0; t < MT; ++t)
      col[u][t] = (MBIR_TAP_ON(NT, t, nt) && (!CHECK || m <= m_hi)) ? rd.get(base[t] + m) : 0.f;
  }
#pragma unroll
  for (int u = 0; u < HB; ++u) {
    const int m = mb + 32 * u;
    if (!CHECK || m <= m_hi) {
      float s = 0.f;
#pragma unroll
      for (int t = 0; t < MT; ++t)
        if (MBIR_TAP_ON(NT, t, nt)) s = fmaf(w[t], col[u][t], s);
      h[m] = __fmul_rn(s, scl);
    }
  }
}

// One warp per (pixel, chunk of 32*SPL slices).  Dynamic shared memory:
// 8 warps x (R + 2 kPad) floats of column buffer, then 8 x 32 ConeRec.
// HBL: rows per lane of a column batch for bands of more than 64 slices
// (8, or 6 where the host's back_long_batch finds 192-row batches leave
// fewer idle row slots on the detector's column than 256-row ones).
template <int CP, int SPL, int NT, typename RD, int HBL = 8>
__device__ __forceinline__ void back_cone_kernel_body(Geo g, const float *__restrict__ vp, int v_start, int v_count, int vpc, RD rd,
                 const int64_t *__restrict__ pix, int P, int slice_start, int band,
                 int slice_chunks, float *__restrict__ out,
                 const ConeFwdRec *__restrict__ recs) {
  MBIR_PDL_ENTRY();
  extern __shared__ float smem[];
  constexpr int MT = MBIR_TAPS(NT);
  const int RT = NT ? (NT - 1) / 2 : g.psf, nt = 2 * RT + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long gw = (long long)blockIdx.x * (kThreads / 32) + warp;
  const int p = (int)(gw / slice_chunks);
  if (p >= P) return;  // whole warp: no block-level barrier in this kernel
  const int sc = (int)(gw - (long long)p * slice_chunks);
  const int hs = g.R + 2 * kPad;
  float *h = smem + warp * hs + kPad;
  ConeRec *tab = reinterpret_cast<ConeRec *>(smem + (kThreads / 32) * hs) + warp * 32;
  for (int i = lane; i < kPad; i += 32) {
    h[i - kPad] = 0.f;
    h[g.R + i] = 0.f;
  }
  const int l0 = sc * 32 * SPL;
  const int l_end = min(band, l0 + 32 * SPL);
  const int chunk = blockIdx.y;
  const int vb = chunk * vpc, ve = min(v_count, vb + vpc);
  float xt, yt;
  pixel_xy(g, (int)pix[p], xt, yt);
  float acc[SPL];
#pragma unroll
  for (int j = 0; j < SPL; ++j) acc[j] = 0.f;
  const float kf = (float)(slice_start + l0);
  const float kl = (float)(slice_start + max(l_end - 1, l0));
  const float mlo_clamp = -(float)(RT + 1), mhi_clamp = (float)(g.R + RT);

  for (int vg = vb; vg < ve; vg += 32) {
    const int nv = min(32, ve - vg);
    __syncwarp();
    if (CP == 1 && MT == 3 && recs != nullptr && lane < nv) {
      // The same values cone_bin_kernel formed for this (view, slot).
      const ConeFwdRec fr = recs[(size_t)(vg + lane) * P + p];
      ConeRec r;
      r.ctr = __float_as_int(fr.c.z);
      r.w[0] = fr.b.y;
      r.w[1] = fr.b.z;
      r.w[2] = fr.b.w;
      r.m0 = fr.a.x;
      r.w_r = fr.a.y;
      r.hw1r = fr.a.z;
      r.lmaxr = fr.a.w;
      r.a0 = fr.c.x;
      r.a1 = fr.c.y;
      tab[lane] = r;
    } else if (lane < nv) {
      const int gv = v_start + vg + lane;
      const float ang = vp[2 * gv];
      const float z_off = __fsub_rn(g.rso, vp[2 * gv + 1]);
      const ConeVP q = cone_vp(g, ang, cosf(ang), sinf(ang), z_off, xt, yt);
      ConeRec r;
      r.ctr = q.ctr;
#pragma unroll
      for (int t = 0; t < MT; ++t) {
        float a = MBIR_TAP_ON(NT, t, nt)
                      ? tap_weight(q.n_p, q.ctr + t - RT, q.half_w1, q.lmax, q.ws, g.C)
                      : 0.f;
        r.w[t] = CP == 2 ? __fmul_rn(a, a) : a;
      }
      r.m0 = q.m0;
      r.w_r = q.w_r;
      r.hw1r = __fdiv_rn(__fadd_rn(q.w_r, 1.f), 2.f);
      r.lmaxr = fminf(q.w_r, 1.f);
      cone_tcoef(g, q.mag, z_off, r.a0, r.a1);
      tab[lane] = r;
    }
    __syncwarp();
    for (int i = 0; i < nv; ++i) {
      const int v = vg + i;
      const ConeRec &r = tab[i];
      const float m0 = r.m0, w_r = r.w_r, hw1r = r.hw1r, lmaxr = r.lmaxr;
      const float a0 = r.a0, a1 = r.a1;
      float w[MT];
      size_t base[MT];
#pragma unroll
      for (int t = 0; t < MT; ++t) {
        w[t] = r.w[t];
        base[t] = rd.base(v, min(max(r.ctr + t - RT, 0), g.C - 1));
      }
      const float scl = rd.scale(v);
      // Rows this chunk's slices reach (the map is affine in k).
      const float ma = fmaf(w_r, kf, m0), mb = fmaf(w_r, kl, m0);
      const float lo = fmaxf(floorf(fminf(ma, mb)) - (float)(RT + 1), 0.f);
      const float hi = fminf(ceilf(fmaxf(ma, mb)) + (float)(RT + 1), (float)(g.R - 1));
      if (lo <= hi) {
        // Column rows in batches of HB per lane, every load of a batch in
        // flight before the first use.  A short band (SPL <= 2, at most 64
        // slices) spans about 64 w_r rows, so its batches are 4 rows deep:
        // fewer predicated-off loads than 8.  A batch's rows past the
        // column's end are predicated off but still issue, so longer bands
        // take the depth HBL that fits the detector's rows (back_long_batch).
        constexpr int HB = NT == 3 ? (SPL <= 2 ? 4 : HBL) : 2;
        const int m_lo = (int)lo, m_hi = (int)hi;
        if constexpr (SPL <= 2) {
          // Short bands: whole batches (every lane's HB rows exist, no row
          // test), then the remaining rows in batches of 2.  (For longer
          // bands the split costs registers and occupancy: the plain loop
          // below is faster there.)
          int g0 = m_lo;
          for (; g0 + 32 * HB - 1 <= m_hi; g0 += 32 * HB)
            column_batch<HB, MT, NT, false>(rd, base, w, scl, g0 + lane, m_hi, h, nt);
          for (; g0 <= m_hi; g0 += 32 * 2)
            column_batch<2, MT, NT, true>(rd, base, w, scl, g0 + lane, m_hi, h, nt);
        } else {
          for (int mb = m_lo + lane; mb <= m_hi; mb += 32 * HB) {
            float col[HB][MT];
#pragma unroll
            for (int u = 0; u < HB; ++u) {
              const int m = mb + 32 * u;
#pragma unroll
              for (int t = 0; t < MT; ++t)
                col[u][t] = (MBIR_TAP_ON(NT, t, nt) && m <= m_hi) ? rd.get(base[t] + m) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < HB; ++u) {
              const int m = mb + 32 * u;
              if (m <= m_hi) {
                float s = 0.f;
#pragma unroll
                for (int t = 0; t < MT; ++t)
                  if (MBIR_TAP_ON(NT, t, nt)) s = fmaf(w[t], col[u][t], s);
                h[m] = __fmul_rn(s, scl);
              }
            }
          }
        }
      }
      __syncwarp();
      if (lmaxr == 1.f)
        back_cone_slices<CP, SPL, NT, true>(acc, h, l0 + lane, band, slice_start, w_r, m0, hw1r,
                                            lmaxr, a0, a1, mlo_clamp, mhi_clamp, RT, nt);
      else
        back_cone_slices<CP, SPL, NT, false>(acc, h, l0 + lane, band, slice_start, w_r, m0, hw1r,
                                             lmaxr, a0, a1, mlo_clamp, mhi_clamp, RT, nt);
      __syncwarp();
    }
  }
  float *o = out + (size_t)chunk * P * band + (size_t)p * band;
#pragma unroll
  for (int j = 0; j < SPL; ++j) {
    const int l = l0 + lane + 32 * j;
    if (l < band) o[l] = acc[j];
  }
}

template <int CP, int SPL, int NT, typename RD, int HBL = 8>
__global__ void __launch_bounds__(kThreads)

back_cone_kernel(Geo g, const float *__restrict__ vp, int v_start, int v_count, int vpc, RD rd,
                 const int64_t *__restrict__ pix, int P, int slice_start, int band,
                 int slice_chunks, float *__restrict__ out,
                 const ConeFwdRec *__restrict__ recs) {
  back_cone_kernel_body<CP, SPL, NT, RD, HBL>(g, vp, v_start, v_count, vpc, rd, pix, P, slice_start, band, slice_chunks, out, recs);
}

// out[i] = sum over chunks of part[chunk * n + i], in chunk order.
__global__ void reduce_chunks_kernel(const float *__restrict__ part, int chunks, size_t n,
                                     float *__restrict__ out) {
  MBIR_PDL_ENTRY();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int c = 0; c < chunks; ++c) s += part[(size_t)c * n + i];
    out[i] = s;
  }
}

// ── forward projection ────────────────────────────────────────────────────
constexpr int kConeFields = 7;  // m0, w_r, hw1r, lmaxr, inv_wr, a0, a1

struct FwdShape {
  int CB;    // channels per CTA
  int TG;    // threads per group (row lanes)
  int RPT;   // rows per thread
  int rows;  // output rows (detector rows; == band for parallel)
  __host__ __device__ int RS() const { return TG * RPT + 1; }
  __host__ __device__ int G() const { return kThreads / TG; }
  size_t smem_bytes() const {
    return sizeof(float) *
           ((size_t)G() * CB * RS() + (size_t)kListCap * (2 + kMaxTaps + kConeFields));
  }
};

// Epilogue: plain store in either sinogram layout.  View v lands in slot
// v - v_base of `out` (the binned kernels hand over absolute views).
struct StoreSino {
  static constexpr bool kViewFastest = true;  // binned grids: views on x
  float *out;
  int layout, C, R;
  int v_base;
  __device__ __forceinline__ bool channel_fastest() const { return layout == MBIR_LAYOUT_VRC; }
  __device__ __forceinline__ void begin(int) {}
  __device__ __forceinline__ void prefetch(int, int, int) {}
  __device__ __forceinline__ void cell(int v, int c, int m, float val) {
    const size_t vs = (size_t)(v - v_base);
    if (layout == MBIR_LAYOUT_VCR)
      out[(vs * C + c) * R + m] = val;
    else
      out[(vs * R + m) * C + c] = val;
  }
  template <int N>
  __device__ __forceinline__ void cells(int v, int c0, int ncb, int m, const float (&acc)[N]) {
#pragma unroll
    for (int j = 0; j < N; ++j)
      if (j < ncb) cell(v, c0 + j, m, acc[j]);
  }
  // Rows m0 .. m0 + 3 of channels c0 .. c0 + ncb - 1; channel j's four sums
  // are acc[j * stride].  In the (V, C, R) layout with R a multiple of 4 and
  // a 16-byte aligned `out`, each channel's four cells are one vector store.
  __device__ __forceinline__ void cells4(int v, int c0, int ncb, int m0,
                                         const float4 *__restrict__ acc, int stride) {
    const size_t vs = (size_t)(v - v_base);
    const bool vec = layout == MBIR_LAYOUT_VCR && (R & 3) == 0 &&
                     (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    for (int j = 0; j < ncb; ++j) {
      const float4 a = acc[j * stride];
      if (vec) {
        *reinterpret_cast<float4 *>(out + (vs * C + c0 + j) * R + m0) = a;
      } else {
        const float q[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (m0 + k < R) cell(v, c0 + j, m0 + k, q[k]);
      }
    }
  }
  // A tile that no pixel reaches is zero.
  __device__ __forceinline__ void empty_tile(int v, int c0, int ncb) {
    for (int i = threadIdx.x; i < ncb * R; i += blockDim.x) {
      if (layout == MBIR_LAYOUT_VCR)
        cell(v, c0 + i / R, i % R, 0.f);
      else
        cell(v, c0 + i % ncb, i / ncb, 0.f);
    }
  }
  __device__ __forceinline__ void end(int) {}
};

template <bool CONE, int NT, typename EPI>
__global__ void __launch_bounds__(kThreads)
forward_kernel(Geo g, const float *__restrict__ vp, int v_start, const float *__restrict__ values,
               int P, int band, int slice_start, const int64_t *__restrict__ pix, FwdShape fs,
               int by_pixel, EPI epi) {
  MBIR_PDL_ENTRY();
  extern __shared__ float sm[];
  constexpr int MT = MBIR_TAPS(NT);
  const int RT = NT ? (NT - 1) / 2 : g.psf, nt = 2 * RT + 1;
  const int TG = fs.TG, G = fs.G(), RS = fs.RS(), CB = fs.CB, RPT = fs.RPT;
  const int rows = fs.rows;
  float *tile = sm;
  int *l_ctr = (int *)(tile + (size_t)G * CB * RS);
  int *l_pix = l_ctr + kListCap;
  float *l_w = (float *)(l_pix + kListCap);
  float *l_c = l_w + kMaxTaps * kListCap;
  __shared__ int s_wcount[kThreads / 32];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int vl = blockIdx.y;
  const int v = v_start + vl;
  const int c0 = blockIdx.x * CB;
  const int ncb = min(CB, g.C - c0);
  const int bp = g.bp;
  const float ang = vp[2 * v];
  const float cs = cosf(ang), sn = sinf(ang);
  const float z_off = __fsub_rn(g.rso, vp[2 * v + 1]);
  ParView pv;
  if (!CONE) pv = parallel_view(g, ang);

  for (int i = tid; i < G * CB * RS; i += kThreads) tile[i] = 0.f;
  const int grp = tid / TG, tg = tid - grp * TG;
  float *mytile = tile + (size_t)grp * CB * RS;

  int pos = 0;
  while (pos < P) {
    int n = 0;
    __syncthreads();
    while (pos < P && n <= kListCap - kThreads) {
      const int p = pos + tid;
      bool keep = false;
      int ctr = 0;
      float n_p = 0.f;
      ConeCenter cc;
      if (p < P) {
        float xt, yt;
        pixel_xy(g, (int)pix[p], xt, yt);
        if (CONE) {
          cc = cone_center(g, cs, sn, xt, yt);
          ctr = cc.ctr;
          n_p = cc.n_p;
        } else {
          n_p = parallel_np(g, pv, xt, yt);
          ctr = (int)fminf(fmaxf(rintf(n_p), -1.0e6f), 1.0e6f);
        }
        keep = (ctr + RT >= c0) && (ctr - RT < c0 + ncb);
      }
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) s_wcount[warp] = __popc(bal);
      __syncthreads();
      int off = n, tot = 0;
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w) {
        const int c = s_wcount[w];
        if (w < warp) off += c;
        tot += c;
      }
      if (keep) {
        const int slot = off + __popc(bal & ((1u << lane) - 1u));
        l_ctr[slot] = ctr;
        l_pix[slot] = by_pixel ? (int)pix[p] : p;  // row of `values` holding the cylinder
        if (CONE) {
          const ConeVP q = cone_finish(g, ang, z_off, cc);
#pragma unroll
          for (int t = 0; t < MT; ++t)
            l_w[t * kListCap + slot] =
                MBIR_TAP_ON(NT, t, nt)
                    ? tap_weight(n_p, ctr + t - RT, q.half_w1, q.lmax, q.ws, g.C) : 0.f;
          float a0, a1;
          cone_tcoef(g, q.mag, z_off, a0, a1);
          l_c[0 * kListCap + slot] = q.m0;
          l_c[1 * kListCap + slot] = q.w_r;
          l_c[2 * kListCap + slot] = __fdiv_rn(__fadd_rn(q.w_r, 1.f), 2.f);
          l_c[3 * kListCap + slot] = fminf(q.w_r, 1.f);
          l_c[4 * kListCap + slot] = 1.f / q.w_r;
          l_c[5 * kListCap + slot] = a0;
          l_c[6 * kListCap + slot] = a1;
        } else {
#pragma unroll
          for (int t = 0; t < MT; ++t)
            l_w[t * kListCap + slot] =
                MBIR_TAP_ON(NT, t, nt)
                    ? tap_weight(n_p, ctr + t - RT, pv.half_w1, pv.lmax, pv.ws, g.C) : 0.f;
        }
      }
      n += tot;
      pos += kThreads;
      __syncthreads();
    }
    // Accumulate the listed pixels: group grp takes entries grp, grp + G, ...
    for (int e = grp; e < n; e += G) {
      const int cb0 = l_ctr[e] - RT - c0;  // tile channel of tap 0
      const float *vrow = values + (size_t)l_pix[e] * band;
      float w[MT];
#pragma unroll
      for (int t = 0; t < MT; ++t) w[t] = l_w[t * kListCap + e];
      float m0 = 0.f, w_r = 0.f, hw1r = 0.f, lmaxr = 0.f, inv_wr = 0.f, a0 = 0.f, a1 = 0.f;
      if (CONE) {
        m0 = l_c[0 * kListCap + e];
        w_r = l_c[1 * kListCap + e];
        hw1r = l_c[2 * kListCap + e];
        lmaxr = l_c[3 * kListCap + e];
        inv_wr = l_c[4 * kListCap + e];
        a0 = l_c[5 * kListCap + e];
        a1 = l_c[6 * kListCap + e];
      }
      for (int j = 0; j < RPT; ++j) {
        const int m = tg + TG * j;
        if (m >= rows) break;
        float det;
        if (!CONE) {
          det = __ldg(vrow + m);
        } else {
          // Detector-side vertical fan (cone_beam.py:203-226): slice taps
          // around k(m) = (m - m0) / w_r, values scaled by 1 / cos(phi).
          const float k_m = ((float)m - m0) * inv_wr;
          const float kc = rintf(fminf(fmaxf(k_m, -1.0e6f), 1.0e6f));
          const float d = w_r * (kc - k_m);
          det = 0.f;
          for (int ko = -bp; ko <= bp; ++ko) {
            const int k_ind = (int)kc + ko;
            const float a = fminf(fmaxf(hw1r - fabsf(fmaf(w_r, (float)ko, d)), 0.f), lmaxr);
            if (a > 0.f && k_ind >= slice_start && k_ind < slice_start + band) {
              const float tk = fmaf(a1, (float)k_ind, a0);
              det = fmaf(a * inv_cos_from_t(tk), __ldg(vrow + (k_ind - slice_start)), det);
            }
          }
        }
        float *col = mytile + m;
#pragma unroll
        for (int t = 0; t < MT; ++t) {
          const int ch = cb0 + t;
          if (MBIR_TAP_ON(NT, t, nt) && ch >= 0 && ch < ncb)
            col[(size_t)ch * RS] = fmaf(w[t], det, col[(size_t)ch * RS]);
        }
      }
    }
  }
  __syncthreads();
  // Epilogue: sum the groups' tiles in group order and hand each cell over.
  epi.begin(vl);
  const int cells = ncb * rows;
  if (epi.channel_fastest()) {
    for (int i = tid; i < cells; i += kThreads) {
      const int ch = i % ncb, m = i / ncb;
      float s = 0.f;
      for (int gg = 0; gg < G; ++gg) s += tile[((size_t)gg * CB + ch) * RS + m];
      epi.cell(vl, c0 + ch, m, s);
    }
  } else {
#pragma unroll 4
    for (int i = tid; i < cells; i += kThreads) {
      const int ch = i / rows, m = i - (i / rows) * rows;
      float s = 0.f;
      for (int gg = 0; gg < G; ++gg) s += tile[((size_t)gg * CB + ch) * RS + m];
      epi.cell(vl, c0 + ch, m, s);
    }
  }
  epi.end(blockIdx.y * gridDim.x + blockIdx.x);
}

// ── forward projection, cone, row-tiled ────────────────────────────────────
// The cone forward for psf radius 1 and up to 1024 detector rows (the
// scanning form of a slice band here; the binned form below shares the row
// loop and, where it applies, stages asynchronously).  A CTA
// owns one view and kFwdCB channels; thread m owns detector row m and its
// kFwdCB channel sums, held in a thread-private column of shared memory
// (kFwdCB + 4 rows so that the three taps of any reaching pixel land
// without a bounds test or a branch on the pixel's channel).  Pixels
// reaching the block are compacted as in forward_kernel, then processed in
// batches of kFwdEB: the batch's cylinders, scaled by 1 / cos(phi) per
// slice, are staged in zero-padded shared memory (one rsqrt per voxel), and
// every thread forms its row's detector-side vertical fan from them
// (cone_beam.py:203-226) and adds the three channel taps.  No atomics; each
// channel's sum is a fixed sequence of FMAs in pixel order.
constexpr int kFwdCB = 16;   // channels per CTA
constexpr int kFwdEB = 16;   // pixels staged per batch
static_assert(kFwdEB <= 32, "fwd_rt_batch tests a batch's pixels one per lane");
constexpr int kFwdVPad = 8;  // zero slices either side of a staged cylinder (>= 2 bp + 1)

// Record capacity of one round (at least one scan chunk); the shared memory
// also holds the stage and (kFwdCB + 4) accumulator rows per thread.  Short
// detectors (fewer than 128 threads) take two scan chunks per round: their
// tiles hold a few tens of records, and a smaller round leaves room for
// more CTAs per SM.
__host__ __device__ inline int fwd_cap(int nthr) {
  return nthr >= 128 ? (nthr > 256 ? nthr : 256) : 2 * nthr;
}

__device__ __forceinline__ ConeFwdRec cone_fwd_record(const Geo &g, float ang, float z_off,
                                                      const ConeCenter &cc, int row) {
  const ConeVP q = cone_finish(g, ang, z_off, cc);
  float a0, a1;
  cone_tcoef(g, q.mag, z_off, a0, a1);
  ConeFwdRec r;
  r.a = make_float4(q.m0, q.w_r, __fdiv_rn(__fadd_rn(q.w_r, 1.f), 2.f), fminf(q.w_r, 1.f));
  r.b = make_float4(1.f / q.w_r,
                    tap_weight(cc.n_p, cc.ctr - 1, q.half_w1, q.lmax, q.ws, g.C),
                    tap_weight(cc.n_p, cc.ctr, q.half_w1, q.lmax, q.ws, g.C),
                    tap_weight(cc.n_p, cc.ctr + 1, q.half_w1, q.lmax, q.ws, g.C));
  r.c = make_float4(a0, a1, __int_as_float(cc.ctr), __int_as_float(row));
  return r;
}

// Channel blocks [b_lo, b_hi] reached by a pixel whose taps are the
// channels ctr - 1 .. ctr + 1 clipped to the detector (-1 when none).
__device__ __forceinline__ void fwd_block_range(int ctr, int C, int &b_lo, int &b_hi) {
  const int lo = max(ctr - 1, 0), hi = min(ctr + 1, C - 1);
  if (lo > hi) {
    b_lo = b_hi = -1;
  } else {
    b_lo = lo / kFwdCB;
    b_hi = hi / kFwdCB;
  }
}

// The pixels of one staged batch for detector row m = threadIdx.x: the
// row's vertical fan over the staged cylinder of each pixel and its three
// channel taps (fwd_rt_round describes the accumulators).  BP = 1 is the
// psf radius 1 with the taps unrolled; BP = 0 takes the radius bp at run
// time.  A tap weight clamp(x, 0, lmax) is formed as min(sat(x), lmax),
// the same value for lmax = min(w_r, 1) <= 1, with no branch on lmax.
//
// The shared records hold -m0 / w_r in a.x and the centre's accumulator
// slot j = ctr - c0 + 1 in c.z (fwd_stage_record), so that the row's centre
// slice k_m = (m - m0) / w_r is one FMA and the slot needs no arithmetic.
// For BP = 1 with sorted records the warp takes the pixels left to walk four
// (or two) at a time: it forms the fans of all of them first, then adds
// them in pixel order, so every sum is the same sequence of FMAs as one
// pixel at a time, with the loads of four pixels in flight together.
template <int BP, bool SORTED>
__device__ __forceinline__ void fwd_rt_batch(const ConeFwdRec *__restrict__ rec, int nb,
                                             const float *__restrict__ stage, int SP, float mf,
                                             float kc_lo, float kc_hi, int slice_start, int bp,
                                             int c0, float *__restrict__ acc_s, int &cj,
                                             float &q0, float &q1, float &q2) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  // A row m reaches the band only when its centre slice k_m lies within
  // [kc_lo, kc_hi]; outside, the clamped centre puts every tap in the zero
  // padding and the row adds an exact zero.  So a warp whose rows
  // [wr0, wr0 + 31], widened by a row either side, all map outside skips the
  // pixel, with the same result.  Lane e tests pixel e of the batch
  // (nb <= kFwdEB <= 32); bit e of `skip` is the answer, and a pixel whose
  // lane does not run (a warp cut short by the detector's last row) is not
  // skipped.  The warp then walks only the pixels left in `todo`, lowest
  // first.
  unsigned todo;
  {
    const int lane = tid & 31;
    const float wr0 = (float)(tid - lane), wr1 = wr0 + 31.f;
    bool out = false;
    if (lane < nb) {
      const float nm = rec[lane].a.x, inv_wr = rec[lane].b.x;
      out = fmaf(wr1 + 1.f, inv_wr, nm) < kc_lo || fmaf(wr0 - 1.f, inv_wr, nm) > kc_hi;
    }
    const unsigned skip = __ballot_sync(__activemask(), out);
    todo = ~skip & (nb >= 32 ? 0xffffffffu : ((1u << nb) - 1u));
  }
  const unsigned rec_s = (unsigned)__cvta_generic_to_shared(rec);
  const unsigned st_s =
      (unsigned)__cvta_generic_to_shared(stage) + 4u * (unsigned)(kFwdVPad - slice_start);
  if (BP == 1 && SORTED) {
    // Pixel e's fan on this row: its slot j, its channel tap weights (rb.y ..
    // rb.w) and the three staged values around the clamped centre slice
    // with their vertical weights.  |kc - k_m| <= 1/2 wherever the taps can
    // meet the band (elsewhere they meet the zero padding), so |d| <= w_r / 2:
    // the outer taps' distances |d -+ w_r| are w_r -+ d.
    auto fan = [&](int e, float4 &rb, int &j) -> float {
      const unsigned ra_s = rec_s + (unsigned)e * (unsigned)sizeof(ConeFwdRec);
      const float4 ra = lds_f32x4(ra_s);
      rb = lds_f32x4(ra_s + 16u);
      j = __float_as_int(lds_f32(ra_s + 40u));  // c.z, in [0, kFwdCB + 1]
      const float nm = ra.x, w_r = ra.y, hw1r = ra.z, lmaxr = ra.w;
      const float k_m = fmaf(mf, rb.x, nm);
      const float kc = fminf(fmaxf(rintf(k_m), kc_lo), kc_hi);
      const float d = w_r * (kc - k_m);
      const unsigned st_a = st_s + 4u * (unsigned)(e * SP + (int)kc);
      const float c1 = hw1r - w_r;
      const float am = fminf(__saturatef(c1 + d), lmaxr);
      const float a0 = fminf(__saturatef(hw1r - fabsf(d)), lmaxr);
      const float ap = fminf(__saturatef(c1 - d), lmaxr);
      return fmaf(ap, lds_f32(st_a + 4u), fmaf(a0, lds_f32(st_a), am * lds_f32(st_a - 4u)));
    };
    // Its three taps into rows j .. j + 2 of the accumulator column, kept in
    // q0..q2 while the slot stays (fwd_rt_round).
    auto add = [&](int j, const float4 &rb, float det) {
      if (j != cj) {  // uniform over the warp; j > cj
        float *a = acc_s + cj * nthr + tid;
        a[0] += q0;
        if (j == cj + 1) {
          q0 = q1;
          q1 = q2;
        } else {
          a[nthr] += q1;
          if (j == cj + 2) {
            q0 = q2;
          } else {
            a[2 * nthr] += q2;
            q0 = 0.f;
          }
          q1 = 0.f;
        }
        q2 = 0.f;
        cj = j;
      }
      q0 = fmaf(rb.y, det, q0);
      q1 = fmaf(rb.z, det, q1);
      q2 = fmaf(rb.w, det, q2);
    };
#pragma unroll 1
    while (todo) {  // uniform over the warp
      const int e0 = __ffs(todo) - 1;
      todo &= todo - 1u;
      if (__popc(todo) >= 3) {
        const int e1 = __ffs(todo) - 1;
        todo &= todo - 1u;
        const int e2 = __ffs(todo) - 1;
        todo &= todo - 1u;
        const int e3 = __ffs(todo) - 1;
        todo &= todo - 1u;
        float4 rb0, rb1, rb2, rb3;
        int j0, j1, j2, j3;
        const float det0 = fan(e0, rb0, j0);
        const float det1 = fan(e1, rb1, j1);
        const float det2 = fan(e2, rb2, j2);
        const float det3 = fan(e3, rb3, j3);
        add(j0, rb0, det0);
        add(j1, rb1, det1);
        add(j2, rb2, det2);
        add(j3, rb3, det3);
      } else if (todo) {
        const int e1 = __ffs(todo) - 1;
        todo &= todo - 1u;
        float4 rb0, rb1;
        int j0, j1;
        const float det0 = fan(e0, rb0, j0);
        const float det1 = fan(e1, rb1, j1);
        add(j0, rb0, det0);
        add(j1, rb1, det1);
      } else {
        float4 rb0;
        int j0;
        const float det0 = fan(e0, rb0, j0);
        add(j0, rb0, det0);
      }
    }
    return;
  }
#pragma unroll 1
  while (todo) {  // uniform over the warp
    const int e = __ffs(todo) - 1;
    todo &= todo - 1u;
    const unsigned ra_s = rec_s + (unsigned)e * (unsigned)sizeof(ConeFwdRec);
    const float4 ra = lds_f32x4(ra_s), rb = lds_f32x4(ra_s + 16u);
    const int j = __float_as_int(lds_f32(ra_s + 40u));  // c.z, in [0, kFwdCB + 1]
    const float nm = ra.x, w_r = ra.y, hw1r = ra.z, lmaxr = ra.w;
    if (SORTED && j != cj) {  // uniform over the warp; j > cj
      float *a = acc_s + cj * nthr + tid;
      a[0] += q0;
      if (j == cj + 1) {
        q0 = q1;
        q1 = q2;
      } else {
        a[nthr] += q1;
        if (j == cj + 2) {
          q0 = q2;
        } else {
          a[2 * nthr] += q2;
          q0 = 0.f;
        }
        q1 = 0.f;
      }
      q2 = 0.f;
      cj = j;
    }
    const float k_m = fmaf(mf, rb.x, nm);
    const float kc = fminf(fmaxf(rintf(k_m), kc_lo), kc_hi);
    const float d = w_r * (kc - k_m);
    const unsigned st_a = st_s + 4u * (unsigned)(e * SP + (int)kc);
    const float *st = stage + e * SP + kFwdVPad + ((int)kc - slice_start);
    float det;
    if (BP == 1) {
      // |kc - k_m| <= 1/2 wherever the taps can meet the band (elsewhere they
      // meet the zero padding), so |d| <= w_r / 2: the outer taps' distances
      // |d -+ w_r| are w_r -+ d.
      const float c1 = hw1r - w_r;
      const float am = fminf(__saturatef(c1 + d), lmaxr);
      const float a0 = fminf(__saturatef(hw1r - fabsf(d)), lmaxr);
      const float ap = fminf(__saturatef(c1 - d), lmaxr);
      det = fmaf(ap, lds_f32(st_a + 4u), fmaf(a0, lds_f32(st_a), am * lds_f32(st_a - 4u)));
    } else {
      det = 0.f;
      for (int ko = -bp; ko <= bp; ++ko) {
        const float a = fminf(__saturatef(hw1r - fabsf(fmaf(w_r, (float)ko, d))), lmaxr);
        det = fmaf(a, st[ko], det);
      }
    }
    // Thread-private accumulator column in shared memory: row r holds
    // channel c0 + r - 2, so tap t of centre slot j lands on row j + t.
    if (SORTED) {
      q0 = fmaf(rb.y, det, q0);
      q1 = fmaf(rb.z, det, q1);
      q2 = fmaf(rb.w, det, q2);
    } else {
      float *a = acc_s + j * nthr + tid;
      a[0] = fmaf(rb.y, det, a[0]);
      a[nthr] = fmaf(rb.z, det, a[nthr]);
      a[2 * nthr] = fmaf(rb.w, det, a[2 * nthr]);
    }
  }
}

// A record as the forward CTA of channel block c0 keeps it in shared
// memory: a.x = -m0 / w_r (the row-to-slice offset) instead of m0, and c.z
// = the centre's accumulator slot ctr - c0 + 1 (int bits) instead of the
// centre channel; the other fields as formed.
__device__ __forceinline__ ConeFwdRec fwd_stage_record(ConeFwdRec r, int c0) {
  r.a.x = -r.a.x * r.b.x;
  r.c.z = __int_as_float(__float_as_int(r.c.z) - c0 + 1);
  return r;
}

// The batches of one round: n records in shared memory, processed kFwdEB at
// a time.  Staging writes the batch's cylinders, scaled by 1 / cos(phi) per
// slice, into the zero-padded stage; then thread m forms detector row m's
// vertical fan for every pixel of the batch and adds its three channel taps
// into its accumulator column acc_s[r * nthr + m], r = 0 .. kFwdCB + 3.
// SORTED: the round's records come in nondecreasing centre channel, so the
// three rows a pixel adds to stay in registers (q0..q2 for rows cj .. cj + 2)
// until the centre moves on; a row that leaves is added into its column
// once.  Every batch ends with all threads past a barrier.
template <bool SORTED>
__device__ __forceinline__ void fwd_rt_round(const ConeFwdRec *__restrict__ rec, int n,
                                             float *__restrict__ stage, int SP,
                                             const float *__restrict__ values, int band,
                                             int slice_start, float kc_lo, float kc_hi, int bp,
                                             int R, int c0, float *__restrict__ acc_s) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  const float mf = (float)tid;
  int cj = SORTED ? __float_as_int(rec[0].c.z) : 0;
  float q0 = 0.f, q1 = 0.f, q2 = 0.f;
  for (int b0 = 0; b0 < n; b0 += kFwdEB) {
    const int nb = min(kFwdEB, n - b0);
    if (2 * band >= nthr) {
      // slice-major: thread t stages slice t (+ nthr ...) of every pixel of
      // the batch, with the batch's loads in flight before the first use.
      // A short batch leaves the unrolled loops early (nb is uniform), so it
      // issues only its own nb slots.
      for (int k = tid; k < band; k += nthr) {
        float val[kFwdEB];
#pragma unroll
        for (int e = 0; e < kFwdEB; ++e) {
          if (e >= nb) break;
          val[e] = __ldg(values + (size_t)__float_as_int(rec[b0 + e].c.w) * band + k);
        }
        const float kf = (float)(slice_start + k);
        float *sk = stage + kFwdVPad + k;
#pragma unroll
        for (int e = 0; e < kFwdEB; ++e) {
          if (e >= nb) break;
          const float4 c = rec[b0 + e].c;
          sk[e * SP] = val[e] * inv_cos_from_t_ftz(fmaf(c.y, kf, c.x));
        }
      }
    } else {
      for (int i = tid; i < nb * band; i += nthr) {
        const int e = i / band, k = i - e * band;
        const float4 c = rec[b0 + e].c;
        stage[e * SP + kFwdVPad + k] =
            __ldg(values + (size_t)__float_as_int(c.w) * band + k) *
            inv_cos_from_t_ftz(fmaf(c.y, (float)(slice_start + k), c.x));
      }
    }
    __syncthreads();
    if (tid < R) {
      if (bp == 1)
        fwd_rt_batch<1, SORTED>(rec + b0, nb, stage, SP, mf, kc_lo, kc_hi, slice_start, bp, c0,
                                acc_s, cj, q0, q1, q2);
      else
        fwd_rt_batch<0, SORTED>(rec + b0, nb, stage, SP, mf, kc_lo, kc_hi, slice_start, bp, c0,
                                acc_s, cj, q0, q1, q2);
    }
    __syncthreads();
  }
  if (SORTED && tid < R) {
    float *a = acc_s + cj * nthr + tid;
    a[0] += q0;
    a[nthr] += q1;
    a[2 * nthr] += q2;
  }
}

// ── asynchronous cylinder staging ─────────────────────────────────────────
// cp.async 16-byte global -> shared copies (L2 only), grouped per batch.
__device__ __forceinline__ void cp_async16(float *dst_smem, const float *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Records per round of the asynchronously staged forward (its two stage
// buffers take the room of the larger record rounds).
__host__ __device__ inline int fwd_cap_async(int nthr) { return min(fwd_cap(nthr), 256); }

// fwd_rt_round<true> with the cylinders staged asynchronously (band a
// multiple of 4, 16-byte aligned cylinder rows), in batches of EB pixels
// (EB <= kFwdEB; a smaller batch keeps the two buffers in the shared memory
// of one synchronous buffer): two stage buffers; the raw
// cylinders of batch b + 1 are copied global -> shared while batch b is
// projected, and each batch is scaled by 1 / cos(phi) in place once it has
// landed.  The staged values and every sum are the same as fwd_rt_round's.
template <int EB>
__device__ __forceinline__ void fwd_rt_round_async(const ConeFwdRec *__restrict__ rec, int n,
                                                   float *__restrict__ stage2, int SP,
                                                   const float *__restrict__ values, int band,
                                                   int slice_start, float kc_lo, float kc_hi,
                                                   int bp, int R, int c0,
                                                   float *__restrict__ acc_s) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  const float mf = (float)tid;
  int cj = __float_as_int(rec[0].c.z);
  float q0 = 0.f, q1 = 0.f, q2 = 0.f;
  const int q4 = band >> 2;  // 16-byte chunks per cylinder (band >= 4)
  const int nbat = (n + EB - 1) / EB;
  // This thread's chunks i = tid, tid + nthr, ... as (pixel e, chunk q),
  // stepped without a division per chunk.
  const int e_step = nthr / q4, q_step = nthr - e_step * q4;
  const int e_first = tid / q4, q_first = tid - e_first * q4;
  auto issue = [&](int b) {
    const int b0 = b * EB, nb = min(EB, n - b0);
    float *buf = stage2 + (b & 1) * EB * SP + kFwdVPad;
    int e = e_first, q = q_first;
    while (e < nb) {
      cp_async16(buf + e * SP + 4 * q,
                 values + (size_t)__float_as_int(rec[b0 + e].c.w) * band + 4 * q);
      e += e_step;
      q += q_step;
      if (q >= q4) {
        q -= q4;
        ++e;
      }
    }
    cp_async_commit();
  };
  issue(0);
  for (int b = 0; b < nbat; ++b) {
    const int b0 = b * EB, nb = min(EB, n - b0);
    if (b + 1 < nbat) {
      issue(b + 1);
      cp_async_wait<1>();  // this thread's copies of batch b have landed
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    float *buf = stage2 + (b & 1) * EB * SP;
    for (int k = tid; k < band; k += nthr) {
      const float kf = (float)(slice_start + k);
      float *sk = buf + kFwdVPad + k;
#pragma unroll
      for (int e = 0; e < EB; ++e) {
        if (e >= nb) break;
        const float4 c = rec[b0 + e].c;
        sk[e * SP] = sk[e * SP] * inv_cos_from_t_ftz(fmaf(c.y, kf, c.x));
      }
    }
    __syncthreads();
    if (tid < R) {
      if (bp == 1)
        fwd_rt_batch<1, true>(rec + b0, nb, buf, SP, mf, kc_lo, kc_hi, slice_start, bp, c0,
                              acc_s, cj, q0, q1, q2);
      else
        fwd_rt_batch<0, true>(rec + b0, nb, buf, SP, mf, kc_lo, kc_hi, slice_start, bp, c0,
                              acc_s, cj, q0, q1, q2);
    }
    __syncthreads();  // before the copy issued next round or batch overwrites buf
  }
  if (tid < R) {
    float *a = acc_s + cj * nthr + tid;
    a[0] += q0;
    a[nthr] += q1;
    a[2 * nthr] += q2;
  }
}

template <typename EPI>
__global__ void __launch_bounds__(1024)
forward_cone_rt_kernel(Geo g, const float *__restrict__ vp, int v_start,
                       const float *__restrict__ values, int P, int band, int slice_start,
                       const int64_t *__restrict__ pix, int by_pixel, EPI epi) {
  MBIR_PDL_ENTRY();
  extern __shared__ float4 sm4[];
  const int nthr = blockDim.x;
  const int cap = fwd_cap(nthr);
  const int SP = band + 2 * kFwdVPad;                     // staged cylinder pitch
  ConeFwdRec *rec = reinterpret_cast<ConeFwdRec *>(sm4);  // cap records
  float *stage = reinterpret_cast<float *>(rec + cap);    // kFwdEB x SP
  float *acc_s = stage + kFwdEB * SP;                     // (kFwdCB + 4) x nthr
  __shared__ int s_wcount[32];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
  const int vl = blockIdx.y;
  const int v = v_start + vl;
  const int c0 = blockIdx.x * kFwdCB;
  const int ncb = min(kFwdCB, g.C - c0);
  const float ang = vp[2 * v];
  const float cs = cosf(ang), sn = sinf(ang);
  const float z_off = __fsub_rn(g.rso, vp[2 * v + 1]);
  const int bp = g.bp;
  // Clamp of the centre slice: a centre outside [ss - bp - 1, ss + band + bp]
  // has no tap inside the band, and the clamped one only meets zero padding
  // (kFwdVPad >= 2 bp + 1).
  const float kc_lo = (float)(slice_start - bp - 1),
              kc_hi = (float)(slice_start + band + bp);

  // Zero padding either side of each staged cylinder (the interiors are
  // written by every batch before they are read).
  for (int i = tid; i < kFwdEB * 2 * kFwdVPad; i += nthr) {
    const int e = i / (2 * kFwdVPad), o = i - e * 2 * kFwdVPad;
    stage[e * SP + (o < kFwdVPad ? o : band + o)] = 0.f;
  }
#pragma unroll
  for (int r = 0; r < kFwdCB + 4; ++r) acc_s[r * nthr + tid] = 0.f;

  int pos = 0;
  while (pos < P) {
    int n = 0;
    __syncthreads();
    while (pos < P && n + nthr <= cap) {
      const int p = pos + tid;
      bool keep = false;
      ConeCenter cc;
      if (p < P) {
        float xt, yt;
        pixel_xy(g, (int)pix[p], xt, yt);
        cc = cone_center(g, cs, sn, xt, yt);
        keep = (cc.ctr + 1 >= c0) && (cc.ctr - 1 < c0 + ncb);
      }
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) s_wcount[warp] = __popc(bal);
      __syncthreads();
      int off = n, tot = 0;
      for (int w = 0; w < nwarps; ++w) {
        const int c = s_wcount[w];
        if (w < warp) off += c;
        tot += c;
      }
      if (keep)
        rec[off + __popc(bal & ((1u << lane) - 1u))] =
            fwd_stage_record(cone_fwd_record(g, ang, z_off, cc, by_pixel ? (int)pix[p] : p), c0);
      n += tot;
      pos += nthr;
      __syncthreads();
    }
    fwd_rt_round<false>(rec, n, stage, SP, values, band, slice_start, kc_lo, kc_hi, bp, g.R, c0,
                        acc_s);
  }
  // Epilogue: thread m hands over its row's cells.
  float acc[kFwdCB];
#pragma unroll
  for (int j = 0; j < kFwdCB; ++j) acc[j] = acc_s[(j + 2) * nthr + tid];
  epi.begin(vl);
  if (tid < g.R) epi.cells(vl, c0, ncb, tid, acc);
  epi.end(blockIdx.y * gridDim.x + blockIdx.x);
}

// ── forward projection, cone, binned ───────────────────────────────────────
// For a pixel subset that several launches use (the VCD gradient, forward
// and positivity re-projection), and for whole volumes a chunk of views at a
// time, the (view, pixel) records are formed once by cone_bin_kernel (or its
// 1024-thread form) and sorted by centre channel, so that each forward CTA
// reads exactly its pixels, in channel order, instead of scanning the subset
// and re-forming every pixel's geometry (atan2, sin/cos, divisions) in each
// of the C / kFwdCB blocks of a view.
//
// cone_bin_kernel: one CTA per view of the chunk [v_start, v_start + gridDim.x).
//   recs[vl * P + p]                     record of subset slot p
//   list[vl * P + ...]                   slots by key = ctr + 1 (ctr in [-1, C]),
//                                        equal keys in increasing slot order
//   offs[vl * (C + 3) + k .. k + 1]      key k's range of list
// A pixel whose centre lies outside [-1, C] has no tap on the detector and
// is in no key.  Channel block b (channels c0 .. c0 + 15) is reached by the
// centres c0 - 1 .. c0 + 16: the keys c0 .. c0 + 17, one contiguous range.
// Slots are placed by a deterministic prefix over (key, warp, lane): no
// atomics decide an order.
__host__ __device__ inline int fwd_nkeys(int C) { return C + 2; }

__device__ __forceinline__ int fwd_key(int ctr, int C) {
  return (ctr >= -1 && ctr <= C) ? ctr + 1 : -1;
}

// Exclusive prefix of a[0 .. n) in place (block-wide; every thread calls
// it); returns the total.  Thread t scans a contiguous run of keys.
__device__ __forceinline__ int block_exclusive_scan(int *a, int n, int *warp_tot) {
  const int nthr = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int per = (n + nthr - 1) / nthr;
  const int lo = min(n, tid * per), hi = min(n, lo + per);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += a[i];
  int x = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int t = lane < (nthr >> 5) ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;  // inclusive over warps
  }
  __syncthreads();
  int run = x - s + (warp > 0 ? warp_tot[warp - 1] : 0);
  const int total = warp_tot[(nthr >> 5) - 1];
  for (int i = lo; i < hi; ++i) {
    const int c = a[i];
    a[i] = run;
    run += c;
  }
  __syncthreads();
  return total;
}

// The parallel-beam record of a (view, pixel): the three channel taps of
// centre ctr (parallel_beam.py:22-53, horizontal_fan.py:51-71) in b.y .. b.w,
// ctr in c.z and the cylinder's row in c.w, the fields the cone record
// keeps in the same places; the vertical-fan fields are unused.
__device__ __forceinline__ ConeFwdRec par_fwd_record(const Geo &g, const ParView &pv, float n_p,
                                                     int ctr, int row) {
  ConeFwdRec r;
  r.a = make_float4(0.f, 0.f, 0.f, 0.f);
  r.b = make_float4(0.f, tap_weight(n_p, ctr - 1, pv.half_w1, pv.lmax, pv.ws, g.C),
                    tap_weight(n_p, ctr, pv.half_w1, pv.lmax, pv.ws, g.C),
                    tap_weight(n_p, ctr + 1, pv.half_w1, pv.lmax, pv.ws, g.C));
  r.c = make_float4(0.f, 0.f, __int_as_float(ctr), __int_as_float(row));
  return r;
}

// One CTA's work of cone_bin_kernel: view vl of the chunk, with bsm the
// (1 + warps) x (C + 2) ints of dynamic shared memory.  Parallel-beam
// geometries (g.cone = 0) are binned the same way, with par_fwd_record.
//
// A stable counting sort in three steps.  Warp w owns the contiguous slots
// [p0, p1) (slot order = warp order, then lane order), so that:
//   1. each warp forms its slots' records and counts them per key into its
//      own row of counters (the leader of each group of equal keys in a
//      32-slot step adds the group's size: no two lanes write one counter);
//   2. the per-key totals are scanned, and each warp's row becomes its
//      starting cursor per key (key-major, then warp order);
//   3. each warp walks its slots again and places them at its cursors.
// Only steps 1 -> 2 -> 3 synchronise the CTA; steps 1 and 3 are warp-local.
// The list is THE stable sort of the slots by key (a stable sort has one
// result), whatever the CTA size.
__device__ __forceinline__ void cone_bin_view(const Geo &g, const float *__restrict__ vp,
                                              int v_start, int vl,
                                              const int64_t *__restrict__ pix, int P,
                                              int by_pixel, ConeFwdRec *__restrict__ recs,
                                              int *__restrict__ list, int *__restrict__ offs,
                                              int *bsm) {
  __shared__ int warp_tot[32];
  const int nthr = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nw = nthr >> 5;
  const int nkeys = fwd_nkeys(g.C);
  int *tot = bsm;             // nkeys: per-key totals, then their exclusive prefix
  int *wc = bsm + nkeys;      // nw x nkeys: per-(warp, key) counts, then cursors
  int *mywc = wc + warp * nkeys;
  const int v = v_start + vl;
  const float ang = vp[2 * v];
  const float cs = cosf(ang), sn = sinf(ang);
  const float z_off = __fsub_rn(g.rso, vp[2 * v + 1]);
  ParView pv;
  if (!g.cone) pv = parallel_view(g, ang);
  ConeFwdRec *vrec = recs + (size_t)vl * P;
  int *vlist = list + (size_t)vl * P;
  int *voffs = offs + (size_t)vl * (nkeys + 1);
  const int per_warp = (P + nw - 1) / nw;
  const int p0 = min(P, warp * per_warp), p1 = min(P, p0 + per_warp);
  const unsigned lt = (1u << lane) - 1u;

  for (int i = tid; i < nkeys * (1 + nw); i += nthr) bsm[i] = 0;
  __syncthreads();
  // 1. records and per-(warp, key) counts
  for (int base = p0; base < p1; base += 32) {
    const int p = base + lane;
    int key = -1;
    if (p < p1) {
      float xt, yt;
      pixel_xy(g, (int)pix[p], xt, yt);
      const int row = by_pixel ? (int)pix[p] : p;
      int ctr;
      if (g.cone) {
        const ConeCenter cc = cone_center(g, cs, sn, xt, yt);
        vrec[p] = cone_fwd_record(g, ang, z_off, cc, row);
        ctr = cc.ctr;
      } else {
        const float n_p = parallel_np(g, pv, xt, yt);
        ctr = (int)fminf(fmaxf(rintf(n_p), -1.0e6f), 1.0e6f);
        vrec[p] = par_fwd_record(g, pv, n_p, ctr, row);
      }
      key = fwd_key(ctr, g.C);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (key >= 0 && (peers & lt) == 0) mywc[key] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // 2. key totals, their prefix, and each warp's cursors
  for (int k = tid; k < nkeys; k += nthr) {
    int t = 0;
    for (int w = 0; w < nw; ++w) t += wc[w * nkeys + k];
    tot[k] = t;
  }
  __syncthreads();
  const int total = block_exclusive_scan(tot, nkeys, warp_tot);
  for (int k = tid; k < nkeys; k += nthr) {
    int run = tot[k];
    voffs[k] = run;
    for (int w = 0; w < nw; ++w) {
      const int c = wc[w * nkeys + k];
      wc[w * nkeys + k] = run;
      run += c;
    }
  }
  if (tid == 0) voffs[nkeys] = total;
  __syncthreads();
  // 3. placement (a lane reads back the record it wrote itself in step 1)
  for (int base = p0; base < p1; base += 32) {
    const int p = base + lane;
    const int key = p < p1 ? fwd_key(__float_as_int(vrec[p].c.z), g.C) : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int pos = key >= 0 ? mywc[key] + __popc(peers & lt) : 0;
    __syncwarp();
    if (key >= 0 && (peers & lt) == 0) mywc[key] += __popc(peers);
    __syncwarp();
    if (key >= 0) vlist[pos] = p;
  }
}

__device__ __forceinline__ void cone_bin_kernel_body(Geo g, const float *__restrict__ vp, int v_start,
                const int64_t *__restrict__ pix, int P, int by_pixel,
                ConeFwdRec *__restrict__ recs, int *__restrict__ list, int *__restrict__ offs) {
  MBIR_PDL_ENTRY();
  extern __shared__ int bsm[];
  cone_bin_view(g, vp, v_start, blockIdx.x, pix, P, by_pixel, recs, list, offs, bsm);
}

__global__ void __launch_bounds__(256)

cone_bin_kernel(Geo g, const float *__restrict__ vp, int v_start,
                const int64_t *__restrict__ pix, int P, int by_pixel,
                ConeFwdRec *__restrict__ recs, int *__restrict__ list, int *__restrict__ offs) {
  cone_bin_kernel_body(g, vp, v_start, pix, P, by_pixel, recs, list, offs);
}

// Whole-volume binning: the same per-view sort with kBinWideThreads threads
// per view (a view then holds every pixel of the volume, a few hundred slots
// per thread at 256 threads).  The list is the same stable sort.
constexpr int kBinWideThreads = 1024;

__global__ void __launch_bounds__(kBinWideThreads)
cone_bin_wide_kernel(Geo g, const float *__restrict__ vp, int v_start,
                     const int64_t *__restrict__ pix, int P, int by_pixel,
                     ConeFwdRec *__restrict__ recs, int *__restrict__ list,
                     int *__restrict__ offs) {
  cone_bin_kernel_body(g, vp, v_start, pix, P, by_pixel, recs, list, offs);
}

// Forward CTA (channel block, view of the chunk) over its bucket.  The
// epilogue sees the absolute view v_start + vl and partial slot
// (v_start + vl) * nblk + block; touched[view * nblk + block] records
// whether any pixel reached the tile.
// AEB > 0: the cylinders are staged asynchronously in batches of AEB pixels
// (fwd_rt_round_async; band a multiple of 4 and 16-byte aligned cylinder
// rows, checked on the host); AEB = 0: synchronously, kFwdEB at a time.
template <typename EPI, int AEB>
__device__ __forceinline__ void forward_cone_binned_kernel_body(Geo g, int v_start, const float *__restrict__ values, int P, int band,
                           int slice_start, const ConeFwdRec *__restrict__ recs,
                           const int *__restrict__ list, const int *__restrict__ offs,
                           unsigned char *__restrict__ touched, EPI epi) {
  MBIR_PDL_ENTRY();
  extern __shared__ float4 sm4[];
  const int nthr = blockDim.x, tid = threadIdx.x;
  constexpr bool ASYNC = AEB > 0;
  const int cap = ASYNC ? fwd_cap_async(nthr) : fwd_cap(nthr);
  const int SP = band + 2 * kFwdVPad;
  constexpr int SEB = ASYNC ? 2 * AEB : kFwdEB;  // staged cylinders (both buffers)
  ConeFwdRec *rec = reinterpret_cast<ConeFwdRec *>(sm4);
  float *stage = reinterpret_cast<float *>(rec + cap);
  float *acc_s = stage + SEB * SP;  // (kFwdCB + 4) x nthr
  // (channel block, view) from the grid: views on x for whole-volume
  // epilogues (EPI::kViewFastest), so that the CTAs in flight are adjacent
  // views of one channel block, whose pixel strips nearly coincide and whose
  // cylinder reads hit L2; channel blocks on x otherwise.
  const bool vf = EPI::kViewFastest;
  const int nblk = vf ? gridDim.y : gridDim.x, blk = vf ? blockIdx.y : blockIdx.x,
            vl = vf ? blockIdx.x : blockIdx.y;
  const int c0 = blk * kFwdCB;
  const int ncb = min(kFwdCB, g.C - c0);
  const int bp = g.bp;
  const float kc_lo = (float)(slice_start - bp - 1),
              kc_hi = (float)(slice_start + band + bp);
  const ConeFwdRec *vrec = recs + (size_t)vl * P;
  const int *vlist = list + (size_t)vl * P;
  const int *voffs = offs + (size_t)vl * (fwd_nkeys(g.C) + 1);
  const int start = voffs[c0];
  const int end = voffs[min(c0 + kFwdCB + 2, fwd_nkeys(g.C))];
  const int v = v_start + vl;
  if (tid == 0) touched[(size_t)v * nblk + blk] = end > start;
  if (end == start) {
    // No pixel reaches the tile: its A x is zero (the VCD epilogue stores
    // nothing; its readers consult `touched`) and the partials are zero.
    epi.empty_tile(v, c0, ncb);
    epi.begin(v);
    epi.end(v * nblk + blk);
    return;
  }

  // Zero padding either side of each staged cylinder (the interiors are
  // written by every batch before they are read).
  for (int i = tid; i < SEB * 2 * kFwdVPad; i += nthr) {
    const int e = i / (2 * kFwdVPad), o = i - e * 2 * kFwdVPad;
    stage[e * SP + (o < kFwdVPad ? o : band + o)] = 0.f;
  }
#pragma unroll
  for (int r = 0; r < kFwdCB + 4; ++r) acc_s[r * nthr + tid] = 0.f;
  // The epilogue's operands (the error sinogram's cells of this tile) are
  // on their way to L2 while the tile is computed.
  epi.prefetch(v, c0, ncb);
  for (int base = start; base < end; base += cap) {
    const int n = min(cap, end - base);
    __syncthreads();
    for (int i = tid; i < n; i += nthr) rec[i] = fwd_stage_record(vrec[vlist[base + i]], c0);
    __syncthreads();
    if constexpr (ASYNC) {
      fwd_rt_round_async<AEB>(rec, n, stage, SP, values, band, slice_start, kc_lo, kc_hi, bp,
                              g.R, c0, acc_s);
      continue;
    }
    // The round's cylinders, 128-byte line by line, toward L1 ahead of the
    // batch staging.
    {
      const int lane = tid & 31, lines = (band + 31) / 32;
      for (int e = tid >> 5; e < n; e += nthr >> 5)
        for (int ln = lane; ln < lines; ln += 32)
          prefetch_l1(values + (size_t)__float_as_int(rec[e].c.w) * band + ln * 32);
    }
    fwd_rt_round<true>(rec, n, stage, SP, values, band, slice_start, kc_lo, kc_hi, bp, g.R, c0,
                       acc_s);
  }
  float acc[kFwdCB];
#pragma unroll
  for (int j = 0; j < kFwdCB; ++j) acc[j] = acc_s[(j + 2) * nthr + tid];
  epi.begin(v);
  if (tid < g.R) epi.cells(v, c0, ncb, tid, acc);
  epi.end(v * nblk + blk);
}

template <typename EPI, int AEB>
__global__ void __launch_bounds__(1024)

forward_cone_binned_kernel(Geo g, int v_start, const float *__restrict__ values, int P, int band,
                           int slice_start, const ConeFwdRec *__restrict__ recs,
                           const int *__restrict__ list, const int *__restrict__ offs,
                           unsigned char *__restrict__ touched, EPI epi) {
  forward_cone_binned_kernel_body<EPI, AEB>(g, v_start, values, P, band, slice_start, recs, list,
                                              offs, touched, epi);
}

// ── forward projection, parallel, binned ───────────────────────────────────
// The parallel-beam counterpart of forward_cone_binned_kernel for a VCD
// subset: one CTA per (channel block of kFwdCB, view), thread m owns
// detector row m (row m of a parallel view is slice m of the band, so its
// value for a pixel is the pixel's cylinder entry m, with no vertical fan).
// The CTA walks its run of the channel-sorted list (keys c0 .. c0 + 17):
// records are staged in shared memory a round at a time, and each thread
// loads the row's values of kParEB pixels at once (coalesced over the rows)
// before accumulating them.  With the pixels in channel order, the three
// channel sums a pixel adds to stay in registers (q0..q2 for accumulator
// rows cj .. cj + 2) and a row that leaves is added into the thread's
// private shared-memory column once.  No atomics: each cell is a fixed
// sequence of FMAs in list order.
constexpr int kParEB = 8;  // pixel values in flight per thread

__device__ __forceinline__ float4 f4_add(float4 a, float4 b) {
  return make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z),
                     __fadd_rn(a.w, b.w));
}

__device__ __forceinline__ float4 f4_fma(float w, float4 x, float4 q) {
  return make_float4(fmaf(w, x.x, q.x), fmaf(w, x.y, q.y), fmaf(w, x.z, q.z), fmaf(w, x.w, q.w));
}

constexpr int kPar4Cap = 128;  // records per round of the four-row forward

__host__ __device__ inline size_t par_binned4_smem(int nthr) {
  return (size_t)kPar4Cap * (sizeof(float4) + sizeof(int)) +
         (size_t)kFwdCB * nthr * sizeof(float4);
}

__host__ __device__ inline size_t par_binned_smem(int nthr) {
  return (size_t)fwd_cap(nthr) * (sizeof(float4) + sizeof(int)) +
         (size_t)(kFwdCB + 4) * nthr * sizeof(float);
}

template <typename EPI>
__device__ __forceinline__ void forward_parallel_binned_kernel_body(Geo g, int v_start, const float *__restrict__ values, int P,
                               int band, const ConeFwdRec *__restrict__ recs,
                               const int *__restrict__ list, const int *__restrict__ offs,
                               unsigned char *__restrict__ touched, EPI epi) {
  MBIR_PDL_ENTRY();
  extern __shared__ float4 sm4[];
  const int nthr = blockDim.x, tid = threadIdx.x;
  const int cap = fwd_cap(nthr);
  float4 *wq = sm4;                                   // cap x (w0, w1, w2, ctr)
  int *rows = reinterpret_cast<int *>(wq + cap);      // cap cylinder rows
  float *acc_s = reinterpret_cast<float *>(rows + cap);  // (kFwdCB + 4) x nthr
  // (channel block, view) from the grid: views on x for whole-volume
  // epilogues (EPI::kViewFastest), so that the CTAs in flight are adjacent
  // views of one channel block, whose pixel strips nearly coincide and whose
  // cylinder reads hit L2; channel blocks on x otherwise.
  const bool vf = EPI::kViewFastest;
  const int nblk = vf ? gridDim.y : gridDim.x, blk = vf ? blockIdx.y : blockIdx.x,
            vl = vf ? blockIdx.x : blockIdx.y;
  const int c0 = blk * kFwdCB;
  const int ncb = min(kFwdCB, g.C - c0);
  const ConeFwdRec *vrec = recs + (size_t)vl * P;
  const int *vlist = list + (size_t)vl * P;
  const int *voffs = offs + (size_t)vl * (fwd_nkeys(g.C) + 1);
  const int start = voffs[c0];
  const int end = voffs[min(c0 + kFwdCB + 2, fwd_nkeys(g.C))];
  const int v = v_start + vl;
  if (tid == 0) touched[(size_t)v * nblk + blk] = end > start;
  if (end == start) {
    epi.empty_tile(v, c0, ncb);
    epi.begin(v);
    epi.end(v * nblk + blk);
    return;
  }
#pragma unroll
  for (int r = 0; r < kFwdCB + 4; ++r) acc_s[r * nthr + tid] = 0.f;
  epi.prefetch(v, c0, ncb);
  const bool mine = tid < band;
  int cj = -1;
  float q0 = 0.f, q1 = 0.f, q2 = 0.f;
  for (int base = start; base < end; base += cap) {
    const int n = min(cap, end - base);
    __syncthreads();
    for (int i = tid; i < n; i += nthr) {
      const ConeFwdRec &r = vrec[vlist[base + i]];
      const float4 b = r.b, c = r.c;
      wq[i] = make_float4(b.y, b.z, b.w, c.z);
      rows[i] = __float_as_int(c.w);
    }
    __syncthreads();
    if (!mine) continue;
    if (cj < 0) cj = __float_as_int(wq[0].w) - c0 + 1;
    for (int e0 = 0; e0 < n; e0 += kParEB) {
      const int nb = min(kParEB, n - e0);
      float val[kParEB];
#pragma unroll
      for (int u = 0; u < kParEB; ++u)
        val[u] = u < nb ? __ldg(values + (size_t)rows[e0 + u] * band + tid) : 0.f;
#pragma unroll
      for (int u = 0; u < kParEB; ++u) {
        if (u >= nb) break;
        const float4 w = wq[e0 + u];
        const int j = __float_as_int(w.w) - c0 + 1;  // in [0, kFwdCB + 1], nondecreasing
        if (j != cj) {
          float *a = acc_s + cj * nthr + tid;
          a[0] += q0;
          if (j == cj + 1) {
            q0 = q1;
            q1 = q2;
          } else {
            a[nthr] += q1;
            if (j == cj + 2) {
              q0 = q2;
            } else {
              a[2 * nthr] += q2;
              q0 = 0.f;
            }
            q1 = 0.f;
          }
          q2 = 0.f;
          cj = j;
        }
        q0 = fmaf(w.x, val[u], q0);
        q1 = fmaf(w.y, val[u], q1);
        q2 = fmaf(w.z, val[u], q2);
      }
    }
  }
  if (mine) {
    float *a = acc_s + cj * nthr + tid;
    a[0] += q0;
    a[nthr] += q1;
    a[2 * nthr] += q2;
  }
  float acc[kFwdCB];
#pragma unroll
  for (int j = 0; j < kFwdCB; ++j) acc[j] = acc_s[(j + 2) * nthr + tid];
  epi.begin(v);
  if (mine) epi.cells(v, c0, ncb, tid, acc);
  epi.end(v * nblk + blk);
}

template <typename EPI>
__global__ void __launch_bounds__(1024)

forward_parallel_binned_kernel(Geo g, int v_start, const float *__restrict__ values, int P,
                               int band, const ConeFwdRec *__restrict__ recs,
                               const int *__restrict__ list, const int *__restrict__ offs,
                               unsigned char *__restrict__ touched, EPI epi) {
  forward_parallel_binned_kernel_body<EPI>(g, v_start, values, P, band, recs, list, offs, touched, epi);
}

// Four rows per thread (band a multiple of 4, at least 128 rows): thread t
// owns detector rows 4t .. 4t + 3, loads their four values of a pixel as one
// 16-byte access and keeps four sets of the three channel sums, so that the
// per-record work (record loads, key test, loop) is shared by four cells.
// The accumulator column holds the tile's kFwdCB channels only (a sum that
// leaves the registers for a channel outside the tile is dropped).  Each
// cell's sum is the same sequence of FMAs as in
// forward_parallel_binned_kernel.
template <typename EPI>
__device__ __forceinline__ void forward_parallel_binned4_kernel_body(Geo g, int v_start, const float *__restrict__ values, int P,
                                int band, const ConeFwdRec *__restrict__ recs,
                                const int *__restrict__ list, const int *__restrict__ offs,
                                unsigned char *__restrict__ touched, EPI epi) {
  MBIR_PDL_ENTRY();
  extern __shared__ float4 sm4[];
  const int nthr = blockDim.x, tid = threadIdx.x;
  float4 *wq = sm4;                                            // kPar4Cap x (w0, w1, w2, ctr)
  int *rows = reinterpret_cast<int *>(wq + kPar4Cap);          // kPar4Cap cylinder rows
  float4 *acc_s = reinterpret_cast<float4 *>(rows + kPar4Cap);  // kFwdCB x nthr
  // (channel block, view) from the grid: views on x for whole-volume
  // epilogues (EPI::kViewFastest), so that the CTAs in flight are adjacent
  // views of one channel block, whose pixel strips nearly coincide and whose
  // cylinder reads hit L2; channel blocks on x otherwise.
  const bool vf = EPI::kViewFastest;
  const int nblk = vf ? gridDim.y : gridDim.x, blk = vf ? blockIdx.y : blockIdx.x,
            vl = vf ? blockIdx.x : blockIdx.y;
  const int c0 = blk * kFwdCB;
  const int ncb = min(kFwdCB, g.C - c0);
  const ConeFwdRec *vrec = recs + (size_t)vl * P;
  const int *vlist = list + (size_t)vl * P;
  const int *voffs = offs + (size_t)vl * (fwd_nkeys(g.C) + 1);
  const int start = voffs[c0];
  const int end = voffs[min(c0 + kFwdCB + 2, fwd_nkeys(g.C))];
  const int v = v_start + vl;
  if (tid == 0) touched[(size_t)v * nblk + blk] = end > start;
  if (end == start) {
    epi.empty_tile(v, c0, ncb);
    epi.begin(v);
    epi.end(v * nblk + blk);
    return;
  }
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int r = 0; r < kFwdCB; ++r) acc_s[r * nthr + tid] = z4;
  epi.prefetch(v, c0, ncb);
  const int m0 = 4 * tid;
  const bool mine = m0 < band;
  // slot r of the register window is channel c0 + r - 2; channel slot
  // r - 2 of acc_s when inside the tile
  auto spill = [&](int r, float4 q) {
    if ((unsigned)(r - 2) < (unsigned)kFwdCB) {
      float4 *a = acc_s + (r - 2) * nthr + tid;
      *a = f4_add(*a, q);
    }
  };
  int cj = -1;
  float4 q0 = z4, q1 = z4, q2 = z4;
  for (int base = start; base < end; base += kPar4Cap) {
    const int n = min(kPar4Cap, end - base);
    __syncthreads();
    for (int i = tid; i < n; i += nthr) {
      const ConeFwdRec &r = vrec[vlist[base + i]];
      const float4 b = r.b, c = r.c;
      wq[i] = make_float4(b.y, b.z, b.w, c.z);
      rows[i] = __float_as_int(c.w);
    }
    __syncthreads();
    if (!mine) continue;
    if (cj < 0) cj = __float_as_int(wq[0].w) - c0 + 1;
    for (int e0 = 0; e0 < n; e0 += kParEB) {
      const int nb = min(kParEB, n - e0);
      float4 val[kParEB];
#pragma unroll
      for (int u = 0; u < kParEB; ++u)
        val[u] = u < nb ? __ldg(reinterpret_cast<const float4 *>(
                              values + (size_t)rows[e0 + u] * band + m0))
                        : z4;
#pragma unroll
      for (int u = 0; u < kParEB; ++u) {
        if (u >= nb) break;
        const float4 w = wq[e0 + u];
        const int j = __float_as_int(w.w) - c0 + 1;  // in [0, kFwdCB + 1], nondecreasing
        if (j != cj) {
          spill(cj, q0);
          if (j == cj + 1) {
            q0 = q1;
            q1 = q2;
          } else {
            spill(cj + 1, q1);
            if (j == cj + 2) {
              q0 = q2;
            } else {
              spill(cj + 2, q2);
              q0 = z4;
            }
            q1 = z4;
          }
          q2 = z4;
          cj = j;
        }
        q0 = f4_fma(w.x, val[u], q0);
        q1 = f4_fma(w.y, val[u], q1);
        q2 = f4_fma(w.z, val[u], q2);
      }
    }
  }
  if (mine) {
    spill(cj, q0);
    spill(cj + 1, q1);
    spill(cj + 2, q2);
  }
  epi.begin(v);
  if (mine) epi.cells4(v, c0, ncb, m0, acc_s + tid, nthr);
  epi.end(v * nblk + blk);
}

template <typename EPI>
__global__ void __launch_bounds__(256)

forward_parallel_binned4_kernel(Geo g, int v_start, const float *__restrict__ values, int P,
                                int band, const ConeFwdRec *__restrict__ recs,
                                const int *__restrict__ list, const int *__restrict__ offs,
                                unsigned char *__restrict__ touched, EPI epi) {
  forward_parallel_binned4_kernel_body<EPI>(g, v_start, values, P, band, recs, list, offs, touched, epi);
}

}  // namespace mbir
