// Projector kernels (parallel and cone; forward and back) for sm_100a.
//
// BACK (gather, adjoint): a TEAM of T lanes owns one pixel's cylinder
// (a chunk of up to T*SPL slices) and walks a contiguous range of views,
// accumulating in registers.  The sinogram is read in the resident VCR
// layout, so every gather along the slice/row axis is unit-stride and
// coalesced.  For cone beam the warp first forms the view's horizontal
// detector column h(m) = sum_tc Wc * sino[v, c + tc, m] for the rows its
// slices reach (shared memory, one buffer per warp), then applies the
// vertical taps per slice -- the separable form of
// cone_beam.py:237-299.  View chunks (grid.y) write partial sums that
// reduce in a fixed order, so results are deterministic.
//
// FORWARD (scatter, expressed as a gather): a CTA owns one view and a block
// of CB detector channels over all rows.  It scans the pixel set, computes
// each pixel's centre channel, keeps the pixels whose footprint reaches its
// channel block (warp-ballot compaction in pixel order) and accumulates
// their taps into shared-memory tiles that each thread group owns
// privately; the groups' tiles are summed in a fixed order.  No atomics
// anywhere, so the forward is bit-reproducible.  The epilogue writes the
// block in either sinogram layout or, for VCD, fuses the line-search
// reductions against the error sinogram.
#pragma once

#include "mbir_common.cuh"

namespace mbir {

constexpr int kThreads = 256;
constexpr int kViewTab = 64;   // views staged per shared-memory table refill
constexpr int kListCap = 512;  // forward: pixel records per processing round

// ── sinogram readers (resident VCR layout) ─────────────────────────────────
struct ReadF32 {
  const float *s;
  int C, R;
  __device__ __forceinline__ float operator()(int v, int c, int m) const {
    return __ldg(s + ((size_t)v * C + c) * R + m);
  }
};

template <typename T>
struct ReadScaled {
  const T *e;
  const float *es;
  int C, R;
  __device__ __forceinline__ float operator()(int v, int c, int m) const {
    return __fmul_rn(to_f32(e[((size_t)v * C + c) * R + m]), __ldg(es + v));
  }
};

// weights * error, the gradient's operand (tomography_model.py:2548-2552).
template <typename T>
struct ReadWeighted {
  const T *e;
  const float *es;
  const T *w;
  const float *ws;
  int C, R;
  __device__ __forceinline__ float operator()(int v, int c, int m) const {
    size_t i = ((size_t)v * C + c) * R + m;
    float wv = __fmul_rn(to_f32(w[i]), __ldg(ws + v));
    float ev = __fmul_rn(to_f32(e[i]), __ldg(es + v));
    return __fmul_rn(wv, ev);
  }
};

struct ConeView {
  float ang, c, s, z_off;
};

// ── back projection: parallel ─────────────────────────────────────────────
template <int CP, int SPL, typename RD>
__global__ void __launch_bounds__(kThreads)
back_parallel_kernel(Geo g, const float *__restrict__ vp, int v_start, int v_count, int vpc,
                     RD rd, const int64_t *__restrict__ pix, int P, int band, int T,
                     int slice_chunks, float *__restrict__ out) {
  __shared__ ParView tab[kViewTab];
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
  const int r = g.psf, ntaps = 2 * g.psf + 1;
  float xt = 0.f, yt = 0.f;
  if (active) pixel_xy(g, (int)pix[p], xt, yt);
  float acc[SPL];
#pragma unroll
  for (int j = 0; j < SPL; ++j) acc[j] = 0.f;

  for (int v0 = vb; v0 < ve; v0 += kViewTab) {
    const int nv = min(kViewTab, ve - v0);
    __syncthreads();
    if (tid < nv) tab[tid] = parallel_view(g, vp[2 * (v_start + v0 + tid)]);
    __syncthreads();
    if (!active) continue;
    for (int i = 0; i < nv; ++i) {
      const ParView pv = tab[i];
      const float n_p = parallel_np(g, pv, xt, yt);
      const int ctr = (int)fminf(fmaxf(rintf(n_p), -1.0e6f), 1.0e6f);
      float w[kMaxTaps];
      int n[kMaxTaps];
#pragma unroll
      for (int t = 0; t < kMaxTaps; ++t) {
        w[t] = 0.f;
        n[t] = 0;
        if (t < ntaps) {
          const int nn = ctr + t - r;
          float a = tap_weight(n_p, nn, pv.half_w1, pv.lmax, pv.ws, g.C);
          if (CP == 2) a = __fmul_rn(a, a);
          w[t] = a;
          n[t] = min(max(nn, 0), g.C - 1);
        }
      }
      const int v = v0 + i;
#pragma unroll
      for (int j = 0; j < SPL; ++j) {
        const int l = l0 + tl + T * j;
        if (l < band) {
          float s = 0.f;
#pragma unroll
          for (int t = 0; t < kMaxTaps; ++t)
            if (t < ntaps && w[t] != 0.f) s = fmaf(w[t], rd(v, n[t], l), s);
          acc[j] += s;
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

// ── back projection: cone ─────────────────────────────────────────────────
// One warp per (pixel, slice chunk of 32*SPL slices).  Dynamic shared memory:
// 8 warps x R floats of detector-column buffer.
template <int CP, int SPL, typename RD>
__global__ void __launch_bounds__(kThreads)
back_cone_kernel(Geo g, const float *__restrict__ vp, int v_start, int v_count, int vpc, RD rd,
                 const int64_t *__restrict__ pix, int P, int slice_start, int band,
                 int slice_chunks, float *__restrict__ out) {
  extern __shared__ float colbuf[];
  __shared__ ConeView tab[kViewTab];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long gw = (long long)blockIdx.x * (kThreads / 32) + warp;
  const int p = (int)(gw / slice_chunks);
  const int sc = (int)(gw - (long long)p * slice_chunks);
  const bool active = p < P;
  const int l0 = sc * 32 * SPL;
  const int l_end = min(band, l0 + 32 * SPL);
  const int chunk = blockIdx.y;
  const int vb = chunk * vpc, ve = min(v_count, vb + vpc);
  const int r = g.psf, ntaps = 2 * g.psf + 1;
  float *h = colbuf + warp * g.R;
  float xt = 0.f, yt = 0.f;
  if (active) pixel_xy(g, (int)pix[p], xt, yt);
  float acc[SPL];
#pragma unroll
  for (int j = 0; j < SPL; ++j) acc[j] = 0.f;
  const float kf = (float)(slice_start + l0);
  const float kl = (float)(slice_start + max(l_end - 1, l0));

  for (int v0 = vb; v0 < ve; v0 += kViewTab) {
    const int nv = min(kViewTab, ve - v0);
    __syncthreads();
    if (tid < nv) {
      const int gv = v_start + v0 + tid;
      ConeView cv;
      cv.ang = vp[2 * gv];
      cv.c = cosf(cv.ang);
      cv.s = sinf(cv.ang);
      cv.z_off = __fsub_rn(g.rso, vp[2 * gv + 1]);
      tab[tid] = cv;
    }
    __syncthreads();
    if (!active) continue;
    for (int i = 0; i < nv; ++i) {
      const ConeView cv = tab[i];
      const ConeVP q = cone_vp(g, cv.ang, cv.c, cv.s, cv.z_off, xt, yt);
      float w[kMaxTaps];
      int n[kMaxTaps];
#pragma unroll
      for (int t = 0; t < kMaxTaps; ++t) {
        w[t] = 0.f;
        n[t] = 0;
        if (t < ntaps) {
          const int nn = q.ctr + t - r;
          float a = tap_weight(q.n_p, nn, q.half_w1, q.lmax, q.ws, g.C);
          if (CP == 2) a = __fmul_rn(a, a);
          w[t] = a;
          n[t] = min(max(nn, 0), g.C - 1);
        }
      }
      const int v = v0 + i;
      // Rows reached by this chunk's slices (the affine map is monotone in k).
      const float ma = __fadd_rn(q.m0, __fmul_rn(q.w_r, kf));
      const float mb = __fadd_rn(q.m0, __fmul_rn(q.w_r, kl));
      const float lo = fmaxf(floorf(fminf(ma, mb)) - (float)(r + 1), 0.f);
      const float hi = fminf(ceilf(fmaxf(ma, mb)) + (float)(r + 1), (float)(g.R - 1));
      if (lo <= hi) {
        const int m_lo = (int)lo, m_hi = (int)hi;
        for (int m = m_lo + lane; m <= m_hi; m += 32) {
          float s = 0.f;
#pragma unroll
          for (int t = 0; t < kMaxTaps; ++t)
            if (t < ntaps && w[t] != 0.f) s = fmaf(w[t], rd(v, n[t], m), s);
          h[m] = s;
        }
        __syncwarp();
        const float half_wr1 = __fdiv_rn(__fadd_rn(q.w_r, 1.f), 2.f);
        const float lmax_r = fminf(q.w_r, 1.f);
#pragma unroll
        for (int j = 0; j < SPL; ++j) {
          const int l = l0 + lane + 32 * j;
          if (l < band) {
            const float k = (float)(slice_start + l);
            const float m_p = __fadd_rn(q.m0, __fmul_rn(q.w_r, k));
            const float mpc = fminf(fmaxf(m_p, -(float)(r + 2)), (float)(g.R + r + 1));
            const int mc = (int)rintf(mpc);
            const float inv_cos = cone_inv_cos(g, q.mag, cv.z_off, k);
            float s = 0.f;
#pragma unroll
            for (int t = 0; t < kMaxTaps; ++t) {
              if (t < ntaps) {
                const int mm = mc + t - r;
                float a = fmaxf(__fsub_rn(half_wr1, fabsf(__fsub_rn(m_p, (float)mm))), 0.f);
                a = __fmul_rn(fminf(a, lmax_r), inv_cos);
                if (CP == 2) a = __fmul_rn(a, a);
                if (mm >= 0 && mm < g.R && a != 0.f) s = fmaf(a, h[mm], s);
              }
            }
            acc[j] += s;
          }
        }
      }
      __syncwarp();
    }
  }
  if (active) {
    float *o = out + (size_t)chunk * P * band + (size_t)p * band;
#pragma unroll
    for (int j = 0; j < SPL; ++j) {
      const int l = l0 + lane + 32 * j;
      if (l < band) o[l] = acc[j];
    }
  }
}

// out[i] = sum over chunks of part[chunk * n + i], in chunk order.
__global__ void reduce_chunks_kernel(const float *__restrict__ part, int chunks, size_t n,
                                     float *__restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int c = 0; c < chunks; ++c) s += part[(size_t)c * n + i];
    out[i] = s;
  }
}

// ── forward projection ────────────────────────────────────────────────────
struct FwdShape {
  int CB;   // channels per CTA
  int TG;   // threads per group (row lanes)
  int RPT;  // rows per thread
  int rows; // output rows (detector rows; == band for parallel)
  __host__ __device__ int RS() const { return TG * RPT + 1; }
  __host__ __device__ int G() const { return kThreads / TG; }
  size_t smem_bytes() const {
    return sizeof(float) * ((size_t)G() * CB * RS() + (size_t)kListCap * (2 + kMaxTaps + 6));
  }
};

// Epilogue: plain store in either sinogram layout.
struct StoreSino {
  float *out;
  int layout, C, R;
  __device__ __forceinline__ bool channel_fastest() const { return layout == MBIR_LAYOUT_VRC; }
  __device__ __forceinline__ void begin() {}
  __device__ __forceinline__ void cell(int v, int c, int m, float val) {
    if (layout == MBIR_LAYOUT_VCR)
      out[((size_t)v * C + c) * R + m] = val;
    else
      out[((size_t)v * R + m) * C + c] = val;
  }
  __device__ __forceinline__ void end(int) {}
};

template <bool CONE, typename EPI>
__global__ void __launch_bounds__(kThreads)
forward_kernel(Geo g, const float *__restrict__ vp, int v_start, const float *__restrict__ values,
               int P, int band, int slice_start, const int64_t *__restrict__ pix, FwdShape fs,
               EPI epi) {
  extern __shared__ float sm[];
  const int TG = fs.TG, G = fs.G(), RS = fs.RS(), CB = fs.CB, RPT = fs.RPT;
  const int rows = fs.rows;
  float *tile = sm;
  int *l_ctr = (int *)(tile + (size_t)G * CB * RS);
  int *l_pix = l_ctr + kListCap;
  float *l_w = (float *)(l_pix + kListCap);
  float *l_c = l_w + kMaxTaps * kListCap;  // cone: m0, w_r, half_wr1, lmax_r, inv_wr, mag
  __shared__ int s_wcount[kThreads / 32];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int vl = blockIdx.y;
  const int v = v_start + vl;
  const int c0 = blockIdx.x * CB;
  const int ncb = min(CB, g.C - c0);
  const int r = g.psf, ntaps = 2 * g.psf + 1, bp = g.bp;
  const float ang = vp[2 * v];
  const float cs = cosf(ang), sn = sinf(ang);
  const float z_off = __fsub_rn(g.rso, vp[2 * v + 1]);
  ParView pv;
  if (!CONE) pv = parallel_view(g, ang);

  for (int i = tid; i < G * CB * RS; i += kThreads) tile[i] = 0.f;
  const int grp = tid / TG, tg = tid - grp * TG;

  int pos = 0;
  while (pos < P) {
    int n = 0;
    __syncthreads();
    while (pos < P && n <= kListCap - kThreads) {
      const int p = pos + tid;
      bool keep = false;
      float xt = 0.f, yt = 0.f;
      int ctr = 0;
      float n_p = 0.f;
      ConeVP q;
      if (p < P) {
        pixel_xy(g, (int)pix[p], xt, yt);
        if (CONE) {
          q = cone_vp(g, ang, cs, sn, z_off, xt, yt);
          ctr = q.ctr;
          n_p = q.n_p;
        } else {
          n_p = parallel_np(g, pv, xt, yt);
          ctr = (int)fminf(fmaxf(rintf(n_p), -1.0e6f), 1.0e6f);
        }
        keep = (ctr + r >= c0) && (ctr - r < c0 + ncb);
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
        l_pix[slot] = p;
        const float hw1 = CONE ? q.half_w1 : pv.half_w1;
        const float lmx = CONE ? q.lmax : pv.lmax;
        const float wsc = CONE ? q.ws : pv.ws;
#pragma unroll
        for (int t = 0; t < kMaxTaps; ++t)
          l_w[t * kListCap + slot] = (t < ntaps) ? tap_weight(n_p, ctr + t - r, hw1, lmx, wsc, g.C) : 0.f;
        if (CONE) {
          l_c[0 * kListCap + slot] = q.m0;
          l_c[1 * kListCap + slot] = q.w_r;
          l_c[2 * kListCap + slot] = __fdiv_rn(__fadd_rn(q.w_r, 1.f), 2.f);
          l_c[3 * kListCap + slot] = fminf(q.w_r, 1.f);
          l_c[4 * kListCap + slot] = 1.f / q.w_r;
          l_c[5 * kListCap + slot] = q.mag;
        }
      }
      n += tot;
      pos += kThreads;
      __syncthreads();
    }
    // Accumulate the listed pixels: group grp takes entries grp, grp + G, ...
    float *mytile = tile + (size_t)grp * CB * RS;
    for (int e = grp; e < n; e += G) {
      const int ctr = l_ctr[e];
      const float *vrow = values + (size_t)l_pix[e] * band;
      float w[kMaxTaps];
#pragma unroll
      for (int t = 0; t < kMaxTaps; ++t) w[t] = l_w[t * kListCap + e];
      float m0 = 0.f, w_r = 0.f, half_wr1 = 0.f, lmax_r = 0.f, inv_wr = 0.f, mag = 0.f;
      if (CONE) {
        m0 = l_c[0 * kListCap + e];
        w_r = l_c[1 * kListCap + e];
        half_wr1 = l_c[2 * kListCap + e];
        lmax_r = l_c[3 * kListCap + e];
        inv_wr = l_c[4 * kListCap + e];
        mag = l_c[5 * kListCap + e];
      }
      for (int j = 0; j < RPT; ++j) {
        const int m = tg + TG * j;
        if (m >= rows) break;
        float det;
        if (!CONE) {
          det = __ldg(vrow + m);
        } else {
          // Detector-side vertical fan (cone_beam.py:203-226).
          const float k_m = __fmul_rn(__fsub_rn((float)m, m0), inv_wr);
          const float kc = rintf(fminf(fmaxf(k_m, -1.0e6f), 1.0e6f));
          const float d = __fmul_rn(w_r, __fsub_rn(kc, k_m));
          det = 0.f;
          for (int ko = -bp; ko <= bp; ++ko) {
            const int k_ind = (int)kc + ko;
            if (k_ind < slice_start || k_ind >= slice_start + band) continue;
            float a = fmaxf(__fsub_rn(half_wr1, fabsf(__fadd_rn(d, __fmul_rn(w_r, (float)ko)))), 0.f);
            a = fminf(a, lmax_r);
            if (a == 0.f) continue;
            const float sv = __fmul_rn(__ldg(vrow + (k_ind - slice_start)),
                                       cone_inv_cos(g, mag, z_off, (float)k_ind));
            det = fmaf(a, sv, det);
          }
        }
        if (det == 0.f) continue;
#pragma unroll
        for (int t = 0; t < kMaxTaps; ++t) {
          const int ch = ctr + t - r - c0;
          if (t < ntaps && ch >= 0 && ch < ncb && w[t] != 0.f) {
            float *cell = mytile + (size_t)ch * RS + m;
            *cell = fmaf(w[t], det, *cell);
          }
        }
      }
    }
  }
  __syncthreads();
  // Epilogue: sum the groups' tiles in group order and hand each cell over.
  epi.begin();
  const int cells = ncb * rows;
  if (epi.channel_fastest()) {
    for (int i = tid; i < cells; i += kThreads) {
      const int ch = i % ncb, m = i / ncb;
      float s = 0.f;
      for (int gg = 0; gg < G; ++gg) s += tile[((size_t)gg * CB + ch) * RS + m];
      epi.cell(vl, c0 + ch, m, s);
    }
  } else {
    for (int i = tid; i < cells; i += kThreads) {
      const int ch = i / rows, m = i - (i / rows) * rows;
      float s = 0.f;
      for (int gg = 0; gg < G; ++gg) s += tile[((size_t)gg * CB + ch) * RS + m];
      epi.cell(vl, c0 + ch, m, s);
    }
  }
  epi.end(blockIdx.y * gridDim.x + blockIdx.x);
}

}  // namespace mbir
