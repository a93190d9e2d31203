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

// ── sinogram readers (resident VCR layout) ─────────────────────────────────
// value(v, c, m) = scale(v) * get(base(v, c) + m)
struct ReadF32 {
  const float *s;
  int C, R;
  __device__ __forceinline__ size_t base(int v, int c) const { return ((size_t)v * C + c) * R; }
  __device__ __forceinline__ float scale(int) const { return 1.f; }
  __device__ __forceinline__ float get(size_t i) const { return __ldg(s + i); }
};

template <typename T>
struct ReadScaled {
  const T *e;
  const float *es;
  int C, R;
  __device__ __forceinline__ size_t base(int v, int c) const { return ((size_t)v * C + c) * R; }
  __device__ __forceinline__ float scale(int v) const { return __ldg(es + v); }
  __device__ __forceinline__ float get(size_t i) const { return to_f32(e[i]); }
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

// ── back projection: parallel ─────────────────────────────────────────────
template <int CP, int SPL, int NT, typename RD>
__global__ void __launch_bounds__(kThreads)
back_parallel_kernel(Geo g, const float *__restrict__ vp, int v_start, int v_count, int vpc,
                     RD rd, const int64_t *__restrict__ pix, int P, int band, int T,
                     int slice_chunks, float *__restrict__ out) {
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
    for (int i = 0; i < nv; ++i) {
      const int v = vg + i;
      const int ctr = mytab[i].ctr;
      float w[MT];
      size_t base[MT];
#pragma unroll
      for (int t = 0; t < MT; ++t) {
        w[t] = mytab[i].w[t];
        base[t] = rd.base(v, min(max(ctr + t - RT, 0), g.C - 1));
      }
      const float scl = rd.scale(v);
#pragma unroll
      for (int j = 0; j < SPL; ++j) {
        const int l = l0 + tl + T * j;
        if (l < band) {
          float s = 0.f;
#pragma unroll
          for (int t = 0; t < MT; ++t)
            if (MBIR_TAP_ON(NT, t, nt)) s = fmaf(w[t], rd.get(base[t] + l), s);
          acc[j] = fmaf(scl, s, acc[j]);
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
// One warp per (pixel, chunk of 32*SPL slices).  Dynamic shared memory:
// 8 warps x (R + 2 kPad) floats of column buffer, then 8 x 32 ConeRec.
template <int CP, int SPL, int NT, typename RD>
__global__ void __launch_bounds__(kThreads)
back_cone_kernel(Geo g, const float *__restrict__ vp, int v_start, int v_count, int vpc, RD rd,
                 const int64_t *__restrict__ pix, int P, int slice_start, int band,
                 int slice_chunks, float *__restrict__ out) {
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
    if (lane < nv) {
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
        const int m_lo = (int)lo, m_hi = (int)hi;
        for (int m = m_lo + lane; m <= m_hi; m += 32) {
          float s = 0.f;
#pragma unroll
          for (int t = 0; t < MT; ++t)
            if (MBIR_TAP_ON(NT, t, nt)) s = fmaf(w[t], rd.get(base[t] + m), s);
          h[m] = __fmul_rn(s, scl);
        }
      }
      __syncwarp();
#pragma unroll
      for (int j = 0; j < SPL; ++j) {
        const int l = l0 + lane + 32 * j;
        if (l < band) {
          const float k = (float)(slice_start + l);
          const float m_p = fminf(fmaxf(fmaf(w_r, k, m0), mlo_clamp), mhi_clamp);
          const float mcf = rintf(m_p);
          const int mc = (int)mcf;
          const float d = m_p - mcf;
          float s = 0.f;
#pragma unroll
          for (int t = 0; t < MT; ++t) {
            if (MBIR_TAP_ON(NT, t, nt)) {
              float a = fminf(fmaxf(hw1r - fabsf(d - (float)(t - RT)), 0.f), lmaxr);
              if (CP == 2) a = a * a;
              s = fmaf(a, h[mc + t - RT], s);
            }
          }
          const float tk = fmaf(a1, k, a0);
          const float ic = CP == 2 ? fmaf(tk, tk, 1.f) : inv_cos_from_t(tk);
          acc[j] = fmaf(ic, s, acc[j]);
        }
      }
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

template <bool CONE, int NT, typename EPI>
__global__ void __launch_bounds__(kThreads)
forward_kernel(Geo g, const float *__restrict__ vp, int v_start, const float *__restrict__ values,
               int P, int band, int slice_start, const int64_t *__restrict__ pix, FwdShape fs,
               int by_pixel, EPI epi) {
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

// ── forward projection, cone, register-tiled ───────────────────────────────
// The cone forward for psf radius 1 and up to 1024 detector rows.  A CTA
// owns one view and kFwdCB channels; thread m owns detector row m and keeps
// the row's kFwdCB channel sums in registers.  Pixels reaching the block are
// compacted as in forward_kernel, then processed in batches of kFwdEB: the
// batch's cylinders, scaled by 1 / cos(phi) per slice, are staged in
// zero-padded shared memory (one rsqrt per voxel), and every thread forms
// its row's detector-side vertical fan from them (cone_beam.py:203-226)
// and adds the three channel taps into registers.  The tap -> register map
// depends on the pixel's centre channel, which is the same for all threads,
// so it is a warp-uniform switch over compile-time register indices: no
// shared-memory read-modify-write chains, no atomics, fixed summation order.
constexpr int kFwdCB = 16;   // channels per CTA
constexpr int kFwdEB = 16;   // pixels staged per batch
constexpr int kFwdVPad = 8;  // zero slices either side of a staged cylinder (>= 2 bp + 1)
constexpr int kFwdRec = 12;  // record words per pixel

// Record capacity of one compaction round: at least one scan chunk.
__host__ __device__ inline int fwd_cap(int nthr) { return nthr > 512 ? nthr : 512; }

template <int J>
__device__ __forceinline__ void fwd_taps(float (&acc)[kFwdCB], float w0, float w1, float w2,
                                         float det) {
  // Case J: the pixel's centre channel is c0 + J - 1, so tap t lands on
  // block channel J - 2 + t.
  if (J - 2 >= 0 && J - 2 < kFwdCB) acc[(J - 2 >= 0 && J - 2 < kFwdCB) ? J - 2 : 0] =
      fmaf(w0, det, acc[(J - 2 >= 0 && J - 2 < kFwdCB) ? J - 2 : 0]);
  if (J - 1 >= 0 && J - 1 < kFwdCB) acc[(J - 1 >= 0 && J - 1 < kFwdCB) ? J - 1 : 0] =
      fmaf(w1, det, acc[(J - 1 >= 0 && J - 1 < kFwdCB) ? J - 1 : 0]);
  if (J >= 0 && J < kFwdCB) acc[(J >= 0 && J < kFwdCB) ? J : 0] =
      fmaf(w2, det, acc[(J >= 0 && J < kFwdCB) ? J : 0]);
}

template <typename EPI>
__global__ void __launch_bounds__(1024)
forward_cone_rt_kernel(Geo g, const float *__restrict__ vp, int v_start,
                       const float *__restrict__ values, int P, int band, int slice_start,
                       const int64_t *__restrict__ pix, int by_pixel, EPI epi) {
  extern __shared__ float sm[];
  const int nthr = blockDim.x;
  const int kFwdCap = fwd_cap(nthr);
  const int SP = band + 2 * kFwdVPad;                 // staged cylinder pitch
  float *stage = sm;                                  // kFwdEB x SP
  int *r_ctr = (int *)(stage + kFwdEB * SP);          // kFwdCap
  int *r_row = r_ctr + kFwdCap;                       // kFwdCap
  float *r_f = (float *)(r_row + kFwdCap);            // 10 x kFwdCap
  __shared__ int s_wcount[32];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
  const int vl = blockIdx.y;
  const int v = v_start + vl;
  const int c0 = blockIdx.x * kFwdCB;
  const int ncb = min(kFwdCB, g.C - c0);
  const float ang = vp[2 * v];
  const float cs = cosf(ang), sn = sinf(ang);
  const float z_off = __fsub_rn(g.rso, vp[2 * v + 1]);
  const int m = tid;
  const float mf = (float)m;
  const int bp = g.bp;
  // Clamp of the centre slice: a centre outside [ss - bp - 1, ss + band + bp]
  // has no tap inside the band, and the clamped one only meets zero padding
  // (kFwdVPad >= 2 bp + 1).
  const float kc_lo = (float)(slice_start - bp - 1),
              kc_hi = (float)(slice_start + band + bp);
  const int R = g.R;

  for (int i = tid; i < kFwdEB * SP; i += nthr) stage[i] = 0.f;
  float acc[kFwdCB];
#pragma unroll
  for (int j = 0; j < kFwdCB; ++j) acc[j] = 0.f;

  int pos = 0;
  while (pos < P) {
    int n = 0;
    __syncthreads();
    while (pos < P && n + nthr <= kFwdCap) {
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
      if (keep) {
        const int s = off + __popc(bal & ((1u << lane) - 1u));
        const ConeVP q = cone_finish(g, ang, z_off, cc);
        float a0, a1;
        cone_tcoef(g, q.mag, z_off, a0, a1);
        r_ctr[s] = cc.ctr - c0 + 1;  // switch case: centre channel + 1, in [0, kFwdCB + 1]
        r_row[s] = by_pixel ? (int)pix[p] : p;
        r_f[0 * kFwdCap + s] = tap_weight(cc.n_p, cc.ctr - 1, q.half_w1, q.lmax, q.ws, g.C);
        r_f[1 * kFwdCap + s] = tap_weight(cc.n_p, cc.ctr, q.half_w1, q.lmax, q.ws, g.C);
        r_f[2 * kFwdCap + s] = tap_weight(cc.n_p, cc.ctr + 1, q.half_w1, q.lmax, q.ws, g.C);
        r_f[3 * kFwdCap + s] = q.m0;
        r_f[4 * kFwdCap + s] = q.w_r;
        r_f[5 * kFwdCap + s] = __fdiv_rn(__fadd_rn(q.w_r, 1.f), 2.f);
        r_f[6 * kFwdCap + s] = fminf(q.w_r, 1.f);
        r_f[7 * kFwdCap + s] = 1.f / q.w_r;
        r_f[8 * kFwdCap + s] = a0;
        r_f[9 * kFwdCap + s] = a1;
      }
      n += tot;
      pos += nthr;
      __syncthreads();
    }
    for (int b0 = 0; b0 < n; b0 += kFwdEB) {
      const int nb = min(kFwdEB, n - b0);
      // Stage the batch's scaled cylinders.
      for (int i = tid; i < nb * band; i += nthr) {
        const int e = i / band, k = i - e * band;
        const int r = b0 + e;
        const float tk = fmaf(r_f[9 * kFwdCap + r], (float)(slice_start + k), r_f[8 * kFwdCap + r]);
        stage[e * SP + kFwdVPad + k] =
            __ldg(values + (size_t)r_row[r] * band + k) * inv_cos_from_t(tk);
      }
      __syncthreads();
      if (m < R) {
        for (int e = 0; e < nb; ++e) {
          const int r = b0 + e;
          const float m0 = r_f[3 * kFwdCap + r], w_r = r_f[4 * kFwdCap + r];
          const float hw1r = r_f[5 * kFwdCap + r], lmaxr = r_f[6 * kFwdCap + r];
          const float inv_wr = r_f[7 * kFwdCap + r];
          const float k_m = (mf - m0) * inv_wr;
          const float kc = fminf(fmaxf(rintf(k_m), kc_lo), kc_hi);
          const float d = w_r * (kc - k_m);
          const float *st = stage + e * SP + kFwdVPad + ((int)kc - slice_start);
          float det;
          if (bp == 1) {
            const float am = fminf(fmaxf(hw1r - fabsf(d - w_r), 0.f), lmaxr);
            const float a0 = fminf(fmaxf(hw1r - fabsf(d), 0.f), lmaxr);
            const float ap = fminf(fmaxf(hw1r - fabsf(d + w_r), 0.f), lmaxr);
            det = fmaf(ap, st[1], fmaf(a0, st[0], am * st[-1]));
          } else {
            det = 0.f;
            for (int ko = -bp; ko <= bp; ++ko) {
              const float a = fminf(fmaxf(hw1r - fabsf(fmaf(w_r, (float)ko, d)), 0.f), lmaxr);
              det = fmaf(a, st[ko], det);
            }
          }
          const float w0 = r_f[0 * kFwdCap + r], w1 = r_f[1 * kFwdCap + r];
          const float w2 = r_f[2 * kFwdCap + r];
          switch (r_ctr[r]) {
            case 0: fwd_taps<0>(acc, w0, w1, w2, det); break;
            case 1: fwd_taps<1>(acc, w0, w1, w2, det); break;
            case 2: fwd_taps<2>(acc, w0, w1, w2, det); break;
            case 3: fwd_taps<3>(acc, w0, w1, w2, det); break;
            case 4: fwd_taps<4>(acc, w0, w1, w2, det); break;
            case 5: fwd_taps<5>(acc, w0, w1, w2, det); break;
            case 6: fwd_taps<6>(acc, w0, w1, w2, det); break;
            case 7: fwd_taps<7>(acc, w0, w1, w2, det); break;
            case 8: fwd_taps<8>(acc, w0, w1, w2, det); break;
            case 9: fwd_taps<9>(acc, w0, w1, w2, det); break;
            case 10: fwd_taps<10>(acc, w0, w1, w2, det); break;
            case 11: fwd_taps<11>(acc, w0, w1, w2, det); break;
            case 12: fwd_taps<12>(acc, w0, w1, w2, det); break;
            case 13: fwd_taps<13>(acc, w0, w1, w2, det); break;
            case 14: fwd_taps<14>(acc, w0, w1, w2, det); break;
            case 15: fwd_taps<15>(acc, w0, w1, w2, det); break;
            case 16: fwd_taps<16>(acc, w0, w1, w2, det); break;
            default: fwd_taps<17>(acc, w0, w1, w2, det); break;
          }
        }
      }
      __syncthreads();
    }
  }
  // Epilogue: thread m hands over its row's cells, channel by channel.
  epi.begin();
  if (m < R) {
#pragma unroll
    for (int j = 0; j < kFwdCB; ++j)
      if (j < ncb) epi.cell(vl, c0 + j, m, acc[j]);
  }
  epi.end(blockIdx.y * gridDim.x + blockIdx.x);
}

}  // namespace mbir
