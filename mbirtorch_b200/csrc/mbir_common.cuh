// Shared device-side definitions for the sm_100a MBIR kernels.
//
// Geometry: the per-(view, pixel) chains of the reference are recomputed
// in-kernel from a handful of per-model constants (struct Geo) instead of
// being materialized per call as the reference's Triton wrappers do
// (triton_cone.py:469-497 charges 48 B per view-pixel for that).  The FP32
// operation order follows the reference torch bodies:
//   parallel  parallel_beam.py:22-53
//   cone      cone_beam.py:59-158
// Scalars that the reference forms in Python double precision before they
// meet an FP32 tensor (e.g. (num_rows - 1) / 2.0, 1.0 / magnification) are
// formed the same way on the host (make_geo) and rounded once to float.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mbir_b200.h"

namespace mbir {

constexpr int kMaxTaps = 2 * MBIR_MAX_TAP_RADIUS + 1;

struct Geo {
  int cone;
  int V, R, C, NR, NC, S;
  int psf, bp, curved;
  float ddc, ddr, offc, offr, dv, dvr, dvs, rso, sdd;
  // derived (host, double -> float)
  float rc_row;      // (NR - 1) / 2
  float rc_col;      // (NC - 1) / 2
  float det_cc;      // (C - 1) / 2
  float det_cr;      // (R - 1) / 2
  float slice_c;     // (S - 1) / 2
  float half_z;      // dvs * (S - 1) / 2
  float inv_M;       // 1 / magnification
  float sid;         // sdd / magnification
  float area;        // dvr * dv
  float inv_sdd;     // 1 / sdd (0 at sdd = inf)
};

inline Geo make_geo(const mbir_geometry &g) {
  Geo o;
  o.cone = g.geometry == MBIR_CONE;
  o.V = g.num_views;
  o.R = g.num_det_rows;
  o.C = g.num_det_channels;
  o.NR = g.num_recon_rows;
  o.NC = g.num_recon_cols;
  o.S = g.num_slices;
  o.psf = g.psf_radius;
  o.bp = g.bp_psf_radius;
  o.curved = g.use_curved_detector;
  o.ddc = g.delta_det_channel;
  o.ddr = g.delta_det_row;
  o.offc = g.det_channel_offset;
  o.offr = g.det_row_offset;
  o.dv = g.delta_voxel;
  o.dvr = g.delta_voxel_row;
  o.dvs = g.delta_voxel_slice;
  o.rso = g.recon_slice_offset;
  o.sdd = g.source_detector_dist;
  o.rc_row = (float)((g.num_recon_rows - 1) / 2.0);
  o.rc_col = (float)((g.num_recon_cols - 1) / 2.0);
  o.det_cc = (float)((g.num_det_channels - 1) / 2.0);
  o.det_cr = (float)((g.num_det_rows - 1) / 2.0);
  o.slice_c = (float)((g.num_slices - 1) / 2.0);
  o.half_z = (float)((double)g.delta_voxel_slice * (g.num_slices - 1) / 2.0);
  o.inv_M = (float)(1.0 / (double)g.magnification);
  o.sid = (float)((double)g.source_detector_dist / (double)g.magnification);
  o.area = (float)((double)g.delta_voxel_row * (double)g.delta_voxel);
  o.inv_sdd = (float)(1.0 / (double)g.source_detector_dist);
  return o;
}

// ── shared-memory loads at 32-bit addresses ────────────────────────────────
// The forward's row loop forms its record and stage addresses as 32-bit
// shared-window offsets (__cvta_generic_to_shared of the CTA's buffers plus
// a byte offset) and loads with ld.shared, which measured fewer integer
// instructions per iteration than indexing the generic pointers.
__device__ __forceinline__ float lds_f32(unsigned a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ float4 lds_f32x4(unsigned a) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(a));
  return v;
}

// ── storage types ──────────────────────────────────────────────────────────
__device__ __forceinline__ float to_f32(float v) { return v; }
__device__ __forceinline__ float to_f32(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_f32(__half v) { return __half2float(v); }

template <typename T> __device__ __forceinline__ T from_f32(float v);
template <> __device__ __forceinline__ float from_f32<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}
template <> __device__ __forceinline__ __half from_f32<__half>(float v) {
  return __float2half_rn(v);
}

// Four consecutive stored values at p (16-byte aligned for FP32, 8-byte for
// 16-bit types) as one vector access.
template <typename T>
__device__ __forceinline__ void load4(const T *p, float (&o)[4]) {
  if constexpr (sizeof(T) == 4) {
    const float4 v = *reinterpret_cast<const float4 *>(p);
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
  } else {
    const uint2 v = *reinterpret_cast<const uint2 *>(p);
    const T *t = reinterpret_cast<const T *>(&v);
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = to_f32(t[k]);
  }
}

template <typename T>
__device__ __forceinline__ void store4(T *p, const T (&s)[4]) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4(s[0], s[1], s[2], s[3]);
  } else {
    uint2 v;
    T *t = reinterpret_cast<T *>(&v);
#pragma unroll
    for (int k = 0; k < 4; ++k) t[k] = s[k];
    *reinterpret_cast<uint2 *>(p) = v;
  }
}

// ── geometry chains ────────────────────────────────────────────────────────
// Un-rotated pixel centre (x, y) relative to iso (note the (i, j) -> (y, x)
// order of the reference).
__device__ __forceinline__ void pixel_xy(const Geo &g, int pix, float &xt, float &yt) {
  int row = pix / g.NC;
  int col = pix - row * g.NC;
  yt = __fmul_rn(g.dvr, __fsub_rn((float)row, g.rc_row));
  xt = __fmul_rn(g.dv, __fsub_rn((float)col, g.rc_col));
}

// Trapezoid weight of channel tap n (horizontal_fan.py:51-71): the overlap
// of the projected voxel with detector cell n, zeroed off the detector.
__device__ __forceinline__ float tap_weight(float n_p, int n, float half_w1, float lmax,
                                            float ws, int C) {
  float a = fmaxf(__fsub_rn(half_w1, fabsf(__fsub_rn(n_p, (float)n))), 0.f);
  a = __fmul_rn(fminf(a, lmax), ws);
  return (n >= 0 && n < C) ? a : 0.f;
}

// Per-view constants of the parallel chain (W and the weight scale depend
// on the view only).
struct ParView {
  float c, s, half_w1, lmax, ws;
};

__device__ __forceinline__ ParView parallel_view(const Geo &g, float angle) {
  ParView o;
  o.c = cosf(angle);
  o.s = sinf(angle);
  float fp = fmaxf(__fmul_rn(fabsf(o.c), g.dv), __fmul_rn(fabsf(o.s), g.dvr));
  float W = __fdiv_rn(fp, g.ddc);
  o.half_w1 = __fdiv_rn(__fadd_rn(W, 1.f), 2.f);
  o.lmax = fminf(W, 1.f);
  o.ws = __fdiv_rn(g.area, fp);
  return o;
}

// Continuous channel coordinate of a pixel in a parallel view.
__device__ __forceinline__ float parallel_np(const Geo &g, const ParView &pv, float xt,
                                             float yt) {
  float x = __fsub_rn(__fmul_rn(pv.c, xt), __fmul_rn(pv.s, yt));
  return __fadd_rn(__fdiv_rn(__fadd_rn(x, g.offc), g.ddc), g.det_cc);
}

// Cone, first half of the chain: rotated pixel, magnification and the
// continuous channel coordinate (all the forward projector's pixel scan
// needs to decide whether a pixel reaches its channel block).
struct ConeCenter {
  float n_p, mag, u, y;
  int ctr;
};

__device__ __forceinline__ ConeCenter cone_center(const Geo &g, float c, float s, float xt,
                                                  float yt) {
  ConeCenter o;
  const float x = __fsub_rn(__fmul_rn(c, xt), __fmul_rn(s, yt));
  o.y = __fadd_rn(__fmul_rn(s, xt), __fmul_rn(c, yt));
  o.mag = __fdiv_rn(1.f, __fsub_rn(g.inv_M, __fdiv_rn(o.y, g.sdd)));
  if (!g.curved)
    o.u = __fmul_rn(o.mag, x);
  else
    o.u = __fmul_rn(g.sdd, atan2f(x, __fsub_rn(g.sid, o.y)));
  o.n_p = __fadd_rn(__fdiv_rn(__fadd_rn(o.u, g.offc), g.ddc), g.det_cc);
  o.ctr = (int)fminf(fmaxf(rintf(o.n_p), -1.0e6f), 1.0e6f);
  return o;
}

// Cone: per (view, pixel) horizontal fan data + the vertical affine pair.
struct ConeVP {
  float n_p, half_w1, lmax, ws;  // horizontal fan
  float mag, m0, w_r;            // vertical fan: m(k) = m0 + w_r * k
  int ctr;
};

// Second half of the chain (cone_beam.py:93-158): footprint, width, weight
// scale and the vertical affine pair.
__device__ __forceinline__ ConeVP cone_finish(const Geo &g, float angle, float z_off,
                                              const ConeCenter &cc) {
  ConeVP o;
  const float theta = !g.curved ? atan2f(cc.u, g.sdd) : __fdiv_rn(cc.u, g.sdd);
  o.n_p = cc.n_p;
  o.ctr = cc.ctr;
  o.mag = cc.mag;
  const float da = __fsub_rn(angle, theta);
  const float fp = fmaxf(__fmul_rn(fabsf(cosf(da)), g.dv), __fmul_rn(fabsf(sinf(da)), g.dvr));
  float W = __fmul_rn(cc.mag, __fdiv_rn(fp, g.ddc));
  if (!g.curved) W = __fdiv_rn(W, cosf(theta));
  o.half_w1 = __fdiv_rn(__fadd_rn(W, 1.f), 2.f);
  o.lmax = fminf(W, 1.f);
  o.ws = __fdiv_rn(g.area, fp);
  o.w_r = __fdiv_rn(__fmul_rn(cc.mag, g.dvs), g.ddr);
  const float z0 = __fsub_rn(z_off, g.half_z);
  o.m0 = __fadd_rn(__fdiv_rn(__fadd_rn(__fmul_rn(cc.mag, z0), g.offr), g.ddr), g.det_cr);
  return o;
}

__device__ __forceinline__ ConeVP cone_vp(const Geo &g, float angle, float c, float s,
                                          float z_off, float xt, float yt) {
  return cone_finish(g, angle, z_off, cone_center(g, c, s, xt, yt));
}

// t(k) = mag * z_k / SDD = a0 + a1 * k for global slice k, the argument of
// 1 / cos(phi) = sqrt(1 + t^2) (cone_beam.py:207-212, 282-286).
__device__ __forceinline__ void cone_tcoef(const Geo &g, float mag, float z_off, float &a0,
                                           float &a1) {
  a1 = __fmul_rn(__fmul_rn(mag, g.dvs), g.inv_sdd);
  a0 = __fmul_rn(__fmul_rn(mag, __fsub_rn(z_off, __fmul_rn(g.dvs, g.slice_c))), g.inv_sdd);
}

// Programmatic dependent launch (sm_90 and later).  A kernel launched with
// programmatic stream serialization may begin while the kernel before it
// in the stream is still running: pdl_wait() returns once that grid has
// completed and its writes are visible (at once for a kernel launched the
// ordinary way), and pdl_release() lets the stream's next kernel begin its
// launch.  MBIR_PDL_ENTRY() opens every kernel that the library may launch
// that way, before the kernel touches global memory.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
#define MBIR_PDL_ENTRY() \
  do {                   \
    pdl_wait();          \
    pdl_release();       \
  } while (0)

// sqrt(1 + t^2) from the fast reciprocal square root (q * rsqrt(q)).
__device__ __forceinline__ float inv_cos_from_t(float t) {
  const float q = fmaf(t, t, 1.f);
  return q * rsqrtf(q);
}

// The same value through the flush-to-zero form of the hardware reciprocal
// square root: q >= 1 is never subnormal, so the result equals
// inv_cos_from_t without rsqrtf's subnormal-input handling.  Used where it
// measured faster (the forward's cylinder staging).
__device__ __forceinline__ float inv_cos_from_t_ftz(float t) {
  const float q = fmaf(t, t, 1.f);
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(q));
  return q * r;
}

// 1 / cos(phi) for the voxel at global slice k of a cone (view, pixel):
// sqrt(1 + (v / SDD)^2) with v = mag * z_k, the same quantity as the
// reference's 1 / cos(atan2(v, SDD)) (exactly 1 at SDD = inf).
__device__ __forceinline__ float cone_inv_cos(const Geo &g, float mag, float z_off, float k) {
  float z = __fadd_rn(__fmul_rn(g.dvs, __fsub_rn(k, g.slice_c)), z_off);
  float t = __fmul_rn(__fmul_rn(mag, z), g.inv_sdd);
  return sqrtf(fmaf(t, t, 1.f));
}

}  // namespace mbir
