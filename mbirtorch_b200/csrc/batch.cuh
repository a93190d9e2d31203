// Cross-job batching of the VCD subset step.
//
// Several reconstructions that share a geometry (a scanner protocol served
// many times) step their subsets together: one launch of each kernel of the
// subset step covers every job, with the job index on grid z.  The kernels
// are the single-job ones: each is a __device__ body (the `*_body`
// functions of projectors.cuh / vcd.cuh) called by its own __global__
// wrapper, and by batched_kernel<B, ...> below, which picks job blockIdx.z's
// arguments out of a table passed by value (up to kMaxBatch jobs; a table of
// a few KB stays well inside the 32 KB kernel-parameter limit).
//
// The host builds the tables by running the single-job launch chain once per
// job in RECORD mode (launchb records instead of launching), then replays
// each recorded launch once for all jobs.  Jobs of one batch take the same
// branches (same geometry, storage and options), so their chains match
// launch for launch; a mismatch is an error.
#pragma once

#include <cstring>
#include <utility>
#include <vector>

#include "vcd.cuh"

namespace mbir {

constexpr int kMaxBatch = MBIR_MAX_BATCH;

// A trivially copyable argument list (kernel arguments are copied byte for
// byte into the parameter table).
template <typename... A> struct ArgPack;
template <> struct ArgPack<> {};
template <typename H, typename... T> struct ArgPack<H, T...> {
  H head;
  ArgPack<T...> tail;
};

template <int I> struct ArgAt {
  template <typename H, typename... T>
  __host__ __device__ static auto get(const ArgPack<H, T...> &a)
      -> decltype(ArgAt<I - 1>::get(a.tail)) {
    return ArgAt<I - 1>::get(a.tail);
  }
};
template <> struct ArgAt<0> {
  template <typename H, typename... T>
  __host__ __device__ static const H &get(const ArgPack<H, T...> &a) {
    return a.head;
  }
};

inline ArgPack<> make_pack() { return ArgPack<>{}; }
template <typename H, typename... T>
ArgPack<H, T...> make_pack(H h, T... t) {
  ArgPack<H, T...> a;
  a.head = h;
  a.tail = make_pack(t...);
  return a;
}

template <typename... K> struct BatchTable {
  ArgPack<K...> job[kMaxBatch];
};

template <typename B, typename... K, size_t... I>
__device__ __forceinline__ void run_job(const ArgPack<K...> &a, std::index_sequence<I...>) {
  B::run(ArgAt<(int)I>::get(a)...);
}

template <typename B, typename... K>
__global__ void __launch_bounds__(B::kMaxThreads, B::kMinBlocks)
batched_kernel(const __grid_constant__ BatchTable<K...> t) {
  run_job<B>(t.job[blockIdx.z], std::index_sequence_for<K...>{});
}

// ── the subset step's kernels as batchable bodies ─────────────────────────
// B::kernel() is the single-job __global__ wrapper, B::run its body.
template <int CP, int SPL, int NT, typename RD> struct BackParallelB {
  static constexpr int kMaxThreads = kThreads, kMinBlocks = 1;
  static auto kernel() { return back_parallel_kernel<CP, SPL, NT, RD>; }
  template <typename... A> __device__ static void run(const A &...a) {
    back_parallel_kernel_body<CP, SPL, NT, RD>(a...);
  }
};
template <int CP, int T, typename RD> struct BackParallel4B {
  static constexpr int kMaxThreads = kThreads, kMinBlocks = 1;
  static auto kernel() { return back_parallel4_kernel<CP, T, RD>; }
  template <typename... A> __device__ static void run(const A &...a) {
    back_parallel4_kernel_body<CP, T, RD>(a...);
  }
};
template <int CP, int SPL, int NT, typename RD, int HBL = 8> struct BackConeB {
  static constexpr int kMaxThreads = kThreads, kMinBlocks = 1;
  static auto kernel() { return back_cone_kernel<CP, SPL, NT, RD, HBL>; }
  template <typename... A> __device__ static void run(const A &...a) {
    back_cone_kernel_body<CP, SPL, NT, RD, HBL>(a...);
  }
};
struct ConeBinB {
  static constexpr int kMaxThreads = 256, kMinBlocks = 1;
  static auto kernel() { return cone_bin_kernel; }
  template <typename... A> __device__ static void run(const A &...a) { cone_bin_kernel_body(a...); }
};
template <typename EPI, int AEB> struct FwdConeBinnedB {
  static constexpr int kMaxThreads = 1024, kMinBlocks = 1;
  static auto kernel() { return forward_cone_binned_kernel<EPI, AEB>; }
  template <typename... A> __device__ static void run(const A &...a) {
    forward_cone_binned_kernel_body<EPI, AEB>(a...);
  }
};
template <typename EPI> struct FwdParBinnedB {
  static constexpr int kMaxThreads = 1024, kMinBlocks = 1;
  static auto kernel() { return forward_parallel_binned_kernel<EPI>; }
  template <typename... A> __device__ static void run(const A &...a) {
    forward_parallel_binned_kernel_body<EPI>(a...);
  }
};
template <typename EPI> struct FwdParBinned4B {
  static constexpr int kMaxThreads = 256, kMinBlocks = 1;
  static auto kernel() { return forward_parallel_binned4_kernel<EPI>; }
  template <typename... A> __device__ static void run(const A &...a) {
    forward_parallel_binned4_kernel_body<EPI>(a...);
  }
};
template <bool DC> struct DirectionB {
  static constexpr int kMaxThreads = kThreads, kMinBlocks = 1;
  static auto kernel() { return vcd_direction_kernel<DC>; }
  template <typename... A> __device__ static void run(const A &...a) {
    vcd_direction_kernel_body<DC>(a...);
  }
};
struct DcSumsB {
  static constexpr int kMaxThreads = 32 * kDcGroups, kMinBlocks = 1;
  static auto kernel() { return vcd_dc_sums_kernel; }
  template <typename... A> __device__ static void run(const A &...a) {
    vcd_dc_sums_kernel_body(a...);
  }
};
struct DcDirectionB {
  static constexpr int kMaxThreads = 256, kMinBlocks = 1;
  static auto kernel() { return vcd_dc_direction_kernel; }
  template <typename... A> __device__ static void run(const A &...a) {
    vcd_dc_direction_kernel_body(a...);
  }
};
struct AlphaB {
  static constexpr int kMaxThreads = kAlphaThreads, kMinBlocks = 1;
  static auto kernel() { return vcd_alpha_kernel; }
  template <typename... A> __device__ static void run(const A &...a) { vcd_alpha_kernel_body(a...); }
};
struct PositivityB {
  static constexpr int kMaxThreads = 256, kMinBlocks = 1;
  static auto kernel() { return vcd_positivity_kernel; }
  template <typename... A> __device__ static void run(const A &...a) {
    vcd_positivity_kernel_body(a...);
  }
};
template <typename T> struct TailB {
  static constexpr int kMaxThreads = 256, kMinBlocks = 6;
  static auto kernel() { return vcd_tail_kernel<T>; }
  template <typename... A> __device__ static void run(const A &...a) { vcd_tail_kernel_body<T>(a...); }
};

}  // namespace mbir
