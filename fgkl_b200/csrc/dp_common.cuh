// Device building blocks shared by the plain and PD PairHMM kernels: arithmetic policies, the
// precision constants, the per-row model of a read position, and record moves between registers,
// global scratch and shared memory.
#pragma once
#include <cuda_pipeline.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <type_traits>

#include "kernels.cuh"

namespace fgkl {

namespace {

constexpr unsigned kFull = 0xffffffffu;
// Warps per block: the default and largest. The first-pass kernels (pairhmm_kernel, pd_kernel) also
// launch with 1 or 2 (a tuning axis); a warp's index comes from blockDim there.
constexpr int kWarpsPerBlock = 4;
__host__ __device__ constexpr int warps_index(int warps) { return warps <= 1 ? 0 : (warps == 2 ? 1 : 2); }

// ---------------------------------------------------------------------------------------------
// Arithmetic policies.
// ---------------------------------------------------------------------------------------------

struct PackedF32 {
  using V = float2;
  using S = float;
  static constexpr int NC = 2;
  static constexpr bool kTransformed = true;
  static constexpr bool kDouble = false;
  __device__ __forceinline__ static V fma(V a, V b, V c) { return __ffma2_rn(a, b, c); }
  __device__ __forceinline__ static V mul(V a, V b) { return __fmul2_rn(a, b); }
  __device__ __forceinline__ static V add(V a, V b) { return __fadd2_rn(a, b); }
  __device__ __forceinline__ static V zero() { return make_float2(0.f, 0.f); }
  __device__ __forceinline__ static V splat(S s) { return make_float2(s, s); }
  __device__ __forceinline__ static S get(const V& v, int c) { return c ? v.y : v.x; }
  __device__ __forceinline__ static void put(V& v, int c, S s) {
    if (c)
      v.y = s;
    else
      v.x = s;
  }
  __device__ __forceinline__ static V up(V v) {
    return make_float2(__shfl_up_sync(kFull, v.x, 1), __shfl_up_sync(kFull, v.y, 1));
  }
  __device__ __forceinline__ static V down(V v) {
    return make_float2(__shfl_down_sync(kFull, v.x, 1), __shfl_down_sync(kFull, v.y, 1));
  }
  __device__ __forceinline__ static V sel(bool m0, bool m1, V a, V b) {
    return make_float2(m0 ? a.x : b.x, m1 ? a.y : b.y);
  }
  __device__ __forceinline__ static V max(V a, V b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
};

struct OneF32 {
  using V = float;
  using S = float;
  static constexpr int NC = 1;
  static constexpr bool kTransformed = true;
  static constexpr bool kDouble = false;
  __device__ __forceinline__ static V fma(V a, V b, V c) { return __fmaf_rn(a, b, c); }
  __device__ __forceinline__ static V mul(V a, V b) { return __fmul_rn(a, b); }
  __device__ __forceinline__ static V add(V a, V b) { return __fadd_rn(a, b); }
  __device__ __forceinline__ static V zero() { return 0.f; }
  __device__ __forceinline__ static V splat(S s) { return s; }
  __device__ __forceinline__ static S get(const V& v, int) { return v; }
  __device__ __forceinline__ static void put(V& v, int, S s) { v = s; }
  __device__ __forceinline__ static V up(V v) { return __shfl_up_sync(kFull, v, 1); }
  __device__ __forceinline__ static V down(V v) { return __shfl_down_sync(kFull, v, 1); }
  __device__ __forceinline__ static V sel(bool m0, bool, V a, V b) { return m0 ? a : b; }
  __device__ __forceinline__ static V max(V a, V b) { return fmaxf(a, b); }
};

struct OneF64 {
  using V = double;
  using S = double;
  static constexpr int NC = 1;
  static constexpr bool kTransformed = false;
  static constexpr bool kDouble = true;
  __device__ __forceinline__ static V fma(V a, V b, V c) { return __fma_rn(a, b, c); }
  __device__ __forceinline__ static V mul(V a, V b) { return __dmul_rn(a, b); }
  __device__ __forceinline__ static V add(V a, V b) { return __dadd_rn(a, b); }
  __device__ __forceinline__ static V zero() { return 0.0; }
  __device__ __forceinline__ static V splat(S s) { return s; }
  __device__ __forceinline__ static S get(const V& v, int) { return v; }
  __device__ __forceinline__ static void put(V& v, int, S s) { v = s; }
  __device__ __forceinline__ static V up(V v) { return __shfl_up_sync(kFull, v, 1); }
  __device__ __forceinline__ static V down(V v) { return __shfl_down_sync(kFull, v, 1); }
  __device__ __forceinline__ static V sel(bool m0, bool, V a, V b) { return m0 ? a : b; }
  __device__ __forceinline__ static V max(V a, V b) { return fmax(a, b); }
};

// Precision constants (fgkl simd.rs:102-154).
template <bool D>
struct Consts;
template <>
struct Consts<false> {
  static constexpr double kInitial = 0x1p120;
  static constexpr double kBackwardScale = 1329227995784915872903807060280344576.0;  // 2^120
  static constexpr double kLog10Initial = 120.0 * 0.301029995663981195213738894724493027;
  static constexpr double kMinAccepted = 1e-28;
  static constexpr double kMinAcceptedJoined = 1e-28;
};
template <>
struct Consts<true> {
  static constexpr double kInitial = 0x1p1020;
  static constexpr double kBackwardScale = 1.0;
  static constexpr double kLog10Initial = 1020.0 * 0.301029995663981195213738894724493027;
  static constexpr double kMinAccepted = 0.0;  // never lost
  static constexpr double kMinAcceptedJoined = 1e24;
};

// ---------------------------------------------------------------------------------------------
// Per-row parameters.
// ---------------------------------------------------------------------------------------------

struct ReadRef {
  int64_t off;  // first byte in the read arrays
  int len;      // 0 = empty component
  int pad;      // 32 * R - len
};

__device__ __forceinline__ double err_prob(const BatchView& v, int q) { return __ldg(v.err_prob + (q > 254 ? 254 : q)); }

__device__ __forceinline__ double match_to_match(const BatchView& v, int a, int b) {
  a = a > 254 ? 254 : a;
  b = b > 254 ? 254 : b;
  const int lo = a <= b ? a : b, hi = a <= b ? b : a;
  return __ldg(v.m2m + ((hi * (hi + 1)) >> 1) + lo);
}

// The f64 model values of read position q (fgkl model.rs:67-83).
struct RowModel {
  double mm, im, mi, md, gc, pm, px;
  double mi_prev, md_prev;  // of position q - 1; 1 above the read
  int oc;                   // prior code the read base matches (kNoCode: none)
  bool read;                // q is a read position
};

__device__ RowModel row_model(const BatchView& v, const ReadRef& r, int q, const uint8_t* codes) {
  RowModel m;
  m.read = r.len > 0 && q >= 0 && q < r.len;
  if (!m.read) {
    m.mm = m.im = m.mi = m.md = m.gc = m.pm = m.px = 0.0;
    m.mi_prev = m.md_prev = 1.0;
    m.oc = kNoCode;
    return m;
  }
  const int64_t o = r.off + q;
  const int base = v.bases[o], qual = v.quals[o], ins = v.ins[o], del = v.del[o], gcp = v.gcp[o];
  m.mm = match_to_match(v, ins, del);
  m.mi = err_prob(v, ins);
  m.md = err_prob(v, del);
  m.gc = err_prob(v, gcp);
  m.im = 1.0 - m.gc;
  const double e = err_prob(v, qual);
  m.pm = 1.0 - e;
  m.px = base == 'N' ? m.pm : e / 3.0;
  m.oc = codes[base];
  m.mi_prev = q > 0 ? err_prob(v, v.ins[o - 1]) : 1.0;
  m.md_prev = q > 0 ? err_prob(v, v.del[o - 1]) : 1.0;
  return m;
}

// Copies `fields` values (a multiple of 16 bytes) from global to shared memory without registers.
template <class V>
__device__ __forceinline__ void prefetch(V* dst_smem, const V* src, int fields) {
  const int chunks = fields * static_cast<int>(sizeof(V)) / 16;
  for (int i = 0; i < chunks; ++i)
    __pipeline_memcpy_async(reinterpret_cast<char*>(dst_smem) + 16 * i, reinterpret_cast<const char*>(src) + 16 * i, 16);
  __pipeline_commit();
}

// Moves a record of N values 16 bytes at a time (records start on 16 bytes; N is a multiple of the
// values per 16 bytes).
template <class V, int N>
__device__ __forceinline__ void store_record(V* dst, const V (&src)[N]) {
  static_assert(N * sizeof(V) % 16 == 0, "record size");
#pragma unroll
  for (int i = 0; i < static_cast<int>(N * sizeof(V) / 16); ++i)
    reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
}
template <class V, int N>
__device__ __forceinline__ void load_record(V (&dst)[N], const V* src) {
#pragma unroll
  for (int i = 0; i < static_cast<int>(N * sizeof(V) / 16); ++i)
    reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
}

__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// The bracket of the match recurrence, which the caller multiplies by the prior. In the FP32 form
// the row's match-to-match factor is folded into its priors (prior * mm) and out of k1 and k2
// (divided by mm), so the diagonal M enters unscaled and k0 is not read: three operations a cell with
// the prior instead of four. A row with mm = 0 makes k1 and k2 infinite and the cell NaN, which the
// acceptance test sends to the FP64 recomputation.
template <class P>
__device__ __forceinline__ typename P::V cell_match(const typename P::V& dM, const typename P::V& dX, const typename P::V& dY,
                                                    const typename P::V& k0, const typename P::V& k1, const typename P::V& k2) {
  if (P::kTransformed) return P::fma(dX, k1, P::fma(dY, k2, dM));
  // fgkl kernel.rs:1011: prior * (y_diag*im + (x_diag*im + m_diag*mm)).
  return P::fma(dY, k1, P::fma(dX, k1, P::mul(dM, k0)));
}

}  // namespace

// Resident blocks per SM of a kernel taking `smem` bytes of dynamic shared memory, resolved once per
// device and kept in `cache` (one per kernel, kMaxDevices entries, blocks + 1, 0 = unresolved): the
// attribute is set and the occupancy queried on the first call only, so each later batch's planning
// makes no CUDA call for it while other batches run.
constexpr int kMaxDevices = 64;
// `smem_limit` (default: `smem`) is the kernel's dynamic shared-memory limit to set, the largest block
// any launch of it uses.
template <class K>
int resident_blocks(K* kernel, size_t smem, int threads, std::atomic<int>* cache, size_t smem_limit = 0) {
  int dev = 0;
  cudaGetDevice(&dev);
  const bool keep = dev >= 0 && dev < kMaxDevices;
  if (keep) {
    const int c = cache[dev].load(std::memory_order_acquire);
    if (c) return c - 1;
  }
  int blocks = 0;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem_limit > smem ? smem_limit : smem));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, smem);
  if (keep) cache[dev].store(blocks + 1, std::memory_order_release);
  return blocks;
}

}  // namespace fgkl
