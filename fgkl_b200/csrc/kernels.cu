// sm_100a PairHMM kernels: one warp per read task, read rows on lanes, columns streamed as an
// anti-diagonal wavefront.
//
// Lane l holds rows l*R .. l*R+R-1 of a 32*R-row block whose LAST row is the read's last row; the
// rows above the read are padding rows whose transitions reproduce row 0 of GATK's matrix (M = X =
// 0 and a constant deletion value of INITIAL / haplotype length), so the row just above the read
// plays row 0 and every read ends on lane 31's last row. At loop step t lane l computes stream
// position t - l (forward) or t - (31 - l) (backward); the row above (below) arrives from the
// neighbouring lane by one shuffle per state value per step.
//
// Forward recurrence per cell (GATK LoglessPairHMM, fgkl kernel.rs:1011-1013):
//   M = prior * (mm*M(i-1,j-1) + im*(X(i-1,j-1) + Y(i-1,j-1)))
//   X = mi*M(i-1,j) + ii*X(i-1,j)          Y = md*M(i,j-1) + dd*Y(i,j-1)
// The single-precision kernels carry X/mi and Y/md instead of X and Y (per-row constants), which
// turns the X and Y updates into one FMA each: 6 FP32 operations per cell instead of 8. Every term
// stays positive, so the change of variables costs no accuracy; an overflow it could cause in
// pathological gap-open ratios surfaces as a non-finite result, which the double-precision
// recomputation replaces. The double-precision kernels use the plain recurrence.
//
// Backward recurrence (suffix sharing, fgkl kernel.rs:1080-1088) per cell, row i from row i+1:
//   into = prior(i+1,j+1) * BM(i+1,j+1);  BX = ii'*BX(i+1,j) + im'*into
//   BY = dd*BY(i,j+1) + im'*into;         BM = md*BY(i,j+1) + mi'*BX(i+1,j) + mm'*into
// with primed transitions those of row i+1, plus BACKWARD_SCALE at the read's last row.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace fgkl {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = 4;

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
};

// Precision constants (fgkl simd.rs:102-154).
template <bool D>
struct Consts;
template <>
struct Consts<false> {
  static constexpr double kBackwardScale = 1329227995784915872903807060280344576.0;  // 2^120
  static constexpr double kLog10Initial = 36.123599479677743;                         // 120*log10(2)
  static constexpr double kMinAccepted = 1e-28;
  static constexpr double kMinAcceptedJoined = 1e-28;
};
template <>
struct Consts<true> {
  static constexpr double kBackwardScale = 1.0;
  static constexpr double kLog10Initial = 307.05059557726084;  // 1020*log10(2)
  static constexpr double kMinAccepted = 0.0;                 // never lost
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

// Forward coefficients of the lane's rows.
template <class P, int R>
struct FwdRows {
  using V = typename P::V;
  using S = typename P::S;
  V c0[R], c1[R], c2[R], c3[R], c4[R], pm[R], px[R];
  int oc[P::NC][R];

  __device__ void load(const BatchView& v, const ReadRef* rd, int lane, const uint8_t* codes) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
      for (int c = 0; c < P::NC; ++c) {
        const int g = lane * R + r;
        const RowModel m = row_model(v, rd[c], g - rd[c].pad, codes);
        double k0, k1, k2, k3, k4;
        if (P::kTransformed) {
          // S = mm*M + (im*mi')*X^ + (im*md')*Y^ with X = mi*X^, Y = md*Y^; X^ = M_up + c3*X^_up; Y^ = M_left + gc*Y^_left.
          if (m.read) {
            k0 = m.mm;
            k1 = m.im * m.mi_prev;
            k2 = m.im * m.md_prev;
            k3 = m.gc * m.mi_prev / m.mi;
            k4 = m.gc;
          } else {
            k0 = k1 = k2 = k3 = 0.0;
            k4 = 1.0;
          }
        } else {
          if (m.read) {
            k0 = m.mm;
            k1 = m.im;
            k2 = m.mi;
            k3 = m.gc;
            k4 = m.md;
          } else {
            k0 = k1 = k2 = k4 = 0.0;
            k3 = 1.0;
          }
        }
        P::put(c0[r], c, static_cast<S>(k0));
        P::put(c1[r], c, static_cast<S>(k1));
        P::put(c2[r], c, static_cast<S>(k2));
        P::put(c3[r], c, static_cast<S>(k3));
        P::put(c4[r], c, static_cast<S>(k4));
        P::put(pm[r], c, static_cast<S>(m.pm));
        P::put(px[r], c, static_cast<S>(m.px));
        oc[c][r] = m.oc;
      }
    }
  }
};

// Backward coefficients: each row's own deletion transitions and the transitions and priors of the
// row below it (rows l*R+1 .. l*R+R; the last comes from the next lane's top row).
template <class P, int R>
struct BwdRows {
  using V = typename P::V;
  using S = typename P::S;
  V md[R], dd[R], mm[R], im[R], mi[R], ii[R], pm[R], px[R];
  int oc[P::NC][R];

  __device__ void load(const BatchView& v, const ReadRef* rd, int lane, const uint8_t* codes) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
      for (int c = 0; c < P::NC; ++c) {
        const int g = lane * R + r;
        const RowModel self = row_model(v, rd[c], g - rd[c].pad, codes);
        const RowModel below = row_model(v, rd[c], g + 1 - rd[c].pad, codes);
        P::put(md[r], c, static_cast<S>(self.read ? self.md : 0.0));
        P::put(dd[r], c, static_cast<S>(self.read ? self.gc : 1.0));
        P::put(mm[r], c, static_cast<S>(below.mm));
        P::put(im[r], c, static_cast<S>(below.im));
        P::put(mi[r], c, static_cast<S>(below.mi));
        P::put(ii[r], c, static_cast<S>(below.gc));
        P::put(pm[r], c, static_cast<S>(below.pm));
        P::put(px[r], c, static_cast<S>(below.px));
        oc[c][r] = below.oc;
      }
    }
  }
};

// ---------------------------------------------------------------------------------------------
// Per-warp scratch: snapshots, backward nodes, segment results.
// ---------------------------------------------------------------------------------------------

template <class P, int R>
struct Scratch {
  using V = typename P::V;
  static constexpr int kSnapFields = 3 * R + 5;  // M, X, Y rows; above-row M, X, Y; acc M, X
  static constexpr int kNodeFields = 2 * R + 1;  // BM, BY rows; below-row BM
  V* snaps;
  V* nodes;
  double* seg_acc;   // [seg][c]
  double* seg_prod;  // [seg][row g][c]

  __device__ Scratch(char* base, int max_slots, int max_nodes, int max_segs) {
    snaps = reinterpret_cast<V*>(base);
    nodes = snaps + static_cast<size_t>(max_slots) * kSnapFields * 32;
    seg_acc = reinterpret_cast<double*>(nodes + static_cast<size_t>(max_nodes) * kNodeFields * 32);
    seg_prod = seg_acc + static_cast<size_t>(max_segs) * P::NC;
  }
  __device__ V* snap(int slot, int f, int lane) { return snaps + (static_cast<size_t>(slot) * kSnapFields + f) * 32 + lane; }
  __device__ V* node(int n, int f, int lane) { return nodes + (static_cast<size_t>(n) * kNodeFields + f) * 32 + lane; }
  __device__ double* prod(int seg, int g, int c) { return seg_prod + (static_cast<size_t>(seg) * 32 * R + g) * P::NC + c; }
};

template <class P, int R>
__host__ __device__ constexpr size_t scratch_size(int max_slots, int max_nodes, int max_segs) {
  using V = typename P::V;
  return static_cast<size_t>(max_slots) * (3 * R + 5) * 32 * sizeof(V) + static_cast<size_t>(max_nodes) * (2 * R + 1) * 32 * sizeof(V) +
         static_cast<size_t>(max_segs) * P::NC * sizeof(double) + static_cast<size_t>(max_segs) * 32 * R * P::NC * sizeof(double);
}

// ---------------------------------------------------------------------------------------------
// Backward pass: every suffix sweep of the program, writing backward nodes.
// ---------------------------------------------------------------------------------------------

template <class P, int R>
__device__ void backward_pass(const LaunchArgs& a, const Program& prog, const ReadRef* rd, const uint8_t* codes, int lane,
                              Scratch<P, R>& sc, unsigned long long& columns) {
  using V = typename P::V;
  BwdRows<P, R> bp;
  bp.load(a.v, rd, lane, codes);
  const V sink = P::splat(lane == 31 ? static_cast<typename P::S>(Consts<P::kDouble>::kBackwardScale) : 0);
  V BM[R], BY[R];
#pragma unroll
  for (int r = 0; r < R; ++r) BM[r] = BY[r] = P::zero();
  V dBM = P::zero(), topBM = P::zero(), topBX = P::zero();
  const uint16_t* stream = a.v.stream + prog.bwd_off;
  const int n = prog.bwd_len;
  int sweep = prog.sweep_off - 1, nodew = prog.nodew_off;
  for (int t = 0; t < n + 31; ++t) {
    V rBM = P::down(topBM), rBX = P::down(topBX);
    if (lane == 31) rBM = rBX = P::zero();
    const int p = t - (31 - lane);
    const bool live = p >= 0 && p < n;
    const uint16_t ev = live ? __ldg(stream + p) : 0;
    if (ev & EV_SWEEP) {
      const int start = a.v.sweep_starts[++sweep];
      if (start < 0) {
#pragma unroll
        for (int r = 0; r < R; ++r) BM[r] = BY[r] = P::zero();
        dBM = P::zero();
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          BM[r] = *sc.node(start, r, lane);
          BY[r] = *sc.node(start, R + r, lane);
        }
        dBM = *sc.node(start, 2 * R, lane);
      }
    }
    if (live) {
      const int code = ev & kCodeMask;
      const bool isN = code == kCodeN;
      V belowX = rBX, diagM = dBM;
#pragma unroll
      for (int r = R - 1; r >= 0; --r) {
        const bool m0 = (code == bp.oc[0][r]) | isN;
        const bool m1 = (code == bp.oc[P::NC - 1][r]) | isN;
        const V prior = P::sel(m0, m1, bp.pm[r], bp.px[r]);
        const V into = P::mul(prior, diagM);
        const V itm = P::mul(into, bp.im[r]);
        V bx = P::fma(belowX, bp.ii[r], itm);
        const V by = P::fma(BY[r], bp.dd[r], itm);
        V bm = P::fma(BY[r], bp.md[r], P::fma(belowX, bp.mi[r], P::mul(into, bp.mm[r])));
        if (r == R - 1) {
          bm = P::add(bm, sink);
          bx = P::add(bx, sink);
        }
        diagM = BM[r];
        BM[r] = bm;
        BY[r] = by;
        belowX = bx;
      }
      topBM = BM[0];
      topBX = belowX;
      dBM = rBM;
      if (lane == 0) ++columns;
    }
    if (ev & EV_NODE) {
      const int node = a.v.node_writes[nodew++];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        *sc.node(node, r, lane) = BM[r];
        *sc.node(node, R + r, lane) = BY[r];
      }
      *sc.node(node, 2 * R, lane) = rBM;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Forward pass.
// ---------------------------------------------------------------------------------------------

template <class P>
__device__ __forceinline__ typename P::V cell_match(const typename P::V& dM, const typename P::V& dX, const typename P::V& dY,
                                                    const typename P::V& k0, const typename P::V& k1, const typename P::V& k2) {
  if (P::kTransformed) return P::fma(dM, k0, P::fma(dX, k1, P::mul(dY, k2)));
  // fgkl kernel.rs:1011: prior * (y_diag*im + (x_diag*im + m_diag*mm)).
  return P::fma(dY, k1, P::fma(dX, k1, P::mul(dM, k0)));
}

template <class P, int R>
__device__ void forward_pass(const LaunchArgs& a, const Program& prog, const ReadRef* rd, const uint8_t* codes, int lane,
                             Scratch<P, R>& sc, unsigned long long& columns) {
  using V = typename P::V;
  using S = typename P::S;
  FwdRows<P, R> fr;
  fr.load(a.v, rd, lane, codes);
  // Which of the lane's rows (and the row above them) are padding, per component.
  unsigned pad_mask[P::NC];
  bool above_pad[P::NC];
#pragma unroll
  for (int c = 0; c < P::NC; ++c) {
    pad_mask[c] = 0;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (lane * R + r < rd[c].pad) pad_mask[c] |= 1u << r;
    above_pad[c] = lane * R - 1 < rd[c].pad;
  }
  // X factor of the read's last row (lane 31), turning the accumulated X^ back into X.
  double last_mi[P::NC];
#pragma unroll
  for (int c = 0; c < P::NC; ++c)
    last_mi[c] = (P::kTransformed && rd[c].len > 0) ? err_prob(a.v, a.v.ins[rd[c].off + rd[c].len - 1]) : 1.0;

  V M[R], X[R], Y[R];
#pragma unroll
  for (int r = 0; r < R; ++r) M[r] = X[r] = Y[r] = P::zero();
  V dM = P::zero(), dX = P::zero(), dY = P::zero();
  V aM = P::zero(), aX = P::zero(), aY = P::zero();  // row above at the segment's start column
  V accM = P::zero(), accX = P::zero();
  V init = P::zero();
  Segment seg{};
  const uint16_t* stream = a.v.stream + prog.fwd_off;
  const int n = prog.fwd_len;
  int seg_i = -1, snap_i = prog.snap_off;
  uint16_t ev_next = (lane == 0 && n > 0) ? __ldg(stream) : 0;
  for (int t = 0; t < n + 31; ++t) {
    V uM = P::up(M[R - 1]), uX = P::up(X[R - 1]), uY = P::up(Y[R - 1]);
    const int p = t - lane;
    const bool live = p >= 0 && p < n;
    const uint16_t ev = ev_next;
    ev_next = (p + 1 >= 0 && p + 1 < n) ? __ldg(stream + p + 1) : 0;
    if (ev & EV_BEGIN) {
      ++seg_i;
      seg = a.v.segs[prog.seg_off + seg_i];
      const S sc_s = P::kDouble ? static_cast<S>(seg.scale_d) : static_cast<S>(seg.scale_f);
      const S in_s = P::kDouble ? static_cast<S>(seg.init_d) : static_cast<S>(seg.init_f);
      init = P::splat(in_s);
      const V scale = P::splat(sc_s);
      if (seg.slot_in < 0) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          M[r] = X[r] = P::zero();
#pragma unroll
          for (int c = 0; c < P::NC; ++c) P::put(Y[r], c, (pad_mask[c] >> r) & 1 ? in_s : S(0));
        }
        aM = aX = P::zero();
#pragma unroll
        for (int c = 0; c < P::NC; ++c) P::put(aY, c, above_pad[c] ? in_s : S(0));
        accM = accX = P::zero();
      } else {
        const int s = seg.slot_in;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          M[r] = P::mul(*sc.snap(s, r, lane), scale);
          X[r] = P::mul(*sc.snap(s, R + r, lane), scale);
          Y[r] = P::mul(*sc.snap(s, 2 * R + r, lane), scale);
#pragma unroll
          for (int c = 0; c < P::NC; ++c)
            if ((pad_mask[c] >> r) & 1) P::put(Y[r], c, in_s);
        }
        aM = P::mul(*sc.snap(s, 3 * R, lane), scale);
        aX = P::mul(*sc.snap(s, 3 * R + 1, lane), scale);
        aY = P::mul(*sc.snap(s, 3 * R + 2, lane), scale);
#pragma unroll
        for (int c = 0; c < P::NC; ++c)
          if (above_pad[c]) P::put(aY, c, in_s);
        accM = P::mul(*sc.snap(s, 3 * R + 3, lane), scale);
        accX = P::mul(*sc.snap(s, 3 * R + 4, lane), scale);
      }
      dM = aM;
      dX = aX;
      dY = aY;
    }
    if (lane == 0) {
      uM = uX = P::zero();
      uY = init;
    }
    if (ev & EV_NOCOMP) {
      uM = aM;
      uX = aX;
      uY = aY;
    }
    if (live && !(ev & EV_NOCOMP)) {
      const int code = ev & kCodeMask;
      const bool isN = code == kCodeN;
      V pM = dM, pX = dX, pY = dY, qM = uM, qX = uX;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const V oM = M[r], oX = X[r], oY = Y[r];
        const bool m0 = (code == fr.oc[0][r]) | isN;
        const bool m1 = (code == fr.oc[P::NC - 1][r]) | isN;
        const V prior = P::sel(m0, m1, fr.pm[r], fr.px[r]);
        const V nM = P::mul(prior, cell_match<P>(pM, pX, pY, fr.c0[r], fr.c1[r], fr.c2[r]));
        V nX, nY;
        if (P::kTransformed) {
          nX = P::fma(qX, fr.c3[r], qM);
          nY = P::fma(oY, fr.c4[r], oM);
        } else {
          nX = P::fma(qX, fr.c3[r], P::mul(qM, fr.c2[r]));
          nY = P::fma(oY, fr.c3[r], P::mul(oM, fr.c4[r]));
        }
        M[r] = nM;
        X[r] = nX;
        Y[r] = nY;
        pM = oM;
        pX = oX;
        pY = oY;
        qM = nM;
        qX = nX;
      }
      dM = uM;
      dX = uX;
      dY = uY;
      accM = P::add(accM, M[R - 1]);
      accX = P::add(accX, X[R - 1]);
      if (lane == 0) ++columns;
    }
    if (ev & EV_SNAP) {
      const int s = a.v.snap_slots[snap_i++];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        *sc.snap(s, r, lane) = M[r];
        *sc.snap(s, R + r, lane) = X[r];
        *sc.snap(s, 2 * R + r, lane) = Y[r];
      }
      *sc.snap(s, 3 * R, lane) = uM;
      *sc.snap(s, 3 * R + 1, lane) = uX;
      *sc.snap(s, 3 * R + 2, lane) = uY;
      *sc.snap(s, 3 * R + 3, lane) = accM;
      *sc.snap(s, 3 * R + 4, lane) = accX;
    }
    if (ev & EV_END) {
      if (lane == 31) {
#pragma unroll
        for (int c = 0; c < P::NC; ++c)
          sc.seg_acc[seg_i * P::NC + c] =
              __dadd_rn(static_cast<double>(P::get(accM, c)), __dmul_rn(last_mi[c], static_cast<double>(P::get(accX, c))));
      }
      if (seg.node >= 0) {
        // Join (fgkl kernel.rs:744-755, :767-791): the cut column's match and deletion values,
        // entered from this column, times the backward node's values, per row in f64.
        const int code = seg.cut_code;
        const bool isN = code == kCodeN;
        V jM = uM, jX = uX, jY = uY;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const bool m0 = (code == fr.oc[0][r]) | isN;
          const bool m1 = (code == fr.oc[P::NC - 1][r]) | isN;
          const V prior = P::sel(m0, m1, fr.pm[r], fr.px[r]);
          const V fM = P::mul(prior, cell_match<P>(jM, jX, jY, fr.c0[r], fr.c1[r], fr.c2[r]));
          const V fY = P::kTransformed ? P::fma(Y[r], fr.c4[r], M[r]) : P::fma(Y[r], fr.c3[r], P::mul(M[r], fr.c4[r]));
          const V bM = *sc.node(seg.node, r, lane);
          const V bY = *sc.node(seg.node, R + r, lane);
          const int g = lane * R + r;
#pragma unroll
          for (int c = 0; c < P::NC; ++c) {
            double yfac = 1.0;
            const int q = g - rd[c].pad;
            if (P::kTransformed && rd[c].len > 0 && q >= 0) yfac = err_prob(a.v, a.v.del[rd[c].off + q]);
            const double fy = __dmul_rn(yfac, static_cast<double>(P::get(fY, c)));
            *sc.prod(seg_i, g, c) = __dadd_rn(__dmul_rn(static_cast<double>(P::get(fM, c)), static_cast<double>(P::get(bM, c))),
                                              __dmul_rn(fy, static_cast<double>(P::get(bY, c))));
          }
          jM = M[r];
          jX = X[r];
          jY = Y[r];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Finalisation: raw results to log10 likelihoods in the caller's layout.
// ---------------------------------------------------------------------------------------------

template <class P, int R>
__device__ void finalize(const LaunchArgs& a, const Task& task, const Region& region, const Program& prog, const ReadRef* rd,
                         int lane, Scratch<P, R>& sc) {
  using C = Consts<P::kDouble>;
  bool lost_any[P::NC];
  unsigned long long lost_count = 0;
#pragma unroll
  for (int c = 0; c < P::NC; ++c) lost_any[c] = false;
  for (int k = lane; k < region.n_haps; k += 32) {
    const HapInfo info = a.v.haps[region.hap_off + k];
    const Segment seg = a.v.segs[prog.seg_off + info.seg];
#pragma unroll
    for (int c = 0; c < P::NC; ++c) {
      if (task.read[c] < 0) continue;
      double raw = sc.seg_acc[info.seg * P::NC + c];
      bool lost;
      if (seg.node >= 0) {
        double sum = 0.0;
        for (int g = rd[c].pad; g < 32 * R; ++g) sum = __dadd_rn(sum, *sc.prod(info.seg, g, c));
        sum = __dadd_rn(sum, *sc.prod(info.seg, rd[c].pad - 1, c));
        raw = __dadd_rn(raw, __ddiv_rn(sum, C::kBackwardScale));
        lost = !(raw >= C::kMinAcceptedJoined);
      } else {
        lost = a.min_accept_plain ? !(raw >= C::kMinAccepted) : (raw != raw);
      }
      if (!P::kDouble) lost |= isinf(raw);
      const double result = lost ? __longlong_as_double(0x7ff8000000000000ll) : log10(raw) - C::kLog10Initial;
      const int read_local = task.read[c] - region.read_off;
      double* dst = a.v.out + region.out_off + static_cast<int64_t>(read_local) * region.n_haps + info.order;
      if (a.rescue) {
        if (isnan(*dst) && !lost) *dst = result;
      } else {
        *dst = result;
        if (lost) {
          lost_any[c] = true;
          ++lost_count;
        }
      }
    }
  }
  if (a.rescue) return;
  if (lost_count) atomicAdd(&a.v.counters->lost_pairs, lost_count);
#pragma unroll
  for (int c = 0; c < P::NC; ++c) {
    const bool any = __any_sync(kFull, lost_any[c]);
    if (any && lane == 0 && a.queue != nullptr) {
      // Queue the read for double-precision recomputation in the bin of its own rows-per-lane.
      int rows = rd[c].len / 32 + 1;
      if (rows > 8) rows = (rows + 1) & ~1;
      const int slot = atomicAdd(a.queue_tail + rows, 1);
      a.queue[a.queue_off[rows] + slot] = Task{task.region, {task.read[c], -1}, rows};
      atomicAdd(&a.v.counters->rescue_reads, 1ull);
    }
  }
}

template <class P, int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) pairhmm_kernel(LaunchArgs a) {
  const int lane = threadIdx.x & 31;
  const int warp = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const int count = a.count ? *a.count : a.n_tasks;
  unsigned long long fcols = 0, bcols = 0;
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(a.task_counter, 1);
    t = __shfl_sync(kFull, t, 0);
    if (t >= count) break;
    const Task task = a.tasks[t];
    const Region region = a.v.regions[task.region];
    const Program prog = a.use_prefix ? region.prefix : region.shared;
    ReadRef rd[P::NC];
#pragma unroll
    for (int c = 0; c < P::NC; ++c) {
      const int id = task.read[c];
      if (id >= 0) {
        rd[c].off = a.v.read_off[id];
        rd[c].len = static_cast<int>(a.v.read_off[id + 1] - rd[c].off);
      } else {
        rd[c].off = 0;
        rd[c].len = 0;
      }
      rd[c].pad = 32 * R - rd[c].len;
    }
    const uint8_t* codes = a.v.code_of_byte + region.code_off;
    Scratch<P, R> sc(a.scratch + static_cast<size_t>(warp) * a.scratch_stride, region.shared.n_slots > region.prefix.n_slots ? region.shared.n_slots : region.prefix.n_slots,
                     region.shared.n_nodes, region.shared.n_segs);
    if (prog.bwd_len > 0) backward_pass<P, R>(a, prog, rd, codes, lane, sc, bcols);
    forward_pass<P, R>(a, prog, rd, codes, lane, sc, fcols);
    __syncwarp();
    finalize<P, R>(a, task, region, prog, rd, lane, sc);
    __syncwarp();
  }
  if (lane == 0 && !a.rescue) {
    atomicAdd(&a.v.counters->fwd_columns, fcols);
    atomicAdd(&a.v.counters->bwd_columns, bcols);
  }
}

template <class P, int R>
void occ(int* blocks, int* threads) {
  *threads = kWarpsPerBlock * 32;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, pairhmm_kernel<P, R>, kWarpsPerBlock * 32, 0);
}

template <class P, int R>
cudaError_t go(int blocks, const LaunchArgs& a, cudaStream_t s) {
  pairhmm_kernel<P, R><<<blocks, kWarpsPerBlock * 32, 0, s>>>(a);
  return cudaGetLastError();
}

template <class P, int R>
struct OccF {
  static int run(int* b, int* t) {
    occ<P, R>(b, t);
    return 0;
  }
};
template <class P, int R>
struct GoF {
  static cudaError_t run(int blocks, const LaunchArgs& a, cudaStream_t s) { return go<P, R>(blocks, a, s); }
};
template <class P, int R>
struct SizeF {
  static size_t run(int slots, int nodes, int segs) { return scratch_size<P, R>(slots, nodes, segs); }
};

// Rows-per-lane dispatch over the instantiated values of each kind: packed FP32 covers 1..8, single
// FP32 the long reads (10, 12, 14, 16), FP64 both.
template <template <class, int> class F, class... Args>
auto dispatch(Kind k, int rows, Args&&... args) -> decltype(F<PackedF32, 1>::run(args...)) {
  using Ret = decltype(F<PackedF32, 1>::run(args...));
#define FGKL_CASE(P, N) \
  case N:               \
    return F<P, N>::run(args...);
  switch (k) {
    case Kind::kPackedF32:
      switch (rows) {
        FGKL_CASE(PackedF32, 1)
        FGKL_CASE(PackedF32, 2)
        FGKL_CASE(PackedF32, 3)
        FGKL_CASE(PackedF32, 4)
        FGKL_CASE(PackedF32, 5)
        FGKL_CASE(PackedF32, 6)
        FGKL_CASE(PackedF32, 7)
        FGKL_CASE(PackedF32, 8)
        default:
          break;
      }
      break;
    case Kind::kOneF32:
      switch (rows) {
        FGKL_CASE(OneF32, 10)
        FGKL_CASE(OneF32, 12)
        FGKL_CASE(OneF32, 14)
        FGKL_CASE(OneF32, 16)
        default:
          break;
      }
      break;
    case Kind::kOneF64:
      switch (rows) {
        FGKL_CASE(OneF64, 1)
        FGKL_CASE(OneF64, 2)
        FGKL_CASE(OneF64, 3)
        FGKL_CASE(OneF64, 4)
        FGKL_CASE(OneF64, 5)
        FGKL_CASE(OneF64, 6)
        FGKL_CASE(OneF64, 7)
        FGKL_CASE(OneF64, 8)
        FGKL_CASE(OneF64, 10)
        FGKL_CASE(OneF64, 12)
        FGKL_CASE(OneF64, 14)
        FGKL_CASE(OneF64, 16)
        default:
          break;
      }
      break;
  }
#undef FGKL_CASE
  return Ret{};
}

bool valid_rows(Kind k, int rows) {
  switch (k) {
    case Kind::kPackedF32:
      return rows >= 1 && rows <= 8;
    case Kind::kOneF32:
      return rows == 10 || rows == 12 || rows == 14 || rows == 16;
    case Kind::kOneF64:
      return (rows >= 1 && rows <= 8) || rows == 10 || rows == 12 || rows == 14 || rows == 16;
  }
  return false;
}

}  // namespace

int max_rows(Kind) { return 16; }

size_t scratch_bytes(Kind k, int rows, int max_slots, int max_nodes, int max_segs) {
  if (!valid_rows(k, rows)) return 0;
  return dispatch<SizeF>(k, rows, max_slots, max_nodes, max_segs);
}

void occupancy(Kind k, int rows, int* blocks, int* threads) {
  *blocks = 0;
  *threads = kWarpsPerBlock * 32;
  if (!valid_rows(k, rows)) return;
  dispatch<OccF>(k, rows, blocks, threads);
}

cudaError_t launch(Kind k, int rows, int blocks, const LaunchArgs& args, cudaStream_t stream) {
  if (!valid_rows(k, rows)) return cudaErrorInvalidValue;
  return dispatch<GoF>(k, rows, blocks, args, stream);
}

}  // namespace fgkl
