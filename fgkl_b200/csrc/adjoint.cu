// sm_100a adjoint kernels: gradients of the summed log10 likelihood with respect to every read
// position's gap-open (insertion, deletion), gap-continuation and base-error probabilities.
//
// One warp per read: for each haplotype of the read's region, in caller order,
//   1. a backward sweep (the reverse wavefront of the suffix-sharing backward pass, right to left
//      over the haplotype) computes B = d(raw)/d(cell state) for M, X and Y, scaled by 2^120 in FP32
//      at the read's last row, and stores each column's values in the warp's scratch; the padding row
//      above the read collects the start mass, so raw = (INITIAL / hap_len) * s / scale is known
//      before any forward value;
//   2. a forward sweep recomputes F (the plain recurrence) and, at every cell, combines the forward
//      values already in registers -- the diagonal, the cell above and the cell to the left -- with
//      the stored B of the cell into the expected-count terms of the gradient:
//        d raw/d dI  += -F_M(diag) p B_M + F_M(up) B_X
//        d raw/d dD  += -F_M(diag) p B_M + F_M(left) B_Y
//        d raw/d eps += -(F_X + F_Y)(diag) p B_M + F_X(up) B_X + F_Y(left) B_Y
//        d raw/d e   += dp/de (F_M(diag) MM + (F_X + F_Y)(diag) IM) B_M,  dp/de = -1 or 1/3
//      each scaled by 1 / (raw ln 10) and accumulated in FP64 per read row.
// The F x B products are formed in FP64 (their FP32 factors can each be near the FP32 range limits).
// A read whose FP32 raw falls below 1e-28 or is not finite for any haplotype is recomputed whole by
// the FP64 instantiation (INITIAL 2^1020, no backward scale), which cannot lose it.
//
// Haplotype bases are compared as bytes: prior code = the byte with 'N' and byte 4 swapped, so N is
// code kCodeN (matches every read base); a read N matches everything through its mismatch prior.
#include <cmath>

#include "adjoint.cuh"
#include "dp_common.cuh"

namespace fgkl {

namespace {

__device__ __forceinline__ uint32_t adj_code(uint32_t b) { return b == 'N' ? kCodeN : (b == kCodeN ? 'N' : b); }

template <class P, int R>
struct AdjRows {
  using V = typename P::V;
  using S = typename P::S;
  // Own row: forward transitions and priors.
  V mm[R], im[R], mi[R], ii[R], md[R], dd[R], pm[R], px[R];
  int oc[R];
  bool readN[R];
  bool real[R];

  __device__ void load(const AdjView& v, int64_t off, int len, int pad, int lane) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int q = lane * R + r - pad;
      real[r] = q >= 0 && q < len;
      if (real[r]) {
        const int64_t o = off + q;
        const double di = v.d_ins[o], dl = v.d_del[o], ep = v.eps[o], e = v.err[o];
        const uint8_t b = v.bases[o];
        mm[r] = static_cast<S>(1.0 - di - dl);
        im[r] = static_cast<S>(1.0 - ep);
        mi[r] = static_cast<S>(di);
        ii[r] = static_cast<S>(ep);
        md[r] = static_cast<S>(dl);
        dd[r] = static_cast<S>(ep);
        pm[r] = static_cast<S>(1.0 - e);
        px[r] = b == 'N' ? pm[r] : static_cast<S>(e / 3.0);
        oc[r] = static_cast<int>(adj_code(b));
        readN[r] = b == 'N';
      } else {
        // Padding rows keep M = X = 0 and Y = INITIAL / hap_len: GATK's row 0.
        mm[r] = im[r] = mi[r] = ii[r] = md[r] = pm[r] = px[r] = P::zero();
        dd[r] = static_cast<S>(1.0);
        oc[r] = -1;
        readN[r] = false;
      }
    }
  }
  __device__ V prior(uint32_t code, int r) const { return (static_cast<int>(code) == oc[r] || code == kCodeN) ? pm[r] : px[r]; }
  __device__ bool match(uint32_t code, int r) const { return static_cast<int>(code) == oc[r] || code == kCodeN || readN[r]; }
};

// The row below each lane row, for the backward recurrence.
template <class P, int R>
struct AdjBelow {
  using V = typename P::V;
  using S = typename P::S;
  V mm[R], im[R], mi[R], ii[R], pm[R], px[R];
  int oc[R];

  __device__ void load(const AdjView& v, int64_t off, int len, int pad, int lane) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int q = lane * R + r + 1 - pad;
      if (q >= 0 && q < len) {
        const int64_t o = off + q;
        const double di = v.d_ins[o], dl = v.d_del[o], ep = v.eps[o], e = v.err[o];
        const uint8_t b = v.bases[o];
        mm[r] = static_cast<S>(1.0 - di - dl);
        im[r] = static_cast<S>(1.0 - ep);
        mi[r] = static_cast<S>(di);
        ii[r] = static_cast<S>(ep);
        pm[r] = static_cast<S>(1.0 - e);
        px[r] = b == 'N' ? pm[r] : static_cast<S>(e / 3.0);
        oc[r] = static_cast<int>(adj_code(b));
      } else {
        mm[r] = im[r] = mi[r] = ii[r] = pm[r] = px[r] = P::zero();
        oc[r] = -1;
      }
    }
  }
  __device__ V prior(uint32_t code, int r) const { return (static_cast<int>(code) == oc[r] || code == kCodeN) ? pm[r] : px[r]; }
};

// Column j's backward values of one lane: a record of BM, BX, BY rows padded to 16 bytes,
// [column][lane][record], so a lane stores and fetches its record with 16-byte moves.
template <class P, int R>
struct AdjCol {
  using V = typename P::V;
  static constexpr int kPer16 = 16 / static_cast<int>(sizeof(V));
  static constexpr int kRec = (3 * R + kPer16 - 1) / kPer16 * kPer16;
  // Columns fetched ahead of the forward sweep into a per-warp shared-memory ring (about 16 KB).
  static constexpr int kDepthRaw = 16384 / (32 * kRec * static_cast<int>(sizeof(V)));
  static constexpr int kDepth = kDepthRaw < 2 ? 2 : (kDepthRaw > 8 ? 8 : kDepthRaw);
  static constexpr size_t kRingBytes = static_cast<size_t>(kDepth) * 32 * kRec * sizeof(V);
  __device__ static V* at(char* scratch, int j, int lane) {
    return reinterpret_cast<V*>(scratch) + (static_cast<size_t>(j) * 32 + lane) * kRec;
  }
};

// The backward sweep's state between two steps: BM and BY rows and the values the next step
// shuffles from the lane below, padded to 16 bytes so a lane saves and restores it with 16-byte moves.
template <class P, int R>
struct AdjBwdState {
  using V = typename P::V;
  static constexpr int kPer16 = 16 / static_cast<int>(sizeof(V));
  static constexpr int kRec = (2 * R + 3 + kPer16 - 1) / kPer16 * kPer16;
  V BM[R], BY[R];
  V dBM, topBM, topBX;
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int r = 0; r < R; ++r) BM[r] = BY[r] = P::zero();
    dBM = topBM = topBX = P::zero();
  }
  __device__ __forceinline__ void save(V* dst) const {
    V rec[kRec];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      rec[r] = BM[r];
      rec[R + r] = BY[r];
    }
    rec[2 * R] = dBM;
    rec[2 * R + 1] = topBM;
    rec[2 * R + 2] = topBX;
#pragma unroll
    for (int i = 2 * R + 3; i < kRec; ++i) rec[i] = P::zero();
    store_record(dst, rec);
  }
  __device__ __forceinline__ void restore(const V* src) {
    V rec[kRec];
    load_record(rec, src);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      BM[r] = rec[r];
      BY[r] = rec[R + r];
    }
    dBM = rec[2 * R];
    topBM = rec[2 * R + 1];
    topBX = rec[2 * R + 2];
  }
};

// Scratch of a pair whose backward columns do not all fit: a block buffer of K backward steps'
// records, then one saved state per block, [block][lane][AdjBwdState::kRec].
template <class P, int R>
struct AdjCkpt {
  using V = typename P::V;
  __device__ static V* block(char* scratch, int i, int lane) {
    return reinterpret_cast<V*>(scratch) + (static_cast<size_t>(i) * 32 + lane) * AdjCol<P, R>::kRec;
  }
  __device__ static V* state(char* scratch, int K, int b, int lane) {
    return reinterpret_cast<V*>(scratch) + static_cast<size_t>(K) * 32 * AdjCol<P, R>::kRec +
           (static_cast<size_t>(b) * 32 + lane) * AdjBwdState<P, R>::kRec;
  }
};

// One step of the backward sweep at lane position p (column m - p): the lane's record of the column
// (BM, BX, BY rows) in `rec`. `md` and `dd` are the lane rows' own deletion transitions.
template <class P, int R>
__device__ __forceinline__ void adj_bwd_step(AdjBwdState<P, R>& s, const AdjBelow<P, R>& bl, const typename P::V (&md)[R],
                                             const typename P::V (&dd)[R], typename P::V sink, uint32_t code, int p,
                                             typename P::V (&rec)[AdjCol<P, R>::kRec]) {
  using V = typename P::V;
  const V rBM = P::down(s.topBM), rBX = P::down(s.topBX);
  if (p == 0) {
    // The all-zero column beyond the haplotype.
#pragma unroll
    for (int r = 0; r < R; ++r) s.BM[r] = s.BY[r] = P::zero();
    s.dBM = P::zero();
  }
  V belowX = rBX, diagM = s.dBM;
#pragma unroll
  for (int r = R - 1; r >= 0; --r) {
    const V into = P::mul(bl.prior(code, r), diagM);
    const V itm = P::mul(into, bl.im[r]);
    V bx = P::fma(belowX, bl.ii[r], itm);
    const V by = P::fma(s.BY[r], dd[r], itm);
    V bm = P::fma(s.BY[r], md[r], P::fma(belowX, bl.mi[r], P::mul(into, bl.mm[r])));
    if (r == R - 1) {
      bm = P::add(bm, sink);
      bx = P::add(bx, sink);
    }
    diagM = s.BM[r];
    s.BM[r] = bm;
    s.BY[r] = by;
    belowX = bx;
    rec[r] = bm;
    rec[R + r] = bx;
    rec[2 * R + r] = by;
  }
#pragma unroll
  for (int i = 3 * R; i < AdjCol<P, R>::kRec; ++i) rec[i] = P::zero();
  s.topBM = s.BM[0];
  s.topBX = belowX;
  s.dBM = rBM;
}

// The base code the backward step at lane position p reads (the diagonal successor's base), none
// beyond the haplotype.
__device__ __forceinline__ uint32_t adj_bwd_code(const uint8_t* hap, int m, int p) {
  const int jj = m - p;
  return (p >= 0 && jj >= 0 && jj < m) ? adj_code(__ldg(hap + jj)) : 0u;
}

// Backward sweep of one pair over steps 0 .. m + 31; returns, in every lane, the padding row's start
// mass s. Without checkpoints (K == 0) it stores every column's record for the forward sweep. With
// checkpoints it stores none and saves, instead, the state entering each block of K steps that the
// forward sweep recomputes (adj_backward_block), block b of forward steps [bK, bK + K) reading
// backward steps [n - (b + 1)K, n - 1 - bK], n = m + 31.
template <class P, int R, bool kCk>
__device__ typename P::V adj_backward(const AdjView& v, const AdjRows<P, R>& own, int64_t off, int len, int pad,
                                      const uint8_t* hap, int m, int lane, char* scratch, int K) {
  using V = typename P::V;
  using S = typename P::S;
  AdjBelow<P, R> bl;
  bl.load(v, off, len, pad, lane);
  const V sink = lane == 31 ? static_cast<S>(Consts<P::kDouble>::kBackwardScale) : P::zero();
  AdjBwdState<P, R> st;
  st.zero();
  const int pad_row = pad - 1;  // the padding row right above the read
  const int pad_lane = pad_row / R, pad_r = pad_row % R;
  const int n = m + 31;
  V start_mass = P::zero();
  uint32_t next_code = adj_bwd_code(hap, m, -(31 - lane));
  for (int t = 0; t < m + 1 + 31; ++t) {
    if (kCk && K > 0 && t > 0 && t < n && (n - t) % K == 0) st.save(AdjCkpt<P, R>::state(scratch, K, (n - t) / K - 1, lane));
    const int p = t - (31 - lane);  // position: column m - p
    const int j = m - p;
    const uint32_t code = next_code;
    next_code = adj_bwd_code(hap, m, p + 1);
    V rec[AdjCol<P, R>::kRec];
    adj_bwd_step<P, R>(st, bl, own.md, own.dd, sink, code, p, rec);
    if ((!kCk || K == 0) && p >= 0 && j >= 1) store_record(AdjCol<P, R>::at(scratch, j, lane), rec);
    if (p == m && lane == pad_lane) {
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (r == pad_r) start_mass = st.BY[r];
    }
  }
  return __shfl_sync(kFull, start_mass, pad_lane);
}

// Recomputes backward steps [t_lo, t_hi] of one pair from the state saved at t_lo (or the initial
// state when t_lo == 0) into the block buffer, record of step t at index t - t_lo. The arithmetic is
// the full sweep's, step for step, so the records are bit-identical to the stored ones. Not inlined:
// the forward sweep's registers are saved around the call, once per block.
template <class P, int R>
__device__ __noinline__ void adj_backward_block(const uint8_t* bases, const double* d_ins, const double* d_del,
                                                const double* eps, const double* err, int64_t off, int len, int pad,
                                                const uint8_t* hap, int m, int lane, char* scratch, int K, int b, int t_lo,
                                                int t_hi) {
  using V = typename P::V;
  using S = typename P::S;
  AdjView pv{};
  pv.bases = bases;
  pv.d_ins = d_ins;
  pv.d_del = d_del;
  pv.eps = eps;
  pv.err = err;
  const AdjView* v = &pv;
  AdjBelow<P, R> bl;
  bl.load(*v, off, len, pad, lane);
  // The lane rows' own deletion transitions, as AdjRows holds them.
  V md[R], dd[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int q = lane * R + r - pad;
    if (q >= 0 && q < len) {
      md[r] = static_cast<S>(v->d_del[off + q]);
      dd[r] = static_cast<S>(v->eps[off + q]);
    } else {
      md[r] = P::zero();
      dd[r] = static_cast<S>(1.0);
    }
  }
  const V sink = lane == 31 ? static_cast<S>(Consts<P::kDouble>::kBackwardScale) : P::zero();
  AdjBwdState<P, R> st;
  if (t_lo > 0)
    st.restore(AdjCkpt<P, R>::state(scratch, K, b, lane));
  else
    st.zero();
  uint32_t next_code = adj_bwd_code(hap, m, t_lo - (31 - lane));
  for (int t = t_lo; t <= t_hi; ++t) {
    const int p = t - (31 - lane);
    const uint32_t code = next_code;
    next_code = adj_bwd_code(hap, m, p + 1);
    V rec[AdjCol<P, R>::kRec];
    adj_bwd_step<P, R>(st, bl, md, dd, sink, code, p, rec);
    store_record(AdjCkpt<P, R>::block(scratch, t - t_lo, lane), rec);
  }
}

// The forward sweep's registers: M, X, Y rows, the row above the lane's top row on the diagonal,
// and the accumulated result.
template <class P, int R>
struct AdjFwdState {
  using V = typename P::V;
  V M[R], X[R], Y[R];
  V dM, dX, dY, acc;
};

// One forward step's arithmetic: the column's forward values from the diagonal (d*), the row above
// (u*) and the lane's own registers, and, for a live step, the gradient terms against the column's
// backward record (bM, bX, bY).
template <class P, int R>
__device__ __forceinline__ void adj_fwd_math(AdjFwdState<P, R>& f, const AdjRows<P, R>& own, uint32_t code, bool live,
                                             const typename P::V (&bM)[R], const typename P::V (&bX)[R],
                                             const typename P::V (&bY)[R], typename P::V uM, typename P::V uX, double norm,
                                             double (&gi)[R], double (&gd)[R], double (&ge)[R], double (&gq)[R]) {
  using V = typename P::V;
  // Match and deletion values from the bottom row up (each row reads the old row above).
#pragma unroll
  for (int r = R - 1; r >= 0; --r) {
    const V pM = r ? f.M[r - 1] : f.dM, pX = r ? f.X[r - 1] : f.dX, pY = r ? f.Y[r - 1] : f.dY;
    const V mOld = f.M[r], yOld = f.Y[r];
    const V prior = own.prior(code, r);
    const V sxy = P::add(pX, pY);
    const V s = P::fma(pM, own.mm[r], P::mul(sxy, own.im[r]));
    f.Y[r] = P::fma(yOld, own.dd[r], P::mul(mOld, own.md[r]));
    f.M[r] = P::mul(prior, s);
    if (live && own.real[r]) {
      const double bm_n = static_cast<double>(bM[r]) * norm, by_n = static_cast<double>(bY[r]) * norm;
      const double bm_p = bm_n * static_cast<double>(prior);
      const double t1 = static_cast<double>(pM) * bm_p;
      gi[r] -= t1;
      gd[r] += static_cast<double>(mOld) * by_n - t1;
      ge[r] += static_cast<double>(yOld) * by_n - static_cast<double>(sxy) * bm_p;
      gq[r] += (own.match(code, r) ? -1.0 : 1.0 / 3.0) * static_cast<double>(s) * bm_n;
    }
  }
  // Insertion values from the top row down (each row reads the new row above).
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const V qM = r ? f.M[r - 1] : uM, qX = r ? f.X[r - 1] : uX;
    f.X[r] = P::fma(qX, own.ii[r], P::mul(qM, own.mi[r]));
    if (live && own.real[r]) {
      const double bx_n = static_cast<double>(bX[r]) * norm;
      gi[r] += static_cast<double>(qM) * bx_n;
      ge[r] += static_cast<double>(qX) * bx_n;
    }
  }
  if (live) f.acc = P::add(f.acc, P::add(f.M[R - 1], f.X[R - 1]));
}

// Column 0 of the forward sweep: the row-0 constant in the padding rows (and in the row above the
// lane's top row when that is padding).
template <class P, int R>
__device__ __forceinline__ void adj_fwd_column0(AdjFwdState<P, R>& f, int pad, int lane, typename P::S init) {
#pragma unroll
  for (int r = 0; r < R; ++r) {
    f.M[r] = f.X[r] = P::zero();
    f.Y[r] = lane * R + r < pad ? init : P::zero();
  }
  f.dM = f.dX = P::zero();
  f.dY = lane * R - 1 < pad ? init : P::zero();
  f.acc = P::zero();
}

// Forward sweep of one pair, accumulating the pair's gradient terms scaled by `norm`; returns the
// raw result (lane 31). Without checkpoints (K == 0) it reads the backward records the backward sweep
// stored; with checkpoints it recomputes them block by block (adj_backward_block) first. Either way
// the records reach the lanes through a shared-memory ring filled D steps ahead by cp.async, one
// commit group per record.
template <class P, int R, bool kCk>
__device__ typename P::V adj_forward(const AdjView& v, const AdjRows<P, R>& own, int64_t off, int len, int pad,
                                     const uint8_t* hap, int m, int lane, char* scratch, typename P::V* ring, int K,
                                     double norm, double (&gi)[R], double (&gd)[R], double (&ge)[R], double (&gq)[R]) {
  using V = typename P::V;
  using S = typename P::S;
  using Col = AdjCol<P, R>;
  constexpr int D = Col::kDepth;
  const S init = static_cast<S>(Consts<P::kDouble>::kInitial / m);
  AdjFwdState<P, R> f;
#pragma unroll
  for (int r = 0; r < R; ++r) f.M[r] = f.X[r] = f.Y[r] = P::zero();
  f.acc = f.dM = f.dX = f.dY = P::zero();
  const int n = m + 31;
  // The lane's record for column k + 1 (k = 0..m-1) sits in ring slot k % D.
  auto slot = [&](int k) { return ring + (static_cast<size_t>(k % D) * 32 + lane) * Col::kRec; };
  auto copy = [&](int k, const V* src) {
    V* dst = slot(k);
#pragma unroll
    for (int i = 0; i < Col::kRec / Col::kPer16; ++i)
      __pipeline_memcpy_async(reinterpret_cast<char*>(dst) + 16 * i, reinterpret_cast<const char*>(src) + 16 * i, 16);
  };
  uint32_t next_code = (m > 0 && lane == 0) ? adj_code(__ldg(hap)) : 0u;
  // One step: the row above's values shuffled down from the lane above (before column 0's reset, as
  // in the unrolled recurrence), column 0's row-0 constant, the arithmetic, and the diagonal kept.
  auto step = [&](int p, const V (&bM)[R], const V (&bX)[R], const V (&bY)[R], bool live, uint32_t code) {
    const V uM = P::up(f.M[R - 1]), uX = P::up(f.X[R - 1]), uY = P::up(f.Y[R - 1]);
    if (p == 0) adj_fwd_column0<P, R>(f, pad, lane, init);
    adj_fwd_math<P, R>(f, own, code, live, bM, bX, bY, uM, uX, norm, gi, gd, ge, gq);
    f.dM = uM;
    f.dX = uX;
    f.dY = uY;
  };
  if (!kCk || K == 0) {
    // Columns fetched D ahead, keyed by the lane position k.
    auto fetch = [&](int k) {
      if (k < m) copy(k, Col::at(scratch, k + 1, lane));
      __pipeline_commit();
    };
#pragma unroll
    for (int k = 0; k < D; ++k) fetch(k);
    for (int t = 0; t < n; ++t) {
      const int p = t - lane;  // column p + 1
      const bool live = p >= 0 && p < m;
      const uint32_t code = next_code;
      next_code = (p + 1 >= 0 && p + 1 < m) ? adj_code(__ldg(hap + p + 1)) : 0u;
      V bM[R], bX[R], bY[R];
      if (live) {
        __pipeline_wait_prior(D - 1);
        V rec[Col::kRec];
        load_record(rec, slot(p));
#pragma unroll
        for (int r = 0; r < R; ++r) {
          bM[r] = rec[r];
          bX[r] = rec[R + r];
          bY[r] = rec[2 * R + r];
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) bM[r] = bX[r] = bY[r] = P::zero();
      }
      step(p, bM, bX, bY, live, code);
      if (live) fetch(p + D);  // into the slot just read (its values are consumed above)
    }
  } else if (kCk) {
    // Block b: forward steps [t0, t1) read backward steps n - 1 - t, recomputed into the block
    // buffer at index n - 1 - t - lo. Every step commits one group, the one for step t + D (empty
    // beyond the block), so the group of a live step is always complete after wait_prior(D - 1).
    for (int t0 = 0; t0 < n; t0 += K) {
      const int t1 = min(t0 + K, n);
      const int lo = max(0, n - t1), hi = n - 1 - t0;
      adj_backward_block<P, R>(v.bases, v.d_ins, v.d_del, v.eps, v.err, off, len, pad, hap, m, lane, scratch, K, t0 / K, lo, hi);
      // The lane's records are fetched back by its own asynchronous copies.
      __threadfence_block();
      __syncwarp();
      auto fetch = [&](int tt) {
        const int k = tt - lane;
        if (tt < t1 && k >= 0 && k < m) copy(k, AdjCkpt<P, R>::block(scratch, n - 1 - tt - lo, lane));
        __pipeline_commit();
      };
      for (int i = 0; i < D; ++i) fetch(t0 + i);
      for (int t = t0; t < t1; ++t) {
        const int p = t - lane;
        const bool live = p >= 0 && p < m;
        const uint32_t code = next_code;
        next_code = (p + 1 >= 0 && p + 1 < m) ? adj_code(__ldg(hap + p + 1)) : 0u;
        V bM[R], bX[R], bY[R];
        if (live) {
          __pipeline_wait_prior(D - 1);
          V rec[Col::kRec];
          load_record(rec, slot(p));
#pragma unroll
          for (int r = 0; r < R; ++r) {
            bM[r] = rec[r];
            bX[r] = rec[R + r];
            bY[r] = rec[2 * R + r];
          }
        } else {
#pragma unroll
          for (int r = 0; r < R; ++r) bM[r] = bX[r] = bY[r] = P::zero();
        }
        step(p, bM, bX, bY, live, code);
        fetch(t + D);
      }
      __pipeline_wait_prior(0);
    }
  }
  __pipeline_wait_prior(0);
  return __shfl_sync(kFull, f.acc, 31);
}

template <class P, int R>
struct AdjMinBlocks {
  static constexpr int value = 1;
};

// kCk: the instantiation for launches whose longest pairs exceed the per-warp scratch, which
// recomputes those pairs' backward columns from checkpoints; the other keeps no checkpoint code.
template <class P, int R, bool kCk>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, (AdjMinBlocks<P, R>::value)) adjoint_kernel(AdjLaunch a) {
  using C = Consts<P::kDouble>;
  extern __shared__ __align__(16) unsigned char adj_smem[];
  const int lane = threadIdx.x & 31;
  const int warp = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  char* scratch = a.scratch + static_cast<size_t>(warp) * a.scratch_stride;
  typename P::V* ring = reinterpret_cast<typename P::V*>(adj_smem + (threadIdx.x >> 5) * AdjCol<P, R>::kRingBytes);
  const int count = a.count ? min(*a.count, a.n_tasks) : a.n_tasks;
  const double ln10 = 2.302585092994045684017991454684364208;
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(a.task_counter, 1);
    t = __shfl_sync(kFull, t, 0);
    if (t >= count) break;
    const int read = a.tasks[t];
    const int g = a.v.read_region[read];
    const int64_t off = a.v.read_off[read];
    const int len = static_cast<int>(a.v.read_off[read + 1] - off);
    const int pad = 32 * R - len;
    const int h0 = a.v.region_hap[g], nh = a.v.region_nhap[g];
    const int read_local = read - a.v.region_read[g];
    AdjRows<P, R> own;
    own.load(a.v, off, len, pad, lane);
    double gi[R], gd[R], ge[R], gq[R];
#pragma unroll
    for (int r = 0; r < R; ++r) gi[r] = gd[r] = ge[r] = gq[r] = 0.0;
    bool lost = false;
    for (int h = 0; h < nh && !lost; ++h) {
      const int64_t hlo = a.v.hap_off[h0 + h];
      const int m = static_cast<int>(a.v.hap_off[h0 + h + 1] - hlo);
      const uint8_t* hap = a.v.hap_bases + hlo;
      // Backward columns stored whole when they fit the warp's scratch, else recomputed from
      // checkpoints block by block (the host sized the scratch so one of the two fits).
      int K = 0;
      const long long cap = static_cast<long long>(a.scratch_stride / (32 * sizeof(typename P::V)));
      if (static_cast<long long>(m + 1) * AdjCol<P, R>::kRec > cap) {
        if (!kCk) {
          lost = true;
          break;
        }
        K = adj_block_steps(cap, m + 31, AdjCol<P, R>::kRec, AdjBwdState<P, R>::kRec, AdjCol<P, R>::kDepth);
        if (K == 0) {
          lost = true;
          break;
        }
      }
      const double s = static_cast<double>(adj_backward<P, R, kCk>(a.v, own, off, len, pad, hap, m, lane, scratch, K));
      // raw = (INITIAL / m) * s / scale: the pair's scaled likelihood, from the backward values.
      const double raw = (C::kInitial / m) * s / C::kBackwardScale;
      if (!P::kDouble && (!(raw >= C::kMinAccepted) || isinf(raw))) {
        lost = true;
        break;
      }
      const double norm = 1.0 / ((C::kInitial / m) * s * ln10);
      // The lane's backward records are fetched back by its own asynchronous copies.
      __threadfence_block();
      __syncwarp();
      const double fwd =
          static_cast<double>(adj_forward<P, R, kCk>(a.v, own, off, len, pad, hap, m, lane, scratch, ring, K, norm, gi, gd, ge, gq));
      if (!P::kDouble && (!(fwd >= C::kMinAccepted) || isinf(fwd))) {
        lost = true;
        break;
      }
      if (lane == 0) a.v.out[a.v.region_out[g] + static_cast<int64_t>(read_local) * nh + h] = log10(fwd) - C::kLog10Initial;
      __syncwarp();
    }
    if (lost) {
      if (lane == 0) {
        atomicAdd(a.v.lost, 1ull);
        if (a.queue) {
          const int bin = adj_rows(len);
          const int slot = atomicAdd(a.queue_tail + bin, 1);
          if (slot < a.queue_off[bin + 1] - a.queue_off[bin]) a.queue[a.queue_off[bin] + slot] = read;
        }
      }
      continue;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (!own.real[r]) continue;
      const int64_t o = off + lane * R + r - pad;
      a.v.g_ins[o] = gi[r];
      a.v.g_del[o] = gd[r];
      a.v.g_eps[o] = ge[r];
      a.v.g_err[o] = gq[r];
    }
  }
}

template <class P, int R, bool kCk>
void adj_occ(int* blocks) {
  static std::atomic<int> cache[kMaxDevices];
  *blocks = resident_blocks(adjoint_kernel<P, R, kCk>, kWarpsPerBlock * AdjCol<P, R>::kRingBytes, kWarpsPerBlock * 32, cache);
}

template <class P, int R, bool kCk>
cudaError_t adj_go(int blocks, const AdjLaunch& a, cudaStream_t s) {
  const size_t smem = kWarpsPerBlock * AdjCol<P, R>::kRingBytes;
  adjoint_kernel<P, R, kCk><<<blocks, kWarpsPerBlock * 32, smem, s>>>(a);
  return cudaGetLastError();
}

template <class F>
auto adj_dispatch_rows(int rows, F&& f) {
  switch (rows) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    case 6: return f(std::integral_constant<int, 6>{});
    case 7: return f(std::integral_constant<int, 7>{});
    case 8: return f(std::integral_constant<int, 8>{});
    case 10: return f(std::integral_constant<int, 10>{});
    case 12: return f(std::integral_constant<int, 12>{});
    case 14: return f(std::integral_constant<int, 14>{});
    case 16: return f(std::integral_constant<int, 16>{});
    case 18: return f(std::integral_constant<int, 18>{});
    default: return f(std::integral_constant<int, 20>{});
  }
}

}  // namespace

namespace {
// Record sizes (values per lane) of an instantiation: backward column, saved state, ring depth.
struct AdjSizes {
  int rec, state, depth;
  size_t value;
};
AdjSizes adj_sizes(bool dbl, int rows) {
  if (dbl)
    return adj_dispatch_rows(rows, [](auto r) {
      constexpr int R = decltype(r)::value;
      return AdjSizes{AdjCol<OneF64, R>::kRec, AdjBwdState<OneF64, R>::kRec, AdjCol<OneF64, R>::kDepth, sizeof(double)};
    });
  return adj_dispatch_rows(rows, [](auto r) {
    constexpr int R = decltype(r)::value;
    return AdjSizes{AdjCol<OneF32, R>::kRec, AdjBwdState<OneF32, R>::kRec, AdjCol<OneF32, R>::kDepth, sizeof(float)};
  });
}
}  // namespace

size_t adj_column_bytes(bool dbl, int rows, int columns) {
  const AdjSizes z = adj_sizes(dbl, rows);
  return static_cast<size_t>(columns) * 32 * z.rec * z.value;
}

size_t adj_scratch_bytes(bool dbl, int rows, int max_hap_len) { return adj_column_bytes(dbl, rows, max_hap_len + 1); }

size_t adj_checkpoint_bytes(bool dbl, int rows, int max_hap_len) {
  const AdjSizes z = adj_sizes(dbl, rows);
  const long long steps = max_hap_len + 31;
  // K * rec + ceil(steps / K) * state is least near K = sqrt(steps * state / rec).
  long long best = -1;
  long long k0 = static_cast<long long>(std::sqrt(static_cast<double>(steps) * z.state / z.rec));
  for (long long K = std::max<long long>(z.depth, k0 - 2); K <= std::max<long long>(z.depth, k0 + 2); ++K) {
    const long long need = K * z.rec + (steps + K - 1) / K * z.state;
    if (best < 0 || need < best) best = need;
  }
  return static_cast<size_t>(best) * 32 * z.value;
}

void adj_occupancy(bool dbl, int rows, bool checkpointed, int* blocks, int* threads) {
  *threads = kWarpsPerBlock * 32;
  *blocks = 0;
  adj_dispatch_rows(rows, [&](auto r) {
    constexpr int R = decltype(r)::value;
    if (dbl)
      checkpointed ? adj_occ<OneF64, R, true>(blocks) : adj_occ<OneF64, R, false>(blocks);
    else
      checkpointed ? adj_occ<OneF32, R, true>(blocks) : adj_occ<OneF32, R, false>(blocks);
    return 0;
  });
}

cudaError_t adj_launch(bool dbl, int rows, bool checkpointed, int blocks, const AdjLaunch& a, cudaStream_t s) {
  return adj_dispatch_rows(rows, [&](auto r) {
    constexpr int R = decltype(r)::value;
    if (dbl) return checkpointed ? adj_go<OneF64, R, true>(blocks, a, s) : adj_go<OneF64, R, false>(blocks, a, s);
    return checkpointed ? adj_go<OneF32, R, true>(blocks, a, s) : adj_go<OneF32, R, false>(blocks, a, s);
  });
}

}  // namespace fgkl
