// sm_100a adjoint kernels: gradients of the summed log10 likelihood with respect to every read
// position's gap-open (insertion, deletion), gap-continuation and base-error probabilities.
//
// One warp per read: for each haplotype of the read's region, in caller order,
//   1. a backward sweep (the reverse wavefront of the suffix-sharing backward pass, right to left
//      over the haplotype) computes B = d(raw)/d(cell state) for M, X and Y, scaled by 2^120 in FP32
//      at the read's last row. It keeps nothing per cell: it saves its state every K steps, and the
//      padding row above the read collects the start mass, so raw = (INITIAL / hap_len) * s / scale
//      is known before any forward value;
//   2. a forward sweep recomputes F (the plain recurrence) in blocks of K steps. Because the two
//      wavefronts are skewed oppositely, forward step t of every lane reads the backward values of
//      backward step n - 1 - t, so before forward block [bK, bK + K) the K backward steps it needs
//      are recomputed from the saved state into shared memory. Each cell then combines the forward
//      values in registers -- the diagonal, the cell above and the cell to the left -- with its
//      backward values into the expected-count terms of the gradient:
//        d raw/d dI  += -F_M(diag) p B_M + F_M(up) B_X
//        d raw/d dD  += -F_M(diag) p B_M + F_M(left) B_Y
//        d raw/d eps += -(F_X + F_Y)(diag) p B_M + F_X(up) B_X + F_Y(left) B_Y
//        d raw/d e   += dp/de (F_M(diag) MM + (F_X + F_Y)(diag) IM) B_M,  dp/de = -1 or 1/3
//      each divided by raw ln 10.
// The products are FP32. The recurrences are linear in their starting values, so F is computed from
// INITIAL * 2^-a / hap_len and the recomputed B from a sink times c = 2^a / (raw * scale * ln 10):
// each product F * B is then the normalised term itself, and a = the mean of log2 raw and log2 of
// the row-0 constant centres the range of F near 1, which keeps both factors of every term that
// matters inside the FP32 range (F runs from the row-0 constant down to about raw, B * c the other
// way). Each lane sums its rows' terms over the forward steps in FP32 and adds the sums into the
// FP64 per-position gradients every 32 steps (atomic adds; a lane alone owns its rows, so the order
// is fixed). A read whose FP32 raw falls below 1e-28 or is not finite for any haplotype is
// recomputed whole by the FP64 instantiation (INITIAL 2^1020, no backward scale, a = 0), which
// cannot lose it.
//
// Reads longer than 620 bases are strip-mined over row blocks of 32 R rows (R = 8), padding at the
// top of the first. The backward sweeps run the blocks bottom to top; lane 31's row below comes
// from the top row the block below stored column by column (its BM and BX). The forward sweeps run
// them top to bottom; lane 0's row above comes from the bottom row the block above stored, or GATK's
// row 0 in the first block.
//
// Haplotype bases are compared as bytes: a haplotype N matches every read base; a read N matches
// everything through its mismatch prior, which equals its match prior.
//
// Most steps of a one-block read are interior: every lane lies strictly inside the haplotype in both
// sweeps (steps 32 .. m - 1). Those steps, block by block, run without the column-0 resets, the
// masks of lanes outside the haplotype and the row-block exchanges.
#include <cmath>
#include <type_traits>

#include "adjoint.cuh"
#include "dp_common.cuh"

namespace fgkl {

namespace {

// Sizes of one instantiation: a lane's record of one backward step (BM, BX, BY rows) and its saved
// backward state (BM, BY rows, the diagonal BM and the two values shuffled from the lane below), in
// 16-byte chunks; the backward steps recomputed per block, as many as about 28 KB of shared memory
// per warp holds (at most 8).
template <class P, int R>
struct AdjSizes {
  using V = typename P::V;
  static constexpr int kPer16 = 16 / static_cast<int>(sizeof(V));
  static constexpr int kRecChunks = (3 * R + kPer16 - 1) / kPer16;
  static constexpr int kRecVals = kRecChunks * kPer16;
  static constexpr int kStateVals = 2 * R + 3;
  static constexpr int kStateChunks = (kStateVals + kPer16 - 1) / kPer16;
  static constexpr int kStepBytes = kRecChunks * 32 * 16;
  static constexpr int kRawK = 28672 / kStepBytes;
  static constexpr int K = kRawK < 1 ? 1 : (kRawK > 8 ? 8 : kRawK);
  // Per warp: the K steps' records, then the next block's checkpoint, fetched a block ahead.
  static constexpr size_t kStageOffset = static_cast<size_t>(K) * kStepBytes;
  static constexpr size_t kSmemPerWarp = kStageOffset + static_cast<size_t>(kStateChunks) * 32 * 16;
};

constexpr int kFlushSteps = 32;  // forward steps between FP64 additions of the FP32 sums

// The lane's rows: their forward transitions and priors, and those of the row below the lane's last
// row, which the backward step of that row reads (the backward step of row r < R - 1 reads row r + 1's
// own). Read row q = lane * R + r - pad, pad relative to the row block (negative below the first).
// Haplotype and read bases are compared as bytes; a haplotype N matches every read base, and a read N
// has equal match and mismatch priors.
template <class P, int R>
struct AdjCoef {
  using V = typename P::V;
  using S = typename P::S;
  V mm[R], im[R], mi[R], ii[R], md[R], dd[R], pm[R], px[R];
  V kqx[R];  // d prior / d e of a mismatch: 1/3, or -1 for a read N (whose prior is 1 - e either way)
  int rb[R];                     // read byte; -1 for a padding row (no haplotype byte matches it)
  V lmm, lim, lmi, lii, lpm, lpx;  // the row below row R - 1
  int lrb;
  uint32_t real;  // bit r: a read row

  struct Row {
    double mm, im, mi, ii, md, dd, pm, px, kqx;
    int rb;
    bool real;
  };
  __device__ static Row row(const AdjView& v, int64_t off, int len, int q) {
    Row w;
    w.real = q >= 0 && q < len;
    if (w.real) {
      const int64_t o = off + q;
      const double di = v.d_ins[o], dl = v.d_del[o], ep = v.eps[o], e = v.err[o];
      const int b = v.bases[o];
      w.mm = 1.0 - di - dl;
      w.im = 1.0 - ep;
      w.mi = di;
      w.ii = ep;
      w.md = dl;
      w.dd = ep;
      w.pm = 1.0 - e;
      w.px = b == 'N' ? w.pm : e / 3.0;
      w.kqx = b == 'N' ? -1.0 : 1.0 / 3.0;
      w.rb = b;
    } else {
      // Padding rows keep M = X = 0 and Y = INITIAL / hap_len: GATK's row 0.
      w.mm = w.im = w.mi = w.ii = w.md = w.pm = w.px = w.kqx = 0.0;
      w.dd = 1.0;
      w.rb = -1;
    }
    return w;
  }

  __device__ void load(const AdjView& v, int64_t off, int len, int pad, int lane) {
    real = 0u;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const Row w = row(v, off, len, lane * R + r - pad);
      mm[r] = static_cast<S>(w.mm);
      im[r] = static_cast<S>(w.im);
      mi[r] = static_cast<S>(w.mi);
      ii[r] = static_cast<S>(w.ii);
      md[r] = static_cast<S>(w.md);
      dd[r] = static_cast<S>(w.dd);
      pm[r] = static_cast<S>(w.pm);
      px[r] = static_cast<S>(w.px);
      kqx[r] = static_cast<S>(w.kqx);
      rb[r] = w.rb;
      if (w.real) real |= 1u << r;
    }
    const Row w = row(v, off, len, lane * R + R - pad);
    lmm = static_cast<S>(w.mm);
    lim = static_cast<S>(w.im);
    lmi = static_cast<S>(w.mi);
    lii = static_cast<S>(w.ii);
    lpm = static_cast<S>(w.pm);
    lpx = static_cast<S>(w.px);
    lrb = w.rb;
  }
  // Coefficients of the row below row r, for the backward step.
  __device__ V bmm(int r) const { return r + 1 < R ? mm[r + 1 < R ? r + 1 : 0] : lmm; }
  __device__ V bim(int r) const { return r + 1 < R ? im[r + 1 < R ? r + 1 : 0] : lim; }
  __device__ V bmi(int r) const { return r + 1 < R ? mi[r + 1 < R ? r + 1 : 0] : lmi; }
  __device__ V bii(int r) const { return r + 1 < R ? ii[r + 1 < R ? r + 1 : 0] : lii; }
  __device__ V bprior(int code, bool hapN, int r) const {
    if (r + 1 < R) {
      const int k = r + 1 < R ? r + 1 : 0;
      return (code == rb[k] || hapN) ? pm[k] : px[k];
    }
    return (code == lrb || hapN) ? lpm : lpx;
  }
};

// The backward sweep's state between two steps. The BM rows are double-buffered: a step reads the
// column's old rows from one set (the diagonal of the row above) and writes the new ones to the
// other, and consecutive steps swap the sets (the step's parity picks them), so no row is copied.
template <class P, int R>
struct AdjBwd {
  using V = typename P::V;
  using Z = AdjSizes<P, R>;
  V BA[R], BB[R], BY[R];
  V dBM, topBM, topBX;

  template <bool kB>
  __device__ __forceinline__ V (&cur())[R] {
    if constexpr (kB)
      return BB;
    else
      return BA;
  }
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int r = 0; r < R; ++r) BA[r] = BB[r] = BY[r] = P::zero();
    dBM = topBM = topBX = P::zero();
  }
  // Saved as [chunk][lane] 16-byte chunks, so each chunk of the warp is 512 contiguous bytes; kB
  // names the set holding the current rows.
  template <bool kB>
  __device__ __forceinline__ void save(V* dst, int lane) {
    V rec[Z::kStateChunks * Z::kPer16];
    const V(&bm)[R] = cur<kB>();
#pragma unroll
    for (int r = 0; r < R; ++r) {
      rec[r] = bm[r];
      rec[R + r] = BY[r];
    }
    rec[2 * R] = dBM;
    rec[2 * R + 1] = topBM;
    rec[2 * R + 2] = topBX;
#pragma unroll
    for (int i = 2 * R + 3; i < Z::kStateChunks * Z::kPer16; ++i) rec[i] = P::zero();
#pragma unroll
    for (int c = 0; c < Z::kStateChunks; ++c)
      reinterpret_cast<uint4*>(dst)[c * 32 + lane] = reinterpret_cast<const uint4*>(rec)[c];
  }
  // Restores a saved state multiplied by `scale` into the first set.
  __device__ __forceinline__ void restore(const V* src, int lane, V scale) {
    V rec[Z::kStateChunks * Z::kPer16];
#pragma unroll
    for (int c = 0; c < Z::kStateChunks; ++c)
      reinterpret_cast<uint4*>(rec)[c] = reinterpret_cast<const uint4*>(src)[c * 32 + lane];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      BA[r] = P::mul(rec[r], scale);
      BY[r] = P::mul(rec[R + r], scale);
    }
    dBM = P::mul(rec[2 * R], scale);
    topBM = P::mul(rec[2 * R + 1], scale);
    topBX = P::mul(rec[2 * R + 2], scale);
  }
};

// One backward step at lane position p (column m - p), reading haplotype byte `code` (the diagonal
// successor's base), from BM set kB to set !kB. `sink` is the scale added at the read's last row
// (lane 31 of the last row block). kGeneral: a step where some lane is at or before column m (p <= 0:
// the all-zero column beyond the haplotype is set at p == 0) or where lane 31 takes the row below from
// the stored top row of the block below (`below`: cBX its BX at this column, cBM its BM, the next
// step's diagonal); without it the step is an interior step of a one-block read and skips both.
// kRec: keep the column's BM, BX, BY rows in `rec`.
template <class P, int R, bool kRec, bool kGeneral, bool kB>
__device__ __forceinline__ void adj_bwd_step(AdjBwd<P, R>& s, const AdjCoef<P, R>& c, typename P::V sink, int code, int p,
                                             bool below, typename P::V cBM, typename P::V cBX,
                                             typename P::V (&rec)[AdjSizes<P, R>::kRecVals]) {
  using V = typename P::V;
  V(&old)[R] = s.template cur<kB>();
  V(&nw)[R] = s.template cur<!kB>();
  V rBM = P::down(s.topBM), rBX = P::down(s.topBX);
  if (kGeneral) {
    if (below) {
      rBM = cBM;
      rBX = cBX;
    }
    if (p == 0) {
#pragma unroll
      for (int r = 0; r < R; ++r) old[r] = s.BY[r] = P::zero();
      s.dBM = P::zero();
    }
  }
  const bool hapN = code == 'N';
  V belowX = rBX;
#pragma unroll
  for (int r = R - 1; r >= 0; --r) {
    const V diagM = r + 1 < R ? old[r + 1 < R ? r + 1 : 0] : s.dBM;
    const V into = P::mul(c.bprior(code, hapN, r), diagM);
    const V itm = P::mul(into, c.bim(r));
    V bx = P::fma(belowX, c.bii(r), itm);
    const V by = P::fma(s.BY[r], c.dd[r], itm);
    V bm = P::fma(s.BY[r], c.md[r], P::fma(belowX, c.bmi(r), P::mul(into, c.bmm(r))));
    if (r == R - 1) {
      bm = P::add(bm, sink);
      bx = P::add(bx, sink);
    }
    nw[r] = bm;
    s.BY[r] = by;
    belowX = bx;
    if (kRec) {
      rec[r] = bm;
      rec[R + r] = bx;
      rec[2 * R + r] = by;
    }
  }
  s.topBM = nw[0];
  s.topBX = belowX;
  s.dBM = rBM;
}

// The haplotype byte the backward step at lane position p reads (the diagonal successor's base),
// 0 beyond the haplotype.
__device__ __forceinline__ int adj_bwd_code(const uint8_t* hap, int m, int p) {
  const int jj = m - p;
  return (p >= 0 && jj >= 0 && jj < m) ? __ldg(hap + jj) : 0;
}

// A pair's per-warp scratch: checkpoints [row block][state][chunk][lane], then the top rows of row
// blocks 1.. [block - 1][column 0..m] (BM, BX), then one bottom row [column] (M, X, Y, 0).
template <class P, int R>
struct AdjScratch {
  using V = typename P::V;
  using Z = AdjSizes<P, R>;
  static constexpr size_t kStateBytes = static_cast<size_t>(Z::kStateChunks) * 32 * 16;
  char* base;
  int n_states;  // per row block
  int m;
  int blocks;

  __host__ __device__ static size_t align(size_t x) { return (x + 255) / 256 * 256; }
  __host__ __device__ static size_t states_bytes(int blocks, int n_states) {
    return align(static_cast<size_t>(blocks) * n_states * kStateBytes);
  }
  __host__ __device__ static size_t up_bytes(int blocks, int m) {
    return align(static_cast<size_t>(blocks > 1 ? blocks - 1 : 0) * (m + 1) * 2 * sizeof(V));
  }
  __host__ __device__ static size_t down_bytes(int blocks, int m) { return blocks > 1 ? align(static_cast<size_t>(m) * 4 * sizeof(V)) : 0; }
  __host__ __device__ static size_t bytes(int read_len, int hap_len) {
    const int blocks = adj_row_blocks(read_len, R);
    const int n = hap_len + 31;
    const int n_states = (n + Z::K - 1) / Z::K;
    return states_bytes(blocks, n_states) + up_bytes(blocks, hap_len) + down_bytes(blocks, hap_len);
  }
  __device__ V* state(int block, int i) const {
    return reinterpret_cast<V*>(base + (static_cast<size_t>(block) * n_states + i) * kStateBytes);
  }
  __device__ V* up(int block, int column) const {  // block >= 1
    return reinterpret_cast<V*>(base + states_bytes(blocks, n_states)) + (static_cast<size_t>(block - 1) * (m + 1) + column) * 2;
  }
  __device__ V* down(int p) const {
    return reinterpret_cast<V*>(base + states_bytes(blocks, n_states) + up_bytes(blocks, m)) + static_cast<size_t>(p) * 4;
  }
};

// Steps where every lane of a one-block read lies strictly inside the haplotype, in both sweeps:
// forward step t (lane positions t - 31 .. t, columns 1 .. m) and backward step t (positions
// t - 31 .. t) are interior for 32 <= t <= m - 1.
constexpr int kAdjInteriorFirst = 32;

// Backward sweep of row block `blk` over steps 0 .. m + 31, saving the state entering every K-th
// step before the end (the state entering backward step n - (i + 1) K as checkpoint i, n = m + 31)
// and, for a block below another, its top row (lane 0) at every column. Returns, in every lane, the
// start mass s of the padding row above the read (first row block only).
template <class P, int R>
__device__ typename P::V adj_backward(const AdjCoef<P, R>& c, const uint8_t* hap, int m, int lane, const AdjScratch<P, R>& sc,
                                      int blk, int pad) {
  using V = typename P::V;
  using S = typename P::S;
  using Z = AdjSizes<P, R>;
  const bool last = blk == sc.blocks - 1;
  const bool single = sc.blocks == 1 && pad >= R;  // one row block, lane 0 all padding
  const V sink = (lane == 31 && last) ? static_cast<S>(Consts<P::kDouble>::kBackwardScale) : P::zero();
  const bool below = lane == 31 && !last;
  AdjBwd<P, R> st;
  st.zero();
  const int pad_row = pad - 1;  // the padding row right above the read (first block)
  const int pad_lane = pad_row >= 0 ? pad_row / R : 0, pad_r = pad_row >= 0 ? pad_row % R : 0;
  const int n = m + 31;
  V start_mass = P::zero();
  int next_code = adj_bwd_code(hap, m, -(31 - lane));
  V cBM = P::zero(), cBX = P::zero();
  V rec[Z::kRecVals];
  auto general = [&](int t) {
    if (t > 0 && t < n && (n - t) % Z::K == 0) {
      if (t & 1)
        st.template save<true>(sc.state(blk, (n - t) / Z::K - 1), lane);
      else
        st.template save<false>(sc.state(blk, (n - t) / Z::K - 1), lane);
    }
    const int p = t - (31 - lane);
    const int code = next_code;
    next_code = adj_bwd_code(hap, m, p + 1);
    if (below) {
      // Lane 31 is at position t: column m - t of the block below's top row.
      if (t <= m) {
        const V* u = sc.up(blk + 1, m - t);
        cBM = u[0];
        cBX = u[1];
      } else {
        cBM = cBX = P::zero();
      }
    }
    if (t & 1)
      adj_bwd_step<P, R, false, true, true>(st, c, sink, code, p, below, cBM, cBX, rec);
    else
      adj_bwd_step<P, R, false, true, false>(st, c, sink, code, p, below, cBM, cBX, rec);
    if (blk > 0 && lane == 0 && p >= 0 && p <= m) {
      V* u = sc.up(blk, m - p);
      u[0] = st.topBM;
      u[1] = st.topBX;
    }
    if (blk == 0 && p == m && lane == pad_lane) {
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (r == pad_r) start_mass = st.BY[r];
    }
  };
  int t = 0;
  const int fast_end = single ? m - 1 : -1;  // last interior step
  for (; t <= n && (t < kAdjInteriorFirst || t > fast_end); ++t) general(t);
  // Interior steps, two at a time from an even step: the next step's byte is in range
  // (m - t + 30 - lane in [0, m - 2]).
  auto interior = [&](int t, auto flip) {
    constexpr bool kB = decltype(flip)::value;
    if ((n - t) % Z::K == 0) st.template save<kB>(sc.state(0, (n - t) / Z::K - 1), lane);
    const int code = next_code;
    next_code = __ldg(hap + (m - t + 30 - lane));
    adj_bwd_step<P, R, false, false, kB>(st, c, sink, code, 0, false, cBM, cBX, rec);
  };
  for (; t + 1 <= fast_end; t += 2) {
    interior(t, std::false_type{});
    interior(t + 1, std::true_type{});
  }
  if (t <= fast_end) interior(t++, std::false_type{});
  for (; t <= n; ++t) general(t);
  return __shfl_sync(kFull, start_mass, pad_lane);
}

// The forward sweep's registers: M, X, Y rows, the row above the lane's top row on the diagonal,
// and the accumulated result.
template <class P, int R>
struct AdjFwd {
  using V = typename P::V;
  V M[R], X[R], Y[R];
  V dM, dX, dY, acc;
};

// One forward step: the column's forward values from the diagonal (d*), the row above (uM, uX) and
// the lane's registers, and the gradient terms against the column's backward values (rec: BM, BX,
// BY rows, already multiplied by c). kMask: steps where some lane lies outside the haplotype, whose
// terms are dropped.
template <class P, int R, bool kMask>
__device__ __forceinline__ void adj_fwd_step(AdjFwd<P, R>& f, const AdjCoef<P, R>& c, int code, bool live,
                                             const typename P::V (&rec)[AdjSizes<P, R>::kRecVals], typename P::V uM,
                                             typename P::V uX, typename P::V (&gi)[R], typename P::V (&gd)[R],
                                             typename P::V (&ge)[R], typename P::V (&gq)[R]) {
  using V = typename P::V;
  using S = typename P::S;
  const V minus_one = static_cast<S>(-1.0);
  const bool hapN = code == 'N';
  // Match and deletion values from the bottom row up (each row reads the old row above).
#pragma unroll
  for (int r = R - 1; r >= 0; --r) {
    const V pM = r ? f.M[r - 1] : f.dM, pX = r ? f.X[r - 1] : f.dX, pY = r ? f.Y[r - 1] : f.dY;
    const V mOld = f.M[r], yOld = f.Y[r];
    const bool match = code == c.rb[r] || hapN;
    const V prior = match ? c.pm[r] : c.px[r];
    const V kq = match ? minus_one : c.kqx[r];
    const V sxy = P::add(pX, pY);
    const V s = P::fma(pM, c.mm[r], P::mul(sxy, c.im[r]));
    f.Y[r] = P::fma(yOld, c.dd[r], P::mul(mOld, c.md[r]));
    f.M[r] = P::mul(prior, s);
    V bm = rec[r], by = rec[2 * R + r];
    if (kMask && !live) bm = by = P::zero();
    const V bmp = P::mul(bm, prior);
    gi[r] = P::fma(-pM, bmp, gi[r]);
    gd[r] = P::fma(-pM, bmp, P::fma(mOld, by, gd[r]));
    ge[r] = P::fma(-sxy, bmp, P::fma(yOld, by, ge[r]));
    gq[r] = P::fma(s, P::mul(bm, kq), gq[r]);
  }
  // Insertion values from the top row down (each row reads the new row above).
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const V qM = r ? f.M[r - 1] : uM, qX = r ? f.X[r - 1] : uX;
    f.X[r] = P::fma(qX, c.ii[r], P::mul(qM, c.mi[r]));
    V bx = rec[R + r];
    if (kMask && !live) bx = P::zero();
    gi[r] = P::fma(qM, bx, gi[r]);
    ge[r] = P::fma(qX, bx, ge[r]);
  }
  if (!kMask || live) f.acc = P::add(f.acc, P::add(f.M[R - 1], f.X[R - 1]));
}

// Adds the lane's FP32 (FP64) sums into the per-position gradients and clears them.
template <class P, int R>
__device__ __forceinline__ void adj_flush(const AdjView& v, const AdjCoef<P, R>& c, int64_t off, int pad, int lane,
                                          typename P::V (&gi)[R], typename P::V (&gd)[R], typename P::V (&ge)[R],
                                          typename P::V (&gq)[R]) {
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if ((c.real >> r) & 1u) {
      const int64_t o = off + lane * R + r - pad;
      atomicAdd(v.g_ins + o, static_cast<double>(gi[r]));
      atomicAdd(v.g_del + o, static_cast<double>(gd[r]));
      atomicAdd(v.g_eps + o, static_cast<double>(ge[r]));
      atomicAdd(v.g_err + o, static_cast<double>(gq[r]));
    }
    gi[r] = gd[r] = ge[r] = gq[r] = P::zero();
  }
}

// Forward sweep of row block `blk`, block by block of K steps with the backward values recomputed
// into shared memory first, accumulating the gradient terms; returns lane 31's accumulated result
// (meaningful in the last row block). `c_fac` scales the recomputed backward values, `init` is the
// row-0 constant of the scaled forward values. Blocks whose steps are all interior steps of a
// one-block read (kAdjInteriorFirst) run both sweeps without the edge and row-block code.
template <class P, int R>
__device__ typename P::V adj_forward(const AdjView& v, const AdjCoef<P, R>& c, int64_t off, int pad, const uint8_t* hap, int m, int lane,
                                     const AdjScratch<P, R>& sc, int blk, typename P::V* smem, typename P::V c_fac,
                                     typename P::V init) {
  using V = typename P::V;
  using S = typename P::S;
  using Z = AdjSizes<P, R>;
  constexpr int K = Z::K;
  const bool first = blk == 0, last = blk == sc.blocks - 1;
  const bool single = sc.blocks == 1 && pad >= R;  // one row block, lane 0 all padding
  const int n = m + 31;
  const V sink = (lane == 31 && last) ? P::mul(static_cast<S>(Consts<P::kDouble>::kBackwardScale), c_fac) : P::zero();
  const bool below = lane == 31 && !last;
  AdjFwd<P, R> f;
#pragma unroll
  for (int r = 0; r < R; ++r) f.M[r] = f.X[r] = f.Y[r] = P::zero();
  f.dM = f.dX = f.dY = f.acc = P::zero();
  V gi[R], gd[R], ge[R], gq[R];
#pragma unroll
  for (int r = 0; r < R; ++r) gi[r] = gd[r] = ge[r] = gq[r] = P::zero();
  uint4* buf = reinterpret_cast<uint4*>(smem);
  V* stage = reinterpret_cast<V*>(reinterpret_cast<char*>(smem) + Z::kStageOffset);
  // The checkpoint a block starts from, copied into shared memory a block ahead (each lane its own
  // chunks), so the restore does not wait on global memory.
  auto fetch_state = [&](int t0n) {
    const int lo_n = max(0, n - min(t0n + K, n));
    if (t0n < n && lo_n > 0) {
      const V* src = sc.state(blk, (n - lo_n) / K - 1);
#pragma unroll
      for (int ch = 0; ch < Z::kStateChunks; ++ch)
        __pipeline_memcpy_async(reinterpret_cast<char*>(stage) + (ch * 32 + lane) * 16,
                                reinterpret_cast<const char*>(src) + (ch * 32 + lane) * 16, 16);
    }
    __pipeline_commit();
  };
  auto store_rec = [&](int slot, V (&rec)[Z::kRecVals]) {
#pragma unroll
    for (int i = 3 * R; i < Z::kRecVals; ++i) rec[i] = P::zero();
#pragma unroll
    for (int ch = 0; ch < Z::kRecChunks; ++ch) buf[(slot * Z::kRecChunks + ch) * 32 + lane] = reinterpret_cast<const uint4*>(rec)[ch];
  };
  auto load_rec = [&](int t, int lo, V (&rec)[Z::kRecVals]) {
    const int slot = n - 1 - t - lo;
#pragma unroll
    for (int ch = 0; ch < Z::kRecChunks; ++ch) reinterpret_cast<uint4*>(rec)[ch] = buf[(slot * Z::kRecChunks + ch) * 32 + lane];
  };
  fetch_state(0);
  int flushed = 0;
  for (int t0 = 0; t0 < n; t0 += K) {
    const int t1 = min(t0 + K, n);
    const int lo = max(0, n - t1), hi = n - 1 - t0;
    const bool interior = single && t0 >= kAdjInteriorFirst && t1 <= m - 1;
    // Backward steps [lo, hi] from the checkpoint entering lo (or the start), scaled by c_fac, into
    // the block buffer [step - lo][chunk][lane].
    {
      AdjBwd<P, R> st;
      __pipeline_wait_prior(0);
      if (lo > 0)
        st.restore(stage, lane, c_fac);
      else
        st.zero();
      fetch_state(t0 + K);
      // Step tb uses BM set (tb - lo) & 1; the restored state is in the first set.
      if (interior) {
        // Backward steps lo..hi are interior (lo >= 32, hi <= m - 2): step tb reads byte
        // m - tb + 31 - lane, inside [2, m - 1].
        int next_code = __ldg(hap + (m - lo + 31 - lane));
        auto rstep = [&](int tb, auto flip) {
          const int code = next_code;
          next_code = __ldg(hap + (m - tb + 30 - lane));
          V rec[Z::kRecVals];
          adj_bwd_step<P, R, true, false, decltype(flip)::value>(st, c, sink, code, 0, false, P::zero(), P::zero(), rec);
          store_rec(tb - lo, rec);
        };
        int tb = lo;
        for (; tb + 1 <= hi; tb += 2) {
          rstep(tb, std::false_type{});
          rstep(tb + 1, std::true_type{});
        }
        if (tb <= hi) rstep(tb, std::false_type{});
      } else {
        int next_code = adj_bwd_code(hap, m, lo - (31 - lane));
        for (int tb = lo; tb <= hi; ++tb) {
          const int p = tb - (31 - lane);
          const int code = next_code;
          next_code = adj_bwd_code(hap, m, p + 1);
          V cBM = P::zero(), cBX = P::zero();
          if (below && tb <= m) {
            const V* u = sc.up(blk + 1, m - tb);
            cBM = P::mul(u[0], c_fac);
            cBX = P::mul(u[1], c_fac);
          }
          V rec[Z::kRecVals];
          if ((tb - lo) & 1)
            adj_bwd_step<P, R, true, true, true>(st, c, sink, code, p, below, cBM, cBX, rec);
          else
            adj_bwd_step<P, R, true, true, false>(st, c, sink, code, p, below, cBM, cBX, rec);
          store_rec(tb - lo, rec);
        }
      }
    }
    __syncwarp();
    if (interior) {
      // Every lane inside the haplotype at every step (step t reads byte t - lane, inside [1, m - 1]),
      // no row block above or below: lane 0's rows are all padding and feed themselves the row-0
      // constant through the shuffle.
      int next_fcode = __ldg(hap + t0 - lane);
      for (int t = t0; t < t1; ++t) {
        const int code = next_fcode;
        next_fcode = __ldg(hap + (t + 1 - lane));
        V rec[Z::kRecVals];
        load_rec(t, lo, rec);
        const V uM = P::up(f.M[R - 1]), uX = P::up(f.X[R - 1]), uY = P::up(f.Y[R - 1]);
        adj_fwd_step<P, R, false>(f, c, code, true, rec, uM, uX, gi, gd, ge, gq);
        f.dM = uM;
        f.dX = uX;
        f.dY = uY;
      }
    } else {
      // The haplotype base of each step, loaded a step ahead.
      int next_fcode = (t0 - lane >= 0 && t0 - lane < m) ? __ldg(hap + t0 - lane) : 0;
      for (int t = t0; t < t1; ++t) {
        const int p = t - lane;  // column p + 1
        const bool live = p >= 0 && p < m;
        const int code = next_fcode;
        next_fcode = (p + 1 >= 0 && p + 1 < m) ? __ldg(hap + p + 1) : 0;
        V rec[Z::kRecVals];
        load_rec(t, lo, rec);
        V uM = P::up(f.M[R - 1]), uX = P::up(f.X[R - 1]), uY = P::up(f.Y[R - 1]);
        if (lane == 0) {
          if (first) {
            uM = uX = P::zero();
            uY = init;
          } else if (p >= 0 && p < m) {
            const V* d = sc.down(p);
            uM = d[0];
            uX = d[1];
            uY = d[2];
          }
        }
        if (p == 0) {
          // Column 0: the row-0 constant in the padding rows (and above the lane's top row when
          // that is padding).
#pragma unroll
          for (int r = 0; r < R; ++r) {
            f.M[r] = f.X[r] = P::zero();
            f.Y[r] = lane * R + r < pad ? init : P::zero();
          }
          f.dM = f.dX = P::zero();
          f.dY = lane * R - 1 < pad ? init : P::zero();
          f.acc = P::zero();
        }
        adj_fwd_step<P, R, true>(f, c, code, live, rec, uM, uX, gi, gd, ge, gq);
        f.dM = uM;
        f.dX = uX;
        f.dY = uY;
        if (!last && lane == 31 && live) {
          V* d = sc.down(p);
          d[0] = f.M[R - 1];
          d[1] = f.X[R - 1];
          d[2] = f.Y[R - 1];
        }
      }
    }
    if (t1 - flushed >= kFlushSteps || t1 == n) {
      adj_flush<P, R>(v, c, off, pad, lane, gi, gd, ge, gq);
      flushed = t1;
    }
    __syncwarp();
  }
  __pipeline_wait_prior(0);
  return __shfl_sync(kFull, f.acc, 31);
}

template <class P, int R>
struct AdjMinBlocks {
  static constexpr int value = P::kDouble ? 1 : (R <= 6 ? 3 : 2);
};

template <class P, int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, (AdjMinBlocks<P, R>::value)) adjoint_kernel(AdjLaunch a) {
  using V = typename P::V;
  using S = typename P::S;
  using C = Consts<P::kDouble>;
  using Z = AdjSizes<P, R>;
  extern __shared__ __align__(16) unsigned char adj_smem[];
  const int lane = threadIdx.x & 31;
  const int warp = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  V* smem = reinterpret_cast<V*>(adj_smem + (threadIdx.x >> 5) * Z::kSmemPerWarp);
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
    const int blocks = adj_row_blocks(len, R);
    const int pad0 = 32 * R * blocks - len;
    const int h0 = a.v.region_hap[g], nh = a.v.region_nhap[g];
    const int read_local = read - a.v.region_read[g];
    bool lost = false;
    for (int h = 0; h < nh && !lost; ++h) {
      const int64_t hlo = a.v.hap_off[h0 + h];
      const int m = static_cast<int>(a.v.hap_off[h0 + h + 1] - hlo);
      const uint8_t* hap = a.v.hap_bases + hlo;
      AdjScratch<P, R> sc;
      sc.base = a.scratch + static_cast<size_t>(warp) * a.scratch_stride;
      sc.m = m;
      sc.blocks = blocks;
      sc.n_states = (m + 31 + Z::K - 1) / Z::K;
      // 1. Backward sweeps, bottom row block first; the first block yields the start mass.
      V s = P::zero();
      for (int blk = blocks - 1; blk >= 0; --blk) {
        AdjCoef<P, R> c;
        c.load(a.v, off, len, pad0 - 32 * R * blk, lane);
        s = adj_backward<P, R>(c, hap, m, lane, sc, blk, pad0 - 32 * R * blk);
        __syncwarp();
      }
      const double init = C::kInitial / m;
      const double raw = init * static_cast<double>(s) / C::kBackwardScale;
      if (!P::kDouble && (!(raw >= C::kMinAccepted) || isinf(raw))) {
        lost = true;
        break;
      }
      // 2. The scale split: F from init * 2^-a, B times 2^a / (raw * scale * ln 10).
      int shift = 0;
      if (!P::kDouble) {
        shift = static_cast<int>(floor(0.5 * (log2(raw) + log2(init))));
        shift = max(0, min(shift, 240));
      }
      const V c_fac = static_cast<S>(ldexp(1.0, shift) / (raw * C::kBackwardScale * ln10));
      const V init_a = static_cast<S>(ldexp(init, -shift));
      // 3. Forward sweeps, top row block first, with the gradient terms.
      V fwd = P::zero();
      for (int blk = 0; blk < blocks; ++blk) {
        AdjCoef<P, R> c;
        const int pad = pad0 - 32 * R * blk;
        c.load(a.v, off, len, pad, lane);
        fwd = adj_forward<P, R>(a.v, c, off, pad, hap, m, lane, sc, blk, smem, c_fac, init_a);
        __syncwarp();
      }
      const double fwd_raw = ldexp(static_cast<double>(fwd), shift);
      if (!P::kDouble && (!(fwd_raw >= C::kMinAccepted) || isinf(fwd_raw))) {
        lost = true;
        break;
      }
      if (lane == 0) a.v.out[a.v.region_out[g] + static_cast<int64_t>(read_local) * nh + h] = log10(fwd_raw) - C::kLog10Initial;
      __syncwarp();
    }
    if (lost) {
      // The FP64 recomputation sums this read's gradients afresh: clear what earlier haplotypes added,
      // each position by the lane that added to it (atomics of one thread to one address keep their
      // order).
      for (int blk = 0; blk < blocks; ++blk)
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int q = lane * R + r - (pad0 - 32 * R * blk);
          if (q < 0 || q >= len) continue;
          atomicExch(reinterpret_cast<unsigned long long*>(a.v.g_ins + off + q), 0ull);
          atomicExch(reinterpret_cast<unsigned long long*>(a.v.g_del + off + q), 0ull);
          atomicExch(reinterpret_cast<unsigned long long*>(a.v.g_eps + off + q), 0ull);
          atomicExch(reinterpret_cast<unsigned long long*>(a.v.g_err + off + q), 0ull);
        }
      __syncwarp();
      if (lane == 0) {
        atomicAdd(a.v.lost, 1ull);
        if (a.queue) {
          const int bin = adj_rows(len);
          const int slot = atomicAdd(a.queue_tail + bin, 1);
          if (slot < a.queue_off[bin + 1] - a.queue_off[bin]) a.queue[a.queue_off[bin] + slot] = read;
        }
      }
    }
  }
}

template <class P, int R>
void adj_occ(int* blocks) {
  static std::atomic<int> cache[kMaxDevices];
  *blocks = resident_blocks(adjoint_kernel<P, R>, kWarpsPerBlock * AdjSizes<P, R>::kSmemPerWarp, kWarpsPerBlock * 32, cache);
}

template <class P, int R>
cudaError_t adj_go(int blocks, const AdjLaunch& a, cudaStream_t s) {
  const size_t smem = kWarpsPerBlock * AdjSizes<P, R>::kSmemPerWarp;
  // resident_blocks set the kernel's dynamic shared-memory limit on this device.
  int per_sm = 0;
  adj_occ<P, R>(&per_sm);
  adjoint_kernel<P, R><<<blocks, kWarpsPerBlock * 32, smem, s>>>(a);
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

size_t adj_scratch_bytes(bool dbl, int rows, int read_len, int hap_len) {
  return adj_dispatch_rows(rows, [&](auto r) {
    constexpr int R = decltype(r)::value;
    return dbl ? AdjScratch<OneF64, R>::bytes(read_len, hap_len) : AdjScratch<OneF32, R>::bytes(read_len, hap_len);
  });
}

void adj_occupancy(bool dbl, int rows, int* blocks, int* threads) {
  *threads = kWarpsPerBlock * 32;
  *blocks = 0;
  adj_dispatch_rows(rows, [&](auto r) {
    constexpr int R = decltype(r)::value;
    if (dbl)
      adj_occ<OneF64, R>(blocks);
    else
      adj_occ<OneF32, R>(blocks);
    return 0;
  });
}

cudaError_t adj_launch(bool dbl, int rows, int blocks, const AdjLaunch& a, cudaStream_t s) {
  return adj_dispatch_rows(rows, [&](auto r) {
    constexpr int R = decltype(r)::value;
    return dbl ? adj_go<OneF64, R>(blocks, a, s) : adj_go<OneF32, R>(blocks, a, s);
  });
}

}  // namespace fgkl
