// sm_100a PairHMM kernels: one warp per read task, read rows on lanes, the region's column stream
// walked as an anti-diagonal wavefront.
//
// Rows. Lane l holds rows l*R .. l*R+R-1 of a 32*R-row block whose LAST row is the read's last row
// and R = ceil(len / 31), so lane 0 holds only padding rows. Padding rows have zero transitions and
// priors and a deletion chain of 1: they keep M = X = 0 and Y = INITIAL / hap_len, i.e. they
// reproduce row 0 of GATK's matrix, the row just above the read plays row 0, and lane 0 feeds
// itself exact row-0 values through the shuffle. At loop step t lane l is at stream position t - l
// (forward) or t - (31 - l) (backward); the row above (below) arrives by one shuffle per value.
//
// Forward recurrence per cell (GATK LoglessPairHMM, fgkl kernel.rs:1011-1013):
//   M = prior * (mm*M(i-1,j-1) + im*(X(i-1,j-1) + Y(i-1,j-1)))
//   X = mi*M(i-1,j) + ii*X(i-1,j)          Y = md*M(i,j-1) + dd*Y(i,j-1)
// The FP32 kernels carry X/mi and Y/md (per-row constants) instead of X and Y: every term stays
// positive, the X and Y updates become one FMA each. They also fold each row's mm into its priors
// (M = (prior*mm) * (M(i-1,j-1) + k1*X^ + k2*Y^)), 5 FP32 operations per cell instead of 8. An
// overflow this could cause for extreme gap-open ratios surfaces as a non-finite result, which is
// recomputed in FP64 with the plain recurrence.
//
// Backward recurrence (suffix sharing, fgkl kernel.rs:1080-1088), row i from row i+1:
//   into = prior(i+1,j+1) * BM(i+1,j+1);  BX = ii'*BX(i+1,j) + im'*into
//   BY = dd*BY(i,j+1) + im'*into;         BM = md*BY(i,j+1) + mi'*BX(i+1,j) + mm'*into
// (primed: transitions of row i+1), plus BACKWARD_SCALE at the read's last row. The padding row
// above the read accumulates fgkl's row-0 start mass `s` in its BY (dd = 1 there).
//
// Events. A lane handles all events of a step in one divergent branch: the stores for the previous
// column (SNAP, END, NODE) and then the loads for its own (BEGIN, SWEEP). Start states come from a
// per-warp staging buffer in shared memory, one record per lane: the previous segment writes it
// directly when it is the snapshot's last writer, otherwise the state is prefetched from global
// scratch with cp.async at the previous segment's BEGIN, after that BEGIN has read the record. Joins only store their forward column; the products
// with the backward node are summed after the sweep, warp-wide, in an order fixed by the read row.
#include <cuda_pipeline.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "dp_common.cuh"
#include "kernels.cuh"

namespace fgkl {

namespace {

// Per-lane field counts of the scratch records, rounded so every record starts on 16 bytes.
template <class P, int R>
struct Layout {
  using V = typename P::V;
  static constexpr int kRound = 16 / static_cast<int>(sizeof(V)) > 1 ? 16 / static_cast<int>(sizeof(V)) : 1;
  static constexpr int up(int x) { return (x + kRound - 1) / kRound * kRound; }
  static constexpr int kSnap = up(3 * R + 4);  // M, X, Y rows; above-row M, X, Y; accumulated result
  static constexpr int kNode = up(2 * R + 1);  // BM, BY rows; below-row BM
  static constexpr int kJoin = up(2 * R);      // cut column M and Y rows
  static constexpr int kStage = kSnap > kNode ? kSnap : kNode;
  // FP32 kernels look priors up in a per-lane table indexed by haplotype code (A, C, G, T, N);
  // regions holding other haplotype bytes run on the FP64 kernel, which compares codes instead.
  static constexpr int kPriorCodes = P::kDouble ? 0 : 5;
  // A lane's priors for one code: its rows padded to whole 16-byte chunks, kPer16 rows a chunk.
  static constexpr int kPer16 = kRound;
  static constexpr int kRp = up(R);
  static constexpr int kChunks = kRp / kPer16;
  static constexpr size_t kStageBytes = 32ull * kStage * sizeof(V);
  static constexpr size_t kSmemPerWarp = kStageBytes + static_cast<size_t>(kPriorCodes) * kRp * 32 * sizeof(V);
  // Element of row r's prior for `code` in the table, [code][chunk][lane][row in chunk]: each chunk of
  // the warp is 512 contiguous bytes, so a step's chunk loads are conflict-free 16-byte loads.
  __device__ static int prior_at(int code, int r, int lane) {
    return ((code * kChunks + r / kPer16) * 32 + lane) * kPer16 + r % kPer16;
  }
};

// Priors of the lane's rows for every haplotype code, in shared memory (Layout::prior_at), times the
// row's match-to-match factor in the FP32 form (cell_match).
template <class P, int R>
__device__ __forceinline__ void put_priors(typename P::V* table, int lane, int r, int c, const RowModel& m) {
  using S = typename P::S;
  const double fold = (P::kTransformed && m.read) ? m.mm : 1.0;
  for (int code = 0; code < Layout<P, R>::kPriorCodes; ++code) {
    const bool match = code == m.oc || code == kCodeN;
    P::put(table[Layout<P, R>::prior_at(code, r, lane)], c, static_cast<S>((match ? m.pm : m.px) * fold));
  }
}

// The lane's priors of every row for `code`, one 16-byte shared-memory load per chunk.
template <class P, int R>
__device__ __forceinline__ void load_priors(const typename P::V* table, int code, int lane,
                                            typename P::V (&pri)[Layout<P, R>::kRp]) {
  using L = Layout<P, R>;
  const uint4* src = reinterpret_cast<const uint4*>(table);
#pragma unroll
  for (int k = 0; k < L::kChunks; ++k) reinterpret_cast<uint4*>(pri)[k] = src[(code * L::kChunks + k) * 32 + lane];
}

// Forward coefficients of the lane's rows.
template <class P, int R>
struct FwdRows {
  using V = typename P::V;
  using S = typename P::S;
  V c0[R], c1[R], c2[R], c3[R], c4[R], pm[R], px[R];
  int oc[P::NC][R];
  const V* table;  // prior table (FP32 kernels)

  __device__ V prior(int code, bool isN, int r, int lane) const {
    if (Layout<P, R>::kPriorCodes) return table[Layout<P, R>::prior_at(code, r, lane)];
    const bool m0 = (code == oc[0][r]) | isN;
    const bool m1 = (code == oc[P::NC - 1][r]) | isN;
    return P::sel(m0, m1, pm[r], px[r]);
  }

  __device__ void load(const BatchView& v, const ReadRef* rd, int lane, const uint8_t* codes, V* ptable) {
    table = ptable;
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
      for (int c = 0; c < P::NC; ++c) {
        const int g = lane * R + r;
        const RowModel m = row_model(v, rd[c], g - rd[c].pad, codes);
        double k0, k1, k2, k3, k4;
        if (P::kTransformed) {
          // S = mm*M + (im*mi')*X^ + (im*md')*Y^ with X = mi*X^, Y = md*Y^, taken as
          // mm * (M + (im*mi'/mm)*X^ + (im*md'/mm)*Y^) with mm in the prior table (cell_match);
          // X^ = M_up + (gc*mi'/mi)*X^_up; Y^ = M_left + gc*Y^_left.
          if (m.read) {
            k0 = m.mm;
            k1 = m.im * m.mi_prev / m.mm;
            k2 = m.im * m.md_prev / m.mm;
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
        put_priors<P, R>(ptable, lane, r, c, m);
      }
    }
  }
};

// Backward coefficients: each row's own deletion transitions and the transitions and priors of the
// row below it (rows l*R+1 .. l*R+R; the last comes from the next lane's top row). In the FP32 form
// the row below's match-to-match factor sits in its prior table (put_priors), so `into` carries it
// and im holds im/mm of the row below.
template <class P, int R>
struct BwdRows {
  using V = typename P::V;
  using S = typename P::S;
  V md[R], dd[R], mm[R], im[R], mi[R], ii[R], pm[R], px[R];
  int oc[P::NC][R];
  const V* table;  // prior table of the rows below (FP32 kernels)

  __device__ V prior(int code, bool isN, int r, int lane) const {
    if (Layout<P, R>::kPriorCodes) return table[Layout<P, R>::prior_at(code, r, lane)];
    const bool m0 = (code == oc[0][r]) | isN;
    const bool m1 = (code == oc[P::NC - 1][r]) | isN;
    return P::sel(m0, m1, pm[r], px[r]);
  }

  __device__ void load(const BatchView& v, const ReadRef* rd, int lane, const uint8_t* codes, V* ptable) {
    table = ptable;
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
        P::put(im[r], c, static_cast<S>(P::kTransformed ? (below.read ? below.im / below.mm : 0.0) : below.im));
        P::put(mi[r], c, static_cast<S>(below.mi));
        P::put(ii[r], c, static_cast<S>(below.gc));
        P::put(pm[r], c, static_cast<S>(below.pm));
        P::put(px[r], c, static_cast<S>(below.px));
        oc[c][r] = below.oc;
        put_priors<P, R>(ptable, lane, r, c, below);
      }
    }
  }
};

// ---------------------------------------------------------------------------------------------
// Scratch: global per-warp records and the shared-memory staging buffers.
// ---------------------------------------------------------------------------------------------

template <class P, int R>
struct Scratch {
  using V = typename P::V;
  using L = Layout<P, R>;
  V* slots;         // [slot][lane][kSnap]
  V* nodes;         // [node][lane][kNode]
  V* joins;         // [seg][lane][kJoin]
  double* seg_raw;  // [seg][c]
  V* stage;         // shared: [buf][lane][kStage]
  V* priors;        // shared: [code][row][lane]

  __device__ Scratch(char* base, V* smem, int n_slots, int n_nodes, int n_segs) {
    slots = reinterpret_cast<V*>(base);
    nodes = slots + static_cast<size_t>(n_slots) * 32 * L::kSnap;
    joins = nodes + static_cast<size_t>(n_nodes) * 32 * L::kNode;
    seg_raw = reinterpret_cast<double*>(joins + static_cast<size_t>(n_segs) * 32 * L::kJoin);
    stage = smem;
    priors = reinterpret_cast<V*>(reinterpret_cast<char*>(smem) + L::kStageBytes);
  }
  __device__ V* slot(int s, int lane) { return slots + (static_cast<size_t>(s) * 32 + lane) * L::kSnap; }
  __device__ V* node(int n, int lane) { return nodes + (static_cast<size_t>(n) * 32 + lane) * L::kNode; }
  __device__ V* join(int seg, int lane) { return joins + (static_cast<size_t>(seg) * 32 + lane) * L::kJoin; }
  // One staging record per lane serves every segment (sweep): a lane writes or prefetches the next
  // segment's start into it only after loading the current segment's start at its BEGIN (SWEEP), and
  // each lane touches its own record alone.
  __device__ V* staged(int, int lane) { return stage + static_cast<size_t>(lane) * L::kStage; }
};

template <class P, int R>
__host__ __device__ constexpr size_t scratch_size(int n_slots, int n_nodes, int n_segs) {
  using V = typename P::V;
  using L = Layout<P, R>;
  return (static_cast<size_t>(n_slots) * 32 * L::kSnap + static_cast<size_t>(n_nodes) * 32 * L::kNode +
          static_cast<size_t>(n_segs) * 32 * L::kJoin) * sizeof(V) + static_cast<size_t>(n_segs) * P::NC * sizeof(double);
}

// Resident blocks per SM each instantiation is compiled for, chosen by timing each bin of the uneven
// workload: four up to 4 rows per lane (R = 4 then spills 8 bytes at 128 registers, and still runs
// 5% faster than at three blocks), three up to 7 (R = 7 spills 8 bytes at 168 and runs 8% faster
// than at two), two at 8 (three spill 76 bytes and run 6% slower).
template <class P, int R>
struct MinBlocks {
  static constexpr int value = P::NC == 2 ? (R <= 4 ? 4 : (R <= 7 ? 3 : 2)) : (P::kDouble ? 1 : 2);
};

// ---------------------------------------------------------------------------------------------
// Backward pass: every suffix sweep of the program, writing backward nodes.
// ---------------------------------------------------------------------------------------------

template <class P, int R>
__device__ void backward_pass(const LaunchArgs& a, const Program& prog, const ReadRef* rd, const uint8_t* codes, int lane,
                              Scratch<P, R>& sc) {
  using V = typename P::V;
  using L = Layout<P, R>;
  BwdRows<P, R> bp;
  bp.load(a.v, rd, lane, codes, sc.priors);
  const V sink = P::splat(lane == 31 ? static_cast<typename P::S>(Consts<P::kDouble>::kBackwardScale) : 0);
  V BM[R], BY[R];
#pragma unroll
  for (int r = 0; r < R; ++r) BM[r] = BY[r] = P::zero();
  V dBM = P::zero(), topBM = P::zero(), topBX = P::zero();
  const int n = prog.bwd_len;
  const uint32_t* stream = a.v.stream + prog.bwd_off - (31 - lane);  // entry of this lane's position at t
  int sweep = -1;
  uint32_t ev_next = __ldg(stream);
  for (int t = 0; t < n + 32; ++t) {
    const V rBM = P::down(topBM), rBX = P::down(topBX);
    const uint32_t ev = ev_next;
    ev_next = __ldg(stream + t + 1);
    if (ev & kEvMask) {
      if (ev & EV_NODE) {
        V rec[L::kNode];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          rec[r] = BM[r];
          rec[R + r] = BY[r];
        }
        rec[2 * R] = dBM;
#pragma unroll
        for (int i = 2 * R + 1; i < L::kNode; ++i) rec[i] = P::zero();
        store_record(sc.node(static_cast<int>(ev >> kPayloadShift), lane), rec);
        if (ev & EV_NSTAGE) store_record(sc.staged(sweep + 1, lane), rec);
      }
      if (ev & EV_SWEEP) {
        ++sweep;
        const Sweep cur = a.v.sweeps[prog.sweep_off + sweep];
        if (sweep + 1 < prog.n_sweeps) prefetch_l1(a.v.sweeps + prog.sweep_off + sweep + 1);
        if (cur.staged) {
          __pipeline_wait_prior(0);
          V rec[L::kNode];
          load_record(rec, sc.staged(sweep, lane));
#pragma unroll
          for (int r = 0; r < R; ++r) {
            BM[r] = rec[r];
            BY[r] = rec[R + r];
          }
          dBM = rec[2 * R];
        } else {
#pragma unroll
          for (int r = 0; r < R; ++r) BM[r] = BY[r] = P::zero();
          dBM = P::zero();
        }
        if (cur.next_node >= 0) prefetch(sc.staged(sweep + 1, lane), sc.node(cur.next_node, lane), L::kNode);
      }
    }
    const int code = ev & kCodeMask;
    const bool isN = code == kCodeN;
    V pri[L::kRp];
    if (L::kPriorCodes) load_priors<P, R>(bp.table, code, lane, pri);
    V belowX = rBX, diagM = dBM;
#pragma unroll
    for (int r = R - 1; r >= 0; --r) {
      const V into = P::mul(L::kPriorCodes ? pri[r] : bp.prior(code, isN, r, lane), diagM);
      const V itm = P::mul(into, bp.im[r]);
      V bx = P::fma(belowX, bp.ii[r], itm);
      const V by = P::fma(BY[r], bp.dd[r], itm);
      V bm = P::fma(BY[r], bp.md[r], P::fma(belowX, bp.mi[r], P::kTransformed ? into : P::mul(into, bp.mm[r])));
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
  }
  __pipeline_wait_prior(0);
}

// ---------------------------------------------------------------------------------------------
// Forward pass.
// ---------------------------------------------------------------------------------------------

// Loop-carried state of the forward sweep of one lane.
template <class P, int R>
struct FwdState {
  using V = typename P::V;
  using S = typename P::S;
  V M[R], X[R], Y[R];
  V acc;
  int seg_i;
  // The next segment's record, loaded a segment ahead so a BEGIN never waits on memory.
  int nx_staged, nx_slot;
  S nx_init;
  // Strip-mined reads: the row above lane 0's top row for this step's column (the previous block's
  // bottom row, or GATK's row 0 in the first block). Read only by forward_step<..., kCarry = true>.
  V cM, cX, cY;

  __device__ void load_next(const BatchView& v, const Program& prog, int seg) {
    if (seg < prog.n_segs) {
      const Segment* rec = v.segs + prog.seg_off + seg;
      nx_staged = rec->staged;
      nx_slot = rec->next_slot;
      nx_init = P::kDouble ? static_cast<S>(rec->init_d) : static_cast<S>(rec->init_f);
    } else {
      nx_staged = 0;
      nx_slot = -1;
      nx_init = S(0);
    }
  }
};

// One forward step: events, then the column. (uM, uX, uY) receive the bottom row of the lane above
// for this column; (dM, dX, dY) hold it for the previous column, the top row's diagonal. The two sets
// alternate between consecutive steps, so no copies are needed. kEv = false compiles the event code
// out, for steps where no lane of the warp has an event. kCarry = true gives lane 0 the row above
// from the state's carry values instead of its own bottom row (strip-mined reads).
template <class P, int R, bool kEv = true, bool kCarry = false>
__device__ __forceinline__ void forward_step(const LaunchArgs& a, const Program& prog, const ReadRef* rd, int lane,
                                             const FwdRows<P, R>& fr, const typename P::V& an, int pad_hi, Scratch<P, R>& sc,
                                             FwdState<P, R>& st, int synth_len, uint32_t ev, typename P::V& uM, typename P::V& uX,
                                             typename P::V& uY, typename P::V& dM, typename P::V& dX, typename P::V& dY) {
  using V = typename P::V;
  using S = typename P::S;
  using L = Layout<P, R>;
  uM = P::up(st.M[R - 1]);
  uX = P::up(st.X[R - 1]);
  uY = P::up(st.Y[R - 1]);
  if (kCarry && lane == 0) {
    uM = st.cM;
    uX = st.cX;
    uY = st.cY;
  }
  // END and ACC act in lane 31 alone (the read's last row); the other lanes pass them by without
  // entering the event code, which every lane otherwise reaches at its own step.
  if (kEv && (ev & (lane == 31 ? kEvMask : (kEvMask & ~(EV_END | EV_ACC))))) {
    if (ev & EV_SNAP) {
      const uint32_t slot = ev >> kPayloadShift;
      V* dst[2] = {slot != kPayloadNone ? sc.slot(static_cast<int>(slot), lane) : nullptr,
                   (ev & EV_STAGE) ? sc.staged(st.seg_i + 1, lane) : nullptr};
      V rec[L::kSnap];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        rec[r] = st.M[r];
        rec[R + r] = st.X[r];
        rec[2 * R + r] = st.Y[r];
      }
      rec[3 * R] = dM;
      rec[3 * R + 1] = dX;
      rec[3 * R + 2] = dY;
      rec[3 * R + 3] = st.acc;
#pragma unroll
      for (int i = 3 * R + 4; i < L::kSnap; ++i) rec[i] = P::zero();
#pragma unroll
      for (int k = 0; k < 2; ++k)
        if (dst[k]) store_record(dst[k], rec);
    }
    if ((ev & EV_END) && lane == 31) {
#pragma unroll
      for (int c = 0; c < P::NC; ++c) sc.seg_raw[st.seg_i * P::NC + c] = static_cast<double>(P::get(st.acc, c));
    }
    if (ev & EV_JOIN) {
      // The cut column's match and deletion rows, joined with the backward node after the sweep
      // (fgkl kernel.rs:744-755).
      V rec[L::kJoin];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        rec[r] = st.M[r];
        rec[R + r] = st.Y[r];
      }
#pragma unroll
      for (int i = 2 * R; i < L::kJoin; ++i) rec[i] = P::zero();
      store_record(sc.join(st.seg_i, lane), rec);
    }
    if (ev & EV_BEGIN) {
      ++st.seg_i;
      // A recomputation stream (FP64 only) has one unshared segment from the origin and no record.
      const bool synth = synth_len > 0;
      const int next_slot = synth ? -1 : st.nx_slot;
      const bool staged = !synth && st.nx_staged;
      const S init = st.nx_init;
      if (!synth) st.load_next(a.v, prog, st.seg_i + 1);
      if (staged) {
        __pipeline_wait_prior(0);
        V s[L::kSnap];
        load_record(s, sc.staged(st.seg_i, lane));
#pragma unroll
        for (int r = 0; r < R; ++r) {
          st.M[r] = s[r];
          st.X[r] = s[R + r];
          st.Y[r] = s[2 * R + r];
        }
        dM = s[3 * R];
        dX = s[3 * R + 1];
        dY = s[3 * R + 2];
        st.acc = s[3 * R + 3];
      } else {
        // The origin: nothing but the row-0 constant, in the padding rows (and the row above the
        // lane when that is padding).
        const S in_s = synth ? static_cast<S>(Consts<P::kDouble>::kInitial / synth_len) : init;
#pragma unroll
        for (int r = 0; r < R; ++r) st.M[r] = st.X[r] = st.Y[r] = P::zero();
        dM = dX = dY = st.acc = P::zero();
        if (lane * R <= pad_hi) {
#pragma unroll
          for (int c = 0; c < P::NC; ++c) {
#pragma unroll
            for (int r = 0; r < R; ++r)
              if (lane * R + r < rd[c].pad) P::put(st.Y[r], c, in_s);
            if (lane * R - 1 < rd[c].pad) P::put(dY, c, in_s);
          }
        }
      }
      if (next_slot >= 0) prefetch(sc.staged(st.seg_i + 1, lane), sc.slot(next_slot, lane), L::kSnap);
    }
    if ((ev & EV_ACC) && lane == 31) {
#pragma unroll
      for (int c = 0; c < P::NC; ++c) sc.seg_raw[st.seg_i * P::NC + c] = static_cast<double>(P::get(st.acc, c));
    }
  }
  const int code = ev & kCodeMask;
  const bool isN = code == kCodeN;
  V pri[L::kRp];
  if (L::kPriorCodes) load_priors<P, R>(fr.table, code, lane, pri);
  // Match and deletion values from the bottom row up: each row reads the old values of the row above
  // (its diagonal) and its own old values (left), so everything updates in place.
#pragma unroll
  for (int r = R - 1; r >= 0; --r) {
    const V pM = r ? st.M[r - 1] : dM, pX = r ? st.X[r - 1] : dX, pY = r ? st.Y[r - 1] : dY;
    const V prior = L::kPriorCodes ? pri[r] : fr.prior(code, isN, r, lane);
    st.Y[r] = P::kTransformed ? P::fma(st.Y[r], fr.c4[r], st.M[r]) : P::fma(st.Y[r], fr.c3[r], P::mul(st.M[r], fr.c4[r]));
    st.M[r] = P::mul(prior, cell_match<P>(pM, pX, pY, fr.c0[r], fr.c1[r], fr.c2[r]));
  }
  // Insertion values from the top row down: each row reads the new values of the row above.
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const V qM = r ? st.M[r - 1] : uM, qX = r ? st.X[r - 1] : uX;
    st.X[r] = P::kTransformed ? P::fma(qX, fr.c3[r], qM) : P::fma(qX, fr.c3[r], P::mul(qM, fr.c2[r]));
  }
  st.acc = P::fma(st.X[R - 1], an, P::add(st.acc, st.M[R - 1]));
}

// Entry p of a recomputation stream: the haplotype's codes, BEGIN on the first column and END after
// the last.
__device__ __forceinline__ uint32_t synth_entry(const uint8_t* seq, int len, int p) {
  if (p < 0 || p > len) return 0u;
  uint32_t e = p < len ? __ldg(seq + p) : 0u;
  if (p == 0) e |= EV_BEGIN;
  if (p == len) e |= EV_END;
  return e;
}

template <class P, int R>
__device__ void forward_pass(const LaunchArgs& a, const Program& prog, const ReadRef* rd, const uint8_t* codes, int lane,
                             Scratch<P, R>& sc, const uint8_t* synth_seq, int synth_len) {
  using V = typename P::V;
  using S = typename P::S;
  FwdRows<P, R> fr;
  fr.load(a.v, rd, lane, codes, sc.priors);
  // X factor of the read's last row (lane 31): the accumulated result is Σ M + mi_n * X^.
  V an;
#pragma unroll
  for (int c = 0; c < P::NC; ++c)
    P::put(an, c, static_cast<S>((P::kTransformed && rd[c].len > 0) ? err_prob(a.v, a.v.ins[rd[c].off + rd[c].len - 1]) : 1.0));
  int pad_hi = 0;
#pragma unroll
  for (int c = 0; c < P::NC; ++c) pad_hi = rd[c].pad > pad_hi ? rd[c].pad : pad_hi;

  FwdState<P, R> st;
#pragma unroll
  for (int r = 0; r < R; ++r) st.M[r] = st.X[r] = st.Y[r] = P::zero();
  st.acc = P::zero();
  st.seg_i = -1;
  st.load_next(a.v, prog, synth_len > 0 ? prog.n_segs : 0);
  V aM = P::zero(), aX = P::zero(), aY = P::zero(), bM = P::zero(), bX = P::zero(), bY = P::zero();
  if (P::kDouble && synth_len > 0) {
    const int n = synth_len;
    for (int t = 0; t < n + 32; t += 2) {
      const uint32_t e0 = synth_entry(synth_seq, n, t - lane), e1 = synth_entry(synth_seq, n, t + 1 - lane);
      forward_step<P, R>(a, prog, rd, lane, fr, an, pad_hi, sc, st, synth_len, e0, aM, aX, aY, bM, bX, bY);
      forward_step<P, R>(a, prog, rd, lane, fr, an, pad_hi, sc, st, synth_len, e1, bM, bX, bY, aM, aX, aY);
    }
  } else {
    const int n = prog.fwd_len;
    const uint32_t* stream = a.v.stream + prog.fwd_off - lane;
    // Four steps an iteration, their stream entries loaded one iteration ahead (the stream carries
    // kStreamPad zero entries past its end, so the last iteration's look-ahead and the up to three
    // steps past n + 31 read no events). An iteration where no lane has an event -- about four in
    // five, as each event column reaches the lanes over 32 steps -- runs a body without event code,
    // which the compiler schedules across the four steps.
    const uint32_t keep = lane == 31 ? kEvMask : (kEvMask & ~(EV_END | EV_ACC));
    uint32_t n0 = __ldg(stream), n1 = __ldg(stream + 1), n2 = __ldg(stream + 2), n3 = __ldg(stream + 3);
    for (int t = 0; t < n + 32; t += 4) {
      const uint32_t e0 = n0, e1 = n1, e2 = n2, e3 = n3;
      n0 = __ldg(stream + t + 4);
      n1 = __ldg(stream + t + 5);
      n2 = __ldg(stream + t + 6);
      n3 = __ldg(stream + t + 7);
      if (__any_sync(kFull, (e0 | e1 | e2 | e3) & keep)) {
        forward_step<P, R>(a, prog, rd, lane, fr, an, pad_hi, sc, st, 0, e0, aM, aX, aY, bM, bX, bY);
        forward_step<P, R>(a, prog, rd, lane, fr, an, pad_hi, sc, st, 0, e1, bM, bX, bY, aM, aX, aY);
        forward_step<P, R>(a, prog, rd, lane, fr, an, pad_hi, sc, st, 0, e2, aM, aX, aY, bM, bX, bY);
        forward_step<P, R>(a, prog, rd, lane, fr, an, pad_hi, sc, st, 0, e3, bM, bX, bY, aM, aX, aY);
      } else {
        forward_step<P, R, false>(a, prog, rd, lane, fr, an, pad_hi, sc, st, 0, e0, aM, aX, aY, bM, bX, bY);
        forward_step<P, R, false>(a, prog, rd, lane, fr, an, pad_hi, sc, st, 0, e1, bM, bX, bY, aM, aX, aY);
        forward_step<P, R, false>(a, prog, rd, lane, fr, an, pad_hi, sc, st, 0, e2, aM, aX, aY, bM, bX, bY);
        forward_step<P, R, false>(a, prog, rd, lane, fr, an, pad_hi, sc, st, 0, e3, bM, bX, bY, aM, aX, aY);
      }
    }
  }
  __pipeline_wait_prior(0);
}

// ---------------------------------------------------------------------------------------------
// Finalisation: joins, thresholds, log10, and the caller's layout.
// ---------------------------------------------------------------------------------------------

template <class P, int R>
__device__ void finalize(const LaunchArgs& a, const Task& task, const Region& region, const Program& prog, const ReadRef* rd,
                         int lane, Scratch<P, R>& sc) {
  using C = Consts<P::kDouble>;
  double* red = reinterpret_cast<double*>(sc.stage);  // [c][row q], the staging buffers are free now
  const int max_rows = 32 * R;
  const int n_join_segs = (P::kDouble && task.hap >= 0) ? 0 : prog.n_segs;
  // Joins (fgkl kernel.rs:767-791): raw = acc + (Σ_rows F_M*B_M + F_Y*B_Y + init*s) / BACKWARD_SCALE,
  // with the row sum taken in an order fixed by the read row so it does not depend on R.
  for (int seg = 0; seg < n_join_segs; ++seg) {
    const int node = a.v.segs[prog.seg_off + seg].node;
    if (node < 0) continue;
    const typename P::V* f = sc.join(seg, lane);
    const typename P::V* b = sc.node(node, lane);
    double row0[P::NC];
#pragma unroll
    for (int c = 0; c < P::NC; ++c) row0[c] = 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const typename P::V fM = f[r], fY = f[R + r], bM = b[r], bY = b[R + r];
#pragma unroll
      for (int c = 0; c < P::NC; ++c) {
        const int q = lane * R + r - rd[c].pad;
        double yfac = 1.0;
        if (P::kTransformed && rd[c].len > 0 && q >= 0) yfac = err_prob(a.v, a.v.del[rd[c].off + q]);
        const double fy = __dmul_rn(yfac, static_cast<double>(P::get(fY, c)));
        const double prod = __dadd_rn(__dmul_rn(static_cast<double>(P::get(fM, c)), static_cast<double>(P::get(bM, c))),
                                      __dmul_rn(fy, static_cast<double>(P::get(bY, c))));
        if (q >= 0) red[c * max_rows + q] = prod;
        if (q == -1) row0[c] = prod;
      }
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < P::NC; ++c) {
      double s = 0.0;
      for (int q = lane; q < rd[c].len; q += 32) s = __dadd_rn(s, red[c * max_rows + q]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s = __dadd_rn(s, __shfl_xor_sync(kFull, s, o));
      // Row 0's start mass lives in one lane.
      const double r0 = __shfl_sync(kFull, row0[c], (rd[c].pad - 1) / R);
      if (lane == 0 && task.read[c] >= 0) {
        double* raw = sc.seg_raw + seg * P::NC + c;
        *raw = __dadd_rn(*raw, __ddiv_rn(__dadd_rn(s, r0), C::kBackwardScale));
      }
    }
    __syncwarp();
  }
  __syncwarp();
  if (P::kDouble && task.hap >= 0) {
    // A recomputation task: its one segment's result goes to the haplotype and its duplicates.
    const double raw = sc.seg_raw[0];
    const bool lost = raw != raw;
    const double result = lost ? __longlong_as_double(0x7ff8000000000000ll) : log10(raw) - C::kLog10Initial;
    const int read_local = task.read[0] - region.read_off;
    for (int k = lane; k < region.n_haps; k += 32) {
      const HapInfo info = a.v.haps[region.hap_off + k];
      if (info.src == task.hap) a.v.out[region.out_off + static_cast<int64_t>(read_local) * region.n_haps + info.order] = result;
    }
    return;
  }
  // A dense read's recomputation (only_lost) fills in only the pairs the first pass lost and counts
  // nothing: the pairs it loses again stay NaN for the unshared sweep that follows it.
  const bool dense = a.only_lost != 0;
  unsigned long long lost_count = 0;
  for (int k = lane; k < region.n_haps; k += 32) {
    const HapInfo info = a.v.haps[region.hap_off + k];
    const Segment* seg = a.v.segs + prog.seg_off + info.seg;
    const bool joined = seg->node >= 0;
    const double factor = seg->factor;
#pragma unroll
    for (int c = 0; c < P::NC; ++c) {
      if (task.read[c] < 0) continue;
      const int read_local = task.read[c] - region.read_off;
      double* dst = a.v.out + region.out_off + static_cast<int64_t>(read_local) * region.n_haps + info.order;
      if (dense && !isnan(*dst)) continue;
      const double raw = __dmul_rn(sc.seg_raw[info.seg * P::NC + c], factor);
      bool lost;
      if (joined)
        lost = !(raw >= C::kMinAcceptedJoined);
      else
        lost = a.min_accept_plain ? !(raw >= C::kMinAccepted) : (raw != raw);
      if (!P::kDouble) lost |= isinf(raw);
      const double result = lost ? __longlong_as_double(0x7ff8000000000000ll) : log10(raw) - C::kLog10Initial;
      *dst = result;
      lost_count += lost;
    }
  }
  if (lost_count && !dense) atomicAdd(&a.v.counters->lost_pairs, lost_count);
}

template <class P, int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, (MinBlocks<P, R>::value)) pairhmm_kernel(LaunchArgs a) {
  using V = typename P::V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int warp_in_block = threadIdx.x >> 5;
  const int warp = blockIdx.x * static_cast<int>(blockDim.x >> 5) + warp_in_block;
  V* smem = reinterpret_cast<V*>(smem_raw + warp_in_block * Layout<P, R>::kSmemPerWarp);
  const int count = a.count ? min(*a.count, a.n_tasks) : a.n_tasks;
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(a.task_counter, 1);
    t = __shfl_sync(kFull, t, 0);
    if (t >= count) break;
    const Task task = a.tasks[t];
    const Region region = a.v.regions[task.region];
    const Program prog = region.prog;
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
    char* scratch = a.scratch + static_cast<size_t>(warp) * a.scratch_stride;
    if (P::kDouble && task.hap >= 0) {
      const HapInfo info = a.v.haps[region.hap_off + task.hap];
      Scratch<P, R> sc(scratch, smem, 0, 0, 1);
      forward_pass<P, R>(a, prog, rd, codes, lane, sc, a.v.hap_codes + region.seq_off + info.seq, info.len);
      __syncwarp();
      finalize<P, R>(a, task, region, prog, rd, lane, sc);
    } else {
      Scratch<P, R> sc(scratch, smem, prog.n_slots, prog.n_nodes, prog.n_segs);
      if (prog.bwd_len > 0) backward_pass<P, R>(a, prog, rd, codes, lane, sc);
      __syncwarp();
      forward_pass<P, R>(a, prog, rd, codes, lane, sc, nullptr, 0);
      __syncwarp();
      finalize<P, R>(a, task, region, prog, rd, lane, sc);
      if (P::kDouble && a.only_lost) {
        // A dense read's shared FP64 sweep can lose a pair again (a joined result below the backward
        // range): each such distinct haplotype is swept once more here without sharing, which
        // cannot lose it (fgkl lib.rs:476-486).
        __syncwarp();
        const double* row = a.v.out + region.out_off + static_cast<int64_t>(task.read[0] - region.read_off) * region.n_haps;
        for (int base = 0; base < region.n_haps; base += 32) {
          const int k = base + lane;
          bool again = false;
          if (k < region.n_haps) {
            const HapInfo info = a.v.haps[region.hap_off + k];
            again = info.src == k && isnan(row[info.order]);
          }
          unsigned mask = __ballot_sync(kFull, again);
          while (mask) {
            Task one = task;
            one.hap = base + __ffs(mask) - 1;
            mask &= mask - 1;
            const HapInfo info = a.v.haps[region.hap_off + one.hap];
            Scratch<P, R> s1(scratch, smem, 0, 0, 1);
            forward_pass<P, R>(a, prog, rd, codes, lane, s1, a.v.hap_codes + region.seq_off + info.seq, info.len);
            __syncwarp();
            finalize<P, R>(a, one, region, prog, rd, lane, s1);
            __syncwarp();
          }
        }
      }
    }
    __syncwarp();
  }
}

// Queues what the first pass lost for FP64 recomputation, in the queue bin of the read's form and
// rows-per-lane (queue_bin), one warp per read. After an FP32 pass, a read of a shared program lost
// against at least a third of its haplotypes (duplicates counted, fgkl lib.rs:495-505) is queued once,
// as a whole-program task that fills in every lost pair of the read with one shared sweep, when that
// sweep is the cheaper one; any other lost pair is queued as (read, distinct sorted haplotype), swept
// unshared. Both are FP64 sweeps of fgkl's recurrence and agree to rounding. One block per region;
// nothing to do (one load per block) when no pair was lost.
__global__ void __launch_bounds__(256) collect_kernel(CollectArgs a) {
  if (a.v.counters->lost_pairs == 0) return;
  const Region region = a.v.regions[blockIdx.x];
  const bool generic = (region.flags & kRegionGeneric) != 0;
  const int lane = threadIdx.x & 31;
  for (int r = threadIdx.x >> 5; r < region.n_reads; r += blockDim.x >> 5) {
    const double* row = a.v.out + region.out_off + static_cast<int64_t>(r) * region.n_haps;
    int lost_all = 0, lost_distinct = 0, lost_steps = 0;
    for (int k = lane; k < region.n_haps; k += 32) {
      const HapInfo info = a.v.haps[region.hap_off + k];
      const bool lost = isnan(row[info.order]);
      lost_all += lost;
      lost_distinct += lost && info.src == k;
      lost_steps += (lost && info.src == k) ? info.len + 32 : 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lost_all += __shfl_xor_sync(kFull, lost_all, o);
      lost_distinct += __shfl_xor_sync(kFull, lost_distinct, o);
      lost_steps += __shfl_xor_sync(kFull, lost_steps, o);
    }
    if (lost_all == 0) continue;
    const int read = region.read_off + r;
    const int len = static_cast<int>(a.v.read_off[read + 1] - a.v.read_off[read]);
    const int bin = queue_bin(len, generic);
    const int rows = queue_bin_rows(bin);
    const int cap = a.queue_off[bin + 1] - a.queue_off[bin];
    // The shared sweep must also cost at most two thirds of the unshared ones in wavefront steps:
    // a program that shares little (most PD regions) runs slower whole, in one warp, than its pairs
    // spread over many.
    const int prog_steps = region.prog.fwd_len + 32 + (region.prog.bwd_len > 0 ? region.prog.bwd_len + 32 : 0);
    if (a.dense && bin < kRowBins && 3 * lost_all >= region.n_haps && 3 * prog_steps <= 2 * lost_steps) {
      if (lane == 0) {
        const int slot = atomicAdd(a.queue_tail + bin, 1);
        if (slot < cap) {
          a.queue[a.queue_off[bin] + slot] = Task{static_cast<int32_t>(blockIdx.x), {read, -1}, rows, -1};
          atomicAdd(&a.v.counters->rescue_reads, static_cast<unsigned long long>(lost_distinct));
        }
      }
      continue;
    }
    for (int k = lane; k < region.n_haps; k += 32) {
      const HapInfo info = a.v.haps[region.hap_off + k];
      if (info.src != k || !isnan(row[info.order])) continue;
      const int slot = atomicAdd(a.queue_tail + bin, 1);
      if (slot < cap) {
        a.queue[a.queue_off[bin] + slot] = Task{static_cast<int32_t>(blockIdx.x), {read, -1}, rows, k};
        atomicAdd(&a.v.counters->rescue_reads, 1ull);
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Strip-mined reads (longer than 620 bases; fgkl sizes its row tables by the batch's longest read,
// kernel.rs:485-577, so any length is accepted): one read against one distinct haplotype, unshared,
// from a stream synthesised from the haplotype's codes (the recomputation form above), with the read's
// rows cut into B = ceil(len / 32R) blocks of 32R rows that the warp runs one after another. The
// padding rows sit at the top of the first block. Lane 0's row above comes from a carry row instead of
// its own bottom row: GATK's row 0 (M = X = 0, Y = INITIAL / hap_len) in the first block, the previous
// block's bottom row after that, which lane 31 writes to the warp's scratch column by column. Lane 0
// reads column j at step j, and lane 31 of the same block overwrites it at step j + 31 with a value
// computed from it through the wavefront, so one carry row serves every block in place.
// ---------------------------------------------------------------------------------------------

// A column of a block's bottom row: M, X, Y (the FP32 kernels' X/mi and Y/md), padded to 16 bytes.
constexpr int kCarryVals = 4;

template <class P>
__host__ __device__ constexpr size_t long_scratch_size(int max_hap_len) {
  return 16 + static_cast<size_t>(max_hap_len) * kCarryVals * sizeof(typename P::V);
}

template <class P, int R>
__device__ __forceinline__ void long_store(typename P::V* carry, const FwdState<P, R>& st, int lane, int t, int n, bool last) {
  const int p = t - 31;  // lane 31's position at step t
  if (!last && lane == 31 && p >= 0 && p < n) {
    typename P::V rec[kCarryVals] = {st.M[R - 1], st.X[R - 1], st.Y[R - 1], P::zero()};
    store_record(carry + static_cast<size_t>(p) * kCarryVals, rec);
  }
}

template <class P, int R>
__device__ __forceinline__ void long_fetch(const typename P::V* carry, typename P::V (&rec)[kCarryVals], int lane, int p, int n,
                                           bool first) {
  if (!first && lane == 0 && p < n) load_record(rec, carry + static_cast<size_t>(p) * kCarryVals);
}

// One block of a strip-mined pair: rd's pad is relative to the block (negative below the first).
template <class P, int R>
__device__ void long_block(const LaunchArgs& a, const ReadRef* rd, int lane, const FwdRows<P, R>& fr, typename P::V an,
                           Scratch<P, R>& sc, const uint8_t* seq, int n, typename P::V* carry, bool first, bool last) {
  using V = typename P::V;
  using S = typename P::S;
  const int pad_hi = rd[0].pad;
  FwdState<P, R> st;
#pragma unroll
  for (int r = 0; r < R; ++r) st.M[r] = st.X[r] = st.Y[r] = P::zero();
  st.acc = P::zero();
  st.seg_i = -1;
  st.nx_staged = 0;
  st.nx_slot = -1;
  st.nx_init = S(0);
  st.cM = st.cX = P::zero();
  st.cY = first ? static_cast<S>(Consts<P::kDouble>::kInitial / n) : P::zero();
  const Program prog{};  // unused: the stream is synthesised
  V aM = P::zero(), aX = P::zero(), aY = P::zero(), bM = P::zero(), bX = P::zero(), bY = P::zero();
  // Lane 0's carry values for the next iteration's two steps, loaded an iteration ahead.
  V n0[kCarryVals], n1[kCarryVals];
#pragma unroll
  for (int i = 0; i < kCarryVals; ++i) n0[i] = n1[i] = P::zero();
  long_fetch<P, R>(carry, n0, lane, 0, n, first);
  long_fetch<P, R>(carry, n1, lane, 1, n, first);
  for (int t = 0; t < n + 32; t += 2) {
    const uint32_t e0 = synth_entry(seq, n, t - lane), e1 = synth_entry(seq, n, t + 1 - lane);
    V c0[kCarryVals], c1[kCarryVals];
#pragma unroll
    for (int i = 0; i < kCarryVals; ++i) {
      c0[i] = n0[i];
      c1[i] = n1[i];
    }
    long_fetch<P, R>(carry, n0, lane, t + 2, n, first);
    long_fetch<P, R>(carry, n1, lane, t + 3, n, first);
    if (!first) {
      st.cM = c0[0];
      st.cX = c0[1];
      st.cY = c0[2];
    }
    forward_step<P, R, true, true>(a, prog, rd, lane, fr, an, pad_hi, sc, st, n, e0, aM, aX, aY, bM, bX, bY);
    long_store<P, R>(carry, st, lane, t, n, last);
    if (!first) {
      st.cM = c1[0];
      st.cX = c1[1];
      st.cY = c1[2];
    }
    forward_step<P, R, true, true>(a, prog, rd, lane, fr, an, pad_hi, sc, st, n, e1, bM, bX, bY, aM, aX, aY);
    long_store<P, R>(carry, st, lane, t + 1, n, last);
  }
}

template <class P, int R>
struct LongMinBlocks {
  static constexpr int value = P::kDouble ? 1 : 2;
};

template <class P, int R>
constexpr size_t long_smem_per_warp() {
  using L = Layout<P, R>;
  return static_cast<size_t>(L::kPriorCodes) * L::kRp * 32 * sizeof(typename P::V);
}

template <class P, int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, (LongMinBlocks<P, R>::value)) long_kernel(LaunchArgs a) {
  using V = typename P::V;
  using S = typename P::S;
  using C = Consts<P::kDouble>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int warp_in_block = threadIdx.x >> 5;
  const int warp = blockIdx.x * kWarpsPerBlock + warp_in_block;
  V* priors = reinterpret_cast<V*>(smem_raw + warp_in_block * long_smem_per_warp<P, R>());
  const int count = a.count ? min(*a.count, a.n_tasks) : a.n_tasks;
  char* scratch = a.scratch + static_cast<size_t>(warp) * a.scratch_stride;
  V* carry = reinterpret_cast<V*>(scratch + 16);
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(a.task_counter, 1);
    t = __shfl_sync(kFull, t, 0);
    if (t >= count) break;
    const Task task = a.tasks[t];
    const Region region = a.v.regions[task.region];
    const HapInfo info = a.v.haps[region.hap_off + task.hap];
    const uint8_t* seq = a.v.hap_codes + region.seq_off + info.seq;
    const int n = info.len;
    ReadRef rd[1];
    rd[0].off = a.v.read_off[task.read[0]];
    rd[0].len = static_cast<int>(a.v.read_off[task.read[0] + 1] - rd[0].off);
    const int blocks = long_blocks(rd[0].len, R);
    const int pad0 = 32 * R * blocks - rd[0].len;
    const uint8_t* codes = a.v.code_of_byte + region.code_off;
    Scratch<P, R> sc(scratch, priors, 0, 0, 0);
    sc.priors = priors;
    // X factor of the read's last row: the accumulated result is the sum of M + mi_n * X^.
    const V an = static_cast<S>(P::kTransformed ? err_prob(a.v, a.v.ins[rd[0].off + rd[0].len - 1]) : 1.0);
    for (int b = 0; b < blocks; ++b) {
      rd[0].pad = pad0 - 32 * R * b;
      FwdRows<P, R> fr;
      fr.load(a.v, rd, lane, codes, priors);
      __syncwarp();
      long_block<P, R>(a, rd, lane, fr, an, sc, seq, n, carry, b == 0, b == blocks - 1);
      __syncwarp();
    }
    // Thresholds of an unshared pair (fgkl kernel.rs:897-914): FP32 results below 1e-28 or not finite
    // go to the FP64 recomputation.
    const double raw = sc.seg_raw[0];
    bool lost = a.min_accept_plain ? !(raw >= C::kMinAccepted) : (raw != raw);
    if (!P::kDouble) lost |= isinf(raw);
    const double result = lost ? __longlong_as_double(0x7ff8000000000000ll) : log10(raw) - C::kLog10Initial;
    const int read_local = task.read[0] - region.read_off;
    unsigned long long lost_count = 0;
    for (int k = lane; k < region.n_haps; k += 32) {
      const HapInfo h = a.v.haps[region.hap_off + k];
      if (h.src != task.hap) continue;
      a.v.out[region.out_off + static_cast<int64_t>(read_local) * region.n_haps + h.order] = result;
      lost_count += lost;
    }
    if (lost_count) atomicAdd(&a.v.counters->lost_pairs, lost_count);
    __syncwarp();
  }
}

template <class P, int R>
void occ(int* blocks, int* threads, int warps) {
  *threads = warps * 32;
  static std::atomic<int> cache[3][kMaxDevices];
  *blocks = resident_blocks(pairhmm_kernel<P, R>, warps * Layout<P, R>::kSmemPerWarp, warps * 32, cache[warps_index(warps)],
                            kWarpsPerBlock * Layout<P, R>::kSmemPerWarp);
}

template <class P, int R>
cudaError_t go(int blocks, const LaunchArgs& a, cudaStream_t s, int warps) {
  const size_t smem = warps * Layout<P, R>::kSmemPerWarp;
  pairhmm_kernel<P, R><<<blocks, warps * 32, smem, s>>>(a);
  return cudaGetLastError();
}

template <class P, int R>
struct OccF {
  static int run(int* b, int* t, int warps) {
    occ<P, R>(b, t, warps);
    return 0;
  }
};
template <class P, int R>
struct GoF {
  static cudaError_t run(int blocks, const LaunchArgs& a, cudaStream_t s, int warps) { return go<P, R>(blocks, a, s, warps); }
};
template <class P, int R>
struct SizeF {
  static size_t run(int slots, int nodes, int segs) { return scratch_size<P, R>(slots, nodes, segs); }
};

// Rows-per-lane dispatch over the instantiated values of each kind: packed FP32 covers 1..8, single
// FP32 the long reads (10..20 rows, even), FP64 both.
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
        FGKL_CASE(OneF32, 18)
        FGKL_CASE(OneF32, 20)
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
        FGKL_CASE(OneF64, 18)
        FGKL_CASE(OneF64, 20)
        default:
          break;
      }
      break;
  }
#undef FGKL_CASE
  return Ret{};
}

bool valid_long_rows(Kind k, int rows) {
  const bool wide = k == Kind::kLongF32;
  for (int i = 0; i < long_rows_count(wide); ++i)
    if (long_rows_value(i, wide) == rows) return true;
  return false;
}

bool valid_rows(Kind k, int rows) {
  if (is_long(k)) return valid_long_rows(k, rows);
  switch (k) {
    case Kind::kPackedF32:
      return rows >= 1 && rows <= 8;
    case Kind::kOneF32:
      return rows >= 10 && rows <= 20 && rows % 2 == 0;
    case Kind::kOneF64:
    case Kind::kOneF32Pd:
    case Kind::kOneF64Pd:
      return (rows >= 1 && rows <= 8) || (rows >= 10 && rows <= 20 && rows % 2 == 0);
    case Kind::kPackedF32Pd:
      return rows >= 1 && rows <= 8;
    default:
      break;
  }
  return false;
}

// Strip-mined plain kinds over the rows-per-lane values of long_rows: 8..16 in FP32, 4..8 in FP64.
template <class F>
auto long_rows_narrow(int rows, F&& f) {
  switch (rows) {
    case 4: return f(std::integral_constant<int, 4>{});
    case 6: return f(std::integral_constant<int, 6>{});
    default: return f(std::integral_constant<int, 8>{});
  }
}
template <class F>
auto long_rows_wide(int rows, F&& f) {
  switch (rows) {
    case 8: return f(std::integral_constant<int, 8>{});
    case 10: return f(std::integral_constant<int, 10>{});
    case 12: return f(std::integral_constant<int, 12>{});
    default: return f(std::integral_constant<int, 16>{});
  }
}

template <class P, int R>
void long_occ(int* blocks) {
  static std::atomic<int> cache[kMaxDevices];
  *blocks = resident_blocks(long_kernel<P, R>, kWarpsPerBlock * long_smem_per_warp<P, R>(), kWarpsPerBlock * 32, cache);
}

template <class P, int R>
cudaError_t long_go(int blocks, const LaunchArgs& a, cudaStream_t s) {
  long_kernel<P, R><<<blocks, kWarpsPerBlock * 32, kWarpsPerBlock * long_smem_per_warp<P, R>(), s>>>(a);
  return cudaGetLastError();
}

}  // namespace

int max_rows(Kind) { return 20; }

size_t long_scratch_bytes(Kind k, int rows, int max_hap_len) {
  if (!is_long(k) || !valid_long_rows(k, rows)) return 0;
  if (is_pd(k)) return pd_long_scratch_bytes(k, rows, max_hap_len);
  return k == Kind::kLongF64 ? long_scratch_size<OneF64>(max_hap_len) : long_scratch_size<OneF32>(max_hap_len);
}

void long_occupancy(Kind k, int rows, int* blocks, int* threads) {
  *blocks = 0;
  *threads = kWarpsPerBlock * 32;
  if (!is_long(k) || !valid_long_rows(k, rows)) return;
  if (is_pd(k)) return pd_long_occupancy(k, rows, blocks, threads);
  if (k == Kind::kLongF64)
    long_rows_narrow(rows, [&](auto r) {
      long_occ<OneF64, decltype(r)::value>(blocks);
      return 0;
    });
  else
    long_rows_wide(rows, [&](auto r) {
      long_occ<OneF32, decltype(r)::value>(blocks);
      return 0;
    });
}

cudaError_t long_launch(Kind k, int rows, int blocks, const LaunchArgs& args, cudaStream_t stream) {
  if (!is_long(k) || !valid_long_rows(k, rows)) return cudaErrorInvalidValue;
  if (is_pd(k)) return pd_long_launch(k, rows, blocks, args, stream);
  if (k == Kind::kLongF64)
    return long_rows_narrow(rows, [&](auto r) { return long_go<OneF64, decltype(r)::value>(blocks, args, stream); });
  return long_rows_wide(rows, [&](auto r) { return long_go<OneF32, decltype(r)::value>(blocks, args, stream); });
}

size_t scratch_bytes(Kind k, int rows, int max_slots, int max_nodes, int max_segs) {
  if (is_long(k) || !valid_rows(k, rows)) return 0;
  if (is_pd(k)) return pd_scratch_bytes(pd_form(k), rows, max_slots, max_segs);
  return dispatch<SizeF>(k, rows, max_slots, max_nodes, max_segs);
}

void occupancy(Kind k, int rows, int* blocks, int* threads, int warps) {
  *blocks = 0;
  *threads = kWarpsPerBlock * 32;
  if (!valid_rows(k, rows) || (warps != 1 && warps != 2 && warps != 4)) return;
  if (is_long(k)) return long_occupancy(k, rows, blocks, threads);
  if (is_pd(k)) return pd_occupancy(pd_form(k), rows, blocks, threads, warps);
  dispatch<OccF>(k, rows, blocks, threads, warps);
}

cudaError_t launch_collect(const CollectArgs& args, int n_regions, cudaStream_t stream) {
  if (n_regions <= 0) return cudaSuccess;
  collect_kernel<<<n_regions, 256, 0, stream>>>(args);
  return cudaGetLastError();
}

cudaError_t launch(Kind k, int rows, int blocks, const LaunchArgs& args, cudaStream_t stream, int warps) {
  if (!valid_rows(k, rows) || (warps != 1 && warps != 2 && warps != 4)) return cudaErrorInvalidValue;
  if (is_long(k)) return long_launch(k, rows, blocks, args, stream);
  if (is_pd(k)) return pd_launch(pd_form(k), rows, blocks, args, stream, warps);
  return dispatch<GoF>(k, rows, blocks, args, stream, warps);
}

// ---------------------------------------------------------------------------------------------
// Allocation-free entry: one region's (read, haplotype) pairs from caller-owned device arrays, each
// pair computed by one warp in FP64 without sharing (the recomputation form of the kernel above),
// with the per-warp scratch -- the segment result the last lane hands to lane 0 -- in a file-scope
// device array instead of an allocated buffer.
// ---------------------------------------------------------------------------------------------

namespace {

constexpr size_t kNoAllocScratchBytes = size_t{2} << 20;  // 2 MiB (FGKL_NOALLOC_SCRATCH_BYTES): header + 8191 warps
constexpr size_t kNoAllocHeader = 256;                    // the 64-bit pair counter (must be 0 at launch)
constexpr size_t kNoAllocPerWarp = 256;                   // one warp's segment result, 256-aligned

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
static __device__ double g_noalloc_err[kMaxQualTable];
static __device__ double g_noalloc_m2m[kM2MTable];
static __device__ uint8_t g_noalloc_codes[256];

struct NoAllocArgs {
  BatchView v;  // read arrays and offsets, tables, read byte -> code table
  const uint8_t* hap_bases;
  const int64_t* hap_off;
  int n_reads, n_haps;
  unsigned long long* counter;  // pairs claimed so far (64-bit: every warp claims one past the last pair)
  char* scratch;  // kNoAllocPerWarp bytes per warp
  double* out;    // n_reads x n_haps, row-major
};

// Prior code of a haplotype byte: the byte itself, with 'N' and byte kCodeN swapped so that N is
// code kCodeN (matches every read base) and the mapping stays one-to-one. The read table holds the
// same permutation, so a read base matches exactly the haplotype bytes equal to it.
__device__ __forceinline__ uint32_t byte_code(uint32_t b) { return b == 'N' ? kCodeN : (b == kCodeN ? 'N' : b); }

__device__ __forceinline__ uint32_t byte_entry(const uint8_t* hap, int len, int p) {
  if (p < 0 || p > len) return 0u;
  uint32_t e = p < len ? byte_code(__ldg(hap + p)) : 0u;
  if (p == 0) e |= EV_BEGIN;
  if (p == len) e |= EV_END;
  return e;
}

template <int R>
__device__ void forward_unshared(const LaunchArgs& a, const ReadRef* rd, int lane, Scratch<OneF64, R>& sc, const uint8_t* hap,
                                 int n) {
  using P = OneF64;
  using V = typename P::V;
  FwdRows<P, R> fr;
  fr.load(a.v, rd, lane, a.v.code_of_byte, sc.priors);
  const V an = 1.0;  // the plain recurrence: the result is the sum of the last row's M and X
  const int pad_hi = rd[0].pad;
  FwdState<P, R> st;
#pragma unroll
  for (int r = 0; r < R; ++r) st.M[r] = st.X[r] = st.Y[r] = 0.0;
  st.acc = 0.0;
  st.seg_i = -1;
  st.nx_staged = 0;
  st.nx_slot = -1;
  st.nx_init = 0.0;
  const Program prog{};  // unused: the stream is synthesised from the haplotype bytes
  V aM = 0.0, aX = 0.0, aY = 0.0, bM = 0.0, bX = 0.0, bY = 0.0;
  for (int t = 0; t < n + 32; t += 2) {
    const uint32_t e0 = byte_entry(hap, n, t - lane), e1 = byte_entry(hap, n, t + 1 - lane);
    forward_step<P, R>(a, prog, rd, lane, fr, an, pad_hi, sc, st, n, e0, aM, aX, aY, bM, bX, bY);
    forward_step<P, R>(a, prog, rd, lane, fr, an, pad_hi, sc, st, n, e1, bM, bX, bY, aM, aX, aY);
  }
}

template <int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 1) noalloc_kernel(NoAllocArgs na) {
  using P = OneF64;
  extern __shared__ __align__(16) unsigned char smem_raw[];  // none requested: nothing is staged
  const int lane = threadIdx.x & 31;
  const int warp = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  LaunchArgs a{};
  a.v = na.v;
  const long long pairs = static_cast<long long>(na.n_reads) * na.n_haps;
  for (;;) {
    unsigned long long claimed = 0;
    if (lane == 0) claimed = atomicAdd(na.counter, 1ull);
    const long long t = static_cast<long long>(__shfl_sync(kFull, claimed, 0));
    if (t >= pairs) break;
    const int r = static_cast<int>(t / na.n_haps), h = static_cast<int>(t % na.n_haps);
    ReadRef rd[1];
    rd[0].off = na.v.read_off[r];
    const int64_t read_len = na.v.read_off[r + 1] - rd[0].off;
    const int64_t hap_lo = na.hap_off[h], hap_len = na.hap_off[h + 1] - hap_lo;
    if (read_len <= 0 || read_len > 31 * R || hap_len <= 0 || hap_len > (int64_t{1} << 30)) {
      // Lengths the call's bounds exclude: the pair has no result.
      if (lane == 0) na.out[t] = __longlong_as_double(0x7ff8000000000000ll);
      continue;
    }
    rd[0].len = static_cast<int>(read_len);
    rd[0].pad = 32 * R - rd[0].len;
    Scratch<P, R> sc(na.scratch + static_cast<size_t>(warp) * kNoAllocPerWarp, reinterpret_cast<double*>(smem_raw), 0, 0, 0);
    forward_unshared<R>(a, rd, lane, sc, na.hap_bases + hap_lo, static_cast<int>(hap_len));
    __syncwarp();
    if (lane == 0) na.out[t] = log10(sc.seg_raw[0]) - Consts<true>::kLog10Initial;
    __syncwarp();
  }
}

template <int R>
cudaError_t noalloc_go(int blocks, const NoAllocArgs& na, cudaStream_t s) {
  noalloc_kernel<R><<<blocks, kWarpsPerBlock * 32, 0, s>>>(na);
  return cudaGetLastError();
}

template <int R>
int noalloc_occupancy() {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, noalloc_kernel<R>, kWarpsPerBlock * 32, 0) != cudaSuccess) return 0;
  return b;
}

template <class F>
auto noalloc_dispatch(int rows, F&& f) {
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

int noalloc_rows(int max_read_len) {
  int rows = (max_read_len + 30) / 31;
  if (rows > 8) rows = (rows + 1) & ~1;
  return rows;
}

cudaError_t noalloc_scratch_address(char** scratch) {
  return cudaGetSymbolAddress(reinterpret_cast<void**>(scratch), g_noalloc_scratch);
}

cudaError_t noalloc_setup(NoAllocDevice* d, const double* err, size_t n_err, const double* m2m, size_t n_m2m,
                          const uint8_t codes[256]) {
  cudaError_t e;
  if (n_err != kMaxQualTable || n_m2m != kM2MTable) return cudaErrorInvalidValue;
  if ((e = cudaGetSymbolAddress(reinterpret_cast<void**>(&d->scratch), g_noalloc_scratch)) != cudaSuccess) return e;
  if ((e = cudaGetSymbolAddress(reinterpret_cast<void**>(&d->err), g_noalloc_err)) != cudaSuccess) return e;
  if ((e = cudaGetSymbolAddress(reinterpret_cast<void**>(&d->m2m), g_noalloc_m2m)) != cudaSuccess) return e;
  if ((e = cudaGetSymbolAddress(reinterpret_cast<void**>(&d->codes), g_noalloc_codes)) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(g_noalloc_err, err, n_err * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(g_noalloc_m2m, m2m, n_m2m * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(g_noalloc_codes, codes, 256)) != cudaSuccess) return e;
  for (int rows = 1; rows <= 20; ++rows) {
    if (rows > 8 && rows % 2) continue;
    d->blocks_per_sm[rows] = noalloc_dispatch(rows, [](auto r) { return noalloc_occupancy<decltype(r)::value>(); });
    if (d->blocks_per_sm[rows] <= 0) return cudaErrorInvalidDeviceFunction;
  }
  d->scratch_bytes = kNoAllocScratchBytes;
  d->header_bytes = kNoAllocHeader;
  d->per_warp_bytes = kNoAllocPerWarp;
  return cudaSuccess;
}

cudaError_t noalloc_launch(const NoAllocDevice& d, const NoAllocCall& c, int rows, int blocks, cudaStream_t stream) {
  NoAllocArgs na{};
  na.v.bases = c.bases;
  na.v.quals = c.quals;
  na.v.ins = c.ins;
  na.v.del = c.del;
  na.v.gcp = c.gcp;
  na.v.read_off = c.read_off;
  na.v.code_of_byte = d.codes;
  na.v.err_prob = d.err;
  na.v.m2m = d.m2m;
  na.hap_bases = c.hap_bases;
  na.hap_off = c.hap_off;
  na.n_reads = c.n_reads;
  na.n_haps = c.n_haps;
  na.counter = reinterpret_cast<unsigned long long*>(d.scratch);
  na.scratch = d.scratch + d.header_bytes;
  na.out = c.out;
  cudaError_t e = cudaMemsetAsync(d.scratch, 0, sizeof(unsigned long long), stream);  // the pair counter starts at zero
  if (e != cudaSuccess) return e;
  return noalloc_dispatch(rows, [&](auto r) { return noalloc_go<decltype(r)::value>(blocks, na, stream); });
}

}  // namespace fgkl
