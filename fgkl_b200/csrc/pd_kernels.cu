// sm_100a PD-HMM kernels (GATK LoglessPDPairHMM for DRAGEN concordance mode; fgkl pd_kernel.rs and
// pd_reference.rs:29-118): the plain kernels' warp wavefront over a prefix-shared column stream,
// with GATK's branch matrices.
//
// Per cell (row i, column j in deletion state s; left = (i, j-1), up = (i-1, j), diag = (i-1, j-1);
// B = branch values, V = (M, X, Y)):
//   B(i,j) = V(left)                 s = NORMAL
//          = B(left)                 s = INSIDE_DEL
//          = max(B(left), V(left))   s = AFTER_DEL
//   M = prior * (mm*D.M + im*(D.X + D.Y)),  D = max(B(diag), V(diag)) after a deletion, else V(diag)
//   Y = md*W.M + dd*W.Y,                    W = max(B(left), V(left)) after a deletion, else V(left)
//   X = mi*U.M + ii*U.X,                    U = max(B(up), V(up)) on a DEL_END column, else V(up)
// The state of a column depends only on the flags and on the state the row started in: NORMAL for
// the read's first row, the state the previous row ended in for the others. The host resolves both
// per column into the stream entry (program.h), with the column's prior code (a match set: its base
// and, on a SNP column, the flagged alternates).
//
// A column right after DEL_END is AFTER_DEL in every row (the state machine sets it from the
// DEL_END flag alone), and there the diagonal and the left cell enter only as max(B, V). So a lane
// takes that max once, at the DEL_END column itself: after computing the column, each row's M, X
// and Y become max(B, V) (row by row down the insertion sweep, so the next row's X reads U =
// max(B(up), V(up)) as GATK's DEL_END rule asks, and the last row after the result has taken its
// unmerged values). Every later reader of those values is a max reader, and the max is idempotent,
// so the AFTER_DEL column itself needs no branch values at all. Branch values are then only the
// lane's own rows: set to V(left) on a column carrying DEL_START or DEL_END (held inside a
// deletion), read on DEL_END columns, stale elsewhere where nothing reads them; the lane above's
// never cross. Columns carrying neither flag (the vast majority) run the plain recurrence.
//
// Priors. A PD region maps its reads' distinct bytes to classes 0..30; each match-set code carries
// the bit set of classes it accepts, so a row's prior is pm or px by one bit test.
//
// FP32 kernels carry X/mi and Y/md per row like the plain kernels; max() commutes with the positive
// per-row scale, so the branch values are kept in the same scale.
#include "dp_common.cuh"
#include "kernels.cuh"

namespace fgkl {

namespace {

template <class P, int R>
struct PdLayout {
  using V = typename P::V;
  static constexpr int kRound = 16 / static_cast<int>(sizeof(V)) > 1 ? 16 / static_cast<int>(sizeof(V)) : 1;
  static constexpr int up(int x) { return (x + kRound - 1) / kRound * kRound; }
  // M, X, Y rows; branch M, X, Y rows; above-row M, X, Y; accumulated result.
  static constexpr int kSnap = up(6 * R + 4);
  static constexpr size_t kStageBytes = 32ull * kSnap * sizeof(V);
  static constexpr size_t kSmemPerWarp = kStageBytes;
};

template <class P, int R>
struct PdScratch {
  using V = typename P::V;
  using L = PdLayout<P, R>;
  V* slots;         // [slot][lane][kSnap]
  double* seg_raw;  // [seg][c]
  V* stage;         // shared: [buf][lane][kSnap]

  __device__ PdScratch(char* base, V* smem, int n_slots) {
    slots = reinterpret_cast<V*>(base);
    seg_raw = reinterpret_cast<double*>(slots + static_cast<size_t>(n_slots) * 32 * L::kSnap);
    stage = smem;
  }
  __device__ V* slot(int s, int lane) { return slots + (static_cast<size_t>(s) * 32 + lane) * L::kSnap; }
  // One staging record per lane serves every segment: a lane writes or prefetches the next
  // segment's start into it only after loading the current one at its BEGIN.
  __device__ V* staged(int, int lane) { return stage + static_cast<size_t>(lane) * L::kSnap; }
};

template <class P, int R>
constexpr size_t pd_scratch_size(int n_slots, int n_segs) {
  return static_cast<size_t>(n_slots) * 32 * PdLayout<P, R>::kSnap * sizeof(typename P::V) +
         static_cast<size_t>(n_segs) * P::NC * sizeof(double);
}

// Forward coefficients of the lane's rows (the plain kernels' FwdRows) and each row's read class.
template <class P, int R>
struct PdRows {
  using V = typename P::V;
  using S = typename P::S;
  V c0[R], c1[R], c2[R], c3[R], c4[R], pm[R], px[R];
  uint32_t cls[P::NC][R];  // bit of the row's read class; 0 for a padding row (no code accepts it)

  __device__ V prior(uint32_t sig, int r) const {
    return P::sel((sig & cls[0][r]) != 0u, (sig & cls[P::NC - 1][r]) != 0u, pm[r], px[r]);
  }

  // Regions whose reads hold more distinct bytes than the class bits cover compare bytes instead:
  // after load_generic, cls holds the row's read byte (bits 0-7), whether it is N (bit 8) and the ALT
  // bit it answers to (bits 9-12), and a stream entry carries the column's haplotype byte (bits 0-7)
  // and its ALT bits (kPdPayloadShift up), so the column accepts the row's base exactly when
  // MatchSet::accepts would (fgkl pd_kernel.rs:196-214).
  __device__ V prior_generic(uint32_t ev, int r) const {
    const uint32_t base = ev & kCodeMask, alts = (ev >> kPdPayloadShift) & 0xFu, c = cls[0][r];
    const bool match = c != 0u && (((c & 0xFFu) == base) || base == 'N' || ((c >> 8) & 1u) || (((c >> 9) & alts) != 0u));
    return match ? pm[r] : px[r];
  }

  __device__ void load(const BatchView& v, const ReadRef* rd, int lane, const uint8_t* classes) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
      for (int c = 0; c < P::NC; ++c) {
        const RowModel m = row_model(v, rd[c], lane * R + r - rd[c].pad, classes);
        double k0, k1, k2, k3, k4;
        if (P::kTransformed) {
          // The match-to-match factor moves into the priors (cell_match).
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
        const double fold = (P::kTransformed && m.read) ? m.mm : 1.0;
        P::put(c0[r], c, static_cast<S>(k0));
        P::put(c1[r], c, static_cast<S>(k1));
        P::put(c2[r], c, static_cast<S>(k2));
        P::put(c3[r], c, static_cast<S>(k3));
        P::put(c4[r], c, static_cast<S>(k4));
        P::put(pm[r], c, static_cast<S>(m.pm * fold));
        P::put(px[r], c, static_cast<S>(m.px * fold));
        cls[c][r] = m.read ? (1u << (m.oc & 31)) : 0u;
      }
    }
  }

  // As load, with the byte-comparison row descriptors of prior_generic in cls (one read).
  __device__ void load_generic(const BatchView& v, const ReadRef* rd, int lane, const uint8_t* classes) {
    load(v, rd, lane, classes);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int q = lane * R + r - rd[0].pad;
      uint32_t d = 0;
      if (rd[0].len > 0 && q >= 0 && q < rd[0].len) {
        const uint32_t b = v.bases[rd[0].off + q];
        const uint32_t alt = (b == 'A' || b == 'a') ? 1u : (b == 'C' || b == 'c') ? 2u : (b == 'G' || b == 'g') ? 4u : (b == 'T' || b == 't') ? 8u : 0u;
        d = b | (b == 'N' ? 1u << 8 : 0u) | (alt << 9) | (1u << 13);  // bit 13: a read row (never 0)
      }
      cls[0][r] = d;
    }
  }
};

template <class P, int R>
struct PdState {
  using V = typename P::V;
  V M[R], X[R], Y[R];
  V BM[R], BX[R], BY[R];
  V acc;
  int seg_i;
  // Strip-mined reads: the row above lane 0's top row for this step's column (read only by
  // pd_step<..., kCarry = true>).
  V cM, cX, cY;
};

// The lane above's bottom row.
template <class P>
struct PdEdge {
  using V = typename P::V;
  V M, X, Y;
};

// One PD forward step: events, then the column. `u` receives the lane above's bottom row for this
// column, `d` holds it for the previous column (the top row's diagonal); the two alternate. kEv = false
// compiles the event code out, for steps where no lane of the warp has an event. kCarry = true gives
// lane 0 the row above from the state's carry values (strip-mined reads); kGeneric = true decides
// priors by comparing bytes (PdRows::prior_generic) instead of by class bits.
template <class P, int R, bool kEv = true, bool kCarry = false, bool kGeneric = false>
__device__ __forceinline__ void pd_step(const LaunchArgs& a, const Program& prog, const ReadRef* rd, int lane,
                                        const PdRows<P, R>& pr, const typename P::V& an, int pad_hi, PdScratch<P, R>& sc,
                                        PdState<P, R>& st, int synth_len, uint32_t ev, uint32_t sig, PdEdge<P>& u,
                                        PdEdge<P>& d) {
  using V = typename P::V;
  using S = typename P::S;
  using L = PdLayout<P, R>;
  u.M = P::up(st.M[R - 1]);
  u.X = P::up(st.X[R - 1]);
  u.Y = P::up(st.Y[R - 1]);
  if (kCarry && lane == 0) {
    u.M = st.cM;
    u.X = st.cX;
    u.Y = st.cY;
  }
  // END and ACC act in lane 31 alone (the read's last row); the other lanes pass them by without
  // entering the event code, which every lane otherwise reaches at its own step.
  if (kEv && (ev & (lane == 31 ? kEvMask : (kEvMask & ~(EV_END | EV_ACC))))) {
    if (ev & EV_SNAP) {
      const uint32_t slot = ev >> kPdPayloadShift;
      V* dst[2] = {slot != kPdPayloadNone ? sc.slot(static_cast<int>(slot), lane) : nullptr,
                   (ev & EV_STAGE) ? sc.staged(st.seg_i + 1, lane) : nullptr};
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        V* o = dst[k];
        if (!o) continue;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          o[r] = st.M[r];
          o[R + r] = st.X[r];
          o[2 * R + r] = st.Y[r];
          o[3 * R + r] = st.BM[r];
          o[4 * R + r] = st.BX[r];
          o[5 * R + r] = st.BY[r];
        }
        o[6 * R] = d.M;
        o[6 * R + 1] = d.X;
        o[6 * R + 2] = d.Y;
        o[6 * R + 3] = st.acc;
      }
    }
    if ((ev & EV_END) && lane == 31) {
#pragma unroll
      for (int c = 0; c < P::NC; ++c) sc.seg_raw[st.seg_i * P::NC + c] = static_cast<double>(P::get(st.acc, c));
    }
    if (ev & EV_BEGIN) {
      ++st.seg_i;
      // A recomputation stream (FP64 only) has one unshared segment from the origin and no record.
      const bool synth = synth_len > 0;
      const Segment* rec = a.v.segs + prog.seg_off + st.seg_i;
      if (!synth && st.seg_i + 1 < prog.n_segs) prefetch_l1(rec + 1);
      const int next_slot = synth ? -1 : rec->next_slot;
      if (!synth && rec->staged) {
        __pipeline_wait_prior(0);
        const V* s = sc.staged(st.seg_i, lane);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          st.M[r] = s[r];
          st.X[r] = s[R + r];
          st.Y[r] = s[2 * R + r];
          st.BM[r] = s[3 * R + r];
          st.BX[r] = s[4 * R + r];
          st.BY[r] = s[5 * R + r];
        }
        d.M = s[6 * R];
        d.X = s[6 * R + 1];
        d.Y = s[6 * R + 2];
        st.acc = s[6 * R + 3];
      } else {
        // The origin: the row-0 constant in the padding rows, zero branch values (GATK never writes
        // branch column zero).
        const S in_s = synth ? static_cast<S>(Consts<P::kDouble>::kInitial / synth_len)
                             : (P::kDouble ? static_cast<S>(rec->init_d) : static_cast<S>(rec->init_f));
#pragma unroll
        for (int r = 0; r < R; ++r) st.M[r] = st.X[r] = st.Y[r] = st.BM[r] = st.BX[r] = st.BY[r] = P::zero();
        d.M = d.X = d.Y = st.acc = P::zero();
        if (lane * R <= pad_hi) {
#pragma unroll
          for (int c = 0; c < P::NC; ++c) {
#pragma unroll
            for (int r = 0; r < R; ++r)
              if (lane * R + r < rd[c].pad) P::put(st.Y[r], c, in_s);
            if (lane * R - 1 < rd[c].pad) P::put(d.Y, c, in_s);
          }
        }
      }
      if (next_slot >= 0) prefetch(sc.staged(st.seg_i + 1, lane), sc.slot(next_slot, lane), L::kSnap);
    }
  }
  // A slow step (some lane at a column carrying DEL_START or DEL_END) runs the branch-value path for
  // the whole warp; it is exact for every column, so lanes do not diverge between it and the plain
  // recurrence.
  const bool slow = __any_sync(kFull, (ev & kPdSlowMask) != 0);
  const bool de = slow && (ev & PD_DE) != 0;
  if (slow) {
    const bool mat = (ev & PD_MAT) != 0;
    const uint32_t s_first = (ev >> kPdFirstShift) & 3u, s_later = (ev >> kPdLaterShift) & 3u;
    if (__all_sync(kFull, s_first == s_later)) {
      // Every row of each lane in one deletion state (the read's first row starts NORMAL, the later
      // rows in the state the row above ended in; the two differ only when a deletion runs to the
      // haplotype's end): a column carrying either flag keeps V(left) as the branch values unless
      // inside a deletion, one predicate a lane.
      const bool keep = mat && s_later != kPdInsideDel;
#pragma unroll
      for (int r = R - 1; r >= 0; --r) {
        const V pM = r ? st.M[r - 1] : d.M, pX = r ? st.X[r - 1] : d.X, pY = r ? st.Y[r - 1] : d.Y;
        if (keep) {
          st.BM[r] = st.M[r];
          st.BX[r] = st.X[r];
          st.BY[r] = st.Y[r];
        }
        const V prior = kGeneric ? pr.prior_generic(ev, r) : pr.prior(sig, r);
        st.Y[r] = P::kTransformed ? P::fma(st.Y[r], pr.c4[r], st.M[r]) : P::fma(st.Y[r], pr.c3[r], P::mul(st.M[r], pr.c4[r]));
        st.M[r] = P::mul(prior, cell_match<P>(pM, pX, pY, pr.c0[r], pr.c1[r], pr.c2[r]));
      }
    } else {
      // Some lane's first read row is in another state than its later rows.
#pragma unroll
      for (int r = R - 1; r >= 0; --r) {
        bool inside[P::NC];
#pragma unroll
        for (int c = 0; c < P::NC; ++c) inside[c] = ((lane * R + r == rd[c].pad) ? s_first : s_later) == kPdInsideDel;
        const V pM = r ? st.M[r - 1] : d.M, pX = r ? st.X[r - 1] : d.X, pY = r ? st.Y[r - 1] : d.Y;
        if (mat) {
          st.BM[r] = P::sel(inside[0], inside[P::NC - 1], st.BM[r], st.M[r]);
          st.BX[r] = P::sel(inside[0], inside[P::NC - 1], st.BX[r], st.X[r]);
          st.BY[r] = P::sel(inside[0], inside[P::NC - 1], st.BY[r], st.Y[r]);
        }
        const V prior = kGeneric ? pr.prior_generic(ev, r) : pr.prior(sig, r);
        st.Y[r] = P::kTransformed ? P::fma(st.Y[r], pr.c4[r], st.M[r]) : P::fma(st.Y[r], pr.c3[r], P::mul(st.M[r], pr.c4[r]));
        st.M[r] = P::mul(prior, cell_match<P>(pM, pX, pY, pr.c0[r], pr.c1[r], pr.c2[r]));
      }
    }
    // Insertion values from the top row down. On a DEL_END column each row's values take the max
    // with its branch values once its X is computed (the last row's after the result below), so
    // the next row's X reads U = max(B(up), V(up)); the lane above's bottom row arrives merged.
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const V qM = r ? st.M[r - 1] : u.M, qX = r ? st.X[r - 1] : u.X;
      st.X[r] = P::kTransformed ? P::fma(qX, pr.c3[r], qM) : P::fma(qX, pr.c3[r], P::mul(qM, pr.c2[r]));
      if (de && r + 1 < R) {
        st.M[r] = P::max(st.BM[r], st.M[r]);
        st.X[r] = P::max(st.BX[r], st.X[r]);
        st.Y[r] = P::max(st.BY[r], st.Y[r]);
      }
    }
  } else {
#pragma unroll
    for (int r = R - 1; r >= 0; --r) {
      const V pM = r ? st.M[r - 1] : d.M, pX = r ? st.X[r - 1] : d.X, pY = r ? st.Y[r - 1] : d.Y;
      const V prior = kGeneric ? pr.prior_generic(ev, r) : pr.prior(sig, r);
      st.Y[r] = P::kTransformed ? P::fma(st.Y[r], pr.c4[r], st.M[r]) : P::fma(st.Y[r], pr.c3[r], P::mul(st.M[r], pr.c4[r]));
      st.M[r] = P::mul(prior, cell_match<P>(pM, pX, pY, pr.c0[r], pr.c1[r], pr.c2[r]));
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const V qM = r ? st.M[r - 1] : u.M, qX = r ? st.X[r - 1] : u.X;
      st.X[r] = P::kTransformed ? P::fma(qX, pr.c3[r], qM) : P::fma(qX, pr.c3[r], P::mul(qM, pr.c2[r]));
    }
  }
  st.acc = P::fma(st.X[R - 1], an, P::add(st.acc, st.M[R - 1]));
  if (de) {
    st.M[R - 1] = P::max(st.BM[R - 1], st.M[R - 1]);
    st.X[R - 1] = P::max(st.BX[R - 1], st.X[R - 1]);
    st.Y[R - 1] = P::max(st.BY[R - 1], st.Y[R - 1]);
  }
}

// Entry p of a recomputation stream: the haplotype's forward entries (code and deletion bits),
// BEGIN on the first column and END after the last.
__device__ __forceinline__ uint32_t pd_synth_entry(const uint32_t* seq, int len, int p) {
  if (p < 0 || p > len) return 0u;
  uint32_t e = p < len ? __ldg(seq + p) : 0u;
  if (p == 0) e |= EV_BEGIN;
  if (p == len) e |= EV_END;
  return e;
}

template <class P, int R>
__device__ void pd_forward_pass(const LaunchArgs& a, const Program& prog, const ReadRef* rd, const uint8_t* classes,
                                const uint32_t* sigs, int lane, PdScratch<P, R>& sc, const uint32_t* synth_seq, int synth_len) {
  using V = typename P::V;
  using S = typename P::S;
  PdRows<P, R> pr;
  pr.load(a.v, rd, lane, classes);
  V an;
#pragma unroll
  for (int c = 0; c < P::NC; ++c)
    P::put(an, c, static_cast<S>((P::kTransformed && rd[c].len > 0) ? err_prob(a.v, a.v.ins[rd[c].off + rd[c].len - 1]) : 1.0));
  int pad_hi = 0;
#pragma unroll
  for (int c = 0; c < P::NC; ++c) pad_hi = rd[c].pad > pad_hi ? rd[c].pad : pad_hi;

  PdState<P, R> st;
#pragma unroll
  for (int r = 0; r < R; ++r) st.M[r] = st.X[r] = st.Y[r] = st.BM[r] = st.BX[r] = st.BY[r] = P::zero();
  st.acc = P::zero();
  st.seg_i = -1;
  PdEdge<P> ea, eb;
  ea.M = ea.X = ea.Y = P::zero();
  eb = ea;
  if (P::kDouble && synth_len > 0) {
    const int n = synth_len;
    for (int t = 0; t < n + 32; t += 2) {
      const uint32_t e0 = pd_synth_entry(synth_seq, n, t - lane), e1 = pd_synth_entry(synth_seq, n, t + 1 - lane);
      pd_step<P, R>(a, prog, rd, lane, pr, an, pad_hi, sc, st, synth_len, e0, __ldg(sigs + (e0 & kCodeMask)), ea, eb);
      pd_step<P, R>(a, prog, rd, lane, pr, an, pad_hi, sc, st, synth_len, e1, __ldg(sigs + (e1 & kCodeMask)), eb, ea);
    }
  } else {
    const int n = prog.fwd_len;
    const uint32_t* stream = a.v.stream + prog.fwd_off - lane;
    // Two steps an iteration; one where no lane has an event runs a body without event code.
    const uint32_t keep = lane == 31 ? kEvMask : (kEvMask & ~(EV_END | EV_ACC));
    uint32_t n0 = __ldg(stream), n1 = __ldg(stream + 1);
    uint32_t g0 = __ldg(sigs + (n0 & kCodeMask)), g1 = __ldg(sigs + (n1 & kCodeMask));
    for (int t = 0; t < n + 32; t += 2) {
      const uint32_t e0 = n0, e1 = n1, s0 = g0, s1 = g1;
      n0 = __ldg(stream + t + 2);
      n1 = __ldg(stream + t + 3);
      g0 = __ldg(sigs + (n0 & kCodeMask));
      g1 = __ldg(sigs + (n1 & kCodeMask));
      if (__any_sync(kFull, (e0 | e1) & keep)) {
        pd_step<P, R>(a, prog, rd, lane, pr, an, pad_hi, sc, st, 0, e0, s0, ea, eb);
        pd_step<P, R>(a, prog, rd, lane, pr, an, pad_hi, sc, st, 0, e1, s1, eb, ea);
      } else {
        pd_step<P, R, false>(a, prog, rd, lane, pr, an, pad_hi, sc, st, 0, e0, s0, ea, eb);
        pd_step<P, R, false>(a, prog, rd, lane, pr, an, pad_hi, sc, st, 0, e1, s1, eb, ea);
      }
    }
  }
  __pipeline_wait_prior(0);
}

// Thresholds, log10 and the caller's layout (fgkl kernel.rs:897-914 via pd_kernel.rs:262-270).
template <class P, int R>
__device__ void pd_finalize(const LaunchArgs& a, const Task& task, const Region& region, const Program& prog, int lane,
                            PdScratch<P, R>& sc) {
  using C = Consts<P::kDouble>;
  __syncwarp();
  if (P::kDouble && task.hap >= 0) {
    const double raw = sc.seg_raw[0];
    const double result = raw != raw ? __longlong_as_double(0x7ff8000000000000ll) : log10(raw) - C::kLog10Initial;
    const int read_local = task.read[0] - region.read_off;
    for (int k = lane; k < region.n_haps; k += 32) {
      const HapInfo info = a.v.haps[region.hap_off + k];
      if (info.src == task.hap) a.v.out[region.out_off + static_cast<int64_t>(read_local) * region.n_haps + info.order] = result;
    }
    return;
  }
  // A dense read's recomputation (only_lost) fills in only the pairs the first pass lost; a PD program
  // has no joins, so in FP64 it loses none.
  const bool dense = a.only_lost != 0;
  unsigned long long lost_count = 0;
  for (int k = lane; k < region.n_haps; k += 32) {
    const HapInfo info = a.v.haps[region.hap_off + k];
    const double factor = a.v.segs[prog.seg_off + info.seg].factor;
#pragma unroll
    for (int c = 0; c < P::NC; ++c) {
      if (task.read[c] < 0) continue;
      const int read_local = task.read[c] - region.read_off;
      double* dst = a.v.out + region.out_off + static_cast<int64_t>(read_local) * region.n_haps + info.order;
      if (dense && !isnan(*dst)) continue;
      const double raw = __dmul_rn(sc.seg_raw[info.seg * P::NC + c], factor);
      bool lost = a.min_accept_plain ? !(raw >= C::kMinAccepted) : (raw != raw);
      if (!P::kDouble) lost |= isinf(raw);
      const double result = lost ? __longlong_as_double(0x7ff8000000000000ll) : log10(raw) - C::kLog10Initial;
      *dst = result;
      lost_count += lost;
    }
  }
  if (lost_count && !dense) atomicAdd(&a.v.counters->lost_pairs, lost_count);
}

// Resident blocks of 4 warps the register budget is cut for (measured on c3): one-read FP32 at 4
// (128 registers, no spill), the FP32x2 form at 2 (up to 255), FP64 at 3 for R <= 5 (168 registers,
// a few spilled values: the recomputation sweeps run faster at 12 warps per SM than at 8), else 1.
template <class P, int R>
struct PdMinBlocks {
  static constexpr int value = P::kDouble ? (R <= 5 ? 3 : 1) : (P::NC == 2 ? 2 : 4);
};

template <class P, int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, (PdMinBlocks<P, R>::value)) pd_kernel(LaunchArgs a) {
  using V = typename P::V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int warp_in_block = threadIdx.x >> 5;
  const int warp = blockIdx.x * static_cast<int>(blockDim.x >> 5) + warp_in_block;
  V* smem = reinterpret_cast<V*>(smem_raw + warp_in_block * PdLayout<P, R>::kSmemPerWarp);
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
    const uint8_t* classes = a.v.code_of_byte + region.code_off;
    const uint32_t* sigs = a.v.pd_sigs + region.sig_off;
    char* scratch = a.scratch + static_cast<size_t>(warp) * a.scratch_stride;
    if (P::kDouble && task.hap >= 0) {
      const HapInfo info = a.v.haps[region.hap_off + task.hap];
      PdScratch<P, R> sc(scratch, smem, 0);
      pd_forward_pass<P, R>(a, prog, rd, classes, sigs, lane, sc, a.v.pd_entries + region.seq_off + info.seq, info.len);
      pd_finalize<P, R>(a, task, region, prog, lane, sc);
    } else {
      PdScratch<P, R> sc(scratch, smem, prog.n_slots);
      pd_forward_pass<P, R>(a, prog, rd, classes, sigs, lane, sc, nullptr, 0);
      pd_finalize<P, R>(a, task, region, prog, lane, sc);
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------------
// Strip-mined PD pairs (reads longer than 620 bases), and every pair of a region whose reads hold
// more distinct bytes than the class bits cover (kGeneric): one read against one distinct
// haplotype, unshared, over the haplotype's forward entries, the rows cut into blocks of 32 R rows
// run one after another. Lane 0's row above comes from a carry row (merged on DEL_END columns like
// every row): GATK's row 0 in the first block (M = X = 0, Y = INITIAL / hap_len), after that
// the previous block's bottom row, written by lane 31 column by column and read by lane 0 31 steps
// before lane 31 of the next block overwrites it (the plain strip-mined kernel's scheme). The
// state a block's top row starts in is the previous row's, which the entries' later-row state
// carries; only the read's first row (in the first block) takes the first-row state.
// ---------------------------------------------------------------------------------------------

constexpr int kPdCarryVals = 4;  // M, X, Y, padded to 16 bytes

template <class P>
constexpr size_t pd_long_scratch_size(int max_hap_len) {
  return 16 + static_cast<size_t>(max_hap_len) * kPdCarryVals * sizeof(typename P::V);
}

template <class P, int R>
__device__ __forceinline__ void pd_long_store(typename P::V* carry, const PdState<P, R>& st, int lane, int t, int n, bool last) {
  const int p = t - 31;
  if (!last && lane == 31 && p >= 0 && p < n) {
    typename P::V rec[kPdCarryVals] = {st.M[R - 1], st.X[R - 1], st.Y[R - 1], P::zero()};
    store_record(carry + static_cast<size_t>(p) * kPdCarryVals, rec);
  }
}

template <class P>
__device__ __forceinline__ void pd_long_fetch(const typename P::V* carry, typename P::V (&rec)[kPdCarryVals], int lane, int p, int n,
                                              bool first) {
  if (!first && lane == 0 && p < n) load_record(rec, carry + static_cast<size_t>(p) * kPdCarryVals);
}

template <class P, int R>
__device__ __forceinline__ void pd_set_carry(PdState<P, R>& st, const typename P::V (&c)[kPdCarryVals]) {
  st.cM = c[0];
  st.cX = c[1];
  st.cY = c[2];
}

template <class P, int R, bool kGeneric>
__device__ void pd_long_block(const LaunchArgs& a, const ReadRef* rd, int lane, const PdRows<P, R>& pr, typename P::V an,
                              PdScratch<P, R>& sc, const uint32_t* seq, const uint32_t* sigs, int n, typename P::V* carry,
                              bool first, bool last) {
  using V = typename P::V;
  using S = typename P::S;
  const int pad_hi = rd[0].pad;
  PdState<P, R> st;
#pragma unroll
  for (int r = 0; r < R; ++r) st.M[r] = st.X[r] = st.Y[r] = st.BM[r] = st.BX[r] = st.BY[r] = P::zero();
  st.acc = P::zero();
  st.seg_i = -1;
  st.cM = st.cX = P::zero();
  st.cY = first ? static_cast<S>(Consts<P::kDouble>::kInitial / n) : P::zero();
  const Program prog{};
  PdEdge<P> ea, eb;
  ea.M = ea.X = ea.Y = P::zero();
  eb = ea;
  V n0[kPdCarryVals], n1[kPdCarryVals];
#pragma unroll
  for (int i = 0; i < kPdCarryVals; ++i) n0[i] = n1[i] = P::zero();
  pd_long_fetch<P>(carry, n0, lane, 0, n, first);
  pd_long_fetch<P>(carry, n1, lane, 1, n, first);
  for (int t = 0; t < n + 32; t += 2) {
    const uint32_t e0 = pd_synth_entry(seq, n, t - lane), e1 = pd_synth_entry(seq, n, t + 1 - lane);
    const uint32_t s0 = kGeneric ? 0u : __ldg(sigs + (e0 & kCodeMask)), s1 = kGeneric ? 0u : __ldg(sigs + (e1 & kCodeMask));
    V c0[kPdCarryVals], c1[kPdCarryVals];
#pragma unroll
    for (int i = 0; i < kPdCarryVals; ++i) {
      c0[i] = n0[i];
      c1[i] = n1[i];
    }
    pd_long_fetch<P>(carry, n0, lane, t + 2, n, first);
    pd_long_fetch<P>(carry, n1, lane, t + 3, n, first);
    if (!first) pd_set_carry<P, R>(st, c0);
    pd_step<P, R, true, true, kGeneric>(a, prog, rd, lane, pr, an, pad_hi, sc, st, n, e0, s0, ea, eb);
    pd_long_store<P, R>(carry, st, lane, t, n, last);
    if (!first) pd_set_carry<P, R>(st, c1);
    pd_step<P, R, true, true, kGeneric>(a, prog, rd, lane, pr, an, pad_hi, sc, st, n, e1, s1, eb, ea);
    pd_long_store<P, R>(carry, st, lane, t + 1, n, last);
  }
}

template <class P, int R, bool kGeneric>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, (P::kDouble ? 1 : 2)) pd_long_kernel(LaunchArgs a) {
  using V = typename P::V;
  using S = typename P::S;
  using C = Consts<P::kDouble>;
  const int lane = threadIdx.x & 31;
  const int warp = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
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
    const uint32_t* seq = a.v.pd_entries + region.seq_off + info.seq;
    const uint32_t* sigs = a.v.pd_sigs + region.sig_off;
    const uint8_t* classes = a.v.code_of_byte + region.code_off;
    const int n = info.len;
    ReadRef rd[1];
    rd[0].off = a.v.read_off[task.read[0]];
    rd[0].len = static_cast<int>(a.v.read_off[task.read[0] + 1] - rd[0].off);
    const int blocks = long_blocks(rd[0].len, R);
    const int pad0 = 32 * R * blocks - rd[0].len;
    PdScratch<P, R> sc(scratch, nullptr, 0);
    const V an = static_cast<S>(P::kTransformed ? err_prob(a.v, a.v.ins[rd[0].off + rd[0].len - 1]) : 1.0);
    for (int b = 0; b < blocks; ++b) {
      rd[0].pad = pad0 - 32 * R * b;
      PdRows<P, R> pr;
      if (kGeneric)
        pr.load_generic(a.v, rd, lane, classes);
      else
        pr.load(a.v, rd, lane, classes);
      pd_long_block<P, R, kGeneric>(a, rd, lane, pr, an, sc, seq, sigs, n, carry, b == 0, b == blocks - 1);
      __syncwarp();
    }
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
void pd_occ(int* blocks, int warps) {
  static std::atomic<int> cache[3][kMaxDevices];
  *blocks = resident_blocks(pd_kernel<P, R>, warps * PdLayout<P, R>::kSmemPerWarp, warps * 32, cache[warps_index(warps)],
                            kWarpsPerBlock * PdLayout<P, R>::kSmemPerWarp);
}

template <class P, int R>
cudaError_t pd_go(int blocks, const LaunchArgs& a, cudaStream_t s, int warps) {
  const size_t smem = warps * PdLayout<P, R>::kSmemPerWarp;
  pd_kernel<P, R><<<blocks, warps * 32, smem, s>>>(a);
  return cudaGetLastError();
}

// Rows-per-lane dispatch over 1..8 and 10..20 (even), FP32 or FP64.
template <class P, class F>
auto pd_rows(int rows, F&& f) {
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


// Rows 1..8 only (the packed two-read form).
template <class F>
auto pd_rows8(int rows, F&& f) {
  switch (rows) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    case 6: return f(std::integral_constant<int, 6>{});
    case 7: return f(std::integral_constant<int, 7>{});
    default: return f(std::integral_constant<int, 8>{});
  }
}

template <class F>
auto pd_long_rows(int rows, F&& f) {
  switch (rows) {
    case 4: return f(std::integral_constant<int, 4>{});
    case 6: return f(std::integral_constant<int, 6>{});
    default: return f(std::integral_constant<int, 8>{});
  }
}

template <class P, int R, bool kGeneric>
void pd_long_occ(int* blocks) {
  static std::atomic<int> cache[kMaxDevices];
  *blocks = resident_blocks(pd_long_kernel<P, R, kGeneric>, 0, kWarpsPerBlock * 32, cache);
}

}  // namespace

size_t pd_long_scratch_bytes(Kind k, int, int max_hap_len) {
  const bool dbl = k == Kind::kLongF64Pd || k == Kind::kGenericF64Pd;
  return dbl ? pd_long_scratch_size<OneF64>(max_hap_len) : pd_long_scratch_size<OneF32>(max_hap_len);
}

void pd_long_occupancy(Kind k, int rows, int* blocks, int* threads) {
  *threads = kWarpsPerBlock * 32;
  *blocks = 0;
  pd_long_rows(rows, [&](auto r) {
    constexpr int R = decltype(r)::value;
    switch (k) {
      case Kind::kLongF32Pd: pd_long_occ<OneF32, R, false>(blocks); break;
      case Kind::kLongF64Pd: pd_long_occ<OneF64, R, false>(blocks); break;
      case Kind::kGenericF32Pd: pd_long_occ<OneF32, R, true>(blocks); break;
      case Kind::kGenericF64Pd: pd_long_occ<OneF64, R, true>(blocks); break;
      default: break;
    }
    return 0;
  });
}

cudaError_t pd_long_launch(Kind k, int rows, int blocks, const LaunchArgs& a, cudaStream_t s) {
  return pd_long_rows(rows, [&](auto r) -> cudaError_t {
    constexpr int R = decltype(r)::value;
    switch (k) {
      case Kind::kLongF32Pd: pd_long_kernel<OneF32, R, false><<<blocks, kWarpsPerBlock * 32, 0, s>>>(a); break;
      case Kind::kLongF64Pd: pd_long_kernel<OneF64, R, false><<<blocks, kWarpsPerBlock * 32, 0, s>>>(a); break;
      case Kind::kGenericF32Pd: pd_long_kernel<OneF32, R, true><<<blocks, kWarpsPerBlock * 32, 0, s>>>(a); break;
      case Kind::kGenericF64Pd: pd_long_kernel<OneF64, R, true><<<blocks, kWarpsPerBlock * 32, 0, s>>>(a); break;
      default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
  });
}

size_t pd_scratch_bytes(PdForm form, int rows, int max_slots, int max_segs) {
  switch (form) {
    case PdForm::kOneF64:
      return pd_rows<OneF64>(rows, [&](auto r) { return pd_scratch_size<OneF64, decltype(r)::value>(max_slots, max_segs); });
    case PdForm::kPackedF32:
      return pd_rows8(rows, [&](auto r) { return pd_scratch_size<PackedF32, decltype(r)::value>(max_slots, max_segs); });
    default:
      return pd_rows<OneF32>(rows, [&](auto r) { return pd_scratch_size<OneF32, decltype(r)::value>(max_slots, max_segs); });
  }
}

void pd_occupancy(PdForm form, int rows, int* blocks, int* threads, int warps) {
  *threads = warps * 32;
  *blocks = 0;
  switch (form) {
    case PdForm::kOneF64:
      pd_rows<OneF64>(rows, [&](auto r) {
        pd_occ<OneF64, decltype(r)::value>(blocks, warps);
        return 0;
      });
      break;
    case PdForm::kPackedF32:
      pd_rows8(rows, [&](auto r) {
        pd_occ<PackedF32, decltype(r)::value>(blocks, warps);
        return 0;
      });
      break;
    default:
      pd_rows<OneF32>(rows, [&](auto r) {
        pd_occ<OneF32, decltype(r)::value>(blocks, warps);
        return 0;
      });
  }
}

cudaError_t pd_launch(PdForm form, int rows, int blocks, const LaunchArgs& a, cudaStream_t s, int warps) {
  switch (form) {
    case PdForm::kOneF64:
      return pd_rows<OneF64>(rows, [&](auto r) { return pd_go<OneF64, decltype(r)::value>(blocks, a, s, warps); });
    case PdForm::kPackedF32:
      return pd_rows8(rows, [&](auto r) { return pd_go<PackedF32, decltype(r)::value>(blocks, a, s, warps); });
    default:
      return pd_rows<OneF32>(rows, [&](auto r) { return pd_go<OneF32, decltype(r)::value>(blocks, a, s, warps); });
  }
}

}  // namespace fgkl
