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

// Backward sweep of one pair; returns, in every lane, the padding row's start mass s.
template <class P, int R>
__device__ typename P::V adj_backward(const AdjView& v, const AdjRows<P, R>& own, int64_t off, int len, int pad,
                                      const uint8_t* hap, int m, int lane, char* scratch) {
  using V = typename P::V;
  using S = typename P::S;
  AdjBelow<P, R> bl;
  bl.load(v, off, len, pad, lane);
  const V sink = lane == 31 ? static_cast<S>(Consts<P::kDouble>::kBackwardScale) : P::zero();
  V BM[R], BY[R];
#pragma unroll
  for (int r = 0; r < R; ++r) BM[r] = BY[r] = P::zero();
  V dBM = P::zero(), topBM = P::zero(), topBX = P::zero();
  const int pad_row = pad - 1;  // the padding row right above the read
  const int pad_lane = pad_row / R, pad_r = pad_row % R;
  V start_mass = P::zero();
  // The base of column j + 1 (the diagonal successor) for position p, none beyond the haplotype;
  // loaded one step ahead.
  auto code_at = [&](int q) -> uint32_t {
    const int jj = m - q;
    return (q >= 0 && jj >= 0 && jj < m) ? adj_code(__ldg(hap + jj)) : 0u;
  };
  uint32_t next_code = code_at(-(31 - lane));
  for (int t = 0; t < m + 1 + 31; ++t) {
    const V rBM = P::down(topBM), rBX = P::down(topBX);
    const int p = t - (31 - lane);  // position: column m - p
    const int j = m - p;
    if (p == 0) {
      // The all-zero column beyond the haplotype.
#pragma unroll
      for (int r = 0; r < R; ++r) BM[r] = BY[r] = P::zero();
      dBM = P::zero();
    }
    const uint32_t code = next_code;
    next_code = code_at(p + 1);
    using Col = AdjCol<P, R>;
    V rec[Col::kRec];
    V belowX = rBX, diagM = dBM;
#pragma unroll
    for (int r = R - 1; r >= 0; --r) {
      const V into = P::mul(bl.prior(code, r), diagM);
      const V itm = P::mul(into, bl.im[r]);
      V bx = P::fma(belowX, bl.ii[r], itm);
      const V by = P::fma(BY[r], own.dd[r], itm);
      V bm = P::fma(BY[r], own.md[r], P::fma(belowX, bl.mi[r], P::mul(into, bl.mm[r])));
      if (r == R - 1) {
        bm = P::add(bm, sink);
        bx = P::add(bx, sink);
      }
      diagM = BM[r];
      BM[r] = bm;
      BY[r] = by;
      belowX = bx;
      rec[r] = bm;
      rec[R + r] = bx;
      rec[2 * R + r] = by;
    }
#pragma unroll
    for (int i = 3 * R; i < Col::kRec; ++i) rec[i] = P::zero();
    if (p >= 0 && j >= 1) store_record(Col::at(scratch, j, lane), rec);
    if (p == m && lane == pad_lane) {
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (r == pad_r) start_mass = BY[r];
    }
    topBM = BM[0];
    topBX = belowX;
    dBM = rBM;
  }
  return __shfl_sync(kFull, start_mass, pad_lane);
}

// Forward sweep of one pair, accumulating the pair's gradient terms scaled by `norm`; returns the
// raw result (lane 31).
template <class P, int R>
__device__ typename P::V adj_forward(const AdjRows<P, R>& own, int pad, const uint8_t* hap, int m, int lane, char* scratch,
                                     typename P::V* ring, double norm, double (&gi)[R], double (&gd)[R], double (&ge)[R],
                                     double (&gq)[R]) {
  using V = typename P::V;
  using S = typename P::S;
  using Col = AdjCol<P, R>;
  constexpr int D = Col::kDepth;
  const S init = static_cast<S>(Consts<P::kDouble>::kInitial / m);
  V M[R], X[R], Y[R];
#pragma unroll
  for (int r = 0; r < R; ++r) M[r] = X[r] = Y[r] = P::zero();
  V acc = P::zero();
  V dM = P::zero(), dX = P::zero(), dY = P::zero();
  // The lane's k-th forward column (k = 0..m-1, column k + 1) sits in ring slot k % D; columns are
  // fetched D ahead with cp.async, one commit group per column.
  auto slot = [&](int k) { return ring + (static_cast<size_t>(k % D) * 32 + lane) * Col::kRec; };
  auto fetch = [&](int k) {
    if (k < m) {
      const V* src = Col::at(scratch, k + 1, lane);
      V* dst = slot(k);
#pragma unroll
      for (int i = 0; i < Col::kRec / Col::kPer16; ++i)
        __pipeline_memcpy_async(reinterpret_cast<char*>(dst) + 16 * i, reinterpret_cast<const char*>(src) + 16 * i, 16);
    }
    __pipeline_commit();
  };
#pragma unroll
  for (int k = 0; k < D; ++k) fetch(k);
  uint32_t next_code = (m > 0 && lane == 0) ? adj_code(__ldg(hap)) : 0u;
  for (int t = 0; t < m + 31; ++t) {
    const V uM = P::up(M[R - 1]), uX = P::up(X[R - 1]), uY = P::up(Y[R - 1]);
    const int p = t - lane;  // column p + 1
    if (p == 0) {
      // Column 0: the row-0 constant in the padding rows (and the row above the lane's top row).
#pragma unroll
      for (int r = 0; r < R; ++r) {
        M[r] = X[r] = P::zero();
        Y[r] = lane * R + r < pad ? init : P::zero();
      }
      dM = dX = P::zero();
      dY = lane * R - 1 < pad ? init : P::zero();
      acc = P::zero();
    }
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
    // Match and deletion values from the bottom row up (each row reads the old row above).
#pragma unroll
    for (int r = R - 1; r >= 0; --r) {
      const V pM = r ? M[r - 1] : dM, pX = r ? X[r - 1] : dX, pY = r ? Y[r - 1] : dY;
      const V mOld = M[r], yOld = Y[r];
      const V prior = own.prior(code, r);
      const V sxy = P::add(pX, pY);
      const V s = P::fma(pM, own.mm[r], P::mul(sxy, own.im[r]));
      Y[r] = P::fma(yOld, own.dd[r], P::mul(mOld, own.md[r]));
      M[r] = P::mul(prior, s);
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
      const V qM = r ? M[r - 1] : uM, qX = r ? X[r - 1] : uX;
      X[r] = P::fma(qX, own.ii[r], P::mul(qM, own.mi[r]));
      if (live && own.real[r]) {
        const double bx_n = static_cast<double>(bX[r]) * norm;
        gi[r] += static_cast<double>(qM) * bx_n;
        ge[r] += static_cast<double>(qX) * bx_n;
      }
    }
    if (live) {
      acc = P::add(acc, P::add(M[R - 1], X[R - 1]));
      fetch(p + D);  // into the slot just read (its values are consumed above)
    }
    dM = uM;
    dX = uX;
    dY = uY;
  }
  __pipeline_wait_prior(0);
  return __shfl_sync(kFull, acc, 31);
}

template <class P, int R>
struct AdjMinBlocks {
  static constexpr int value = 1;
};

template <class P, int R>
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
      const double s = static_cast<double>(adj_backward<P, R>(a.v, own, off, len, pad, hap, m, lane, scratch));
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
      const double fwd = static_cast<double>(adj_forward<P, R>(own, pad, hap, m, lane, scratch, ring, norm, gi, gd, ge, gq));
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

template <class P, int R>
void adj_occ(int* blocks) {
  static std::atomic<int> cache[kMaxDevices];
  *blocks = resident_blocks(adjoint_kernel<P, R>, kWarpsPerBlock * AdjCol<P, R>::kRingBytes, kWarpsPerBlock * 32, cache);
}

template <class P, int R>
cudaError_t adj_go(int blocks, const AdjLaunch& a, cudaStream_t s) {
  const size_t smem = kWarpsPerBlock * AdjCol<P, R>::kRingBytes;
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

size_t adj_scratch_bytes(bool dbl, int rows, int max_hap_len) {
  const size_t rec = dbl ? adj_dispatch_rows(rows, [](auto r) { return static_cast<size_t>(AdjCol<OneF64, decltype(r)::value>::kRec); })
                         : adj_dispatch_rows(rows, [](auto r) { return static_cast<size_t>(AdjCol<OneF32, decltype(r)::value>::kRec); });
  return static_cast<size_t>(max_hap_len + 1) * 32 * rec * (dbl ? sizeof(double) : sizeof(float));
}

void adj_occupancy(bool dbl, int rows, int* blocks, int* threads) {
  *threads = kWarpsPerBlock * 32;
  *blocks = 0;
  if (dbl)
    adj_dispatch_rows(rows, [&](auto r) {
      adj_occ<OneF64, decltype(r)::value>(blocks);
      return 0;
    });
  else
    adj_dispatch_rows(rows, [&](auto r) {
      adj_occ<OneF32, decltype(r)::value>(blocks);
      return 0;
    });
}

cudaError_t adj_launch(bool dbl, int rows, int blocks, const AdjLaunch& a, cudaStream_t s) {
  if (dbl) return adj_dispatch_rows(rows, [&](auto r) { return adj_go<OneF64, decltype(r)::value>(blocks, a, s); });
  return adj_dispatch_rows(rows, [&](auto r) { return adj_go<OneF32, decltype(r)::value>(blocks, a, s); });
}

}  // namespace fgkl
