// sm_100a Smith-Waterman: GATK's SmithWatermanJavaAligner (fgkl crates/smithwaterman/src/reference.rs,
// lib.rs) over a batch of (reference, alternate) pairs, one warp per pair.
//
// Rows are reference positions, on lanes: lane l holds rows l*8+1 .. l*8+8 of a 256-row block, and a
// longer reference runs as consecutive blocks. Columns are alternate positions, walked as an
// anti-diagonal wavefront: at step t lane l is at column t - l + 1, and the row above arrives from
// lane l - 1 by shuffle (lane 0 takes GATK's row 0, or, below the first block, the bottom row the
// block above stored per column). Per cell (reference.rs:69-110), in integers:
//   diag  = H(i-1, j-1) + (ref[i] == alt[j] ? match : mismatch)
//   F(i, j) = max over the vertical gap: F(i-1, j) + extend, or H(i-1, j) + open when that is larger
//   E(i, j) = the same along the row from (i, j-1)
//   H = diag when diag >= F and diag >= E, else E when E >= F, else F; never below -1e8.
// Each cell keeps one traceback byte: the direction (diagonal, horizontal, vertical) and whether its
// vertical and its horizontal gap extend the neighbour's (not opened here), from which the traceback
// recovers GATK's gap lengths. The bytes are stored anti-diagonal-major ([block][step][lane][8
// rows]), so each step's stores are one contiguous 256-byte run. After the fill, lane 0 picks the
// end cell from the last column and last row with GATK's tie rules and walks back (reference.rs:
// 113-203). For the SoftClip and Ignore strategies an alternate that occurs exactly in the
// reference short-circuits to one match (lib.rs:602-607, the last occurrence), found first by the
// warp testing 32 start positions at a time.
#include <climits>
#include <cstdint>

#include "dp_common.cuh"
#include "sw.cuh"

namespace fgkl {

namespace {

constexpr int kBlockRows = 32 * kSwRows;
constexpr int kCutoff = -100000000;  // GATK's MATRIX_MIN_CUTOFF
constexpr int kLowInit = INT_MIN / 2;  // GATK's lowInitValue
constexpr uint32_t kExtV = 4, kExtH = 8;

__host__ __device__ inline size_t sw_align256(size_t x) { return (x + 255) / 256 * 256; }

// A pair's per-warp scratch.
struct SwScratch {
  uint8_t* tb;         // [block][step][lane][8 rows]
  int32_t* last_col;   // H(i, m), i = 1..n
  int32_t* last_row;   // H(n, j), j = 1..m
  int2* carry;         // bottom row of a block: (H, F) per column
  int m;

  __host__ __device__ static size_t tb_bytes(int64_t n, int64_t m) {
    return sw_align256(static_cast<size_t>((n + kBlockRows - 1) / kBlockRows) * static_cast<size_t>(m + 31) * kBlockRows);
  }
  __host__ __device__ static size_t bytes(int64_t n, int64_t m) {
    return tb_bytes(n, m) + sw_align256(4 * static_cast<size_t>(n)) + sw_align256(4 * static_cast<size_t>(m)) +
           sw_align256(8 * static_cast<size_t>(m));
  }
  __device__ SwScratch(char* base, int n, int m_) : m(m_) {
    tb = reinterpret_cast<uint8_t*>(base);
    last_col = reinterpret_cast<int32_t*>(base + tb_bytes(n, m_));
    last_row = reinterpret_cast<int32_t*>(base + tb_bytes(n, m_) + sw_align256(4 * static_cast<size_t>(n)));
    carry = reinterpret_cast<int2*>(base + tb_bytes(n, m_) + sw_align256(4 * static_cast<size_t>(n)) +
                                    sw_align256(4 * static_cast<size_t>(m_)));
  }
  // Traceback byte of cell (i, j), 1 <= i <= n, 1 <= j <= m.
  __device__ uint32_t at(int i, int j) const {
    const int b = (i - 1) / kBlockRows, rl = (i - 1) - b * kBlockRows, ln = rl / kSwRows, r = rl % kSwRows;
    const size_t t = static_cast<size_t>(j - 1) + ln;
    return tb[((static_cast<size_t>(b) * (m + 31) + t) * 32 + ln) * kSwRows + r];
  }
};

__global__ void __launch_bounds__(kWarpsPerBlock * 32, 8) sw_kernel(SwArgs a) {
  const int lane = threadIdx.x & 31;
  const int warp = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  char* const base = a.scratch + static_cast<size_t>(warp) * a.stride;
  const bool edge = a.strategy == kSwIndel || a.strategy == kSwLeadingIndel;
  const int open = a.open, extend = a.extend;
  // H of row 0 at column x, and of column 0 at row x (reference.rs:50-62).
  auto edge_val = [&](int x) { return (edge && x >= 1) ? open + (x - 1) * extend : 0; };
  for (;;) {
    int task = 0;
    if (lane == 0) task = atomicAdd(a.counter, 1);
    task = __shfl_sync(kFull, task, 0);
    if (task >= a.n_pairs) break;
    const int k = a.order ? a.order[task] : task;
    const uint8_t* ref = a.ref + a.ref_off[k];
    const uint8_t* alt = a.alt + a.alt_off[k];
    const int n = static_cast<int>(a.ref_off[k + 1] - a.ref_off[k]);
    const int m = static_cast<int>(a.alt_off[k + 1] - a.alt_off[k]);
    uint32_t* cig = a.cigar + a.cigar_slot[k];

    // The exact-substring shortcut (reference.rs:15-23): the last occurrence of the alternate.
    if ((a.strategy == kSwSoftClip || a.strategy == kSwIgnore) && m <= n) {
      int found = -1;
      for (int start = n - m; start >= 0; start -= 32) {
        const int s = start - lane;
        bool ok = s >= 0;
        for (int q = 0; ok && q < m; ++q) ok = __ldg(ref + s + q) == __ldg(alt + q);
        const unsigned hits = __ballot_sync(kFull, ok);
        if (hits) {
          found = start - (__ffs(hits) - 1);
          break;
        }
      }
      if (found >= 0) {
        if (lane == 0) {
          cig[0] = (static_cast<uint32_t>(m) << 4) | kSwOpM;
          a.count[k] = 1;
          a.offset[k] = found;
        }
        __syncwarp();
        continue;
      }
    }

    // The fill, one row block after another.
    SwScratch sc(base, n, m);
    const int blocks = (n + kBlockRows - 1) / kBlockRows;
    for (int b = 0; b < blocks; ++b) {
      const int top = b * kBlockRows + lane * kSwRows + 1;  // the lane's first row (1-based)
      int rb[kSwRows], H[kSwRows], E[kSwRows];
#pragma unroll
      for (int r = 0; r < kSwRows; ++r) {
        rb[r] = top + r <= n ? static_cast<int>(__ldg(ref + top + r - 1)) : -1;
        H[r] = 0;
        E[r] = kLowInit;
      }
      const int last_r = (n - top >= 0 && n - top < kSwRows) ? n - top : -1;  // row n among the lane's rows
      int dH = 0;                  // H of the row above at the previous column (the top row's diagonal)
      int bH = 0, bF = kLowInit;   // this lane's bottom row at its last column, for the lane below
      uint8_t* tbb = sc.tb + static_cast<size_t>(b) * (m + 31) * kBlockRows;
      for (int t = 0; t < m + 31; ++t) {
        const int j = t - lane + 1;
        int uH = __shfl_up_sync(kFull, bH, 1), uF = __shfl_up_sync(kFull, bF, 1);
        const bool active = j >= 1 && j <= m;
        if (lane == 0) {
          if (b == 0) {
            uH = edge_val(j);
            uF = kLowInit;
          } else if (active) {
            const int2 c = sc.carry[j - 1];
            uH = c.x;
            uF = c.y;
          }
        }
        if (j == 1) {
          // Column 0: GATK's edge values, no horizontal gap yet.
#pragma unroll
          for (int r = 0; r < kSwRows; ++r) {
            H[r] = edge_val(top + r);
            E[r] = kLowInit;
          }
          dH = edge_val(top - 1);
        }
        uint32_t lo = 0, hi = 0;
        if (active) {
          const int ab = __ldg(alt + j - 1);
          int upH = uH, upF = uF, dg = dH;
#pragma unroll
          for (int r = 0; r < kSwRows; ++r) {
            const int sd = dg + (rb[r] == ab ? a.match : a.mismatch);
            // A gap extends the neighbour's unless opening here scores strictly more. H is the largest
            // of the three: the diagonal when it is at least both gaps, else the horizontal gap when it
            // is at least the vertical one (so max(sd, max(E, F)) and one compare decide it).
            const int fe = upF + extend, fo = upH + open;
            const int F = max(fe, fo);
            const int ee = E[r] + extend, eo = H[r] + open;
            E[r] = max(ee, eo);
            const int gap = max(E[r], F);
            const uint32_t dir = sd >= gap ? 0u : (E[r] >= F ? 1u : 2u);
            int h = max(sd, gap);
            h = h > kCutoff ? h : kCutoff;
            const uint32_t byte = dir | (fe >= fo ? kExtV : 0u) | (ee >= eo ? kExtH : 0u);
            if (r < 4)
              lo |= byte << (8 * r);
            else
              hi |= byte << (8 * (r - 4));
            dg = H[r];
            H[r] = h;
            upH = h;
            upF = F;
          }
          bH = upH;
          bF = upF;
          // The last row and the last column, for the end cell: the lane holding the reference's last
          // row stores its H at every column, and each lane stores its rows once, at the last column.
          // Kept out of the row loop, where they were a compare and a predicated store per cell.
          if (last_r >= 0) {
            int v = H[0];
#pragma unroll
            for (int r = 1; r < kSwRows; ++r)
              if (r == last_r) v = H[r];
            sc.last_row[j - 1] = v;
          }
          if (j == m) {
#pragma unroll
            for (int r = 0; r < kSwRows; ++r)
              if (top + r <= n) sc.last_col[top + r - 1] = H[r];
          }
          if (lane == 31 && b + 1 < blocks) sc.carry[j - 1] = make_int2(bH, bF);
        }
        dH = uH;
        *reinterpret_cast<uint2*>(tbb + (static_cast<size_t>(t) * 32 + lane) * kSwRows) = make_uint2(lo, hi);
      }
      __syncwarp();
    }
    __threadfence_block();
    __syncwarp();

    // End cell (reference.rs:113-143), by the warp: the best of the last column, ties to the lowest
    // row (the scan runs down the column and keeps the last of equal values), then, unless the
    // strategy is LeadingIndel, the last row's cells, each taking over when higher, or equal and
    // nearer the diagonal (|n - j| below the current |p1 - p2|, ties to the earlier column). Each
    // lane scans a strided share; the shares combine in the scan's order.
    int p1 = 0, p2 = m, seg = 0;
    if (a.strategy == kSwIndel) {
      p1 = n;
    } else {
      int cv = INT_MIN, ci = 0;
      for (int i = lane + 1; i <= n; i += 32) {
        const int cur = sc.last_col[i - 1];
        if (cur >= cv) {
          cv = cur;
          ci = i;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const int ov = __shfl_xor_sync(kFull, cv, o), oi = __shfl_xor_sync(kFull, ci, o);
        if (ov > cv || (ov == cv && oi > ci)) {
          cv = ov;
          ci = oi;
        }
      }
      p1 = ci;
      if (a.strategy != kSwLeadingIndel) {
        int rv = INT_MIN, rj = 0, rd = INT_MAX;
        for (int j = lane + 1; j <= m; j += 32) {
          const int cur = sc.last_row[j - 1], d = abs(n - j);
          if (cur > rv || (cur == rv && d < rd)) {
            rv = cur;
            rj = j;
            rd = d;
          }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const int ov = __shfl_xor_sync(kFull, rv, o), oj = __shfl_xor_sync(kFull, rj, o), od = __shfl_xor_sync(kFull, rd, o);
          if (ov > rv || (ov == rv && (od < rd || (od == rd && oj < rj)))) {
            rv = ov;
            rj = oj;
            rd = od;
          }
        }
        if (rv > cv || (rv == cv && rd < abs(ci - m))) {
          p1 = n;
          p2 = rj;
          seg = m - rj;
        }
      }
    }

    // Traceback (reference.rs:144-203), lane 0.
    if (lane == 0) {
      // Elements last to first, reversed at the end.
      int e = 0;
      if (seg > 0 && a.strategy == kSwSoftClip) {
        cig[e++] = (static_cast<uint32_t>(seg) << 4) | kSwOpS;
        seg = 0;
      }
      uint32_t state = kSwOpM;
      do {
        const uint32_t byte = sc.at(p1, p2);
        const uint32_t dir = byte & 3u;
        uint32_t next;
        int step = 1;
        if (dir == 2) {
          next = kSwOpD;
          // GATK's gap length: one more than the run of extending cells above (row 1 always opens).
          for (int q = p1; q > 1 && (sc.at(q, p2) & kExtV); --q) ++step;
          p1 -= step;
        } else if (dir == 1) {
          next = kSwOpI;
          for (int q = p2; q > 1 && (sc.at(p1, q) & kExtH); --q) ++step;
          p2 -= step;
        } else {
          next = kSwOpM;
          p1 -= 1;
          p2 -= 1;
        }
        if (next == state) {
          seg += step;
        } else {
          if (seg > 0) cig[e++] = (static_cast<uint32_t>(seg) << 4) | state;
          seg = step;
          state = next;
        }
      } while (p1 > 0 && p2 > 0);
      int off = 0;
      if (a.strategy == kSwSoftClip) {
        cig[e++] = (static_cast<uint32_t>(seg) << 4) | state;
        if (p2 > 0) cig[e++] = (static_cast<uint32_t>(p2) << 4) | kSwOpS;
        off = p1;
      } else if (a.strategy == kSwIgnore) {
        cig[e++] = (static_cast<uint32_t>(seg + p2) << 4) | state;
        off = p1 - p2;
      } else {
        cig[e++] = (static_cast<uint32_t>(seg) << 4) | state;
        if (p1 > 0)
          cig[e++] = (static_cast<uint32_t>(p1) << 4) | kSwOpD;
        else if (p2 > 0)
          cig[e++] = (static_cast<uint32_t>(p2) << 4) | kSwOpI;
      }
      for (int x = 0, y = e - 1; x < y; ++x, --y) {
        const uint32_t tmp = cig[x];
        cig[x] = cig[y];
        cig[y] = tmp;
      }
      a.count[k] = e;
      a.offset[k] = off;
    }
    __syncwarp();
  }
}

// Packs every pair's CIGAR elements (counts[k] of them from cigar_slot[k]) into one dense run,
// pair after pair, so the host downloads only the elements the batch produced rather than every
// slot's capacity. One block: each thread sums a contiguous share of the counts, the block scans the
// 1024 sums, each thread then copies its share's pairs.
constexpr int kCompactThreads = 1024;
__global__ void __launch_bounds__(kCompactThreads) sw_compact_kernel(const uint32_t* cigar, const int64_t* slot, const int32_t* count,
                                                                     int n_pairs, uint32_t* packed) {
  __shared__ int64_t warp_sum[kCompactThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int64_t share = (static_cast<int64_t>(n_pairs) + kCompactThreads - 1) / kCompactThreads;
  const int64_t lo = min(static_cast<int64_t>(n_pairs), tid * share), hi = min(static_cast<int64_t>(n_pairs), lo + share);
  int64_t own = 0;
  for (int64_t k = lo; k < hi; ++k) own += count[k];
  // Exclusive scan of the per-thread sums: within each warp, then over the warps.
  int64_t incl = own;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t v = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_sum[w] = incl;
  __syncthreads();
  if (w == 0) {
    int64_t ws = warp_sum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t v = __shfl_up_sync(kFull, ws, o);
      if (lane >= o) ws += v;
    }
    warp_sum[lane] = ws;  // inclusive over the warps
  }
  __syncthreads();
  int64_t pos = (w > 0 ? warp_sum[w - 1] : 0) + incl - own;
  for (int64_t k = lo; k < hi; ++k) {
    const uint32_t* src = cigar + slot[k];
    for (int i = 0; i < count[k]; ++i) packed[pos + i] = src[i];
    pos += count[k];
  }
}

}  // namespace

size_t sw_scratch_bytes(int64_t ref_len, int64_t alt_len) { return SwScratch::bytes(ref_len, alt_len); }

cudaError_t sw_compact(const uint32_t* cigar, const int64_t* slot, const int32_t* count, int n_pairs, uint32_t* packed,
                       cudaStream_t stream) {
  if (n_pairs <= 0) return cudaSuccess;
  sw_compact_kernel<<<1, kCompactThreads, 0, stream>>>(cigar, slot, count, n_pairs, packed);
  return cudaGetLastError();
}

void sw_occupancy(int* blocks_per_sm, int* threads_per_block) {
  *threads_per_block = kWarpsPerBlock * 32;
  static std::atomic<int> cache[kMaxDevices];
  *blocks_per_sm = resident_blocks(sw_kernel, 0, kWarpsPerBlock * 32, cache);
}

cudaError_t sw_launch(int blocks, const SwArgs& a, cudaStream_t stream) {
  sw_kernel<<<blocks, kWarpsPerBlock * 32, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace fgkl
