// Device-program layout shared by the host planner and the sm_100a kernels.
//
// A region (one PairHMM call: R reads x H haplotypes) is planned on the host into a "program": a
// column stream that every read of the region walks through, one warp per read task. Each stream
// entry is one DP column of one sorted haplotype (forward) or one backward column of one suffix
// sweep (backward); its low byte is the prior code of the haplotype base the column emits and its
// high byte carries the events the lane handles at that column. Per-segment and per-sweep details
// live in side tables consumed in stream order, so a lane only needs running counters.
#pragma once
#include <cstdint>

namespace fgkl {

// ---- stream entry bits (uint16_t) ----
constexpr uint16_t kCodeMask = 0x00FF;
constexpr uint16_t EV_BEGIN = 1u << 8;   // forward: load the segment's start column before computing
constexpr uint16_t EV_SNAP = 1u << 9;    // forward: store the column into the next snapshot slot
constexpr uint16_t EV_END = 1u << 10;    // forward: finish the segment (result or join) after computing
constexpr uint16_t EV_NOCOMP = 1u << 11; // forward: zero-length segment, no column computed
constexpr uint16_t EV_SWEEP = 1u << 12;  // backward: load the sweep's start node before computing
constexpr uint16_t EV_NODE = 1u << 13;   // backward: store a backward node after computing
constexpr uint16_t kEvMask = 0xFF00;

// Prior code of haplotype 'N' (codes 0..4 are A, C, G, T, N; extra bytes follow in first-seen
// order, kernel.rs:27-107).
constexpr int kCodeN = 4;
constexpr uint8_t kNoCode = 0xFF;

// One forward run of a distinct sorted haplotype: columns start+1..=stop, resumed from a snapshot
// slot (or the origin) and either finished or joined with a backward node at column stop+1.
struct Segment {
  int32_t slot_in;   // snapshot slot holding column `start`; -1 = origin (column 0)
  int32_t node;      // backward node joined at the cut; -1 = no cut
  int32_t hap;       // sorted haplotype index
  int32_t cut_code;  // prior code of the haplotype base at the cut column
  float scale_f;     // src_len / hap_len, narrowed like kernel.rs:641
  float init_f;      // 2^120 / hap_len narrowed to f32 (kernel.rs:640)
  double scale_d;    // src_len / hap_len in f64
  double init_d;     // 2^1020 / hap_len
};

// Offsets of one program inside the batch-global arrays.
struct Program {
  int32_t fwd_off, fwd_len;    // forward stream entries
  int32_t bwd_off, bwd_len;    // backward stream entries (0 = no suffix sharing)
  int32_t seg_off, n_segs;     // segments, forward stream order
  int32_t snap_off, n_snaps;   // snapshot slot ids written, forward stream order
  int32_t nodew_off, n_nodew;  // backward node ids written, backward stream order
  int32_t sweep_off, n_sweeps; // start node per sweep (-1 = the all-zero column beyond the end)
  int32_t n_slots, n_nodes;
};

struct Region {
  Program shared;   // prefix + suffix sharing (first pass)
  Program prefix;   // prefix sharing only (double-precision recomputation)
  int32_t hap_off;  // into the HapInfo array
  int32_t n_haps;
  int32_t read_off; // first global read index
  int32_t n_reads;
  int64_t out_off;  // first output element (row-major n_reads x n_haps, caller order)
  int32_t code_off; // 256-entry byte -> prior code table
  int32_t pad_;
};

// Per sorted haplotype: where its result goes and where it comes from.
struct HapInfo {
  int32_t order;  // caller's index of the sorted haplotype
  int32_t seg;    // segment of the first copy (duplicates share it)
  int32_t src;    // sorted index of the first copy
  int32_t pad_;
};

// One warp's unit of work: one or two reads of a region, with R rows per lane (32 * R > length).
struct Task {
  int32_t region;
  int32_t read[2];  // global read indices; read[1] = -1 when the task holds one read
  int32_t rows;     // R
};

// Per-pass counters written by the kernels.
struct Counters {
  unsigned long long lost_pairs;   // pairs handed to the double-precision recomputation
  unsigned long long fwd_columns;  // forward stream positions processed (per read)
  unsigned long long bwd_columns;  // backward stream positions processed (per read)
  unsigned long long rescue_reads; // reads queued for recomputation
};

// Flattened batch: everything a kernel needs, as device pointers.
struct BatchView {
  const uint8_t* bases;
  const uint8_t* quals;
  const uint8_t* ins;
  const uint8_t* del;
  const uint8_t* gcp;
  const int64_t* read_off;   // global read -> first byte
  const Region* regions;
  const HapInfo* haps;
  const uint16_t* stream;
  const Segment* segs;
  const int32_t* snap_slots;
  const int32_t* node_writes;
  const int32_t* sweep_starts;
  const uint8_t* code_of_byte;
  const double* err_prob;     // 255 entries
  const double* m2m;          // triangular table, 32640 entries
  double* out;
  Counters* counters;
};

}  // namespace fgkl
