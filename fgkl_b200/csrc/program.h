// Device-program layout shared by the host planner and the sm_100a kernels.
//
// A region (one PairHMM call: R reads x H haplotypes) is planned on the host into a program that
// every read of the region walks, one warp per read task. The forward stream holds one 32-bit entry
// per DP column of each distinct sorted haplotype; the backward stream one per backward column of
// each suffix sweep. An entry's low byte is the prior code of the haplotype base the column emits;
// its flags name the events a lane handles when it reaches the entry: events that load or keep state
// before the entry's own column is computed (BEGIN, ACC, SWEEP), and events that store the state of
// the PREVIOUS column (SNAP, END, JOIN, NODE). Deferring the stores by one column lets the lane handle every event of a step
// in one branch before computing. Each stream is padded with kStreamPad zero entries on both sides
// so lanes ahead of or behind the wavefront read harmless entries without bounds checks.
#pragma once
#include <cstdint>

namespace fgkl {

constexpr int kStreamPad = 64;

// ---- stream entry bits (uint32_t) ----
constexpr uint32_t kCodeMask = 0xFFu;
// forward
constexpr uint32_t EV_BEGIN = 1u << 8;    // load the segment's start column before computing this one
constexpr uint32_t EV_ACC = 1u << 9;      // this column is a cut column: keep the result so far first
constexpr uint32_t EV_SNAP = 1u << 10;    // the previous column is a snapshot (payload: slot, staging)
constexpr uint32_t EV_END = 1u << 11;     // the previous column ended the segment
constexpr uint32_t EV_STAGE = 1u << 12;   // the snapshot also goes to the staging buffer of the next segment
constexpr uint32_t EV_JOIN = 1u << 13;    // the previous column is a cut column: keep its M and Y rows
// backward
constexpr uint32_t EV_SWEEP = 1u << 8;    // load the sweep's start node before computing this column
constexpr uint32_t EV_NODE = 1u << 10;    // the previous column is a backward node (payload: node id)
constexpr uint32_t EV_NSTAGE = 1u << 12;  // the node also goes to the staging buffer of the next sweep
constexpr uint32_t kEvMask = 0x3F00u;
constexpr int kPayloadShift = 14;
constexpr uint32_t kPayloadNone = (1u << (32 - kPayloadShift)) - 1;  // no global slot

// PD-HMM forward entries (no suffix sharing, so ACC, JOIN and the backward events are unused) also
// carry the column's deletion handling, which depends only on the flags (fgkl pd_kernel.rs:1-22):
// the deletion state of the column in the read's first row and in every later row (rows after the
// first start in the state the previous row ended in), whether the column carries DEL_END, and
// whether it carries DEL_START or DEL_END, so its branch values must be kept. Their slot payload
// starts higher up.
constexpr uint32_t PD_MAT = 1u << 14;  // keep the column's branch values (DEL_START or DEL_END)
constexpr uint32_t PD_DE = 1u << 15;   // DEL_END: insertion from the branch values above
constexpr int kPdFirstShift = 16;      // 2 bits: deletion state in the read's first row
constexpr int kPdLaterShift = 18;      // 2 bits: deletion state in the later rows
constexpr uint32_t kPdNormal = 0, kPdInsideDel = 1, kPdAfterDel = 2;
// Any column a PD lane cannot compute with the plain recurrence. The column after DEL_END (AFTER_DEL
// in every row) is not one of them: its max merges are taken at the DEL_END column itself.
constexpr uint32_t kPdSlowMask = PD_MAT | PD_DE;
constexpr int kPdPayloadShift = 20;
constexpr uint32_t kPdPayloadNone = (1u << (32 - kPdPayloadShift)) - 1;
// Read bytes a PD region distinguishes (classes 0..30; 31 marks a padding row).
constexpr int kPdMaxReadClasses = 31;

// Prior code of haplotype 'N' (codes 0..4 are A, C, G, T, N; extra bytes follow in first-seen
// order, fgkl kernel.rs:27-107).
constexpr int kCodeN = 4;
constexpr uint8_t kNoCode = 0xFF;

// One forward run of a distinct sorted haplotype: columns start+1..=stop resumed from its start
// column (the origin or a staged snapshot), then either finished or, for a cut, continued through
// the cut column, whose match and deletion rows are joined with backward node `node`.
//
// The recurrence is linear in the row-0 constant INITIAL / length. fgkl rescales a snapshot at every
// resume (kernel.rs:641, :673-678). Here a sharing tree (a segment from the origin and every segment
// that resumes from it, directly or not) runs at one constant, INITIAL / tree_len with tree_len its
// longest haplotype's length, and each raw result is multiplied by tree_len / hap_len at the end, so
// a resume costs nothing (rescaling at each resume, inside the event windows, cost 5.5% on 4096
// uneven regions). No value then exceeds what its own haplotype's recurrence reaches, so nothing
// overflows that fgkl's does not. A tree kept at its first haplotype's constant overflows when that
// one is much shorter (a one-base haplotype prefixing a long one, with short reads). A member shorter
// than its tree's longest runs that ratio below fgkl's scale. That matters only where 2^1020 L is an
// FP64 subnormal (log10 L below -614.7), where fgkl's own value has lost precision too; equal lengths
// run at fgkl's own scale.
struct Segment {
  double factor;      // tree_len / hap_len
  float init_f;       // 2^120 / tree_len narrowed to f32 (kernel.rs:640), for origin segments
  int32_t staged;     // 1: start from the staging buffer; 0: from the origin (column 0)
  double init_d;      // 2^1020 / tree_len
  int32_t next_slot;  // global snapshot slot to prefetch for the NEXT segment at this BEGIN, or -1
  int32_t node;       // backward node joined at the cut; -1 = no cut
  int32_t hap;        // sorted haplotype index
  int32_t pad_;
};

// One backward sweep (the first of a program computes node 0 from the all-zero column).
struct Sweep {
  int32_t staged;     // 1: start from the staging buffer; 0: all-zero start column
  int32_t next_node;  // global node to prefetch for the NEXT sweep at this SWEEP, or -1
};

// Offsets of one program inside the batch-global arrays (stream offsets point at entry 0).
struct Program {
  int32_t fwd_off, fwd_len;
  int32_t bwd_off, bwd_len;  // bwd_len 0 = no suffix sharing
  int32_t seg_off, n_segs;
  int32_t sweep_off, n_sweeps;
  int32_t n_slots, n_nodes;  // global snapshot slots and backward nodes one read needs
};

struct Region {
  Program prog;     // the first pass: prefix (and, when enabled, suffix) sharing
  int32_t hap_off;  // into the HapInfo array
  int32_t n_haps;
  int32_t read_off; // first global read index
  int32_t n_reads;
  int64_t out_off;  // first output element (row-major n_reads x n_haps, caller order)
  int32_t code_off; // 256-entry byte -> prior code table (PD: read byte -> read class)
  int32_t seq_off;  // sorted haplotypes' prior codes (PD: forward entries), concatenated (recomputation streams)
  int32_t sig_off;  // PD: per match-set code, the bit set of read classes it accepts
  int32_t flags;    // kRegion* bits
};

// Region flags.
constexpr int32_t kRegionGeneric = 1;  // PD: prior by byte comparison (more read bytes than class bits)

// Per sorted haplotype: where its result goes and where it comes from.
struct HapInfo {
  int32_t order;  // caller's index of the sorted haplotype
  int32_t seg;    // segment of the first copy (duplicates share it)
  int32_t src;    // sorted index of the first copy
  int32_t len;    // bases; its codes start at region.seq_off + seq
  int32_t seq;
  int32_t pad_[3];
};

// One warp's unit of work: one or two reads of a region, with R rows per lane (31 * R >= length).
// A recomputation task (hap >= 0) runs one read against one distinct haplotype from the origin,
// without sharing, from a stream synthesised from the haplotype's codes.
struct Task {
  int32_t region;
  int32_t read[2];  // global read indices; read[1] = -1 when the task holds one read
  int32_t rows;     // R
  int32_t hap;      // sorted haplotype of a recomputation task, else -1
};

// Per-pass counters written by the kernels.
struct Counters {
  unsigned long long lost_pairs;   // pairs handed to the double-precision recomputation
  unsigned long long rescue_reads; // (read, distinct haplotype) pairs queued for recomputation
  unsigned long long pad_[2];
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
  const uint32_t* stream;
  const Segment* segs;
  const Sweep* sweeps;
  const uint8_t* code_of_byte;
  const uint8_t* hap_codes;  // sorted haplotypes' codes per region
  const uint32_t* pd_entries;  // PD: sorted haplotypes' forward entries (code and deletion bits) per region
  const uint32_t* pd_sigs;     // PD: accepted read classes per match-set code
  const double* err_prob;     // 255 entries
  const double* m2m;          // triangular table, 32640 entries
  double* out;
  Counters* counters;
};

}  // namespace fgkl
