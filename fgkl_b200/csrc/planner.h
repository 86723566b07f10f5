// Host-side haplotype sorter and sharing planner.
//
// Restates, bit for bit, fgkl's plain-kernel planning:
//   SortedHaps::new        crates/pairhmm/src/kernel.rs:53-81   (stable lexicographic sort, LCP,
//                                                                duplicate flags, prior codes)
//   SuffixPlan::new        crates/pairhmm/src/plan.rs:61-89     (cut depths, backward sweeps, node
//                                                                numbering; MIN_SAVING = 4)
//   SharedColumns          crates/pairhmm/src/plan.rs:93-113
//   SortedPdHaps::new      crates/pairhmm/src/pd_kernel.rs:61-136 (sort by row-end deletion state,
//                                                                then interleaved bases and flags; LCP
//                                                                only between equal end states;
//                                                                match-set codes)
//   segments, MatchSet     crates/pairhmm/src/pd_kernel.rs:699-723, :196-214
// and turns the result into the column stream the sm_100a kernels walk (program.h).
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

#include "program.h"

namespace fgkl {

struct HapView {
  const uint8_t* bases;
  int32_t len;
};

struct Cut {
  int32_t column;  // forward sweep stops at column - 1 and joins backward node `node` at `column`
  int32_t node;
};

struct BackwardSweep {
  int32_t hap;     // sorted index of the haplotype whose bases the sweep follows
  int32_t resume;  // depth of the start node
  int32_t need;    // deepest depth computed
  int32_t start;   // node holding depth `resume`
  std::vector<std::pair<int32_t, int32_t>> writes;  // (depth, node), ascending
};

struct SuffixPlan {
  std::vector<Cut> cuts;  // per sorted haplotype; column == -1 means no cut
  std::vector<BackwardSweep> sweeps;
  int32_t nodes = 1;
};

struct SharedColumns {
  uint64_t prefix_only = 0, forward = 0, backward = 0;
};

// PD flag bits of a haplotype base (fgkl pd.rs:13-27).
constexpr uint8_t kPdSnp = 1, kPdDelStart = 2, kPdDelEnd = 4, kPdAltA = 8, kPdAltC = 16, kPdAltG = 32, kPdAltT = 64;

// Whether a read base matches the alternates a flag byte names (pd.rs:99-110).
bool base_matches_pd(uint8_t read_base, uint8_t flags);

// The read bases a PD column accepts: its own base and, with SNP, the flagged alternates
// (pd_kernel.rs:196-214).
struct MatchSet {
  uint8_t base;
  uint8_t alts;  // ALT bits; zero without SNP
  static MatchSet of(uint8_t base, uint8_t flag);
  bool accepts(uint8_t read_base) const;
  bool operator==(const MatchSet& o) const { return base == o.base && alts == o.alts; }
};

// Deletion state of each of a row's `len` columns when the row starts in `state` (kPdNormal,
// kPdInsideDel, kPdAfterDel); returns the state carried out of the last column
// (pd_kernel.rs:699-723).
uint8_t pd_row_states(const uint8_t* flags, int32_t len, uint8_t state, uint8_t* out);

struct SortedHaps {
  std::vector<int32_t> order;  // order[k] = caller index of sorted haplotype k
  std::vector<HapView> bases;  // sorted
  std::vector<std::vector<uint8_t>> codes;
  std::vector<int32_t> lcp;
  std::vector<uint8_t> dup;
  std::vector<uint8_t> extra_bases;  // bytes outside ACGTN, first-seen order over sorted haplotypes
  int32_t max_len = 0;
  SuffixPlan plan;
  // PD-HMM sets only (make_pd): codes index match_sets; pd_bits holds each column's deletion bits
  // as forward-entry bits (program.h); end_state is the state every row after the first starts in.
  bool pd = false;
  std::vector<const uint8_t*> flags;
  std::vector<MatchSet> match_sets;
  std::vector<std::vector<uint32_t>> pd_bits;
  std::vector<uint8_t> end_state;
  // More than 256 distinct match sets: codes do not fit the stream's code byte and are left zero;
  // such a region compares bytes instead (the entries then carry base and ALT bits).
  bool too_many_sets = false;

  static SortedHaps make(const std::vector<HapView>& haps, bool share_suffixes);
  // Prefix sharing only, as fgkl's PD kernel.
  static SortedHaps make_pd(const std::vector<HapView>& haps, const std::vector<const uint8_t*>& flags);
  int num_codes() const { return pd ? static_cast<int>(match_sets.size()) : 5 + static_cast<int>(extra_bases.size()); }
  uint8_t byte_of_code(int code) const;
  SharedColumns columns() const;
};

// Host copy of one program (program.h), before it is concatenated into a batch. Streams hold only
// the entries of positions 0..n (the last carries the post events of the final column); the
// kStreamPad zero entries around them are added when the batch is assembled.
struct ProgramBuild {
  std::vector<uint32_t> fwd, bwd;
  std::vector<Segment> segs;
  std::vector<Sweep> sweeps;
  int32_t n_slots = 0, n_nodes = 0;
  // Σ(forward columns) and Σ(backward columns) per read row, for the computed-cell count.
  uint64_t fwd_columns = 0, bwd_columns = 0;
};

// The forward (and, with `with_suffix`, backward) column stream of a sorted haplotype set.
//
// Snapshot placement: a segment resuming at column q reads the value the LAST earlier segment
// passing q wrote (the semantics of fgkl's per-column snapshot array, kernel.rs:254-259, :656-662),
// so each snapshot is written once, by that last writer: into the staging buffer when the very next
// segment reads it, and into a global slot when a later one does (prefetched into staging at the
// BEGIN of the segment before its reader).
void emit_program(const SortedHaps& s, bool with_suffix, ProgramBuild& out);

// 256-entry byte -> prior code table of a sorted set (kNoCode for bytes no haplotype holds that
// are not A, C, G, T or N).
void code_table(const SortedHaps& s, uint8_t out[256]);

}  // namespace fgkl
