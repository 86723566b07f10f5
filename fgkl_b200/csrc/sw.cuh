// Launch interface of the sm_100a Smith-Waterman kernel (sw.cu): GATK's SmithWatermanJavaAligner
// as fgkl restates it (crates/smithwaterman/src/reference.rs:9-203, lib.rs), over a batch of
// (reference, alternate) pairs.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace fgkl {

// Overhang strategies, numbered as fgkl's JNI entry numbers them (crates/jni/src/lib.rs:290-296).
enum SwStrategy : int { kSwSoftClip = 0, kSwIndel = 1, kSwLeadingIndel = 2, kSwIgnore = 3 };

// CIGAR element: length << 4 | operation, operations numbered as in BAM.
constexpr uint32_t kSwOpM = 0, kSwOpI = 1, kSwOpD = 2, kSwOpS = 4;

constexpr int kSwRows = 8;  // reference rows per lane; a row block is 32 * 8 = 256 rows

struct SwArgs {
  const uint8_t* ref;
  const int64_t* ref_off;  // n_pairs + 1
  const uint8_t* alt;
  const int64_t* alt_off;  // n_pairs + 1
  const int32_t* order;    // pairs, costliest first
  int n_pairs;
  int match, mismatch, open, extend;  // GATK's SWParameters
  int strategy;
  char* scratch;           // per warp: sw_scratch_bytes of the batch's largest pair
  size_t stride;
  uint32_t* cigar;         // pair k's elements from cigar_slot[k] (capacity ref + alt + 2)
  const int64_t* cigar_slot;
  int32_t* count;          // elements per pair
  int32_t* offset;         // GATK's alignmentOffset per pair
  int* counter;            // zero before the launch
};

// Per-warp scratch for a pair of a `ref_len` reference and `alt_len` alternate: the traceback bytes
// of every row block, the last column and last row scores, and the row one block hands the next.
size_t sw_scratch_bytes(int64_t ref_len, int64_t alt_len);
void sw_occupancy(int* blocks_per_sm, int* threads_per_block);
cudaError_t sw_launch(int blocks, const SwArgs& a, cudaStream_t stream);
// Packs the pairs' CIGAR elements, pair after pair, into `packed` (as many elements as the counts
// sum to), after sw_launch on the same stream.
cudaError_t sw_compact(const uint32_t* cigar, const int64_t* slot, const int32_t* count, int n_pairs, uint32_t* packed,
                       cudaStream_t stream);

}  // namespace fgkl
