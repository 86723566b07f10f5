// The benchmark workload generators (fgkl_b200/csrc/synthetic.cpp, which restate fgkl's SplitMix64
// region generators, crates/pairhmm/src/synthetic.rs) compiled into the oracle library, so that the
// timed CPU reference builds its workload without loading the CUDA library. TEST AND BENCHMARK
// INFRASTRUCTURE ONLY.
#include <cstdint>
#include <exception>

#include "synthetic.h"

#define OR_API __attribute__((visibility("default")))

extern "C" {

// The workload `which` (0-4, see synthetic.h); NULL on a bad argument.
OR_API void* or_synth_config(int32_t which, uint64_t seed, int32_t regions, int32_t threads) {
  try {
    return new fgkl::SynthBatch(fgkl::config_batch(which, seed, regions, threads));
  } catch (const std::exception&) {
    return nullptr;
  }
}

// ptrs: region_reads, region_haps, bases, quals, ins, del, gcp, read_off, hap_bases, hap_flags (NULL
// for plain workloads), hap_off. sizes: regions, reads, read bytes, haplotypes, haplotype bytes.
OR_API void or_synth_arrays(const void* h, const void** ptrs, int64_t* sizes) {
  const auto& b = *static_cast<const fgkl::SynthBatch*>(h);
  ptrs[0] = b.region_reads.data();
  ptrs[1] = b.region_haps.data();
  ptrs[2] = b.bases.data();
  ptrs[3] = b.quals.data();
  ptrs[4] = b.ins.data();
  ptrs[5] = b.del.data();
  ptrs[6] = b.gcp.data();
  ptrs[7] = b.read_off.data();
  ptrs[8] = b.hap_bases.data();
  ptrs[9] = b.pd ? b.hap_flags.data() : nullptr;
  ptrs[10] = b.hap_off.data();
  sizes[0] = static_cast<int64_t>(b.region_reads.size());
  sizes[1] = static_cast<int64_t>(b.read_off.size()) - 1;
  sizes[2] = static_cast<int64_t>(b.bases.size());
  sizes[3] = static_cast<int64_t>(b.hap_off.size()) - 1;
  sizes[4] = static_cast<int64_t>(b.hap_bases.size());
}

OR_API void or_synth_free(void* h) { delete static_cast<fgkl::SynthBatch*>(h); }

}  // extern "C"
