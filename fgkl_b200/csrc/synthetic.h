// Deterministic synthetic assembly regions.
//
// `reference_region` and `reference_pd_region` restate fgkl's generators exactly (SplitMix64 and
// the same sequence of draws, crates/pairhmm/src/synthetic.rs:10-41, :84-153, :199-289, :312-334),
// so the regions the reference's own tests use can be rebuilt here from their seeds. The
// `config_*` generators build the benchmark workloads (one function per workload shape).
#pragma once
#include <cstdint>
#include <vector>

namespace fgkl {

class Rng {
 public:
  explicit Rng(uint64_t seed) : s_(seed) {}
  uint64_t next_u64() {
    s_ += 0x9E3779B97F4A7C15ull;
    uint64_t z = s_;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  size_t below(size_t n) { return static_cast<size_t>(next_u64() % static_cast<uint64_t>(n)); }
  bool chance(double p) { return static_cast<double>(next_u64() >> 11) / static_cast<double>(1ull << 53) < p; }
  uint8_t base() { return "ACGT"[below(4)]; }

 private:
  uint64_t s_;
};

struct SynthRead {
  std::vector<uint8_t> bases, quals, ins, del, gcp;
};

struct SynthRegion {
  std::vector<SynthRead> reads;
  std::vector<std::vector<uint8_t>> haps;
  std::vector<std::vector<uint8_t>> flags;  // empty for plain regions
};

// A batch of regions in the flattened layout of the batch API.
struct SynthBatch {
  std::vector<uint8_t> bases, quals, ins, del, gcp;
  std::vector<int64_t> read_off{0};
  std::vector<uint8_t> hap_bases, hap_flags;
  std::vector<int64_t> hap_off{0};
  std::vector<int32_t> region_reads, region_haps;
  bool pd = false;
  void append(const SynthRegion& r);
};

SynthRegion reference_region(uint64_t seed, size_t num_reads, size_t read_len, size_t num_haps, size_t hap_len);
SynthRegion reference_pd_region(uint64_t seed, size_t num_reads, size_t read_len, size_t num_haps, size_t hap_len);
std::vector<uint8_t> reference_edited(Rng& rng, const std::vector<uint8_t>& alphabet, const std::vector<uint8_t>& base);

// Benchmark workloads; `which` selects the shape:
//   0: one region, 32 reads x 151, 4 haplotypes x 300 (0-3 SNPs, 0-2 indels of 1-5 bp each)
//   1: uneven regions: 8-256 reads (75% of length 151, else 50-250) x 2-32 haplotypes whose
//      reference window is the longest read plus 50-400
//   2: 200 reads x 151 against 128 SNP-edited haplotypes of 400 with variants in [200, 340)
//   3: partially determined: 64 reads x 151 against 16 flagged haplotypes of 350
//   4: 64 reads x 151 against 8 haplotypes of 350 (gradient workload)
// `regions` overrides the region count (0 keeps the default: 1, 4096, 512, 1024, 256).
SynthBatch config_batch(int which, uint64_t seed, int regions, int threads);

}  // namespace fgkl
