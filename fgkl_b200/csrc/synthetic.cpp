#include "synthetic.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <thread>

#include "tables.h"

namespace fgkl {

namespace {

constexpr uint8_t kSnp = 1, kDelStart = 2, kDelEnd = 4, kAltA = 8, kAltC = 16, kAltG = 32, kAltT = 64;

// sample_read, synthetic.rs:312-334.
SynthRead sample_read(Rng& rng, const std::vector<uint8_t>& source, size_t read_len) {
  size_t len = read_len;
  if (rng.chance(0.3)) len = 1 + rng.below(read_len);
  len = std::min(len, source.size());
  const size_t start = rng.below(source.size() - len + 1);
  SynthRead r;
  r.bases.assign(source.begin() + static_cast<long>(start), source.begin() + static_cast<long>(start + len));
  for (auto& b : r.bases) {
    if (rng.chance(0.002))
      b = 'N';
    else if (rng.chance(0.01))
      b = rng.base();
    r.quals.push_back(static_cast<uint8_t>(rng.chance(0.05) ? 2 + rng.below(15) : 20 + rng.below(21)));
    r.ins.push_back(static_cast<uint8_t>(rng.chance(0.1) ? 20 + rng.below(30) : 45));
    r.del.push_back(static_cast<uint8_t>(rng.chance(0.1) ? 20 + rng.below(30) : 45));
  }
  r.gcp.assign(len, 10);
  return r;
}

// A read of exactly `len` bases at a random offset of `hap`, qualities uniform 10-40, substitution
// errors at the Phred rate, gap-open 45 and gap continuation 10.
SynthRead phred_read(Rng& rng, const std::vector<uint8_t>& hap, size_t len) {
  len = std::min(len, hap.size());
  const size_t off = rng.below(hap.size() - len + 1);
  SynthRead r;
  r.bases.assign(hap.begin() + static_cast<long>(off), hap.begin() + static_cast<long>(off + len));
  for (auto& b : r.bases) {
    const int q = 10 + static_cast<int>(rng.below(31));
    r.quals.push_back(static_cast<uint8_t>(q));
    if (rng.chance(std::pow(10.0, -q / 10.0))) {
      uint8_t nb = rng.base();
      while (nb == b) nb = rng.base();
      b = nb;
    }
  }
  r.ins.assign(len, 45);
  r.del.assign(len, 45);
  r.gcp.assign(len, 10);
  return r;
}

std::vector<uint8_t> random_window(Rng& rng, size_t len) {
  std::vector<uint8_t> w(len);
  for (auto& b : w) b = rng.base();
  return w;
}

// The reference window with 0-3 SNPs and 0-2 indels of 1-5 bp.
std::vector<uint8_t> variant_hap(Rng& rng, const std::vector<uint8_t>& ref) {
  std::vector<uint8_t> h = ref;
  const size_t snps = rng.below(4), indels = rng.below(3);
  for (size_t s = 0; s < snps; ++s) {
    const size_t pos = rng.below(h.size());
    uint8_t nb = rng.base();
    while (nb == h[pos]) nb = rng.base();
    h[pos] = nb;
  }
  for (size_t i = 0; i < indels; ++i) {
    const size_t l = 1 + rng.below(5);
    if (rng.chance(0.5)) {
      const size_t pos = rng.below(h.size() + 1);
      std::vector<uint8_t> ins(l);
      for (auto& b : ins) b = rng.base();
      h.insert(h.begin() + static_cast<long>(pos), ins.begin(), ins.end());
    } else if (h.size() > l + 1) {
      const size_t pos = rng.below(h.size() - l + 1);
      h.erase(h.begin() + static_cast<long>(pos), h.begin() + static_cast<long>(pos + l));
    }
  }
  return h;
}

uint64_t region_seed(uint64_t seed, uint64_t region) {
  Rng r(seed * 0x2545F4914F6CDD1Dull + region * 0x9E3779B97F4A7C15ull + 0x1234567ull);
  return r.next_u64();
}

SynthRegion gen_plain(Rng& rng, size_t n_reads, const std::vector<size_t>& read_lens, size_t n_haps, size_t ref_len) {
  SynthRegion reg;
  const auto ref = random_window(rng, ref_len);
  for (size_t h = 0; h < n_haps; ++h) reg.haps.push_back(variant_hap(rng, ref));
  for (size_t r = 0; r < n_reads; ++r) {
    const auto& hap = reg.haps[rng.below(n_haps)];
    reg.reads.push_back(phred_read(rng, hap, read_lens[r]));
  }
  return reg;
}

SynthRegion gen_region(int which, uint64_t seed) {
  Rng rng(seed);
  switch (which) {
    case 0:
      return gen_plain(rng, 32, std::vector<size_t>(32, 151), 4, 300);
    case 4:
      return gen_plain(rng, 64, std::vector<size_t>(64, 151), 8, 350);
    case 1: {
      const size_t n_reads = 8 + rng.below(249), n_haps = 2 + rng.below(31);
      std::vector<size_t> lens(n_reads);
      size_t max_len = 0;
      for (auto& l : lens) {
        l = rng.chance(0.75) ? 151 : 50 + rng.below(201);
        max_len = std::max(max_len, l);
      }
      return gen_plain(rng, n_reads, lens, n_haps, max_len + 50 + rng.below(351));
    }
    case 2: {
      SynthRegion reg;
      const auto ref = random_window(rng, 400);
      reg.haps.push_back(ref);
      while (reg.haps.size() < 128) {
        auto h = ref;
        const size_t snps = 1 + rng.below(3);
        for (size_t s = 0; s < snps; ++s) {
          const size_t pos = 200 + rng.below(140);
          uint8_t nb = rng.base();
          while (nb == h[pos]) nb = rng.base();
          h[pos] = nb;
        }
        reg.haps.push_back(std::move(h));
      }
      for (size_t r = 0; r < 200; ++r) reg.reads.push_back(phred_read(rng, reg.haps[rng.below(128)], 151));
      return reg;
    }
    case 3: {
      SynthRegion reg;
      const auto ref = random_window(rng, 350);
      std::vector<std::vector<uint8_t>> realized;
      for (size_t k = 0; k < 16; ++k) {
        auto bases = ref;
        if (k > 0 && rng.chance(0.5)) {
          const size_t pos = rng.below(bases.size());
          uint8_t nb = rng.base();
          while (nb == bases[pos]) nb = rng.base();
          bases[pos] = nb;
        }
        const size_t n = bases.size();
        std::vector<uint8_t> flags(n, 0), alt = bases;
        std::vector<bool> deleted(n, false);
        for (size_t p = 0; p < n; ++p) {
          if (flags[p] != 0) continue;
          const double u = static_cast<double>(rng.next_u64() >> 11) / static_cast<double>(1ull << 53);
          if (u < 0.05) {
            const int mask = 1 + static_cast<int>(rng.below(15));
            uint8_t f = kSnp;
            const uint8_t alts[4] = {kAltA, kAltC, kAltG, kAltT};
            std::vector<uint8_t> choices;
            for (int bit = 0; bit < 4; ++bit)
              if (mask & (1 << bit)) {
                f |= alts[bit];
                choices.push_back("ACGT"[bit]);
              }
            flags[p] = f;
            alt[p] = choices[rng.below(choices.size())];
          } else if (u < 0.07) {
            const size_t len = std::min<size_t>(1 + rng.below(10), n - p);
            bool free_span = true;
            for (size_t q = p; q < p + len; ++q) free_span &= flags[q] == 0;
            if (!free_span) continue;
            flags[p] |= kDelStart;
            flags[p + len - 1] |= kDelEnd;
            for (size_t q = p; q < p + len; ++q) deleted[q] = true;
            p += len - 1;
          }
        }
        std::vector<uint8_t> allele;
        for (size_t p = 0; p < n; ++p)
          if (!deleted[p]) allele.push_back(alt[p]);
        realized.push_back(allele.empty() ? bases : allele);
        reg.haps.push_back(std::move(bases));
        reg.flags.push_back(std::move(flags));
      }
      for (size_t r = 0; r < 64; ++r) {
        const size_t k = rng.below(16);
        const auto& src = rng.chance(0.5) ? realized[k] : reg.haps[k];
        reg.reads.push_back(phred_read(rng, src, 151));
      }
      return reg;
    }
    default:
      throw std::invalid_argument("unknown workload");
  }
}

}  // namespace

void SynthBatch::append(const SynthRegion& r) {
  for (const auto& rd : r.reads) {
    bases.insert(bases.end(), rd.bases.begin(), rd.bases.end());
    quals.insert(quals.end(), rd.quals.begin(), rd.quals.end());
    ins.insert(ins.end(), rd.ins.begin(), rd.ins.end());
    del.insert(del.end(), rd.del.begin(), rd.del.end());
    gcp.insert(gcp.end(), rd.gcp.begin(), rd.gcp.end());
    read_off.push_back(static_cast<int64_t>(bases.size()));
  }
  for (size_t h = 0; h < r.haps.size(); ++h) {
    hap_bases.insert(hap_bases.end(), r.haps[h].begin(), r.haps[h].end());
    if (!r.flags.empty()) {
      hap_flags.insert(hap_flags.end(), r.flags[h].begin(), r.flags[h].end());
      pd = true;
    } else {
      hap_flags.insert(hap_flags.end(), r.haps[h].size(), 0);
    }
    hap_off.push_back(static_cast<int64_t>(hap_bases.size()));
  }
  region_reads.push_back(static_cast<int32_t>(r.reads.size()));
  region_haps.push_back(static_cast<int32_t>(r.haps.size()));
}

std::vector<uint8_t> reference_edited(Rng& rng, const std::vector<uint8_t>& alphabet, const std::vector<uint8_t>& base) {
  std::vector<uint8_t> hap = base;
  const size_t edits = 1 + rng.below(3);
  for (size_t e = 0; e < edits; ++e) {
    const size_t pos = rng.below(hap.size());
    switch (rng.below(3)) {
      case 0:
        hap[pos] = alphabet[rng.below(alphabet.size())];
        break;
      case 1:
        hap.insert(hap.begin() + static_cast<long>(pos), alphabet[rng.below(alphabet.size())]);
        break;
      default:
        if (hap.size() > 1) hap.erase(hap.begin() + static_cast<long>(pos));
        break;
    }
  }
  return hap;
}

SynthRegion reference_region(uint64_t seed, size_t num_reads, size_t read_len, size_t num_haps, size_t hap_len) {
  Rng rng(seed);
  SynthRegion reg;
  std::vector<uint8_t> reference(hap_len);
  for (auto& b : reference) b = rng.base();
  reg.haps.push_back(reference);
  while (reg.haps.size() < num_haps) {
    if (reg.haps.size() > 1 && rng.chance(0.1)) {
      auto dup = reg.haps[rng.below(reg.haps.size())];
      reg.haps.push_back(std::move(dup));
      continue;
    }
    auto hap = reference;
    const size_t edits = 1 + rng.below(3);
    for (size_t e = 0; e < edits; ++e) {
      const size_t pos = rng.below(hap.size());
      switch (rng.below(3)) {
        case 0: {
          const uint8_t old = hap[pos];
          uint8_t nb = rng.base();
          while (nb == old) nb = rng.base();
          hap[pos] = nb;
          break;
        }
        case 1: {
          const size_t n = 1 + rng.below(5);
          std::vector<uint8_t> ins(n);
          for (auto& b : ins) b = rng.base();
          hap.insert(hap.begin() + static_cast<long>(pos), ins.begin(), ins.end());
          break;
        }
        default: {
          const size_t end = std::min(pos + 1 + rng.below(5), hap.size());
          if (hap.size() - (end - pos) >= 1) hap.erase(hap.begin() + static_cast<long>(pos), hap.begin() + static_cast<long>(end));
          break;
        }
      }
    }
    reg.haps.push_back(std::move(hap));
  }
  for (size_t r = 0; r < num_reads; ++r) {
    const auto& hap = reg.haps[rng.below(reg.haps.size())];
    reg.reads.push_back(sample_read(rng, hap, read_len));
  }
  return reg;
}

SynthRegion reference_pd_region(uint64_t seed, size_t num_reads, size_t read_len, size_t num_haps, size_t hap_len) {
  Rng rng(seed);
  SynthRegion reg;
  std::vector<uint8_t> reference(hap_len);
  for (auto& b : reference) b = rng.base();
  std::vector<std::vector<uint8_t>> realized;
  for (size_t k = 0; k < num_haps; ++k) {
    auto bases = reference;
    if (k > 0) {
      const size_t edits = rng.below(3);
      for (size_t e = 0; e < edits; ++e) {
        const size_t pos = rng.below(bases.size());
        switch (rng.below(3)) {
          case 0:
            bases[pos] = rng.base();
            break;
          case 1: {
            const size_t n = 1 + rng.below(5);
            std::vector<uint8_t> ins(n);
            for (auto& b : ins) b = rng.base();
            bases.insert(bases.begin() + static_cast<long>(pos), ins.begin(), ins.end());
            break;
          }
          default: {
            const size_t end = std::min(pos + 1 + rng.below(5), bases.size());
            if (bases.size() - (end - pos) >= 2) bases.erase(bases.begin() + static_cast<long>(pos), bases.begin() + static_cast<long>(end));
            break;
          }
        }
      }
    }
    const size_t n = bases.size();
    std::vector<uint8_t> flags(n, 0), alt = bases;
    std::vector<bool> deleted(n, false);
    const size_t events = 1 + rng.below(4);
    for (size_t e = 0; e < events; ++e) {
      const size_t pos = rng.below(n);
      if (flags[pos] != 0) continue;
      if (rng.chance(0.5)) {
        size_t mask;
        do {
          mask = rng.below(16);
        } while (mask == 0);
        uint8_t flag = kSnp;
        const uint8_t alts[4] = {kAltA, kAltC, kAltG, kAltT};
        std::vector<uint8_t> choices;
        for (int bit = 0; bit < 4; ++bit)
          if (mask & (1u << bit)) {
            flag |= alts[bit];
            choices.push_back("ACGT"[bit]);
          }
        flags[pos] = flag;
        alt[pos] = choices[rng.below(choices.size())];
      } else {
        const size_t len = std::min<size_t>(1 + rng.below(8), n - pos);
        bool busy = false;
        for (size_t q = pos; q < pos + len; ++q) busy |= flags[q] != 0;
        if (busy) continue;
        flags[pos] |= kDelStart;
        flags[pos + len - 1] |= kDelEnd;
        for (size_t q = pos; q < pos + len; ++q) deleted[q] = true;
      }
    }
    std::vector<uint8_t> allele;
    for (size_t p = 0; p < n; ++p)
      if (!deleted[p]) allele.push_back(alt[p]);
    realized.push_back(allele.empty() ? bases : allele);
    reg.haps.push_back(std::move(bases));
    reg.flags.push_back(std::move(flags));
  }
  for (size_t r = 0; r < num_reads; ++r) {
    const size_t k = rng.below(num_haps);
    const auto& source = rng.chance(0.5) ? realized[k] : reg.haps[k];
    reg.reads.push_back(sample_read(rng, source, read_len));
  }
  return reg;
}

SynthBatch config_batch(int which, uint64_t seed, int regions, int threads) {
  static const int kDefault[5] = {1, 4096, 512, 1024, 256};
  if (which < 0 || which > 4) throw std::invalid_argument("unknown workload");
  const int n = regions > 0 ? regions : kDefault[which];
  std::vector<SynthRegion> out(static_cast<size_t>(n));
  if (threads < 1) threads = 1;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      for (int g = t; g < n; g += threads)
        out[static_cast<size_t>(g)] = gen_region(which, n == 1 ? seed : region_seed(seed, static_cast<uint64_t>(g)));
    });
  for (auto& th : pool) th.join();
  SynthBatch b;
  for (const auto& r : out) b.append(r);
  b.pd = (which == 3);
  return b;
}

}  // namespace fgkl
