#include "planner.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <stdexcept>

namespace fgkl {

namespace {

constexpr uint8_t kStandard[5] = {'A', 'C', 'G', 'T', 'N'};
// A backward sweep must skip at least this many forward columns to pay for its join (plan.rs:9).
constexpr int32_t kMinSaving = 4;

// Byte -> ACGTN code (0..4), -1 for any other byte: one table load per haplotype base.
struct StandardCodes {
  int8_t code[256];
  StandardCodes() {
    for (int b = 0; b < 256; ++b) code[b] = -1;
    for (int i = 0; i < 5; ++i) code[kStandard[i]] = static_cast<int8_t>(i);
  }
};
const StandardCodes kStandardCodes;

int standard_code(uint8_t b) { return kStandardCodes.code[b]; }

bool lex_less(const HapView& a, const HapView& b) {
  return std::lexicographical_compare(a.bases, a.bases + a.len, b.bases, b.bases + b.len);
}

// Ordering of the reversed byte strings (plan.rs:128).
bool rev_less(const HapView& a, const HapView& b) {
  const int32_t n = std::min(a.len, b.len);
  for (int32_t i = 0; i < n; ++i) {
    const uint8_t x = a.bases[a.len - 1 - i], y = b.bases[b.len - 1 - i];
    if (x != y) return x < y;
  }
  return a.len < b.len;
}

int32_t common_prefix(const HapView& a, const HapView& b) {
  const int32_t n = std::min(a.len, b.len);
  int32_t i = 0;
  while (i < n && a.bases[i] == b.bases[i]) ++i;
  return i;
}

int32_t common_suffix(const HapView& a, const HapView& b) {
  const int32_t n = std::min(a.len, b.len);
  int32_t i = 0;
  while (i < n && a.bases[a.len - 1 - i] == b.bases[b.len - 1 - i]) ++i;
  return i;
}

bool same(const HapView& a, const HapView& b) {
  return a.len == b.len && std::memcmp(a.bases, b.bases, a.len) == 0;
}

// Distinct haplotypes ordered by reversed bases (plan.rs:116-144).
struct SuffixOrder {
  std::vector<int32_t> order, lcs, pos;

  SuffixOrder(const std::vector<HapView>& bases, const std::vector<int32_t>& distinct) {
    order = distinct;
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t b) { return rev_less(bases[a], bases[b]); });
    lcs.assign(order.size(), 0);
    for (size_t r = 1; r < order.size(); ++r) lcs[r] = common_suffix(bases[order[r - 1]], bases[order[r]]);
    pos.assign(bases.size(), 0);
    for (size_t r = 0; r < order.size(); ++r) pos[order[r]] = static_cast<int32_t>(r);
  }

  int32_t longest_shared(int32_t r) const {
    const int32_t next = (static_cast<size_t>(r) + 1 < lcs.size()) ? lcs[r + 1] : 0;
    return std::max(lcs[r], next);
  }
};

// Node numbering in call order (plan.rs:200-235); ids are deterministic because they depend only on
// the order of node_for calls.
struct NodeNumbering {
  std::map<std::pair<int32_t, int32_t>, int32_t> ids;

  int32_t node_for(const std::vector<BackwardSweep>& sweeps, const std::vector<int32_t>& sweep_at,
                   const std::vector<int32_t>& lcs, int32_t r, int32_t depth) {
    if (depth == 0) return 0;
    int32_t p = r;
    int32_t shared = std::numeric_limits<int32_t>::max();
    for (;;) {
      const int32_t s = sweep_at[p];
      if (s >= 0 && sweeps[s].resume < depth && depth <= sweeps[s].need) {
        auto key = std::make_pair(s, depth);
        auto it = ids.find(key);
        if (it != ids.end()) return it->second;
        const int32_t next = static_cast<int32_t>(ids.size()) + 1;
        ids.emplace(key, next);
        return next;
      }
      shared = std::min(shared, lcs[p]);
      if (!(p > 0 && shared >= depth)) throw std::logic_error("backward depth is never computed");
      --p;
    }
  }
};

SuffixPlan forward_only(size_t n) {
  SuffixPlan p;
  p.cuts.assign(n, Cut{-1, -1});
  p.nodes = 1;
  return p;
}

// SuffixPlan::new, plan.rs:61-89.
SuffixPlan suffix_plan(const std::vector<HapView>& bases, const std::vector<int32_t>& lcp,
                       const std::vector<uint8_t>& dup) {
  const size_t n = bases.size();
  std::vector<int32_t> distinct;
  for (size_t k = 0; k < n; ++k)
    if (!dup[k]) distinct.push_back(static_cast<int32_t>(k));
  SuffixOrder suffixes(bases, distinct);

  // cut_depths, plan.rs:148-168.
  std::vector<int32_t> depth(n, 0);
  for (size_t t = 0; t < distinct.size(); ++t) {
    const int32_t k = distinct[t];
    const int32_t next_lcp = (t + 1 < distinct.size()) ? lcp[distinct[t + 1]] : 0;
    const int32_t shared_prefix = std::max(lcp[k], next_lcp);
    const int32_t len = bases[k].len;
    if (shared_prefix < len) {
      const int32_t d = std::min(suffixes.longest_shared(suffixes.pos[k]), len - shared_prefix - 1);
      if (d >= kMinSaving) depth[k] = d;
    }
  }

  // backward_sweeps, plan.rs:173-196.
  SuffixPlan plan;
  std::vector<int32_t> sweep_at(suffixes.order.size(), -1);
  int32_t reach = 0;
  for (size_t r = 0; r < suffixes.order.size(); ++r) {
    const int32_t k = suffixes.order[r];
    const int32_t resume = std::min(suffixes.lcs[r], reach);
    if (depth[k] > resume) {
      sweep_at[r] = static_cast<int32_t>(plan.sweeps.size());
      plan.sweeps.push_back(BackwardSweep{k, resume, depth[k], 0, {}});
    }
    reach = std::max(resume, depth[k]);
  }

  NodeNumbering numbering;
  std::vector<int32_t> starts;
  for (const auto& s : plan.sweeps)
    starts.push_back(numbering.node_for(plan.sweeps, sweep_at, suffixes.lcs, suffixes.pos[s.hap], s.resume));
  plan.cuts.assign(n, Cut{-1, -1});
  for (int32_t k : distinct) {
    if (depth[k] > 0) {
      const int32_t node = numbering.node_for(plan.sweeps, sweep_at, suffixes.lcs, suffixes.pos[k], depth[k]);
      plan.cuts[k] = Cut{bases[k].len - depth[k], node};
    }
  }
  for (size_t i = 0; i < plan.sweeps.size(); ++i) plan.sweeps[i].start = starts[i];
  for (const auto& [key, node] : numbering.ids) plan.sweeps[key.first].writes.emplace_back(key.second, node);
  for (auto& s : plan.sweeps) std::sort(s.writes.begin(), s.writes.end());
  plan.nodes = static_cast<int32_t>(numbering.ids.size()) + 1;
  return plan;
}

}  // namespace

SortedHaps SortedHaps::make(const std::vector<HapView>& haps, bool share_suffixes) {
  SortedHaps s;
  const size_t n = haps.size();
  s.order.resize(n);
  for (size_t i = 0; i < n; ++i) s.order[i] = static_cast<int32_t>(i);
  std::stable_sort(s.order.begin(), s.order.end(), [&](int32_t a, int32_t b) { return lex_less(haps[a], haps[b]); });
  s.bases.reserve(n);
  for (int32_t i : s.order) s.bases.push_back(haps[i]);
  for (const auto& h : s.bases)
    for (int32_t j = 0; j < h.len; ++j) {
      const uint8_t b = h.bases[j];
      if (standard_code(b) < 0 && std::find(s.extra_bases.begin(), s.extra_bases.end(), b) == s.extra_bases.end())
        s.extra_bases.push_back(b);
    }
  if (s.extra_bases.size() > 250) throw std::invalid_argument("more than 250 distinct non-ACGTN haplotype bytes");
  s.codes.resize(n);
  for (size_t k = 0; k < n; ++k) {
    const HapView& h = s.bases[k];
    s.codes[k].resize(h.len);
    for (int32_t j = 0; j < h.len; ++j) {
      const uint8_t b = h.bases[j];
      const int c = standard_code(b);
      s.codes[k][j] = c >= 0 ? static_cast<uint8_t>(c)
                             : static_cast<uint8_t>(5 + (std::find(s.extra_bases.begin(), s.extra_bases.end(), b) -
                                                         s.extra_bases.begin()));
    }
  }
  s.lcp.assign(n, 0);
  s.dup.assign(n, 0);
  for (size_t k = 1; k < n; ++k) {
    s.lcp[k] = common_prefix(s.bases[k - 1], s.bases[k]);
    s.dup[k] = same(s.bases[k - 1], s.bases[k]) ? 1 : 0;
  }
  for (const auto& h : s.bases) s.max_len = std::max(s.max_len, h.len);
  s.plan = share_suffixes ? suffix_plan(s.bases, s.lcp, s.dup) : forward_only(n);
  return s;
}

bool base_matches_pd(uint8_t read_base, uint8_t flags) {
  if (!(flags & kPdSnp)) return false;
  switch (read_base) {
    case 'A':
    case 'a':
      return flags & kPdAltA;
    case 'C':
    case 'c':
      return flags & kPdAltC;
    case 'G':
    case 'g':
      return flags & kPdAltG;
    case 'T':
    case 't':
      return flags & kPdAltT;
    default:
      return false;
  }
}

MatchSet MatchSet::of(uint8_t base, uint8_t flag) {
  const uint8_t alts = (flag & kPdSnp) ? static_cast<uint8_t>(flag & (kPdAltA | kPdAltC | kPdAltG | kPdAltT)) : 0;
  return MatchSet{base, alts};
}

bool MatchSet::accepts(uint8_t read_base) const {
  return read_base == base || read_base == 'N' || base == 'N' || (alts != 0 && base_matches_pd(read_base, kPdSnp | alts));
}

uint8_t pd_row_states(const uint8_t* flags, int32_t len, uint8_t state, uint8_t* out) {
  for (int32_t j = 0; j < len; ++j) {
    if (out) out[j] = state;
    if (state == kPdAfterDel) state = kPdNormal;
    if (flags[j] & kPdDelStart) state = kPdInsideDel;
    if (flags[j] & kPdDelEnd) state = kPdAfterDel;
  }
  return state;
}

SortedHaps SortedHaps::make_pd(const std::vector<HapView>& haps, const std::vector<const uint8_t*>& flags) {
  SortedHaps s;
  s.pd = true;
  const size_t n = haps.size();
  std::vector<uint8_t> ends(n);
  for (size_t i = 0; i < n; ++i) ends[i] = pd_row_states(flags[i], haps[i].len, kPdNormal, nullptr);
  // (row-end state, interleaved (base, flag) pairs), pairs compared lexicographically, a prefix
  // first; the sort is stable.
  auto pairs_less = [&](int32_t a, int32_t b) {
    const int32_t m = std::min(haps[a].len, haps[b].len);
    for (int32_t j = 0; j < m; ++j) {
      const uint8_t xa = haps[a].bases[j], xb = haps[b].bases[j];
      if (xa != xb) return xa < xb;
      const uint8_t fa = flags[a][j], fb = flags[b][j];
      if (fa != fb) return fa < fb;
    }
    return haps[a].len < haps[b].len;
  };
  s.order.resize(n);
  for (size_t i = 0; i < n; ++i) s.order[i] = static_cast<int32_t>(i);
  std::stable_sort(s.order.begin(), s.order.end(), [&](int32_t a, int32_t b) {
    if (ends[a] != ends[b]) return ends[a] < ends[b];
    return pairs_less(a, b);
  });
  s.codes.resize(n);
  s.pd_bits.resize(n);
  std::vector<uint8_t> first, later;
  for (size_t k = 0; k < n; ++k) {
    const int32_t i = s.order[k];
    const HapView& h = haps[i];
    const uint8_t* f = flags[i];
    s.bases.push_back(h);
    s.flags.push_back(f);
    s.end_state.push_back(ends[i]);
    s.codes[k].resize(h.len);
    for (int32_t j = 0; j < h.len && !s.too_many_sets; ++j) {
      const MatchSet set = MatchSet::of(h.bases[j], f[j]);
      auto it = std::find(s.match_sets.begin(), s.match_sets.end(), set);
      if (it == s.match_sets.end()) {
        if (s.match_sets.size() >= 256) {
          s.too_many_sets = true;
          break;
        }
        s.match_sets.push_back(set);
        it = s.match_sets.end() - 1;
      }
      s.codes[k][j] = static_cast<uint8_t>(it - s.match_sets.begin());
    }
    first.assign(static_cast<size_t>(h.len), 0);
    later.assign(static_cast<size_t>(h.len), 0);
    pd_row_states(f, h.len, kPdNormal, first.data());
    const uint8_t later_end = pd_row_states(f, h.len, ends[i], later.data());
    if (later_end != ends[i]) throw std::logic_error("row end state not fixed by the flags");
    s.pd_bits[k].resize(h.len);
    for (int32_t j = 0; j < h.len; ++j) {
      uint32_t b = (static_cast<uint32_t>(first[j]) << kPdFirstShift) | (static_cast<uint32_t>(later[j]) << kPdLaterShift);
      if (f[j] & (kPdDelStart | kPdDelEnd)) b |= PD_MAT;
      if (f[j] & kPdDelEnd) b |= PD_DE;
      s.pd_bits[k][j] = b;
    }
  }
  s.lcp.assign(n, 0);
  s.dup.assign(n, 0);
  for (size_t k = 1; k < n; ++k) {
    if (s.end_state[k] != s.end_state[k - 1]) continue;
    const HapView &a = s.bases[k - 1], &b = s.bases[k];
    const int32_t m = std::min(a.len, b.len);
    int32_t j = 0;
    while (j < m && a.bases[j] == b.bases[j] && s.flags[k - 1][j] == s.flags[k][j]) ++j;
    s.lcp[k] = j;
    s.dup[k] = (a.len == b.len && j == a.len) ? 1 : 0;
  }
  for (const auto& h : s.bases) s.max_len = std::max(s.max_len, h.len);
  s.plan = forward_only(n);
  return s;
}

uint8_t SortedHaps::byte_of_code(int code) const {
  return code < 5 ? kStandard[code] : extra_bases[code - 5];
}

SharedColumns SortedHaps::columns() const {
  SharedColumns c;
  for (size_t k = 0; k < bases.size(); ++k) {
    if (dup[k]) continue;
    const int32_t len = bases[k].len;
    const int32_t stop = plan.cuts[k].column >= 0 ? plan.cuts[k].column - 1 : len;
    c.prefix_only += static_cast<uint64_t>(len - lcp[k]);
    c.forward += static_cast<uint64_t>(stop - lcp[k]);
  }
  for (const auto& s : plan.sweeps) c.backward += static_cast<uint64_t>(s.need - s.resume);
  return c;
}

void code_table(const SortedHaps& s, uint8_t out[256]) {
  std::memset(out, kNoCode, 256);
  for (int c = 0; c < s.num_codes(); ++c) out[s.byte_of_code(c)] = static_cast<uint8_t>(c);
}

void emit_program(const SortedHaps& s, bool with_suffix, ProgramBuild& out) {
  const size_t n = s.bases.size();
  const double init_f64 = std::ldexp(1.0, 1020);
  const double init_f32 = std::ldexp(1.0, 120);

  // ---- forward: one segment per distinct sorted haplotype ----
  struct Seg {
    int32_t hap, start, stop, len;
    Cut cut;
  };
  std::vector<Seg> segs;
  for (size_t k = 0; k < n; ++k) {
    if (s.dup[k]) continue;
    const int32_t len = s.bases[k].len;
    const Cut cut = with_suffix ? s.plan.cuts[k] : Cut{-1, -1};
    const int32_t stop = cut.column >= 0 ? cut.column - 1 : len;
    if (stop < s.lcp[k]) throw std::logic_error("cut before the shared prefix");
    segs.push_back(Seg{static_cast<int32_t>(k), s.lcp[k], stop, len, cut});
  }
  const int32_t m = static_cast<int32_t>(segs.size());
  // The last earlier segment passing each reader's start column wrote the value it resumes from.
  std::vector<int32_t> writer(m, -1);
  for (int32_t i = 1; i < m; ++i) {
    const int32_t q = segs[i].start;
    if (q == 0) continue;
    for (int32_t j = i - 1; j >= 0; --j)
      if (segs[j].start < q && q <= segs[j].stop) {
        writer[i] = j;
        break;
      }
    if (writer[i] < 0) throw std::logic_error("snapshot read before written");
  }
  // Writes keyed by (writer, column): staged for the next segment, and/or a global slot.
  std::map<std::pair<int32_t, int32_t>, std::pair<bool, int32_t>> writes;
  for (int32_t i = 1; i < m; ++i)
    if (writer[i] >= 0) writes[{writer[i], segs[i].start}] = {false, -1};
  int32_t n_slots = 0;
  for (int32_t i = 1; i < m; ++i) {
    if (writer[i] < 0) continue;
    auto& w = writes[{writer[i], segs[i].start}];
    if (writer[i] == i - 1)
      w.first = true;
    else if (w.second < 0)
      w.second = n_slots++;
  }
  // The writes of each segment in column order (the map iterates by writer, then column), so the
  // column loop below meets them with one comparison a column instead of a lookup.
  std::vector<std::vector<std::pair<int32_t, std::pair<bool, int32_t>>>> writes_of(static_cast<size_t>(m));
  for (const auto& [key, w] : writes) writes_of[static_cast<size_t>(key.first)].push_back({key.second, w});
  uint32_t pending = 0;  // post events of the previous column, carried by the next entry
  auto push = [&](std::vector<uint32_t>& v, uint32_t e) {
    v.push_back(e | pending);
    pending = 0;
  };
  // Each sharing tree runs at the constant of its longest haplotype (program.h, Segment).
  std::vector<int32_t> root(m, 0), tree_len(m, 0);
  for (int32_t i = 0; i < m; ++i) {
    root[i] = segs[i].start > 0 ? root[writer[i]] : i;
    tree_len[root[i]] = std::max(tree_len[root[i]], segs[i].len);
  }
  for (int32_t i = 0; i < m; ++i) {
    const Seg& g = segs[i];
    const double t_len = static_cast<double>(tree_len[root[i]]);
    Segment rec{};
    rec.hap = g.hap;
    rec.node = g.cut.column >= 0 ? g.cut.node : -1;
    rec.staged = g.start > 0 ? 1 : 0;
    rec.factor = t_len / static_cast<double>(g.len);
    rec.init_d = init_f64 / t_len;
    rec.init_f = static_cast<float>(init_f32 / t_len);
    rec.next_slot = -1;
    if (i + 1 < m && writer[i + 1] >= 0 && writer[i + 1] < i) rec.next_slot = writes.at({writer[i + 1], segs[i + 1].start}).second;
    out.segs.push_back(rec);
    // A cut segment also computes its cut column (stop + 1) as an ordinary column.
    const int32_t last = g.cut.column >= 0 ? g.cut.column : g.stop;
    const auto& mine = writes_of[static_cast<size_t>(i)];
    size_t next_write = 0;
    out.fwd.reserve(out.fwd.size() + static_cast<size_t>(last - g.start) + 1);
    for (int32_t j = g.start + 1; j <= last; ++j) {
      const bool is_cut = g.cut.column >= 0 && j == g.cut.column;
      const uint32_t pd_bits = s.pd ? s.pd_bits[g.hap][j - 1] : 0u;
      push(out.fwd, s.codes[g.hap][j - 1] | pd_bits | (j == g.start + 1 ? EV_BEGIN : 0u) | (is_cut ? EV_ACC : 0u));
      if (!is_cut && next_write < mine.size() && mine[next_write].first == j) {
        const auto& w = mine[next_write++].second;
        const uint32_t none = s.pd ? kPdPayloadNone : kPayloadNone;
        const uint32_t slot = w.second >= 0 ? static_cast<uint32_t>(w.second) : none;
        if (w.second >= 0 && slot >= none) throw std::invalid_argument("too many snapshot slots for the stream payload");
        pending |= EV_SNAP | (w.first ? EV_STAGE : 0u) | (slot << (s.pd ? kPdPayloadShift : kPayloadShift));
      }
    }
    if (next_write != mine.size()) throw std::logic_error("snapshot column outside its writer");
    pending |= g.cut.column >= 0 ? EV_JOIN : EV_END;
    out.fwd_columns += static_cast<uint64_t>(last - g.start);
  }
  push(out.fwd, 0);
  out.n_slots = n_slots;

  // ---- backward: node 0 from the all-zero column beyond the end, then the plan's sweeps ----
  out.n_nodes = 0;
  if (!with_suffix || s.plan.sweeps.empty()) return;
  const auto& plan = s.plan;
  const int32_t S = static_cast<int32_t>(plan.sweeps.size()) + 1;
  std::vector<int32_t> node_writer(static_cast<size_t>(plan.nodes), -1);
  node_writer[0] = 0;
  for (int32_t t = 1; t < S; ++t)
    for (const auto& w : plan.sweeps[t - 1].writes) node_writer[w.second] = t;
  auto start_of = [&](int32_t t) { return t == 0 ? -1 : plan.sweeps[t - 1].start; };
  pending = 0;
  for (int32_t t = 0; t < S; ++t) {
    Sweep rec{};
    rec.staged = t > 0 ? 1 : 0;
    rec.next_node = -1;
    if (t + 1 < S) {
      const int32_t nxt = start_of(t + 1);
      if (node_writer[nxt] < 0 || node_writer[nxt] > t) throw std::logic_error("sweep starts from an unwritten node");
      if (node_writer[nxt] < t) rec.next_node = nxt;
    }
    out.sweeps.push_back(rec);
    auto node_flags = [&](int32_t node) {
      const bool stage = t + 1 < S && start_of(t + 1) == node;
      return EV_NODE | (stage ? EV_NSTAGE : 0u) | (static_cast<uint32_t>(node) << kPayloadShift);
    };
    if (t == 0) {
      push(out.bwd, EV_SWEEP);
      pending |= node_flags(0);
      continue;
    }
    const auto& sw = plan.sweeps[t - 1];
    const int32_t len = s.bases[sw.hap].len;
    const int32_t right = len - sw.resume, left = len - sw.need;
    size_t w = 0;
    for (int32_t j = right - 1; j >= left; --j) {
      // Base at column j + 1, emitted moving down-right from column j.
      push(out.bwd, s.codes[sw.hap][j] | (j == right - 1 ? EV_SWEEP : 0u));
      if (w < sw.writes.size() && len - sw.writes[w].first == j) {
        pending |= node_flags(sw.writes[w].second);
        ++w;
      }
    }
    if (w != sw.writes.size()) throw std::logic_error("backward write outside its sweep");
    out.bwd_columns += static_cast<uint64_t>(sw.need - sw.resume);
  }
  push(out.bwd, 0);
  out.n_nodes = plan.nodes;
}

}  // namespace fgkl
