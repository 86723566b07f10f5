#include "tables.h"

#include <cmath>
#include <mutex>

namespace fgkl {

namespace {
constexpr double kJacobianMaxTolerance = 8.0;
constexpr double kJacobianStep = 0.0001;

// MathUtils.fastRound: truncation after adding +-0.5 (model.rs:104-106).
int64_t fast_round(double d) { return d > 0.0 ? static_cast<int64_t>(d + 0.5) : static_cast<int64_t>(d - 0.5); }

double jacobian(double diff) {
  const int64_t k = fast_round(diff * (1.0 / kJacobianStep));
  return std::log10(1.0 + std::pow(10.0, -static_cast<double>(k) * kJacobianStep));
}

Tables build() {
  Tables t{};
  for (int q = 0; q <= kMaxQual; ++q) t.error_prob[q] = std::pow(10.0, static_cast<double>(q) / -10.0);
  const double inv_ln10 = 1.0 / std::log(10.0);
  int offset = 0;
  for (int i = 0; i <= kMaxQual; ++i) {
    for (int j = 0; j <= i; ++j) {
      const double s = approximate_log10_sum_log10(-0.1 * i, -0.1 * j);
      const double p = std::fmin(std::pow(10.0, s), 1.0);
      t.m2m[offset + j] = std::pow(10.0, std::log1p(-p) * inv_ln10);
    }
    offset += i + 1;
  }
  return t;
}
}  // namespace

double approximate_log10_sum_log10(double a, double b) {
  if (a > b) return approximate_log10_sum_log10(b, a);
  if (a == -INFINITY) return b;
  const double diff = b - a;
  return diff < kJacobianMaxTolerance ? b + jacobian(diff) : b;
}

double Tables::match_to_match(int ins, int del) const {
  const int a = ins > kMaxQual ? kMaxQual : ins, b = del > kMaxQual ? kMaxQual : del;
  const int lo = a <= b ? a : b, hi = a <= b ? b : a;
  return m2m[((hi * (hi + 1)) >> 1) + lo];
}

void Tables::transitions(int ins, int del, int gcp, double t[6]) const {
  const double gc = err(gcp);
  t[kMM] = match_to_match(ins, del);
  t[kMI] = err(ins);
  t[kMD] = err(del);
  t[kIM] = 1.0 - gc;
  t[kII] = gc;
  t[kDD] = gc;
}

const Tables& tables() {
  static const Tables t = build();
  return t;
}

}  // namespace fgkl
