// Phred-quality probability tables, computed on the host in f64 exactly as fgkl's model.rs:37-102
// (GATK's QualityUtils / PairHMMModel with the quantized Jacobian log-sum), then uploaded once per
// device. Kernels narrow them per read row.
#pragma once
#include <array>
#include <cstdint>

namespace fgkl {

constexpr int kMaxQual = 254;
constexpr int kM2MSize = ((kMaxQual + 1) * (kMaxQual + 2)) / 2;

// Transition indices, model.rs:15-21.
enum Trans { kMM = 0, kIM = 1, kMI = 2, kII = 3, kMD = 4, kDD = 5 };

struct Tables {
  std::array<double, kMaxQual + 1> error_prob;
  std::array<double, kM2MSize> m2m;

  double err(int q) const { return error_prob[q > kMaxQual ? kMaxQual : q]; }
  double match_to_match(int ins, int del) const;
  void transitions(int ins, int del, int gcp, double t[6]) const;
};

const Tables& tables();

// GATK's approximateLog10SumLog10 through the quantized Jacobian (model.rs:87-96).
double approximate_log10_sum_log10(double a, double b);

}  // namespace fgkl
