// Shared pieces of the drop-in command-line drivers.
#pragma once

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/chsga.h"

namespace cli {

inline uint64_t env_u64(const char* name, uint64_t dflt) {
  const char* v = std::getenv(name);
  if (!v || !*v) return dflt;
  return std::strtoull(v, nullptr, 10);
}

[[noreturn]] inline void die(const std::string& what, const char* detail) {
  std::cerr << what << (detail && *detail ? ": " : "") << (detail ? detail : "") << "\n";
  std::exit(EXIT_FAILURE);
}

// print_mean_with_moe of src/ParSGAoverrides/csr_align.hpp:84-99: mean and
// t-critical 95% margin of the per-read times, skipping the first read.
inline void print_mean_with_moe_t(const std::string& label, const std::vector<double>& v) {
  if (v.size() <= 1) {
    std::cout << label << ": insufficient data (need >1 after skipping first)\n";
    return;
  }
  static const std::unordered_map<int, double> t95 = {
      {1, 12.706}, {2, 4.303},  {3, 3.182},  {4, 2.776},  {5, 2.571},  {6, 2.447},  {7, 2.365},
      {8, 2.306},  {9, 2.262},  {10, 2.228}, {11, 2.201}, {12, 2.179}, {13, 2.160}, {14, 2.145},
      {15, 2.131}, {16, 2.120}, {17, 2.110}, {18, 2.101}, {19, 2.093}, {20, 2.086}};
  const size_t n = v.size() - 1;
  double m = 0;
  for (size_t i = 1; i < v.size(); ++i) m += v[i];
  m /= (double)n;
  double sd = 0;
  if (v.size() > 2) {
    for (size_t i = 1; i < v.size(); ++i) sd += (v[i] - m) * (v[i] - m);
    sd = std::sqrt(sd / (double)(n - 1));
  }
  const int df = (int)n - 1;
  const double tc = df <= 0 ? 0.0 : t95.at(std::min(df, 20));
  const double moe = tc * sd / std::sqrt((double)n);
  std::cout << std::fixed << std::setprecision(4);
  std::cout << label << ": " << m << " ± " << moe << " sec (n=" << n << ", df=" << df << ")\n";
}

// print_mean_with_moe of src/ConSGA_traceback.cpp:26-51 (1.96 x SE).
inline void print_mean_with_moe_z(const char* label, const std::vector<double>& times) {
  if (times.size() <= 1) {
    std::cout << " " << label << ":        " << (times.empty() ? 0.0 : times[0]) << " sec\n";
    return;
  }
  const size_t n = times.size() - 1;
  double mean = 0;
  for (size_t i = 1; i < times.size(); ++i) mean += times[i];
  mean /= (double)n;
  double var = 0;
  for (size_t i = 1; i < times.size(); ++i) var += (times[i] - mean) * (times[i] - mean);
  var /= (double)(n - 1);
  const double moe = 1.96 * std::sqrt(var / (double)n);
  std::cout << " " << label << ":        " << std::fixed << std::setprecision(4) << mean << " ± "
            << moe << " sec (n=" << n << ", df=" << (n - 1) << ")\n";
}

inline void check(chsga_status s, chsga_ctx* ctx, const char* what) {
  if (s != CHSGA_OK) die(what, ctx ? chsga_last_error(ctx) : chsga_last_error_global());
}

// Scoring of this binary: the ConSGA_*matchN_dag builds define
// CHSGA_MATCH_N (the reference's ALPHABET_SIZE=4), the *mismatchN_dag builds
// do not (ALPHABET_SIZE=5).
inline uint32_t scoring_flags() {
#ifdef CHSGA_MATCH_N
  return CHSGA_FLAG_MATCH_N;
#else
  return 0;
#endif
}

}  // namespace cli
