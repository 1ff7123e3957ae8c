// Compiled kernel variants of the resident 2D engine for fixed line lengths.
//
// Each fixed length N has one or more register-resident kernels (threads per CTA, FFT radices,
// CTAs per line); the batch engine picks one per length, by measurement when autotuning is on
// (see Batch2D::set_autotune), else the first listed.
#pragma once

#include <cstddef>
#include <vector>

namespace bwpm {

struct FixedVariant {
  int n;                     // line length
  int nt;                    // threads per CTA
  int cluster;               // CTAs per line (1: one CTA owns the line)
  std::vector<int> radices;  // FFT stages (each divides the values per thread)
  const void* fn;            // kernel entry
  std::size_t smem;          // dynamic shared memory per CTA, bytes
};

// every compiled variant, grouped by length in increasing order
const std::vector<FixedVariant>& fixed_variants();

// Run-time-length kernels: E values per thread, any length n = E·nt whose radices (2, 3, 4, 5,
// 8) all divide E, nt ≤ 512 threads (256 for E > 8); ordered by increasing E.
struct RtVariant {
  int e;
  const void* fn;
  int max_threads;  // the instance's thread limit (rg::rt_max_threads(e), or 512: wide form)
};
const std::vector<RtVariant>& rt_variants();

// parts of the registry compiled in separate translation units
void add_variants_small(std::vector<FixedVariant>& v);
void add_variants_large(std::vector<FixedVariant>& v);

}  // namespace bwpm
