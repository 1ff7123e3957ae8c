// Kernel variants of the resident 2D engine for lengths 256-1536 (see variants.hpp).
#include "resident2d.cuh"
#include "variants.hpp"

namespace bwpm {

namespace {
using rf::Radices;

template <int N, int NT, int... R>
FixedVariant fixed() {
  return {N, NT, 1, {R...}, (const void*)k_resident2d_fixed<N, NT, Radices<R...>>, fixed_smem_bytes<N>()};
}

}  // namespace

void add_variants_small(std::vector<FixedVariant>& v) {
  // per length, only variants that no other variant beats in both per-step latency and SM time
  // (measured on a B200: 1 item, tilted slab, 400 slabs)
  v.push_back(fixed<256, 32, 8, 8, 4>());
  v.push_back(fixed<384, 32, 4, 4, 4, 3, 2>());
  v.push_back(fixed<512, 64, 8, 8, 8>());
  v.push_back(fixed<768, 64, 4, 4, 4, 4, 3>());
  v.push_back(fixed<1024, 128, 8, 8, 8, 2>());
  v.push_back(fixed<1536, 192, 8, 8, 8, 3>());  // radix 3 as a gather stage
  v.push_back(fixed<1536, 128, 4, 4, 4, 4, 2, 3>());
}

const std::vector<FixedVariant>& fixed_variants() {
  static const std::vector<FixedVariant> all = [] {
    std::vector<FixedVariant> v;
    add_variants_small(v);
    add_variants_large(v);
    return v;
  }();
  return all;
}

}  // namespace bwpm
