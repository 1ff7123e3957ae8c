// Kernel variants of the resident 2D engine for lengths 2048-8192 (see variants.hpp).
#include "cluster2d.cuh"
#include "resident2d.cuh"
#include "variants.hpp"

namespace bwpm {

namespace {
using rf::Radices;

template <int N, int NT, int... R>
FixedVariant fixed() {
  return {N, NT, 1, {R...}, (const void*)k_resident2d_fixed<N, NT, Radices<R...>>, fixed_smem_bytes<N>()};
}

// one line over a cluster of C CTAs, G passes per inverse exchange
template <int N, int C, int NT, int G, int... R>
FixedVariant cluster_g() {
  return {N, NT, C, {R...}, (const void*)k_resident2d_cluster<N, C, NT, Radices<R...>, G>,
          r2c::cluster_smem_bytes<N, C, G>()};
}
template <int N, int C, int NT, int... R>
FixedVariant cluster() {
  return cluster_g<N, C, NT, r2c::cluster_group<N, C>(), R...>();
}
}  // namespace

void add_variants_large(std::vector<FixedVariant>& v) {
  // per length, only variants that no other variant beats in both per-step latency and SM time
  // (measured on a B200: 1 item, tilted slab, 400 slabs); the first is the default
  v.push_back(fixed<2048, 256, 8, 8, 8, 4>());
  v.push_back(fixed<3072, 256, 4, 4, 4, 4, 4, 3>());
  v.push_back(fixed<4096, 256, 16, 16, 16>());
  v.push_back(cluster<4096, 2, 256, 8, 8, 8, 4>());
  v.push_back(cluster<4096, 4, 128, 8, 8, 8, 2>());
  v.push_back(cluster<4096, 8, 64, 8, 8, 8>());
  v.push_back(cluster<6144, 2, 256, 4, 4, 4, 4, 4, 3>());
  v.push_back(fixed<6144, 256, 8, 8, 8, 4, 3>());
  v.push_back(cluster<6144, 4, 192, 8, 8, 8, 3>());  // radix 3 as a gather stage
  v.push_back(cluster<8192, 4, 256, 8, 8, 8, 4>());
  v.push_back(fixed<8192, 512, 8, 8, 8, 8, 2>());
  v.push_back(cluster<8192, 8, 128, 8, 8, 8, 2>());
}

}  // namespace bwpm
