// Run-time-length register-resident kernels of the resident 2D engine (see rgen.cuh).
#include "rgen.cuh"
#include "variants.hpp"

namespace bwpm {

const std::vector<RtVariant>& rt_variants() {
  using rg::rt_max_threads;
  static const std::vector<RtVariant> v = {
      {8, (const void*)k_resident2d_rt<8>, rt_max_threads(8)},
      {9, (const void*)k_resident2d_rt<9>, rt_max_threads(9)},
      {10, (const void*)k_resident2d_rt<10>, rt_max_threads(10)},
      {12, (const void*)k_resident2d_rt<12>, rt_max_threads(12)},
      {15, (const void*)k_resident2d_rt<15>, rt_max_threads(15)},
      {16, (const void*)k_resident2d_rt<16>, rt_max_threads(16)},
      {20, (const void*)k_resident2d_rt<20>, rt_max_threads(20)},
      {24, (const void*)k_resident2d_rt<24>, rt_max_threads(24)},
      {30, (const void*)k_resident2d_rt<30>, rt_max_threads(30)},
      // wide forms (512 threads, 128 registers) for lines beyond the default thread limit
      {9, (const void*)k_resident2d_rt<9, 512>, 512},
      {10, (const void*)k_resident2d_rt<10, 512>, 512},
      {12, (const void*)k_resident2d_rt<12, 512>, 512}};
  return v;
}

}  // namespace bwpm
