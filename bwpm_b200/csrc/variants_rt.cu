// Run-time-length register-resident kernels of the resident 2D engine (see rgen.cuh).
#include "rgen.cuh"
#include "variants.hpp"

namespace bwpm {

const std::vector<RtVariant>& rt_variants() {
  static const std::vector<RtVariant> v = {
      {8, (const void*)k_resident2d_rt<8>},   {9, (const void*)k_resident2d_rt<9>},
      {10, (const void*)k_resident2d_rt<10>}, {12, (const void*)k_resident2d_rt<12>},
      {15, (const void*)k_resident2d_rt<15>}, {16, (const void*)k_resident2d_rt<16>},
      {20, (const void*)k_resident2d_rt<20>}, {24, (const void*)k_resident2d_rt<24>},
      {30, (const void*)k_resident2d_rt<30>}};
  return v;
}

}  // namespace bwpm
