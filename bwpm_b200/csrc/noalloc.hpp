// Allocation-free 2D slab step (see noalloc.cu).
#pragma once

#include <cstddef>
#include <cstdint>

#include "common.cuh"

namespace bwpm {

// Largest lateral size the fixed scratch array holds, and the array's size in bytes.
constexpr int kNoAllocMaxN = 8192;
constexpr std::size_t kNoAllocScratchBytes =
    256 + 2ull * kNoAllocMaxN * sizeof(cd) + static_cast<std::size_t>(kNoAllocMaxN) * sizeof(cd);

// One FP64 forward transmission step of a 2D field; all arrays are device pointers.
void step2d_noalloc(int device, std::size_t ny, double dy, double dz, double k0, const cd* indices,
                    std::size_t m, const std::int32_t* labels_before, const std::int32_t* labels_after,
                    cd index_before, const double* mask, const cd* field_in, cd* field_out,
                    cudaStream_t stream);

}  // namespace bwpm
