// Set-up of the plane engine on the device: per slab step, the label pairs present, the pair-id
// plane (which pair each pixel selects) and the sorted list of interface pixels, from a uint8
// label volume in device memory.
//
// This is the per-step analysis of cpp/src/solver.cpp:384-417 and :419-459 (pairs of a step in
// std::set order, the I_r,s selection, reflection sources where ñ(plane p) ≠ ñ(plane p + 1)),
// done once per solve for all steps at once instead of per slab on the host: codes
// (r + 1)·m + s sort like the pairs, a presence bitmask per step gives the pairs in order, and
// one CTA per step compacts the interface pixels in pixel order with ballot/popc scans.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace bwpm {

constexpr int kSetupThreads = 1024;

struct SetupVolume {
  const std::uint8_t* labels;  // (nz, ny, nx) labels, device
  long long nn;                // ny·nx
  int nz, ny, nx, m;           // m materials; codes (r + 1)·m + s, r = −1: before the volume
  int words;                   // presence words per step: ⌈(m + 1)·m / 32⌉
};

__device__ __forceinline__ int setup_code(const SetupVolume& v, int p, long long q) {
  const int r = p == 0 ? -1 : static_cast<int>(v.labels[(p - 1) * v.nn + q]);
  const int s = v.labels[p * v.nn + q];
  return (r + 1) * v.m + s;
}

// grid (blocks per step, nz): presence bits of the codes and the number of interface pixels
// (code_iface[code] ≠ 0) per step; bits/count zeroed by the caller.
__global__ void __launch_bounds__(256)
    k_setup_presence(SetupVolume v, const std::uint8_t* code_iface, unsigned* bits,
                     unsigned long long* iface_count) {
  extern __shared__ unsigned s_bits[];
  __shared__ unsigned s_count;
  const int p = blockIdx.y;
  for (int w = threadIdx.x; w < v.words; w += blockDim.x) s_bits[w] = 0u;
  if (threadIdx.x == 0) s_count = 0u;
  __syncthreads();
  unsigned local = 0;
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < v.nn;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int code = setup_code(v, p, q);
    atomicOr(&s_bits[code >> 5], 1u << (code & 31));
    local += code_iface[code];
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(&s_count, local);
  __syncthreads();
  for (int w = threadIdx.x; w < v.words; w += blockDim.x)
    if (s_bits[w]) atomicOr(&bits[static_cast<long long>(p) * v.words + w], s_bits[w]);
  if (threadIdx.x == 0 && s_count) atomicAdd(&iface_count[p], static_cast<unsigned long long>(s_count));
}

// grid (blocks per step, steps listed in `steps`): pid[q] = code_id[table row][code] for the
// steps with more than one pair.
__global__ void k_setup_pid(SetupVolume v, const int* steps, const long long* pid_off,
                            const std::uint8_t* code_id, int ncode, std::uint8_t* pid_pool) {
  const int k = blockIdx.y;
  const int p = steps[k];
  std::uint8_t* out = pid_pool + pid_off[k];
  const std::uint8_t* table = code_id + static_cast<long long>(k) * ncode;
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < v.nn;
       q += static_cast<long long>(gridDim.x) * blockDim.x)
    out[q] = table[setup_code(v, p, q)];
}

// one CTA per listed step: its interface pixels in increasing pixel order at iface_off[k], and
// (3D, rowoff_off[k] ≥ 0) the offset of each row's first entry, ny + 1 values.
__global__ void __launch_bounds__(kSetupThreads)
    k_setup_iface(SetupVolume v, const int* steps, const long long* iface_off,
                  const long long* rowoff_off, const std::uint8_t* code_iface, int* iface_pool,
                  int* rowoff_pool) {
  __shared__ int s_warp[kSetupThreads / 32];
  __shared__ int s_total;
  const int k = blockIdx.x;
  const int p = steps[k];
  int* out = iface_pool + iface_off[k];
  int* rowoff = rowoff_off[k] >= 0 ? rowoff_pool + rowoff_off[k] : nullptr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int running = 0;  // entries written so far (uniform across the CTA)
  const int row_len = rowoff ? v.nx : static_cast<int>(v.nn < (1LL << 30) ? v.nn : (1LL << 30));
  const int rows = rowoff ? v.ny : 1;
  for (int y = 0; y < rows; ++y) {
    if (rowoff && threadIdx.x == 0) rowoff[y] = running;
    const long long base = rowoff ? static_cast<long long>(y) * v.nx : 0;
    for (int c0 = 0; c0 < row_len; c0 += kSetupThreads) {
      const int x = c0 + threadIdx.x;
      const long long q = base + x;
      const bool flag = x < row_len && code_iface[setup_code(v, p, q)];
      const unsigned ballot = __ballot_sync(0xffffffffu, flag);
      if (lane == 0) s_warp[warp] = __popc(ballot);
      __syncthreads();
      if (threadIdx.x == 0) {  // exclusive scan of the warp counts
        int acc = 0;
        for (int w = 0; w < kSetupThreads / 32; ++w) {
          const int c = s_warp[w];
          s_warp[w] = acc;
          acc += c;
        }
        s_total = acc;
      }
      __syncthreads();
      if (flag) out[running + s_warp[warp] + __popc(ballot & ((1u << lane) - 1u))] = static_cast<int>(q);
      running += s_total;
      __syncthreads();
    }
  }
  if (rowoff && threadIdx.x == 0) rowoff[rows] = running;
}

// int32 labels → uint8 (device); sets *bad when a label is outside [0, m).
__global__ void k_labels_to_u8(const std::int32_t* in, std::uint8_t* out, long long count, int m,
                               int* bad) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const std::int32_t v = in[i];
    if (v < 0 || v >= m) {
      *bad = 1;
      out[i] = 0;
    } else {
      out[i] = static_cast<std::uint8_t>(v);
    }
  }
}

}  // namespace bwpm
