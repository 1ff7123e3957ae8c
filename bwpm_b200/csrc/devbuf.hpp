// RAII device allocation.
#pragma once

#include <utility>

#include "common.cuh"

namespace bwpm {

template <typename U>
struct DevBuf {
  U* ptr = nullptr;
  std::size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(std::size_t count) { alloc(count); }
  void alloc(std::size_t count) {
    release();
    n = count;
    if (count) check_cuda(cudaMalloc(&ptr, count * sizeof(U)), "cudaMalloc");
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
  }
  ~DevBuf() { release(); }
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), n(o.n) {
    o.ptr = nullptr;
    o.n = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    std::swap(ptr, o.ptr);
    std::swap(n, o.n);
    return *this;
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  std::size_t bytes() const { return n * sizeof(U); }
  void upload(const U* host, std::size_t count) {
    if (count) check_cuda(cudaMemcpy(ptr, host, count * sizeof(U), cudaMemcpyHostToDevice), "upload");
  }
};

}  // namespace bwpm
