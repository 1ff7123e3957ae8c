// RAII device allocation.
//
// A buffer is either a plain cudaMalloc allocation or a stream-ordered one (cudaMallocAsync /
// cudaFreeAsync on the owner's stream). Stream-ordered buffers never synchronise the device when
// they are freed, so several solvers can allocate, run and free concurrently on one GPU; their
// owner must keep the stream alive until the buffer is released (declare the stream first).
#pragma once

#include <utility>

#include "common.cuh"

namespace bwpm {

template <typename U>
struct DevBuf {
  U* ptr = nullptr;
  std::size_t n = 0;
  cudaStream_t stream = nullptr;  // stream of a stream-ordered allocation
  bool ordered = false;
  DevBuf() = default;
  explicit DevBuf(std::size_t count) { alloc(count); }
  DevBuf(std::size_t count, cudaStream_t s) { alloc(count, s); }
  void alloc(std::size_t count) {
    release();
    n = count;
    if (count) check_cuda(cudaMalloc(&ptr, count * sizeof(U)), "cudaMalloc");
  }
  void alloc(std::size_t count, cudaStream_t s) {
    release();
    n = count;
    stream = s;
    ordered = true;
    if (count) check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&ptr), count * sizeof(U), s), "cudaMallocAsync");
  }
  void release() {
    if (ptr) {
      if (ordered)
        cudaFreeAsync(ptr, stream);
      else
        cudaFree(ptr);
    }
    ptr = nullptr;
    n = 0;
    ordered = false;
    stream = nullptr;
  }
  ~DevBuf() { release(); }
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), n(o.n), stream(o.stream), ordered(o.ordered) {
    o.ptr = nullptr;
    o.n = 0;
    o.ordered = false;
    o.stream = nullptr;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    std::swap(ptr, o.ptr);
    std::swap(n, o.n);
    std::swap(stream, o.stream);
    std::swap(ordered, o.ordered);
    return *this;
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  std::size_t bytes() const { return n * sizeof(U); }
  // Stream-ordered buffers copy on their stream and wait for that stream only (the host data may
  // be released on return; other streams of the device keep running).
  void upload(const U* host, std::size_t count) {
    if (!count) return;
    if (ordered) {
      check_cuda(cudaMemcpyAsync(ptr, host, count * sizeof(U), cudaMemcpyHostToDevice, stream), "upload");
      check_cuda(cudaStreamSynchronize(stream), "upload");
    } else
      check_cuda(cudaMemcpy(ptr, host, count * sizeof(U), cudaMemcpyHostToDevice), "upload");
  }
  void zero() {
    if (!n) return;
    if (ordered)
      check_cuda(cudaMemsetAsync(ptr, 0, bytes(), stream), "memset");
    else
      check_cuda(cudaMemset(ptr, 0, bytes()), "memset");
  }
};

// RAII page-locked host allocation (cudaHostAlloc).
template <typename U>
struct PinnedBuf {
  U* ptr = nullptr;
  std::size_t n = 0;
  PinnedBuf() = default;
  void alloc(std::size_t count) {
    release();
    n = count;
    if (count)
      check_cuda(cudaHostAlloc(reinterpret_cast<void**>(&ptr), count * sizeof(U), cudaHostAllocDefault),
                 "cudaHostAlloc");
  }
  void release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    n = 0;
  }
  ~PinnedBuf() { release(); }
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
};

// RAII CUDA event without timing.
struct OwnedEvent {
  cudaEvent_t e = nullptr;
  OwnedEvent() = default;
  void create() {
    if (!e) check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
  }
  ~OwnedEvent() {
    if (e) cudaEventDestroy(e);
  }
  OwnedEvent(const OwnedEvent&) = delete;
  OwnedEvent& operator=(const OwnedEvent&) = delete;
  operator cudaEvent_t() const { return e; }
};

// RAII CUDA graph and its executable form.
struct OwnedGraph {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t exec = nullptr;
  OwnedGraph() = default;
  ~OwnedGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (g) cudaGraphDestroy(g);
  }
  OwnedGraph(const OwnedGraph&) = delete;
  OwnedGraph& operator=(const OwnedGraph&) = delete;
};

// A non-blocking stream owned by a solver; declared before the solver's buffers so that it is
// destroyed after them.
struct OwnedStream {
  cudaStream_t s = nullptr;
  OwnedStream() = default;
  void create() { check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate"); }
  ~OwnedStream() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
  OwnedStream(const OwnedStream&) = delete;
  OwnedStream& operator=(const OwnedStream&) = delete;
  operator cudaStream_t() const { return s; }
};

// Keeps freed stream-ordered memory in the device's default pool (no return to the driver
// between solves); process-local, set once per device.
inline void keep_pool_memory(int device) {
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return;
  unsigned long long keep = ~0ull;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
}

// Device memory free for new allocations: what the driver reports free plus what the device's
// default pool holds reserved but unused (kept by keep_pool_memory, so a process that freed
// buffers does not see its own cached memory as taken).
inline std::size_t free_device_bytes(int device) {
  std::size_t free_b = 0, total_b = 0;
  check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    unsigned long long reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
        reserved > used)
      free_b += static_cast<std::size_t>(reserved - used);
  }
  return free_b;
}

}  // namespace bwpm
