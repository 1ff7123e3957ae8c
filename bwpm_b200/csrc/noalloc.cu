// Allocation-free 2D slab step: bwpm_step2d_noalloc (declared in include/bwpm_b200.h).
//
// Some callers cannot allocate device memory at the point where they need a slab step: a host
// framework that owns all device memory through its own arena, a real-time loop that must not
// allocate after start-up, or a plugin whose memory budget was fixed when it was loaded. This
// entry point takes the caller's device buffers for inputs and outputs and keeps its own
// scratch (the spectrum of the incoming field and the FFT twiddles) in one file-scope device
// array of fixed size, so it never calls cudaMalloc or cudaFree.
//
// The step is one forward transmission step of the 2D FPWPM in FP64, the same operation as one
// slab of bwpm_solver_run with iterations = 0: out = mask · Σ_(r,s) I_r,s F⁻¹{T_r,s e^{i k_z,s dz}
// F{e}}. The operator values are evaluated on the fly (no tables), so nothing has to be built.
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "fft.cuh"
#include "interface.cuh"
#include "noalloc.hpp"

namespace bwpm {
namespace {

constexpr int kMaxMaterials = 32;
constexpr int kMaxPairCodes = (kMaxMaterials + 1) * kMaxMaterials;  // (r ∈ −1…m−1, s ∈ 0…m−1)
constexpr int kNoAllocThreads = 512;
constexpr int kMaxDevices = 64;

// Scratch layout (bytes): [0, 256) status word; spectrum of both components (2·kNoAllocMaxN
// complex128); twiddles (kNoAllocMaxN entries of 16 bytes).
constexpr std::size_t kStatusBytes = 256;
constexpr std::size_t kSpectrumBytes = 2ull * kNoAllocMaxN * sizeof(cd);
constexpr std::size_t kTwiddleBytes = static_cast<std::size_t>(kNoAllocMaxN) * sizeof(Tw<double>);
constexpr std::size_t kScratchBytes = kStatusBytes + kSpectrumBytes + kTwiddleBytes;
static_assert(kScratchBytes == kNoAllocScratchBytes, "scratch size");

// Shared by every call on a device and kept from the last call; see bwpm_step2d_noalloc.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

struct Materials {
  cd index[kMaxMaterials];
  cd index_before;
  int m;
};

// twiddles of `plan` (forward sign), FP64: exp(−2πi·(r·k mod L·R)/(L·R))
__global__ void k_noalloc_twiddles(Tw<double>* tw, FftPlan plan) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= plan.ntw) return;
  int s = plan.nstages - 1;
  while (s > 0 && plan.twoff[s] > i) --s;
  const int r = plan.radix[s], len = plan.len[s];
  const int local = i - plan.twoff[s];
  const int j = local / len + 1, k = local % len;  // r-major: entry (j − 1)·L + k
  const long long lr = static_cast<long long>(len) * r;
  const long long m = (static_cast<long long>(j) * k) % lr;
  double sn, cs;
  sincospi(-2.0 * static_cast<double>(m) / static_cast<double>(lr), &sn, &cs);
  tw[i].hi = cd{cs, sn};
}

// EPT: complex values a thread stages per FFT stage. 16 serves most lengths; lengths whose
// radix-3/5/7 stages would need more than kNoAllocThreads threads at 16 (7203, 7350, 7560, 7776,
// 7840, 7875, 7938, 8000, 8064, 8100) run the EPT = 32 instance.
template <int EPT>
__global__ void __launch_bounds__(kNoAllocThreads)
    k_noalloc_step2d(unsigned char* scratch, const cd* in, cd* out, const std::int32_t* lab_before,
                     const std::int32_t* lab_after, const double* mask, Materials mat, int n,
                     double dy, double dz, double k0, FftPlan plan) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* buf = reinterpret_cast<cd*>(smem_raw);
  __shared__ unsigned s_codes[(kMaxPairCodes + 31) / 32];
  __shared__ int s_bad;
  int* status = reinterpret_cast<int*>(scratch);
  cd* spec = reinterpret_cast<cd*>(scratch + kStatusBytes) + static_cast<long long>(blockIdx.x) * n;
  const Tw<double>* tw = reinterpret_cast<const Tw<double>*>(scratch + kStatusBytes + kSpectrumBytes);
  const int c = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  // distinct (r, s) pairs, lexicographic like the reference's std::set (cpp/src/solver.cpp:389-390)
  for (int i = tid; i < (kMaxPairCodes + 31) / 32; i += nt) s_codes[i] = 0u;
  if (tid == 0) s_bad = 0;
  __syncthreads();
  for (int q = tid; q < n; q += nt) {
    const int r = lab_before ? lab_before[q] : -1, s = lab_after[q];
    if (r < -1 || r >= mat.m || s < 0 || s >= mat.m) {
      s_bad = 1;
      continue;
    }
    const int code = (r + 1) * mat.m + s;
    atomicOr(&s_codes[code >> 5], 1u << (code & 31));
  }
  for (int q = tid; q < n; q += nt) buf[q] = in[2 * q + c];
  __syncthreads();
  if (s_bad) {
    if (tid == 0) atomicExch(status, 1);
    return;
  }
  fft_smem<-1, EPT>(buf, plan, tw, 1, tid, nt);
  for (int q = tid; q < n; q += nt) spec[q] = buf[q];
  __syncthreads();
  const double inv_n = 1.0 / static_cast<double>(n);
  const int ncode = (mat.m + 1) * mat.m;
  for (int code = 0; code < ncode; ++code) {
    if (!(s_codes[code >> 5] & (1u << (code & 31)))) continue;
    const int r = code / mat.m - 1, s = code % mat.m;
    const cd nr = r < 0 ? mat.index_before : mat.index[r], ns = mat.index[s];
    for (int q = tid; q < n; q += nt) {
      cd m3[3];
      operator_matrix(kFwdT, 0.0, fftfreq(q, n, dy), nr, ns, k0, dz, m3);
      buf[q] = spec[q] * m3[c == 0 ? 0 : 2];
    }
    __syncthreads();
    fft_smem<+1, EPT>(buf, plan, tw, 1, tid, nt);
    for (int q = tid; q < n; q += nt) {
      const int lr = lab_before ? lab_before[q] : -1;
      if (lr != r || lab_after[q] != s) continue;
      cd v = buf[q] * inv_n;
      if (mask) v = v * mask[q];
      out[2 * q + c] = v;
    }
    __syncthreads();
  }
}

// Radix plan without heap allocation (the same radix choice as make_plan in plan.hpp).
bool plan_fixed(int n, FftPlan& p) {
  int radix[kMaxStages];
  int count = 0, m = n, twos = 0;
  while (m % 2 == 0) {
    m /= 2;
    ++twos;
  }
  for (int f : {3, 5, 7})
    while (m % f == 0) {
      if (count == kMaxStages) return false;
      radix[count++] = f;
      m /= f;
    }
  for (int f = 11; m > 1 && f <= kMaxGenericRadix; f += 2)
    while (m % f == 0) {
      if (count == kMaxStages) return false;
      radix[count++] = f;
      m /= f;
    }
  if (m > 1) return false;
  auto push = [&](int r) {
    if (count == kMaxStages) return false;
    radix[count++] = r;
    return true;
  };
  if (twos % 3 == 1 && twos >= 4) {
    for (int i = 0; i < (twos - 4) / 3; ++i)
      if (!push(8)) return false;
    if (!push(4) || !push(4)) return false;
  } else {
    for (int i = 0; i < twos / 3; ++i)
      if (!push(8)) return false;
    if (twos % 3 == 2 && !push(4)) return false;
    if (twos % 3 == 1 && !push(2)) return false;
  }
  p = FftPlan{};
  p.n = n;
  p.nstages = count;
  int len = 1, off = 0;
  for (int s = 0; s < count; ++s) {
    p.radix[s] = radix[s];
    p.len[s] = len;
    p.twoff[s] = off;
    off += len * (radix[s] - 1);
    len *= radix[s];
  }
  p.rootoff = off;
  p.ntw = off;
  for (int s = 0; s < count; ++s)
    if (radix[s] > 8) return false;  // the on-device twiddle kernel covers radices 2-8 only
  return true;
}

int threads_fixed(const FftPlan& p, int ept) {
  long long need = 32;
  for (int s = 0; s < p.nstages; ++s) {
    const long long total = p.n / p.radix[s];
    const long long k = kmax_for(p.radix[s], ept);
    need = std::max(need, (total + k - 1) / k);
  }
  return static_cast<int>((need + 31) / 32 * 32);
}

}  // namespace

void step2d_noalloc(int device, std::size_t ny, double dy, double dz, double k0, const cd* indices,
                    std::size_t m, const std::int32_t* labels_before, const std::int32_t* labels_after,
                    cd index_before, const double* mask, const cd* field_in, cd* field_out,
                    cudaStream_t stream) {
  if (ny < 2 || ny > static_cast<std::size_t>(kNoAllocMaxN))
    throw invalid_argument("ny must be in [2, " + std::to_string(kNoAllocMaxN) +
                           "] for the allocation-free step (its scratch is sized for that)");
  if (m < 1 || m > static_cast<std::size_t>(kMaxMaterials))
    throw invalid_argument("the allocation-free step takes 1 to " + std::to_string(kMaxMaterials) +
                           " materials");
  if (!indices || !labels_after || !field_in || !field_out)
    throw invalid_argument("null array");
  if (device < 0 || device >= kMaxDevices) throw invalid_argument("device out of range");
  FftPlan plan;
  if (!plan_fixed(static_cast<int>(ny), plan))
    throw invalid_argument("ny must factor into 2, 3, 5 and 7 for the allocation-free step");
  const bool wide = threads_fixed(plan, 16) > kNoAllocThreads;
  const int threads = std::max(64, threads_fixed(plan, wide ? 32 : 16));
  if (threads > kNoAllocThreads) throw invalid_argument("ny too large for the allocation-free step");
  // the caller's current device is restored on every exit path (the call selects `device`)
  struct DeviceGuard {
    int prev = -1;
    DeviceGuard() {
      if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    }
    ~DeviceGuard() {
      if (prev >= 0) cudaSetDevice(prev);
    }
  } guard;
  check_cuda(cudaSetDevice(device), "cudaSetDevice");
  unsigned char* scratch = nullptr;
  {  // set-up once per device, with that device current: the scratch array's device address
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[device]) {
      void* ptr = nullptr;
      check_cuda(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress");
      for (const void* k : {(const void*)k_noalloc_step2d<16>, (const void*)k_noalloc_step2d<32>})
        check_cuda(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(kNoAllocMaxN * sizeof(cd))),
                   "cudaFuncSetAttribute");
      g_scratch_ptr[device] = ptr;
    }
    scratch = static_cast<unsigned char*>(g_scratch_ptr[device]);
  }
  Materials mat{};
  for (std::size_t i = 0; i < m; ++i) mat.index[i] = indices[i];
  mat.index_before = index_before;
  mat.m = static_cast<int>(m);
  // the status word must start at zero; spectrum and twiddles are fully rewritten by every call
  check_cuda(cudaMemsetAsync(scratch, 0, sizeof(int), stream), "cudaMemsetAsync");
  Tw<double>* tw = reinterpret_cast<Tw<double>*>(scratch + kStatusBytes + kSpectrumBytes);
  if (plan.ntw > 0) {
    k_noalloc_twiddles<<<ceil_div(plan.ntw, 256), 256, 0, stream>>>(tw, plan);
    check_cuda(cudaGetLastError(), "k_noalloc_twiddles");
  }
  if (wide)
    k_noalloc_step2d<32><<<2, threads, ny * sizeof(cd), stream>>>(
        scratch, field_in, field_out, labels_before, labels_after, mask, mat, static_cast<int>(ny),
        dy, dz, k0, plan);
  else
    k_noalloc_step2d<16><<<2, threads, ny * sizeof(cd), stream>>>(
        scratch, field_in, field_out, labels_before, labels_after, mask, mat, static_cast<int>(ny),
        dy, dz, k0, plan);
  check_cuda(cudaGetLastError(), "k_noalloc_step2d");
  int status = 0;
  check_cuda(cudaMemcpyAsync(&status, scratch, sizeof(int), cudaMemcpyDeviceToHost, stream), "status");
  check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
  if (status) throw invalid_argument("labels must index into `indices`");
}

}  // namespace bwpm
