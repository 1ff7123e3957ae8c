// Mixed-radix Stockham FFT in shared memory (radix 2, 3, 4, 5, 7, 8 and generic odd primes).
//
// A transform of length N runs as stages s = 0 … S−1 with radix R_s and sub-length L_s
// (L_0 = 1, L_{s+1} = L_s·R_s). Stage s, butterfly i ∈ [0, N/R): k = i mod L,
//   u_r = x[i + r·N/R]·w^{r·k},  w = exp(∓2πi/(L·R)),  u ← DFT_R(u),
//   x'[(i − k)·R + k + r·L] = u_r,
// which leaves the result in natural order (autosort). The stages run in place: every thread
// loads its butterflies into registers, the block synchronises, then stores.
//
// Data layout in shared memory is point-major with B interleaved batch lanes: point n of lane b
// sits at buf[n·B + b]. Twiddles come from a per-stage table tw[off_s + k·(R−1) + r−1] =
// exp(−2πi·r·k/(L·R)) built in FP64 on the host (forward); the inverse uses the conjugate.
// Inverse transforms are unnormalised.
//
// Precision of FP32 transforms: every constant (twiddles and the radix-3/5/7/8 butterfly
// constants) is carried as an unevaluated pair hi + lo of floats, and a product with a constant
// folds the lo part into its FMA chain before the single final rounding. A constant rounded to
// FP32 alone is a fixed relative error per mode that recurs in every slab step, so it grows
// linearly along a chain of thousands of steps (≈ 5e-8 per step); with the pairs the per-step
// error is the unbiased arithmetic rounding only, ≈ 20× smaller after 1000 steps.
#pragma once

#include "common.cuh"

namespace bwpm {

constexpr int kMaxStages = 20;
constexpr int kMaxGenericRadix = 61;

struct FftPlan {
  int n = 1;
  int nstages = 0;
  int radix[kMaxStages] = {};
  int len[kMaxStages] = {};     // L_s
  int twoff[kMaxStages] = {};   // offset of the stage's twiddles
  int rootoff = 0;              // offset of the N-th roots exp(−2πi m/N), m < N (generic radix)
  int ntw = 0;                  // total twiddle entries
};

// Butterflies a thread stages per stage: EPT complex values per thread (radix ≤ 8), one
// butterfly for the generic radix.
__host__ __device__ constexpr int kmax_for(int r, int ept = 16) {
  return r <= 8 ? (ept / r > 0 ? ept / r : 1) : 1;
}

// Twiddle storage: FP64 transforms keep one double value, FP32 transforms a (hi, lo) pair.
template <typename T>
struct Tw {
  cx<T> hi;
};
template <>
struct Tw<float> {
  cf hi, lo;
};

// u·w (DIR < 0) or u·conj(w) (DIR > 0).
template <int DIR>
__device__ __forceinline__ cd twmul(cd u, const Tw<double>& w) {
  const double wi = DIR < 0 ? w.hi.im : -w.hi.im;
  return {fma(u.re, w.hi.re, -u.im * wi), fma(u.re, wi, u.im * w.hi.re)};
}
template <int DIR>
__device__ __forceinline__ cf twmul(cf u, const Tw<float>& w) {
  const float hr = w.hi.re, hi = DIR < 0 ? w.hi.im : -w.hi.im;
  const float lr = w.lo.re, li = DIR < 0 ? w.lo.im : -w.lo.im;
  const float re = fmaf(u.re, hr, fmaf(-u.im, hi, fmaf(u.re, lr, -u.im * li)));
  const float im = fmaf(u.re, hi, fmaf(u.im, hr, fmaf(u.re, li, u.im * lr)));
  return {re, im};
}

// x·c for a real constant c = hi + lo (the lo part only matters in FP32).
template <typename T>
__device__ __forceinline__ cx<T> kmul(cx<T> x, double c) {
  if constexpr (sizeof(T) == sizeof(double)) {
    return {x.re * c, x.im * c};
  } else {
    const float h = static_cast<float>(c);
    const float l = static_cast<float>(c - static_cast<double>(h));
    return {fmaf(x.re, h, x.re * l), fmaf(x.im, h, x.im * l)};
  }
}

// Products with a complex table value given as (hi, lo) pairs in FP32, or one FP64 value.
__device__ __forceinline__ cf pmul(cf u, cf hi, cf lo) {
  const float re = fmaf(u.re, hi.re, fmaf(-u.im, hi.im, fmaf(u.re, lo.re, -u.im * lo.im)));
  const float im = fmaf(u.re, hi.im, fmaf(u.im, hi.re, fmaf(u.re, lo.im, u.im * lo.re)));
  return {re, im};
}

namespace fftdetail {

// Cosines/sines of 2π/5, 4π/5, 2π/7, 4π/7, 6π/7 and √3/2, √½ (mathematical constants).
constexpr double kC51 = 0.30901699437494742410, kC52 = -0.80901699437494742410;
constexpr double kS51 = 0.95105651629515357212, kS52 = 0.58778525229247312917;
constexpr double kC71 = 0.62348980185873353053, kC72 = -0.22252093395631440429,
                 kC73 = -0.90096886790241912624;
constexpr double kS71 = 0.78183148246802980871, kS72 = 0.97492791218182360702,
                 kS73 = 0.43388373911755812048;
constexpr double kS3 = 0.86602540378443864676;
constexpr double kR2 = 0.70710678118654752440;

template <int DIR, typename T>
__device__ __forceinline__ void dft2(cx<T>* u) {
  const cx<T> a = u[0], b = u[1];
  u[0] = a + b;
  u[1] = a - b;
}

template <int DIR, typename T>
__device__ __forceinline__ void dft4(cx<T>& a0, cx<T>& a1, cx<T>& a2, cx<T>& a3) {
  const cx<T> t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = mul_i<DIR>(a1 - a3);
  a0 = t0 + t2;
  a2 = t0 - t2;
  a1 = t1 + t3;
  a3 = t1 - t3;
}

template <int DIR, typename T>
__device__ __forceinline__ void dft8(cx<T>* u) {
  cx<T> e0 = u[0], e1 = u[2], e2 = u[4], e3 = u[6];
  cx<T> o0 = u[1], o1 = u[3], o2 = u[5], o3 = u[7];
  dft4<DIR>(e0, e1, e2, e3);
  dft4<DIR>(o0, o1, o2, o3);
  // w8^1 = (1 ∓ i)/√2, w8^2 = ∓i, w8^3 = (−1 ∓ i)/√2
  const cx<T> w1o = kmul<T>(DIR < 0 ? cx<T>{o1.re + o1.im, o1.im - o1.re}
                                    : cx<T>{o1.re - o1.im, o1.im + o1.re}, kR2);
  const cx<T> w2o = mul_i<DIR>(o2);
  const cx<T> w3o = kmul<T>(DIR < 0 ? cx<T>{o3.im - o3.re, -(o3.re + o3.im)}
                                    : cx<T>{-(o3.re + o3.im), o3.re - o3.im}, kR2);
  u[0] = e0 + o0;
  u[4] = e0 - o0;
  u[1] = e1 + w1o;
  u[5] = e1 - w1o;
  u[2] = e2 + w2o;
  u[6] = e2 - w2o;
  u[3] = e3 + w3o;
  u[7] = e3 - w3o;
}

template <int DIR, typename T>
__device__ __forceinline__ void dft3(cx<T>* u) {
  const cx<T> t1 = u[1] + u[2];
  const cx<T> t2 = u[0] - t1 * static_cast<T>(0.5);
  const cx<T> t3 = kmul<T>(mul_i<DIR>(u[1] - u[2]), kS3);
  u[0] = u[0] + t1;
  u[1] = t2 + t3;
  u[2] = t2 - t3;
}

template <int DIR, typename T>
__device__ __forceinline__ void dft5(cx<T>* u) {
  const cx<T> b1 = u[1] + u[4], b2 = u[2] + u[3], d1 = u[1] - u[4], d2 = u[2] - u[3];
  const cx<T> a0 = u[0];
  const cx<T> t1 = a0 + kmul<T>(b1, kC51) + kmul<T>(b2, kC52);
  const cx<T> t2 = a0 + kmul<T>(b1, kC52) + kmul<T>(b2, kC51);
  const cx<T> v1 = mul_i<DIR>(kmul<T>(d1, kS51) + kmul<T>(d2, kS52));
  const cx<T> v2 = mul_i<DIR>(kmul<T>(d1, kS52) - kmul<T>(d2, kS51));
  u[0] = a0 + b1 + b2;
  u[1] = t1 + v1;
  u[4] = t1 - v1;
  u[2] = t2 + v2;
  u[3] = t2 - v2;
}

template <int DIR, typename T>
__device__ __forceinline__ void dft7(cx<T>* u) {
  const cx<T> b1 = u[1] + u[6], b2 = u[2] + u[5], b3 = u[3] + u[4];
  const cx<T> d1 = u[1] - u[6], d2 = u[2] - u[5], d3 = u[3] - u[4];
  const cx<T> a0 = u[0];
  const cx<T> t1 = a0 + kmul<T>(b1, kC71) + kmul<T>(b2, kC72) + kmul<T>(b3, kC73);
  const cx<T> t2 = a0 + kmul<T>(b1, kC72) + kmul<T>(b2, kC73) + kmul<T>(b3, kC71);
  const cx<T> t3 = a0 + kmul<T>(b1, kC73) + kmul<T>(b2, kC71) + kmul<T>(b3, kC72);
  const cx<T> v1 = mul_i<DIR>(kmul<T>(d1, kS71) + kmul<T>(d2, kS72) + kmul<T>(d3, kS73));
  const cx<T> v2 = mul_i<DIR>(kmul<T>(d1, kS72) - kmul<T>(d2, kS73) - kmul<T>(d3, kS71));
  const cx<T> v3 = mul_i<DIR>(kmul<T>(d1, kS73) - kmul<T>(d2, kS71) + kmul<T>(d3, kS72));
  u[0] = a0 + b1 + b2 + b3;
  u[1] = t1 + v1;
  u[6] = t1 - v1;
  u[2] = t2 + v2;
  u[5] = t2 - v2;
  u[3] = t3 + v3;
  u[4] = t3 - v3;
}

template <int DIR, int R, typename T>
__device__ __forceinline__ void dft(cx<T>* u) {
  if constexpr (R == 2) dft2<DIR>(u);
  if constexpr (R == 3) dft3<DIR>(u);
  if constexpr (R == 4) dft4<DIR>(u[0], u[1], u[2], u[3]);
  if constexpr (R == 5) dft5<DIR>(u);
  if constexpr (R == 7) dft7<DIR>(u);
  if constexpr (R == 8) dft8<DIR>(u);
}


// One stage of radix R on `batch` lanes (point stride `batch`), in place; a thread stages up to
// EPT values (kmax_for(R, EPT) butterflies).
template <int DIR, int R, int EPT, typename T>
__device__ __forceinline__ void stage_body(cx<T>* buf, int n, int len,
                                           const Tw<T>* __restrict__ tw, int batch, int tid,
                                           int nthreads) {
  constexpr int K = kmax_for(R, EPT);
  const int nb = n / R;
  const int total = nb * batch;
  cx<T> u[K][R];
  int dst[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = tid + k * nthreads;
    dst[k] = -1;
    if (t < total) {
      const int b = t % batch, i = t / batch;
      const int kk = i % len;
#pragma unroll
      for (int r = 0; r < R; ++r) u[k][r] = buf[(i + r * nb) * batch + b];
      if (len > 1) {
        // r-major layout: consecutive k (consecutive threads) read consecutive entries
#pragma unroll
        for (int r = 1; r < R; ++r) u[k][r] = twmul<DIR>(u[k][r], tw[(r - 1) * len + kk]);
      }
      dft<DIR, R>(u[k]);
      dst[k] = ((i - kk) * R + kk) * batch + b;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (dst[k] >= 0) {
#pragma unroll
      for (int r = 0; r < R; ++r) buf[dst[k] + r * len * batch] = u[k][r];
    }
  __syncthreads();
}

template <int DIR, int R, int EPT, typename T>
__device__ __noinline__ void stage(cx<T>* buf, int n, int len, const Tw<T>* __restrict__ tw,
                                   int batch, int tid, int nthreads) {
  stage_body<DIR, R, EPT>(buf, n, len, tw, batch, tid, nthreads);
}

// Generic odd radix R ≤ kMaxGenericRadix by the symmetric real-cosine form; one butterfly
// per thread (the planner guarantees nthreads ≥ batch·N/R).
template <int DIR, typename T>
__device__ __noinline__ void stage_generic(cx<T>* buf, int n, int len, int R,
                                           const Tw<T>* __restrict__ tw,
                                           const Tw<T>* __restrict__ roots, int batch, int tid,
                                           int nthreads) {
  const int nb = n / R;
  const int total = nb * batch;
  cx<T> u[kMaxGenericRadix];
  cx<T> y[kMaxGenericRadix];
  int dst = -1;
  if (tid < total) {
    const int b = tid % batch, i = tid / batch;
    const int kk = i % len;
    for (int r = 0; r < R; ++r) u[r] = buf[(i + r * nb) * batch + b];
    if (len > 1)
      for (int r = 1; r < R; ++r) u[r] = twmul<DIR>(u[r], tw[(r - 1) * len + kk]);
    const int step = n / R;  // roots[j·step] = exp(−2πi j/R)
    for (int m = 0; m < R; ++m) {
      cx<T> acc = u[0];
      for (int j = 1; j < R; ++j) {
        const int e = (j * m) % R;
        acc = acc + twmul<DIR>(u[j], roots[e * step]);
      }
      y[m] = acc;
    }
    dst = ((i - kk) * R + kk) * batch + b;
  }
  __syncthreads();
  if (dst >= 0)
    for (int r = 0; r < R; ++r) buf[dst + r * len * batch] = y[r];
  __syncthreads();
}

}  // namespace fftdetail

// Full in-place transform of `batch` lanes of length plan.n in shared memory.
// DIR = −1 forward (exp(−2πi…)), +1 inverse (unnormalised). The launch must provide
// threads_needed(plan, batch, EPT) threads.
template <int DIR, int EPT = 16, typename T>
__device__ __noinline__ void fft_smem(cx<T>* buf, const FftPlan& plan, const Tw<T>* __restrict__ tw,
                         int batch, int tid, int nthreads) {
  using namespace fftdetail;
  for (int s = 0; s < plan.nstages; ++s) {
    const int r = plan.radix[s], len = plan.len[s];
    const Tw<T>* w = tw + plan.twoff[s];
    switch (r) {
      case 2: stage<DIR, 2, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      case 3: stage<DIR, 3, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      case 4: stage<DIR, 4, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      case 5: stage<DIR, 5, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      case 7: stage<DIR, 7, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      case 8: stage<DIR, 8, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      default:
        stage_generic<DIR>(buf, plan.n, len, r, w, tw + plan.rootoff, batch, tid, nthreads);
    }
  }
}

// The same transform with the radix 2-8 stages expanded in the caller. A call of a stage
// function saves and restores the caller's live registers through local memory at every stage;
// the 3D plane kernels, whose threads hold pixel data and table values across their
// transforms, use this form. The generic radix stays a call.
template <int DIR, int EPT = 16, typename T>
__device__ __forceinline__ void fft_smem_inline(cx<T>* buf, const FftPlan& plan,
                                                const Tw<T>* __restrict__ tw, int batch, int tid,
                                                int nthreads) {
  using namespace fftdetail;
  for (int s = 0; s < plan.nstages; ++s) {
    const int r = plan.radix[s], len = plan.len[s];
    const Tw<T>* w = tw + plan.twoff[s];
    switch (r) {
      case 2: stage_body<DIR, 2, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      case 3: stage_body<DIR, 3, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      case 4: stage_body<DIR, 4, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      case 5: stage_body<DIR, 5, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      case 7: stage_body<DIR, 7, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      case 8: stage_body<DIR, 8, EPT>(buf, plan.n, len, w, batch, tid, nthreads); break;
      default:
        stage_generic<DIR>(buf, plan.n, len, r, w, tw + plan.rootoff, batch, tid, nthreads);
    }
  }
}

}  // namespace bwpm
