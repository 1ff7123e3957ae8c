// Register-resident FFT for lines of a compile-time length N (complex64, split constants).
//
// NT threads, E = N/NT values per thread. Thread t owns positions t + m·NT (m < E): the
// "owned pattern". In the Stockham stage of radix R (sub-length L) the thread's butterflies are
// i = t + j·NT (j < E/R); their inputs x[i + r·N/R] = x[t + (j + r·E/R)·NT] are exactly owned
// positions, and in the last stage (L = N/R) the outputs x'[i + r·L] are owned positions too.
// So a transform takes its input from registers and leaves its output in registers (natural
// order, owned pattern); between stages the values go through shared memory once
// (write scattered, barrier, read owned), alternating two buffers so one barrier suffices.
// Buffers are padded by one element per 16 (pad()), which makes the scattered writes of every
// power-of-two stride and the owned reads free of bank conflicts.
//
// Twiddles: the per-stage r-major tables of plan.hpp (entry (r − 1)·L + k of stage s at offset
// Σ_{s'<s} L_s'·(R_s' − 1)), stored as FP32 (hi, lo) pairs; see fft.cuh for why every constant is
// carried as a pair.
#pragma once

#include "fft.cuh"

namespace bwpm {
namespace rf {

template <int... Rs>
struct Radices {};

__device__ __forceinline__ int pad(int a) { return a + (a >> 4); }
__host__ __device__ constexpr int padded(int n) { return n + n / 16 + 1; }

// x·exp(DIR·2πi·e/16) with exact (±1, ±i) cases and split constants otherwise.
template <int DIR, int EXP>
__device__ __forceinline__ cf w16mul(cf x) {
  constexpr int e = EXP % 16;
  if constexpr (e == 0) {
    return x;
  } else if constexpr (e == 4) {
    return mul_i<DIR>(x);
  } else if constexpr (e == 8) {
    return -x;
  } else if constexpr (e == 12) {
    return mul_i<-DIR>(x);
  } else {
    constexpr double pi = 3.141592653589793238462643383279502884;
    // cos and sin of 2πe/16 for e = 1, 2, 3, 5, 6, 7, 9, … from the octant values
    constexpr double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173;
    constexpr double r2 = 0.70710678118654752440;
    constexpr double cs[16][2] = {{1, 0},   {c1, s1},   {r2, r2},   {s1, c1},
                                  {0, 1},   {-s1, c1},  {-r2, r2},  {-c1, s1},
                                  {-1, 0},  {-c1, -s1}, {-r2, -r2}, {-s1, -c1},
                                  {0, -1},  {s1, -c1},  {r2, -r2},  {c1, -s1}};
    (void)pi;
    constexpr double c = cs[e][0], s = DIR * cs[e][1];
    const cf hi{static_cast<float>(c), static_cast<float>(s)};
    const cf lo{static_cast<float>(c - static_cast<double>(static_cast<float>(c))),
                static_cast<float>(s - static_cast<double>(static_cast<float>(s)))};
    return pmul(x, hi, lo);
  }
}

template <int DIR>
__device__ __forceinline__ void dft16(cf* u) {
  // n = 4·n1 + n2, m = m1 + 4·m2: DFT4 over n1, twiddle w16^(n2·m1), DFT4 over n2
  cf a[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    cf x0 = u[n2], x1 = u[n2 + 4], x2 = u[n2 + 8], x3 = u[n2 + 12];
    fftdetail::dft4<DIR>(x0, x1, x2, x3);
    a[n2][0] = x0;
    a[n2][1] = x1;
    a[n2][2] = x2;
    a[n2][3] = x3;
  }
  a[1][1] = w16mul<DIR, 1>(a[1][1]);
  a[1][2] = w16mul<DIR, 2>(a[1][2]);
  a[1][3] = w16mul<DIR, 3>(a[1][3]);
  a[2][1] = w16mul<DIR, 2>(a[2][1]);
  a[2][2] = w16mul<DIR, 4>(a[2][2]);
  a[2][3] = w16mul<DIR, 6>(a[2][3]);
  a[3][1] = w16mul<DIR, 3>(a[3][1]);
  a[3][2] = w16mul<DIR, 6>(a[3][2]);
  a[3][3] = w16mul<DIR, 9>(a[3][3]);
#pragma unroll
  for (int m1 = 0; m1 < 4; ++m1) {
    cf x0 = a[0][m1], x1 = a[1][m1], x2 = a[2][m1], x3 = a[3][m1];
    fftdetail::dft4<DIR>(x0, x1, x2, x3);
    u[m1] = x0;
    u[m1 + 4] = x1;
    u[m1 + 8] = x2;
    u[m1 + 12] = x3;
  }
}

template <int DIR, int R>
__device__ __forceinline__ void dft(cf* u) {
  if constexpr (R == 16)
    dft16<DIR>(u);
  else
    fftdetail::dft<DIR, R>(u);
}

// One stage; v holds the owned values on entry (stage input) and on exit (next stage's input,
// or the transform's output after the last stage).
template <int DIR, int N, int NT, int R, int L, int OFF, bool LAST>
__device__ __forceinline__ void stage(cf (&v)[N / NT], cf* buf, const Tw<float>* __restrict__ tw,
                                      int t) {
  constexpr int E = N / NT, K = E / R;
  static_assert(E % R == 0, "radix must divide the values per thread");
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const int i = t + j * NT;
    const int k = i % L;
    cf u[R];
#pragma unroll
    for (int r = 0; r < R; ++r) u[r] = v[j + r * K];
    if constexpr (L > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) u[r] = twmul<DIR>(u[r], tw[OFF + (r - 1) * L + k]);
    }
    dft<DIR, R>(u);
    if constexpr (LAST) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[j + r * K] = u[r];
    } else {
      const int base = (i - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[pad(base + r * L)] = u[r];
    }
    // compiler-only fence: one butterfly's twiddles and temporaries are dead before the next
    // butterfly's loads are issued (keeps the live registers of a stage at one butterfly)
    asm volatile("" ::: "memory");
  }
  if constexpr (!LAST) {
    __syncthreads();
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = buf[pad(t + m * NT)];
  }
}

// A stage whose radix does not divide the values per thread E: the owned values go to in_buf,
// each thread gathers whole butterflies i = t + j·NT < N/R (the last round partly idle), writes
// their outputs to out_buf and reads back its owned values. Two barriers instead of one; the
// caller leaves `phase` as it was (both buffers were used, the last reads were from out_buf).
template <int DIR, int N, int NT, int R, int L, int OFF>
__device__ __forceinline__ void stage_gather(cf (&v)[N / NT], cf* in_buf, cf* out_buf,
                                             const Tw<float>* __restrict__ tw, int t) {
  constexpr int E = N / NT, NB = N / R, KG = (NB + NT - 1) / NT;
#pragma unroll
  for (int m = 0; m < E; ++m) in_buf[pad(t + m * NT)] = v[m];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < KG; ++j) {
    const int i = t + j * NT;
    if (NB % NT == 0 || i < NB) {
      const int k = i % L;
      cf u[R];
#pragma unroll
      for (int r = 0; r < R; ++r) u[r] = in_buf[pad(i + r * NB)];
      if constexpr (L > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) u[r] = twmul<DIR>(u[r], tw[OFF + (r - 1) * L + k]);
      }
      dft<DIR, R>(u);
      const int base = (i - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) out_buf[pad(base + r * L)] = u[r];
    }
    asm volatile("" ::: "memory");
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < E; ++m) v[m] = out_buf[pad(t + m * NT)];
}

template <int DIR, int N, int NT, int L, int OFF, int R, int... Rest>
__device__ __forceinline__ void stages(cf (&v)[N / NT], cf* b0, cf* b1, int& phase,
                                       const Tw<float>* __restrict__ tw, int t) {
  constexpr bool last = sizeof...(Rest) == 0;
  if constexpr ((N / NT) % R == 0) {
    stage<DIR, N, NT, R, L, OFF, last>(v, phase ? b1 : b0, tw, t);
    if constexpr (!last) phase ^= 1;
  } else {
    stage_gather<DIR, N, NT, R, L, OFF>(v, phase ? b1 : b0, phase ? b0 : b1, tw, t);
  }
  if constexpr (!last) stages<DIR, N, NT, L * R, OFF + L * (R - 1), Rest...>(v, b0, b1, phase, tw, t);
}

// In-register transform of the owned values (DIR −1 forward, +1 inverse unnormalised).
// `phase` selects the exchange buffer and must be uniform across the block; the buffer it
// points to after the transform is free for the caller (no thread still reads it).
template <int DIR, int N, int NT, int... Rs>
__device__ __forceinline__ void fft(cf (&v)[N / NT], cf* b0, cf* b1, int& phase,
                                   const Tw<float>* __restrict__ tw, int t, Radices<Rs...>) {
  static_assert((1 * ... * Rs) == N, "radices must multiply to N");
  stages<DIR, N, NT, 1, 0, Rs...>(v, b0, b1, phase, tw, t);
}

}  // namespace rf
}  // namespace bwpm
