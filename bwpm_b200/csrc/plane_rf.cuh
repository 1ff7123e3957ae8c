// Fixed-length complex64 3D slab-step kernels: register-resident transforms (rfft.cuh) for
// lateral sizes 256, 384, 512, 768 and 1024.
//
// Same step as k_cols_step_bulk + k_rows_select (plane_kernels.cuh), the path of
// cpp/src/solver_cuda.cu:140-330 (FFT → operator × propagator → inverse FFT → selection by pair
// id → mask), with the transforms held in registers: a thread owns the positions t + m·NT
// (m < E = N/NT) of both field components of its line, a stage exchanges through shared memory
// once (two buffers per line, one barrier), and the two components share each twiddle load. The
// general kernels stage every radix-2..8 pass through shared memory twice with two barriers and
// hold up to 16 values per thread in flight, which left them latency-bound with spills.
//
// Data layouts are those of the general kernels, so both families mix within one run: xbuf and
// the work planes x-major (pixel (x, y) at (x·ny + y)·2 + c), `out`, pair ids and masks
// row-major. The twiddles are the per-stage tables of plan.hpp for this file's radix order.
#pragma once

#include <vector>

#include "plane_kernels.cuh"
#include "rfft.cuh"

namespace bwpm {

// Radix order and threads per line of each length: E = N/NT values per thread and component
// (8, or 12 for 3·2^k), every radix divides E (no gather stages). These are the orders the
// resident 2D engine measured fastest for its single-line kernels of the same lengths.
template <int N>
struct PlaneRf;
template <>
struct PlaneRf<256> {
  static constexpr int NT = 32;
  using R = rf::Radices<8, 8, 4>;
};
template <>
struct PlaneRf<384> {
  static constexpr int NT = 32;
  using R = rf::Radices<4, 4, 4, 3, 2>;
};
template <>
struct PlaneRf<512> {
  static constexpr int NT = 64;
  using R = rf::Radices<8, 8, 8>;
};
template <>
struct PlaneRf<768> {
  static constexpr int NT = 64;
  using R = rf::Radices<4, 4, 4, 4, 3>;
};
template <>
struct PlaneRf<1024> {
  static constexpr int NT = 128;
  using R = rf::Radices<8, 8, 8, 2>;
};

constexpr int kRfThreads = 256;  // threads per CTA of both kernels

// Lines per CTA (columns of the column kernel, rows of the row kernel).
template <int N>
constexpr int rf_lines() {
  return kRfThreads / PlaneRf<N>::NT;
}

// Shared memory of a CTA: per line two components × two exchange buffers.
template <int N>
constexpr std::size_t rf_smem() {
  return static_cast<std::size_t>(rf_lines<N>()) * 4 * rf::padded(N) * sizeof(cf);
}

namespace rfp {

// One stage on both components (a, b) of a line: rf::stage with the twiddle shared.
template <int DIR, int N, int NT, int R, int L, int OFF, bool LAST>
__device__ __forceinline__ void stage2(cf (&a)[N / NT], cf (&b)[N / NT], cf* bufa, cf* bufb,
                                       const Tw<float>* __restrict__ tw, int t) {
  constexpr int E = N / NT, K = E / R;
  static_assert(E % R == 0, "radix must divide the values per thread");
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const int i = t + j * NT;
    const int k = i % L;
    cf u[R], v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      u[r] = a[j + r * K];
      v[r] = b[j + r * K];
    }
    if constexpr (L > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const Tw<float> w = tw[OFF + (r - 1) * L + k];
        u[r] = twmul<DIR>(u[r], w);
        v[r] = twmul<DIR>(v[r], w);
      }
    }
    rf::dft<DIR, R>(u);
    rf::dft<DIR, R>(v);
    if constexpr (LAST) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        a[j + r * K] = u[r];
        b[j + r * K] = v[r];
      }
    } else {
      const int base = (i - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        bufa[rf::pad(base + r * L)] = u[r];
        bufb[rf::pad(base + r * L)] = v[r];
      }
    }
    asm volatile("" ::: "memory");
  }
  if constexpr (!LAST) {
    __syncthreads();
#pragma unroll
    for (int m = 0; m < E; ++m) {
      a[m] = bufa[rf::pad(t + m * NT)];
      b[m] = bufb[rf::pad(t + m * NT)];
    }
  }
}

template <int DIR, int N, int NT, int L, int OFF, int R, int... Rest>
__device__ __forceinline__ void stages2(cf (&a)[N / NT], cf (&b)[N / NT], cf* const (&buf)[2][2],
                                        int& phase, const Tw<float>* __restrict__ tw, int t) {
  constexpr bool last = sizeof...(Rest) == 0;
  stage2<DIR, N, NT, R, L, OFF, last>(a, b, buf[phase][0], buf[phase][1], tw, t);
  if constexpr (!last) {
    phase ^= 1;
    stages2<DIR, N, NT, L * R, OFF + L * (R - 1), Rest...>(a, b, buf, phase, tw, t);
  }
}

// Transform of both components of a line in registers (DIR −1 forward, +1 inverse
// unnormalised). buf[phase][c] are the line's exchange buffers; after the call the buffers of
// buf[phase] are free (no thread of the block still reads them).
template <int DIR, int N, int... Rs>
__device__ __forceinline__ void fft2(cf (&a)[N / PlaneRf<N>::NT], cf (&b)[N / PlaneRf<N>::NT],
                                     cf* const (&buf)[2][2], int& phase,
                                     const Tw<float>* __restrict__ tw, int t, rf::Radices<Rs...>) {
  static_assert((1 * ... * Rs) == N, "radices must multiply to N");
  stages2<DIR, N, PlaneRf<N>::NT, 1, 0, Rs...>(a, b, buf, phase, tw, t);
}

}  // namespace rfp

// y transform of each column, per pass the operator product and the inverse y transform into
// the pass's work plane (k_cols_step_bulk's contract; a.cols is unused). CTA: rf_lines<NY>()
// columns, NT threads each. One CTA per SM at full registers: the spectrum is held across the
// passes' transforms, and at 128 registers (two CTAs) it spilled; 512² microlens 38.3 → 35.6 µs
// per slab pass, 1024² 260 → 254 µs.
template <int NY>
__global__ void __launch_bounds__(kRfThreads, 1)
    k_cols_rf(ColStep<float> a, const PassRec* __restrict__ ps, int npass,
              const Tw<float>* __restrict__ tw) {
  constexpr int NT = PlaneRf<NY>::NT, E = NY / NT, P = rf::padded(NY);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cf* sm = reinterpret_cast<cf*>(smem_raw);
  const int line = threadIdx.x / NT, t = threadIdx.x % NT;
  cf* base = sm + static_cast<long long>(line) * 4 * P;
  cf* const buf[2][2] = {{base, base + P}, {base + 2 * P, base + 3 * P}};
  const int nx = a.nx;
  const long long n = static_cast<long long>(NY) * nx;
  const int x = blockIdx.x * rf_lines<NY>() + line;  // the host launches nx / lines CTAs
  cf sx[E], sy[E];
#pragma unroll
  for (int m = 0; m < E; ++m)
    ld_px(a.in + (static_cast<long long>(x) * NY + t + m * NT) * 2, sx[m], sy[m]);
  int phase = 0;
  rfp::fft2<-1, NY>(sx, sy, buf, phase, tw, t, typename PlaneRf<NY>::R{});
  if (a.spec_out)
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const long long q = static_cast<long long>(t + m * NT) * nx + x;
      a.spec_out[2 * q] = sx[m];
      a.spec_out[2 * q + 1] = sy[m];
    }
  for (int j = 0; j < npass; ++j) {
    const PassRec pr = ps[j];
    const cf* tab = static_cast<const cf*>(pr.tab);
    cf wx[E], wy[E];
    if (pr.scalar) {
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const long long q = static_cast<long long>(x) * NY + t + m * NT;
        const cf hi = tab[q], lo = tab[n + q];
        wx[m] = pmul(sx[m], hi, lo);
        wy[m] = pmul(sy[m], hi, lo);
      }
    } else {
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const long long q = static_cast<long long>(x) * NY + t + m * NT;
        cf tv[6];
#pragma unroll
        for (int b = 0; b < 6; ++b) tv[b] = tab[b * n + q];
        wx[m] = tmul_v(sx[m], tv, 0) + tmul_v(sy[m], tv, 1);
        wy[m] = tmul_v(sx[m], tv, 1) + tmul_v(sy[m], tv, 2);
        // the table values of four points in flight at a time
        if (m % 4 == 3) asm volatile("" ::: "memory");
      }
    }
    rfp::fft2<+1, NY>(wx, wy, buf, phase, tw, t, typename PlaneRf<NY>::R{});
    cf* w = a.work + static_cast<long long>(j) * 2 * n;
#pragma unroll
    for (int m = 0; m < E; ++m)
      st_px(w + (static_cast<long long>(x) * NY + t + m * NT) * 2, wx[m], wy[m]);
  }
}

// Per CTA rf_lines<NX>() rows: per pass the inverse x transform of the work planes' rows, the
// selection by pair id, mask and reflection gather; then the sparse sources, the output rows and
// (with xnext) their forward x transform, stored x-major (k_rows_select's contract; a.rows,
// a.group unused). Every pixel belongs to exactly one transmission pass (its pair's). The host
// launches ny / lines CTAs (ny a multiple of the lines). The lines of a CTA interleave within a
// warp (line = thread mod lines), so one warp access covers the whole x-major run of the CTA's
// rows at each of its x (whole 32-byte sectors): with one line per warp, every sector was
// requested by as many warps as lines (512² microlens: 43.0 → 36.9 µs per slab pass).
template <int NX>
__global__ void __launch_bounds__(kRfThreads, 2)
    k_rows_rf(RowSelect<float> a, const PassRec* __restrict__ ps, int npass,
              const Tw<float>* __restrict__ tw) {
  constexpr int NT = PlaneRf<NX>::NT, E = NX / NT, P = rf::padded(NX), LN = rf_lines<NX>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cf* sm = reinterpret_cast<cf*>(smem_raw);
  const int line = threadIdx.x % LN, t = threadIdx.x / LN;
  cf* base = sm + static_cast<long long>(line) * 4 * P;
  cf* const buf[2][2] = {{base, base + P}, {base + 2 * P, base + 3 * P}};
  const int ny = a.ny;
  const long long n = static_cast<long long>(ny) * NX;
  const int y0 = blockIdx.x * LN, y = y0 + line;
  const long long row = static_cast<long long>(y) * NX;
  const int k0 = a.iface ? a.rowoff[y0] : 0, k1 = a.iface ? a.rowoff[y0 + LN] : 0;
  cf ox[E], oy[E];
#pragma unroll
  for (int m = 0; m < E; ++m) ox[m] = oy[m] = cf{0.f, 0.f};
  int phase = 0;
  for (int j = 0; j < npass; ++j) {
    const PassRec pr = ps[j];
    const cf* w = a.work + static_cast<long long>(j) * 2 * n;
    cf wx[E], wy[E];
#pragma unroll
    for (int m = 0; m < E; ++m)
      ld_px(w + (static_cast<long long>(t + m * NT) * ny + y) * 2, wx[m], wy[m]);
    rfp::fft2<+1, NX>(wx, wy, buf, phase, tw, t, typename PlaneRf<NX>::R{});
    if (!pr.refl) {
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const long long q = row + t + m * NT;
        if (!a.pid || a.pid[q] == pr.pair) {
          ox[m] = wx[m] * a.inv_n;
          oy[m] = wy[m] * a.inv_n;
        }
      }
    } else {
      // the gather reads other threads' values: through the free buffers, natural order
      cf* gx = buf[phase][0];
      cf* gy = buf[phase][1];
#pragma unroll
      for (int m = 0; m < E; ++m) {
        gx[rf::pad(t + m * NT)] = wx[m];
        gy[rf::pad(t + m * NT)] = wy[m];
      }
      __syncthreads();
      for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        const int q = a.iface[k];
        if (a.pid && a.pid[q] != pr.pair) continue;
        const int qy = q / NX, qx = q - qy * NX;
        const cf* lb = sm + static_cast<long long>(qy - y0) * 4 * P + (phase ? 2 * P : 0);
        a.refl_out[2 * k] = lb[rf::pad(qx)] * a.inv_n;
        a.refl_out[2 * k + 1] = lb[P + rf::pad(qx)] * a.inv_n;
      }
      __syncthreads();  // the next transform writes these buffers first
    }
  }
  if (a.mask)
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const long long q = row + t + m * NT;
      ox[m] = mmul(ox[m], a.mask, q, n);
      oy[m] = mmul(oy[m], a.mask, q, n);
    }
  if (a.add && k1 > k0) {  // sparse sources (distinct pixels) through the free buffers
    cf* gx = buf[phase][0];
    cf* gy = buf[phase][1];
#pragma unroll
    for (int m = 0; m < E; ++m) {
      gx[rf::pad(t + m * NT)] = ox[m];
      gy[rf::pad(t + m * NT)] = oy[m];
    }
    __syncthreads();
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
      const int q = a.iface[k];
      const int qy = q / NX, qx = q - qy * NX;
      cf* lb = sm + static_cast<long long>(qy - y0) * 4 * P + (phase ? 2 * P : 0);
      lb[rf::pad(qx)] = lb[rf::pad(qx)] + a.add[2 * k];
      lb[P + rf::pad(qx)] = lb[P + rf::pad(qx)] + a.add[2 * k + 1];
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < E; ++m) {
      ox[m] = gx[rf::pad(t + m * NT)];
      oy[m] = gy[rf::pad(t + m * NT)];
    }
    __syncthreads();  // the next transform writes these buffers first
  }
  if (a.store_out || !a.xnext)
#pragma unroll
    for (int m = 0; m < E; ++m) st_px(a.out + 2 * (row + t + m * NT), ox[m], oy[m]);
  if (a.xnext) {
    rfp::fft2<-1, NX>(ox, oy, buf, phase, tw, t, typename PlaneRf<NX>::R{});
#pragma unroll
    for (int m = 0; m < E; ++m)
      st_px(a.xnext + (static_cast<long long>(t + m * NT) * ny + y) * 2, ox[m], oy[m]);
  }
}

// ---- host side: kernel, shared memory and radix order per run-time length ------------------

using ColsRfFn = void (*)(ColStep<float>, const PassRec*, int, const Tw<float>*);
using RowsRfFn = void (*)(RowSelect<float>, const PassRec*, int, const Tw<float>*);

struct RfKernels {
  ColsRfFn cols = nullptr;
  RowsRfFn rows = nullptr;
  int lines = 0;          // lines per CTA
  std::size_t smem = 0;   // shared memory per CTA
  std::vector<int> radices;
};

template <int... Rs>
inline std::vector<int> radix_list(rf::Radices<Rs...>) {
  return {Rs...};
}

template <int N>
inline RfKernels rf_kernels_of() {
  return {k_cols_rf<N>, k_rows_rf<N>, rf_lines<N>(), rf_smem<N>(),
          radix_list(typename PlaneRf<N>::R{})};
}

// The fixed-length kernels of length n (cols/rows null when there are none).
inline RfKernels rf_kernels(int n) {
  switch (n) {
    case 256: return rf_kernels_of<256>();
    case 384: return rf_kernels_of<384>();
    case 512: return rf_kernels_of<512>();
    case 768: return rf_kernels_of<768>();
    case 1024: return rf_kernels_of<1024>();
    default: return {};
  }
}

}  // namespace bwpm
