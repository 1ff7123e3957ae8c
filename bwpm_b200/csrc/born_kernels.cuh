// Born-step kernels of the plane engine: weak index fluctuations δn in one host medium per slab.
//
// Restates cpp/src/solver.cpp:215-382 (CUDA twin cpp/src/solver_cuda.cu:190-350):
//   G_d·S = i dz/(2k_z)·[P(k_d)·F{V·F⁻¹(Ŝ⊥, Ŝ_z)}]⊥,  Ŝ_z = −d·k⊥·Ŝ⊥/k_z,  V = 2ñ₀k₀²δn,
//   Cayley step: x = P_½Ê, (1 − G/2)·y = G·x (GMRES), ΔÊ = P_½^{±}·y,
//   sources Ŝ_m = F{V·E_m} at the Gauss points ζ_m = (1 ∓ 1/√3)/2·dz,
//   emission Σ_m ½·e^{i d′k_z(dz−ζ_m)}·i dz/(2k_z)·[P(k_d′)·Ŝ_m]⊥,
// on propagating, non-grazing waves only. Per-point quantities (k⊥, k_z, propagation flag) are
// evaluated in FP64 from the grid; fields are stored in the engine's type T.
#pragma once

#include "fft.cuh"
#include "interface.cuh"
#include "plane_kernels.cuh"

namespace bwpm {

struct BornGrid {
  cd host;       // ñ₀ of the slab
  double k0, dz, dy, dx;
  int ny, nx;
};

struct BornPoint {
  double kx, ky;
  cd kz;
  bool prop;
};

__device__ __forceinline__ BornPoint born_point(const BornGrid& g, long long q) {
  BornPoint p;
  p.kx = fftfreq(q % g.nx, g.nx, g.dx);
  p.ky = fftfreq(q / g.nx, g.ny, g.dy);
  const double kp2 = p.kx * p.kx + p.ky * p.ky;
  p.kz = kz_of(g.host, g.k0, kp2);
  const cd host2k2 = ((g.host * g.host) * g.k0) * g.k0;  // as cpp/src/solver.cpp:221
  p.prop = born_propagating(host2k2, kp2);
  return p;
}

// a·x + b·y in FP64, stored in T (the vector update of k_axpby).
template <typename T>
__device__ __forceinline__ cx<T> axpby_at(cd a, cx<T> x, cd b, cx<T> y) {
  return cast<T>(a * cast<double>(x) + b * cast<double>(y));
}

// out = in · e^{i·sign·k_z·dz/2} on propagating waves, 0 elsewhere (P_½ and its inverse).
template <typename T>
__device__ __forceinline__ void born_half_at(long long q, const cx<T>* in, cx<T>* out,
                                             const BornGrid& g, double sign) {
  const BornPoint p = born_point(g, q);
  cd f{0.0, 0.0};
  if (p.prop) f = cexp(cd{0.0, sign} * p.kz * (g.dz / 2.0));
  out[2 * q] = cast<T>(cast<double>(in[2 * q]) * f);
  out[2 * q + 1] = cast<T>(cast<double>(in[2 * q + 1]) * f);
}

template <typename T>
__global__ void k_born_half(const cx<T>* in, cx<T>* out, BornGrid g, double sign) {
  const long long n = static_cast<long long>(g.ny) * g.nx;
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q < n) born_half_at(q, in, out, g, sign);
}

// The Born slab of the current step in device memory (grid with the slab's host index,
// direction, potential plane): the operator kernels of the GMRES cycle graph, captured once per
// solver, read it here, so one graph serves every slab and both directions.
template <typename T>
struct BornCur {
  BornGrid g;
  int dir;
  const cx<T>* pot;
};

template <typename T>
__global__ void k_set_born_cur(BornCur<T>* cur, BornCur<T> v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *cur = v;
}

// w3 = (Ŝ_x, Ŝ_y, −d·k⊥·Ŝ⊥/k_z)·e^{i k_z s} on propagating waves (s = 0: no phase), 0 elsewhere.
template <typename T>
__device__ __forceinline__ void born_prepare_at(long long q, const cx<T>* spec, cx<T>* w3,
                                                const BornGrid& g, int direction,
                                                double distance) {
  const BornPoint p = born_point(g, q);
  if (!p.prop) {
    w3[3 * q] = w3[3 * q + 1] = w3[3 * q + 2] = cx<T>{0, 0};
    return;
  }
  const cd ex = cast<double>(spec[2 * q]), ey = cast<double>(spec[2 * q + 1]);
  const cd ez = cdiv(-static_cast<double>(direction) * (p.kx * ex + p.ky * ey), p.kz);
  cd ph{1.0, 0.0};
  if (distance != 0.0) ph = cexp(cd{0.0, 1.0} * p.kz * distance);
  w3[3 * q] = cast<T>(ex * ph);
  w3[3 * q + 1] = cast<T>(ey * ph);
  w3[3 * q + 2] = cast<T>(ez * ph);
}

template <typename T>
__global__ void k_born_prepare(const cx<T>* spec, cx<T>* w3, BornGrid g, int direction,
                               double distance) {
  const long long n = static_cast<long long>(g.ny) * g.nx;
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q < n) born_prepare_at(q, spec, w3, g, direction, distance);
}

// P_½ (signed = 0) or P_½^{±} with the sign of the current slab's direction (signed = 1).
template <typename T>
__global__ void k_born_half_cur(const cx<T>* in, cx<T>* out, const BornCur<T>* cur, int signed_) {
  const BornGrid g = cur->g;
  const long long n = static_cast<long long>(g.ny) * g.nx;
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q < n) born_half_at(q, in, out, g, signed_ && cur->dir <= 0 ? -1.0 : 1.0);
}

template <typename T>
__global__ void k_born_prepare_cur(const cx<T>* spec, cx<T>* w3, const BornCur<T>* cur) {
  const BornGrid g = cur->g;
  const long long n = static_cast<long long>(g.ny) * g.nx;
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q < n) born_prepare_at(q, spec, w3, g, cur->dir, 0.0);
}

// w3 *= V·(1/N) in real space, V = 2ñ₀k₀²δn precomputed per pixel.
template <typename T>
__global__ void k_born_potential(cx<T>* w3, const cx<T>* v, long long n, T inv_n) {
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q >= n) return;
  const cx<T> s = v[q] * inv_n;
  for (int c = 0; c < 3; ++c) w3[3 * q + c] = s * w3[3 * q + c];
}

template <typename T>
__global__ void k_born_potential_cur(cx<T>* w3, const BornCur<T>* cur, long long n, T inv_n) {
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q >= n) return;
  const cx<T> s = cur->pot[q] * inv_n;
  for (int c = 0; c < 3; ++c) w3[3 * q + c] = s * w3[3 * q + c];
}

// out = i dz/(2k_z)·(Ŝ⊥ − k⊥·(k⊥·Ŝ⊥ + d·k_z·Ŝ_z)/k²) on propagating waves, 0 elsewhere.
template <typename T>
__device__ __forceinline__ void born_finish_at(long long q, const cx<T>* w3, cx<T>* out,
                                               const BornGrid& g, int direction) {
  const BornPoint p = born_point(g, q);
  if (!p.prop) {
    out[2 * q] = out[2 * q + 1] = cx<T>{0, 0};
    return;
  }
  const cd k = g.host * g.k0;
  const cd k2 = k * k;
  const cd green = cdiv(cd{0.0, g.dz}, 2.0 * p.kz);
  const cd s0 = cast<double>(w3[3 * q]), s1 = cast<double>(w3[3 * q + 1]),
           s2 = cast<double>(w3[3 * q + 2]);
  const cd lon = cdiv(p.kx * s0 + p.ky * s1 + (static_cast<double>(direction) * p.kz) * s2, k2);
  out[2 * q] = cast<T>(green * (s0 - p.kx * lon));
  out[2 * q + 1] = cast<T>(green * (s1 - p.ky * lon));
}

template <typename T>
__global__ void k_born_finish(const cx<T>* w3, cx<T>* out, BornGrid g, int direction) {
  const long long n = static_cast<long long>(g.ny) * g.nx;
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q < n) born_finish_at(q, w3, out, g, direction);
}

// With `in` (the operator of the Cayley step, A = 1 − G/2): out = in − G·in/2, in the
// arithmetic of k_axpby(out ← in, G·in, −½, 1) on G·in stored in T.
template <typename T>
__global__ void k_born_finish_cur(const cx<T>* w3, cx<T>* out, const BornCur<T>* cur,
                                  const cx<T>* in) {
  const BornGrid g = cur->g;
  const long long n = static_cast<long long>(g.ny) * g.nx;
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q >= n) return;
  born_finish_at(q, w3, out, g, cur->dir);
  if (in)
    for (int c = 0; c < 2; ++c)
      out[2 * q + c] = axpby_at(cd{-0.5, 0.0}, out[2 * q + c], cd{1.0, 0.0}, in[2 * q + c]);
}

// total = Σ_m ½·e^{i d′k_z(1−ζ_m)dz}·i dz/(2k_z)·[P(k_d′)·Ŝ_m]⊥ (spectrum), sources (2, N, 3).
template <typename T>
__global__ void k_born_emit(const cx<T>* sources, cx<T>* total, BornGrid g, int direction) {
  const long long n = static_cast<long long>(g.ny) * g.nx;
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q >= n) return;
  const BornPoint p = born_point(g, q);
  if (!p.prop) {
    total[2 * q] = total[2 * q + 1] = cx<T>{0, 0};
    return;
  }
  const double r3 = 0.57735026918962576451;  // 1/√3
  const double gauss[2] = {(1.0 - r3) / 2.0, (1.0 + r3) / 2.0};
  const cd skz = static_cast<double>(direction) * p.kz;
  const cd k = g.host * g.k0;
  const cd k2 = k * k;
  cd t0{0.0, 0.0}, t1{0.0, 0.0};
  for (int m = 0; m < 2; ++m) {
    const cd green = (0.5 * cexp(cd{0.0, 1.0} * skz * ((1.0 - gauss[m]) * g.dz))) *
                     cdiv(cd{0.0, g.dz}, 2.0 * p.kz);
    const cx<T>* s = sources + 3 * n * m + 3 * q;
    const cd s0 = cast<double>(s[0]), s1 = cast<double>(s[1]), s2 = cast<double>(s[2]);
    const cd lon = cdiv(p.kx * s0 + p.ky * s1 + skz * s2, k2);
    t0 = t0 + green * (s0 - p.kx * lon);
    t1 = t1 + green * (s1 - p.ky * lon);
  }
  total[2 * q] = cast<T>(t0);
  total[2 * q + 1] = cast<T>(t1);
}

// ---- vector operations for GMRES (length m complex) ---------------------------------------

template <typename T>
__global__ void k_axpby(cx<T>* y, const cx<T>* x, cd a, cd b, long long m) {
  // y = a·x + b·y
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i >= m) return;
  y[i] = axpby_at(a, x[i], b, y[i]);
}

// ---- transforms of planes with ncomp interleaved components ---------------------------------

// nx = 1: one CTA per component, the whole line in shared memory. A launch has ncomp CTAs, so
// a transform's latency is the cost: the stages are expanded in the kernel (no register saves
// through local memory per stage), 128 registers, and EPT values per thread (8 where the
// threads allow it: twice the warps of 16).
template <int DIR, typename T, int EPT = 16>
__global__ void __launch_bounds__(kPlaneThreads, 1)
    k_line_fft(const cx<T>* in, cx<T>* out, int n, int ncomp, const __grid_constant__ FftPlan plan,
               const Tw<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* buf = reinterpret_cast<cx<T>*>(smem_raw);
  const int c = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  for (int q = tid; q < n; q += nt) buf[q] = in[static_cast<long long>(q) * ncomp + c];
  __syncthreads();
  fft_smem_inline<DIR, EPT>(buf, plan, tw, 1, tid, nt);
  for (int q = tid; q < n; q += nt) out[static_cast<long long>(q) * ncomp + c] = buf[q];
}

// y transform of `cols` columns × ncomp components per CTA; smem [y][col][comp].
template <int DIR, typename T>
__global__ void __launch_bounds__(kPlaneThreads, kPlaneMinBlocks<T>)
    k_cols_fft(const cx<T>* in, cx<T>* out, int ny, int nx, int ncomp, int cols,
               const __grid_constant__ FftPlan plan, const Tw<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* buf = reinterpret_cast<cx<T>*>(smem_raw);
  const int x0 = blockIdx.x * cols;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = cols * ncomp, tile = ny * lane;
  for (int idx = tid; idx < tile; idx += nt) {
    const int y = idx / lane, rem = idx - y * lane;
    const int x = x0 + rem / ncomp, c = rem % ncomp;
    buf[idx] = x < nx ? in[(static_cast<long long>(y) * nx + x) * ncomp + c] : cx<T>{0, 0};
  }
  __syncthreads();
  fft_smem_inline<DIR>(buf, plan, tw, lane, tid, nt);
  for (int idx = tid; idx < tile; idx += nt) {
    const int y = idx / lane, rem = idx - y * lane;
    const int x = x0 + rem / ncomp, c = rem % ncomp;
    if (x < nx) out[(static_cast<long long>(y) * nx + x) * ncomp + c] = buf[idx];
  }
}

}  // namespace bwpm
