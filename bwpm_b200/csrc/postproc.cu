// Post-processing of transverse fields on the device, FP64 with compensated sums:
// - port_power: Poynting flux through a port plane, Σ Re k_z (|Ê_x|² + |Ê_y|² + |Ê_z|²)·dx·dy/N
//   with Ê_z = −direction·(k_x Ê_x + k_y Ê_y)/k_z (src/bwpm/adapter.py:267-284); with nx = 1 and
//   dx = 1 it is the 2D power flux of src/bwpm/fpwpm.py:205-216 (the facade's energy residual);
// - plane_power: n Σ cos θ (|E_s|² + |E_p|²) over the propagating modes
//   (src/bwpm/pilot_imc3d.py:24-67);
// - axial_focus: the on-axis intensity Σ_c |Σ_k A_c(k) e^{i k_z d}|²/(nx·ny)² of the propagating
//   modes, E_z = −k⊥·E⊥/k_z, at each offset d (src/bwpm/pilot_imc3d.py:96-131).
// The angular spectrum is this library's FP64 FFT (unnormalised forward transform, like
// numpy.fft.fft2); k grids follow numpy.fft.fftfreq with the reference's rounding.
#include <algorithm>
#include <cmath>

#include "born_kernels.cuh"
#include "devbuf.hpp"
#include "plan.hpp"
#include "plane_kernels.cuh"
#include "postproc.hpp"

namespace bwpm {
namespace {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 296;  // 2 per SM
constexpr double kGrazingCos = 1e-9;  // src/bwpm/pilot_imc3d.py:18

struct Kahan {
  double s = 0.0, c = 0.0;
  __device__ void add(double v) {
    const double y = v - c;
    const double t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

// Block sum of one double per thread (compensated over the warps); thread 0 gets the total.
__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  Kahan k;
  if (threadIdx.x == 0)
    for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) k.add(red[i]);
  __syncthreads();
  return k.s;
}

struct Modes {
  const cd* spec;  // (ny, nx, 2) unnormalised spectrum
  int ny, nx;
  double dy, dx, k0;
};

__device__ __forceinline__ void k_of(const Modes& m, long long q, double& kx, double& ky) {
  kx = fftfreq(q % m.nx, m.nx, m.dx);
  ky = fftfreq(q / m.nx, m.ny, m.dy);
}

// cos θ of mode (kx, ky) in a medium of real index n, 0 for non-propagating and grazing modes
__device__ __forceinline__ double cos_theta(double kx, double ky, double n, double k0) {
  const double k = n * k0;
  const double cos_sq = 1.0 - (kx * kx + ky * ky) / (k * k);
  const double c = sqrt(fmax(cos_sq, 0.0));
  return c > kGrazingCos ? c : 0.0;
}

__device__ __forceinline__ double norm2(cd a) { return a.re * a.re + a.im * a.im; }

// kind 0: port power terms; kind 1: plane power terms. One partial per block.
__global__ void __launch_bounds__(kRedThreads)
    k_power_terms(Modes m, int kind, cd index, int direction, double* partial) {
  __shared__ double red[kRedThreads / 32];
  const long long n = static_cast<long long>(m.ny) * m.nx;
  Kahan acc;
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    double kx, ky;
    k_of(m, q, kx, ky);
    const cd a0 = m.spec[2 * q], a1 = m.spec[2 * q + 1];
    if (kind == 0) {
      const cd kz = kz_of(index, m.k0, kx * kx + ky * ky);
      const cd ez = cdiv(-static_cast<double>(direction) * (kx * a0 + ky * a1), kz);
      acc.add(kz.re * (norm2(a0) + norm2(a1) + norm2(ez)));
    } else {
      const double ct = cos_theta(kx, ky, index.re, m.k0);
      const double kp = hypot(kx, ky);
      const double safe = kp > 0.0 ? kp : 1.0;
      const double sx = kp > 0.0 ? -ky / safe : 0.0, sy = kp > 0.0 ? kx / safe : 1.0;
      const double px = kp > 0.0 ? kx / safe : 1.0, py = kp > 0.0 ? ky / safe : 0.0;
      const cd es = a0 * sx + a1 * sy;
      const cd ep = (a0 * px + a1 * py) / (ct > kGrazingCos ? ct : 1.0);
      acc.add(ct * (norm2(es) + norm2(ep)));
    }
  }
  const double s = block_sum(acc.s, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void k_sum_partials(const double* partial, int count, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Kahan k;
  for (int i = 0; i < count; ++i) k.add(partial[i]);
  *out = k.s;
}

// Axial focus, stage 1: per mode the three on-axis amplitudes A_c (spectrum referred to the grid
// centre) and k_z, zero for modes outside the propagating set.
__global__ void k_focus_modes(Modes m, double n, double na, cd* amp, double* kz_out) {
  const long long total = static_cast<long long>(m.ny) * m.nx;
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q >= total) return;
  double kx, ky;
  k_of(m, q, kx, ky);
  const double ct = cos_theta(kx, ky, n, m.k0);
  bool prop = ct > 0.0;
  if (na > 0.0) prop = prop && hypot(kx, ky) <= na * m.k0;
  if (!prop) {
    amp[3 * q] = amp[3 * q + 1] = amp[3 * q + 2] = cd{0.0, 0.0};
    kz_out[q] = 0.0;
    return;
  }
  const double arg = kx * static_cast<double>(m.nx / 2) * m.dx + ky * static_cast<double>(m.ny / 2) * m.dy;
  double sn, cs;
  sincos(arg, &sn, &cs);
  const cd shift{cs, sn};
  const cd ax = m.spec[2 * q] * shift, ay = m.spec[2 * q + 1] * shift;
  const double kz = n * m.k0 * ct;
  amp[3 * q] = ax;
  amp[3 * q + 1] = ay;
  amp[3 * q + 2] = -(kx * ax + ky * ay) / kz;
  kz_out[q] = kz;
}

// Stage 2: grid (offset, chunk); Σ over the chunk's modes of A_c e^{i k_z d} for c = x, y, z.
__global__ void __launch_bounds__(kRedThreads)
    k_focus_sums(const cd* amp, const double* kz, long long total, const double* offsets,
                 int chunks, double* partial) {
  __shared__ double red[kRedThreads / 32];
  const int d_idx = blockIdx.x / chunks, chunk = blockIdx.x % chunks;
  const double d = offsets[d_idx];
  const long long per = (total + chunks - 1) / chunks;
  const long long q0 = chunk * per, q1 = min(total, q0 + per);
  Kahan acc[6];
  for (long long q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
    const double k = kz[q];
    if (k == 0.0) continue;
    double sn, cs;
    sincos(k * d, &sn, &cs);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const cd a = amp[3 * q + c];
      acc[2 * c].add(a.re * cs - a.im * sn);
      acc[2 * c + 1].add(a.re * sn + a.im * cs);
    }
  }
  for (int j = 0; j < 6; ++j) {
    const double s = block_sum(acc[j].s, red);
    if (threadIdx.x == 0) partial[static_cast<long long>(blockIdx.x) * 6 + j] = s;
  }
}

// Stage 3: intensity per offset from the chunk sums.
__global__ void k_focus_intensity(const double* partial, int noff, int chunks, double norm,
                                  double* intensity) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= noff) return;
  double total = 0.0;
  for (int c = 0; c < 3; ++c) {
    Kahan re, im;
    for (int k = 0; k < chunks; ++k) {
      const double* p = partial + (static_cast<long long>(d) * chunks + k) * 6;
      re.add(p[2 * c]);
      im.add(p[2 * c + 1]);
    }
    total += re.s * re.s + im.s * im.s;
  }
  intensity[d] = total / norm;
}

}  // namespace

// FP64 angular spectrum (unnormalised forward 2D FFT) of a device field (ny, nx, 2) into `out`
// (device, same shape); `tmp` is a scratch plane of the same size (unused for nx = 1).
void field_spectrum(const cd* field, cd* out, cd* tmp, int ny, int nx, cudaStream_t stream) {
  const HostPlan hy = make_plan(ny);
  DevBuf<Tw<double>> twy, twx;
  auto upload = [&](const HostPlan& hp, DevBuf<Tw<double>>& d) {
    const std::vector<Tw<double>> t = twiddles_for<double>(hp);
    d.alloc(std::max<std::size_t>(1, t.size()), stream);
    if (!t.empty())
      check_cuda(cudaMemcpyAsync(d.ptr, t.data(), t.size() * sizeof(Tw<double>),
                                 cudaMemcpyHostToDevice, stream), "twiddles");
  };
  upload(hy, twy);
  const std::size_t smem_max = 227 * 1024;
  if (nx == 1) {
    const int threads = std::max(64, threads_needed(hy.plan, 1));
    if (threads > kPlaneThreads || ny * sizeof(cd) > smem_max)
      throw invalid_argument("ny too large for the line transform");
    check_cuda(cudaFuncSetAttribute(k_line_fft<-1, double>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), "smem");
    k_line_fft<-1, double><<<2, threads, ny * sizeof(cd), stream>>>(field, out, ny, 2, hy.plan, twy.ptr);
    check_cuda(cudaGetLastError(), "k_line_fft");
  } else {
    const HostPlan hx = make_plan(nx);
    upload(hx, twx);
    int rows = std::max(1, std::min<int>(8, static_cast<int>(49152 / (nx * 2 * sizeof(cd)))));
    while (rows > 1 && threads_needed(hx.plan, rows * 2) > kPlaneThreads) --rows;
    const int rthreads = std::max(64, threads_needed(hx.plan, rows * 2));
    int cols = 2;
    while (cols > 1 && (ny * cols * 2 * sizeof(cd) > 98304 ||
                        threads_needed(hy.plan, cols * 2) > kPlaneThreads))
      --cols;
    const int cthreads = std::max(64, threads_needed(hy.plan, cols * 2));
    if (rthreads > kPlaneThreads || cthreads > kPlaneThreads ||
        nx * rows * 2 * sizeof(cd) > smem_max || ny * cols * 2 * sizeof(cd) > smem_max)
      throw invalid_argument("plane too large for the spectrum transform");
    check_cuda(cudaFuncSetAttribute(k_rows_fft<-1, double>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), "smem");
    check_cuda(cudaFuncSetAttribute(k_cols_fft<-1, double>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), "smem");
    k_rows_fft<-1, double><<<ceil_div(ny, rows), rthreads, rows * nx * 2 * sizeof(cd), stream>>>(
        field, tmp, ny, nx, 2, rows, hx.plan, twx.ptr);
    check_cuda(cudaGetLastError(), "k_rows_fft");
    k_cols_fft<-1, double><<<ceil_div(nx, cols), cthreads, ny * cols * 2 * sizeof(cd), stream>>>(
        tmp, out, ny, nx, 2, cols, hy.plan, twy.ptr);
    check_cuda(cudaGetLastError(), "k_cols_fft");
  }
}

namespace {

void check_grid(const PlaneGeometry& g) {
  if (g.ny < 1 || g.nx < 1) throw invalid_argument("ny and nx must be positive");
  if (!(g.dy > 0.0) || !(g.dx > 0.0) || !(g.k0 > 0.0))
    throw invalid_argument("dy, dx and k0 must be positive");
}

// Spectrum of a host or device field in FP64 on `stream` (spec: 2·N complex device values).
void spectrum_of(const PlaneGeometry& g, const cd* field, bool on_device, DevBuf<cd>& spec,
                 cudaStream_t stream) {
  const std::size_t n2 = 2 * static_cast<std::size_t>(g.ny) * g.nx;
  DevBuf<cd> in, tmp;
  const cd* src = field;
  if (!on_device) {
    in.alloc(n2, stream);
    check_cuda(cudaMemcpyAsync(in.ptr, field, n2 * sizeof(cd), cudaMemcpyHostToDevice, stream),
               "field upload");
    src = in.ptr;
  }
  spec.alloc(n2, stream);
  if (g.nx > 1) tmp.alloc(n2, stream);
  field_spectrum(src, spec.ptr, tmp.ptr, g.ny, g.nx, stream);
}

double power_sum(const PlaneGeometry& g, const cd* field, bool on_device, int kind, cd index,
                 int direction, cudaStream_t stream) {
  check_grid(g);
  DevBuf<cd> spec;
  spectrum_of(g, field, on_device, spec, stream);
  DevBuf<double> partial(kRedBlocks + 1, stream);
  const Modes m{spec.ptr, g.ny, g.nx, g.dy, g.dx, g.k0};
  k_power_terms<<<kRedBlocks, kRedThreads, 0, stream>>>(m, kind, index, direction, partial.ptr);
  check_cuda(cudaGetLastError(), "k_power_terms");
  k_sum_partials<<<1, 32, 0, stream>>>(partial.ptr, kRedBlocks, partial.ptr + kRedBlocks);
  check_cuda(cudaGetLastError(), "k_sum_partials");
  double out = 0.0;
  check_cuda(cudaMemcpyAsync(&out, partial.ptr + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost,
                             stream), "download");
  check_cuda(cudaStreamSynchronize(stream), "synchronize");
  return out;
}

}  // namespace

double port_power(const PlaneGeometry& g, const cd* field, bool on_device, cd index, int direction,
                  cudaStream_t stream) {
  if (direction != 1 && direction != -1) throw invalid_argument("direction must be +1 or -1");
  const double s = power_sum(g, field, on_device, 0, index, direction, stream);
  return s * g.dx * g.dy / (static_cast<double>(g.ny) * g.nx);
}

double plane_power(const PlaneGeometry& g, const cd* field, bool on_device, double index,
                   cudaStream_t stream) {
  if (!(index > 0.0)) throw invalid_argument("index must be positive");
  return index * power_sum(g, field, on_device, 1, cd{index, 0.0}, 1, stream);
}

void axial_focus(const PlaneGeometry& g, const cd* field, bool on_device, double index,
                 const double* offsets, std::size_t noff, double na, double* best, double* peak,
                 double* intensity_out, cudaStream_t stream) {
  check_grid(g);
  if (!(index > 0.0)) throw invalid_argument("index must be positive");
  if (noff == 0) throw invalid_argument("offsets must not be empty");
  DevBuf<cd> spec;
  spectrum_of(g, field, on_device, spec, stream);
  const long long total = static_cast<long long>(g.ny) * g.nx;
  DevBuf<cd> amp(3 * total, stream);
  DevBuf<double> kz(total, stream), d_off(noff, stream), d_int(noff, stream);
  const Modes m{spec.ptr, g.ny, g.nx, g.dy, g.dx, g.k0};
  k_focus_modes<<<ceil_div(total, 256), 256, 0, stream>>>(m, index, na, amp.ptr, kz.ptr);
  check_cuda(cudaGetLastError(), "k_focus_modes");
  check_cuda(cudaMemcpyAsync(d_off.ptr, offsets, noff * sizeof(double), cudaMemcpyHostToDevice,
                             stream), "offsets");
  const int chunks = static_cast<int>(std::max<long long>(
      1, std::min<long long>(ceil_div(total, 4096), std::max<long long>(1, 1184 / static_cast<long long>(noff)))));
  DevBuf<double> partial(noff * chunks * 6, stream);
  k_focus_sums<<<static_cast<unsigned>(noff * chunks), kRedThreads, 0, stream>>>(
      amp.ptr, kz.ptr, total, d_off.ptr, chunks, partial.ptr);
  check_cuda(cudaGetLastError(), "k_focus_sums");
  const double norm = static_cast<double>(total) * static_cast<double>(total);
  k_focus_intensity<<<ceil_div(noff, 128), 128, 0, stream>>>(partial.ptr, static_cast<int>(noff),
                                                            chunks, norm, d_int.ptr);
  check_cuda(cudaGetLastError(), "k_focus_intensity");
  std::vector<double> inten(noff);
  check_cuda(cudaMemcpyAsync(inten.data(), d_int.ptr, noff * sizeof(double), cudaMemcpyDeviceToHost,
                             stream), "download");
  check_cuda(cudaStreamSynchronize(stream), "synchronize");
  // the first offset with the largest intensity (src/bwpm/pilot_imc3d.py:125-131)
  double b = 0.0, p = -1.0;
  for (std::size_t i = 0; i < noff; ++i)
    if (inten[i] > p) {
      b = offsets[i];
      p = inten[i];
    }
  *best = b;
  *peak = p;
  if (intensity_out) std::copy(inten.begin(), inten.end(), intensity_out);
}

}  // namespace bwpm
