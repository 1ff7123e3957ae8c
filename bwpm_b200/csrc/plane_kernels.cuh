// Slab-step kernels of the plane engine (general ny × nx planes, FP64 or FP32 complex).
//
// One slab step (cpp/src/solver.cpp:384-417, "apply") for a field e of shape (ny, nx, 2):
//   out = mask · Σ_(r,s) I_r,s · F⁻¹{M_rs · F{e}}   (transmission kinds)
//   vals[j] = [Σ_(r,s), ñ_r≠ñ_s I_r,s · F⁻¹{R_rs · F{e}}](iface[j])   (reflection kinds)
// The forward transform is shared by the reflection and the transmission of the same step
// (the reference computes it twice), every (pair, kind) is one "pass" of spectral multiply and
// inverse transform, and the pixel selection I_r,s, the mask, the gather of reflection sources
// at interface pixels and the sparse source add of cpp/src/solver.cpp:419-441 run in the
// epilogue of the inverse transform.
//
// 2D (nx = 1): the matrices are diagonal (k_x = 0 exactly), so E_x and E_y are independent;
// k_step2d runs one CTA per component and does the whole step in shared memory.
// 3D: k_rows_fft (x transform), k_cols_step (y transform, passes, inverse y transform) and
// k_rows_select (inverse x transform + epilogue).
#pragma once

#include "bulk.cuh"
#include "fft.cuh"
#include "interface.cuh"

namespace bwpm {

constexpr int kMaxPasses = 128;
constexpr int kPlaneThreads = 512;  // CTA width limit of the plane kernels (128 registers)
// Register budget of the 3D step kernels, as CTAs of kPlaneThreads per SM: complex64 runs
// faster with two (64 registers, some spills, twice the warps), FP64 with one (128 registers;
// its butterflies hold twice the bytes). Measured per slab pass on the 512² microlens:
// complex64 64.3 µs (two) against 73.4 µs (one), FP64 115.8 against 99.1 µs.
template <typename T>
constexpr int kPlaneMinBlocks = sizeof(T) == sizeof(double) ? 1 : 2;

// Table entry times field value. FP64 tables hold one value per entry; FP32 tables hold the
// FP64 value as hi + lo with the lo block `lo` entries after the hi block (see fft.cuh on why
// constants recurring in every slab step are carried as pairs).
template <typename T>
__device__ __forceinline__ cx<T> tmul(cx<T> u, const cx<T>* m, long long q, long long lo) {
  if constexpr (sizeof(T) == sizeof(double)) {
    return u * m[q];
  } else {
    return pmul(u, m[q], m[lo + q]);
  }
}

// Table entry e (0: m00, 1: m01, 2: m11) from a point's loaded table values (kB of them: FP64
// one value per entry; FP32 hi values then lo values), times a field value; as tmul.
template <typename T, int KB>
__device__ __forceinline__ cx<T> tmul_v(cx<T> u, const cx<T> (&tv)[KB], int e) {
  if constexpr (sizeof(T) == sizeof(double)) {
    return u * tv[e];
  } else {
    return pmul(u, tv[e], tv[3 + e]);
  }
}

// Field value times the mask (FP32 masks hold hi values then lo values, `n` apart).
template <typename T>
__device__ __forceinline__ cx<T> mmul(cx<T> v, const T* mask, long long q, long long n) {
  if constexpr (sizeof(T) == sizeof(double)) {
    return v * mask[q];
  } else {
    return {fmaf(v.re, mask[q], v.re * mask[n + q]), fmaf(v.im, mask[q], v.im * mask[n + q])};
  }
}

// Operator tables: 3 entries (m00, m01, m11) of N values; FP32 tables add the 3 lo blocks.
template <typename T>
constexpr int table_blocks() {
  return sizeof(T) == sizeof(double) ? 3 : 6;
}

// One pass of a step: operator table ((m00, m01, m11) SoA, 3·N entries of cx<T>, FP32 tables
// followed by their lo blocks), pair index (into the step's pair-id plane), reflection flag. The
// records of every step live in device memory (a per-solve pool built once), so a kernel reads
// pass j as one uniform load instead of indexing a by-value parameter array.
// `scalar`: a complex64 transmission between equal indices in 3D, whose operator is the
// propagator e^{i k_z dz} times the identity (T = 1 for ñ_r = ñ_s): its table holds only that
// value (hi block, then lo block: 2·N entries) and both components are multiplied by it.
struct PassRec {
  const void* tab;
  int pair;
  int refl;
  int scalar;
};

template <typename T>
struct Step2D {
  const cx<T>* in;          // (N, 2)
  cx<T>* out;               // (N, 2)
  cx<T>* spec;              // (N, 2) spectrum scratch F{e}
  const uint8_t* pid;       // (N) pair id per pixel, or null when the step has one pair
  const T* mask;            // (N) or null
  const int* iface;         // sorted interface pixels of the step, or null
  int niface;
  cx<T>* refl_out;          // (niface, 2) gathered reflection sources, or null
  const cx<T>* add;         // (niface, 2) sparse sources added after the step, or null
  int n;
  int store_spec;           // keep F{e} in `spec` even for a single pass (Born)
  T inv_n;
};

// Two CTAs per launch: the per-CTA latency is the cost, so the stages are expanded in the
// kernel, 128 registers, and EPT values per thread (8 where the threads allow it). Against the
// stage calls at 64 registers and 16 values: 2D FP64 per-solve runs 2.0× faster.
template <typename T, int EPT = 16>
__global__ void __launch_bounds__(kPlaneThreads, 1) k_step2d(Step2D<T> a, const PassRec* __restrict__ ps, int npass, const __grid_constant__ FftPlan plan, const Tw<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* buf = reinterpret_cast<cx<T>*>(smem_raw);
  const int c = blockIdx.x;
  const int n = a.n, tid = threadIdx.x, nt = blockDim.x;
  for (int q = tid; q < n; q += nt) buf[q] = a.in[2 * q + c];
  __syncthreads();
  fft_smem_inline<-1, EPT>(buf, plan, tw, 1, tid, nt);
  cx<T>* spec = a.spec;  // interleaved (N, 2), like the field
  const bool keep_spec = npass > 1 || a.store_spec;
  if (keep_spec) {
    for (int q = tid; q < n; q += nt) spec[2 * q + c] = buf[q];
    __syncthreads();
  }
  const long long e = c == 0 ? 0 : 2LL * n;  // m00 for E_x, m11 for E_y
  for (int j = 0; j < npass; ++j) {
    const cx<T>* m = static_cast<const cx<T>*>(ps[j].tab) + e;
    if (keep_spec)
      for (int q = tid; q < n; q += nt) buf[q] = tmul(spec[2 * q + c], m, q, 3LL * n);
    else
      for (int q = tid; q < n; q += nt) buf[q] = tmul(buf[q], m, q, 3LL * n);
    __syncthreads();
    fft_smem_inline<+1, EPT>(buf, plan, tw, 1, tid, nt);
    const int pair = ps[j].pair;
    if (!ps[j].refl) {
      for (int q = tid; q < n; q += nt)
        if (!a.pid || a.pid[q] == pair) {
          cx<T> v = buf[q] * a.inv_n;
          if (a.mask) v = mmul(v, a.mask, q, n);
          a.out[2 * q + c] = v;
        }
    } else {
      for (int k = tid; k < a.niface; k += nt) {
        const int q = a.iface[k];
        if (!a.pid || a.pid[q] == pair) a.refl_out[2 * k + c] = buf[q] * a.inv_n;
      }
    }
    __syncthreads();
  }
  if (a.add)
    for (int k = tid; k < a.niface; k += nt) {
      const int q = a.iface[k];
      a.out[2 * q + c] = a.out[2 * q + c] + a.add[2 * k + c];
    }
}

// x transform of `rows` rows × ncomp interleaved components per CTA; smem [x][row][comp].
// TOUT: the output is stored transposed, out[(x·ny + y)·ncomp + c] (the layout the column
// kernel of a slab step reads contiguously); otherwise row-major like the input.
template <int DIR, typename T, bool TOUT = false>
__global__ void __launch_bounds__(kPlaneThreads, kPlaneMinBlocks<T>) k_rows_fft(const cx<T>* in, cx<T>* out, int ny, int nx, int ncomp, int rows,
                           const __grid_constant__ FftPlan plan, const Tw<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* buf = reinterpret_cast<cx<T>*>(smem_raw);
  const int y0 = blockIdx.x * rows;
  const int here = min(rows, ny - y0);
  const int tid = threadIdx.x, nt = blockDim.x;
  const int per_row = nx * ncomp;
  const int total = rows * per_row;
  for (int idx = tid; idx < total; idx += nt) {
    const int row = idx / per_row, rem = idx - row * per_row;
    const int x = rem / ncomp, c = rem - x * ncomp;
    buf[(x * rows + row) * ncomp + c] =
        row < here ? in[(static_cast<long long>(y0 + row) * nx + x) * ncomp + c] : cx<T>{0, 0};
  }
  __syncthreads();
  fft_smem_inline<DIR>(buf, plan, tw, rows * ncomp, tid, nt);
  if constexpr (TOUT) {  // per x a run of `here` rows × ncomp, contiguous in both memories
    const int run = here * ncomp;
    for (int idx = tid; idx < nx * run; idx += nt) {
      const int x = idx / run, rem = idx - x * run;
      out[(static_cast<long long>(x) * ny + y0) * ncomp + rem] = buf[x * rows * ncomp + rem];
    }
  } else {
    for (int idx = tid; idx < here * per_row; idx += nt) {
      const int row = idx / per_row, rem = idx - row * per_row;
      const int x = rem / ncomp, c = rem - x * ncomp;
      out[(static_cast<long long>(y0 + row) * nx + x) * ncomp + c] = buf[(x * rows + row) * ncomp + c];
    }
  }
}

template <typename T>
struct ColStep {
  const cx<T>* in;      // x-transformed field, transposed: in[(x·ny + y)·2 + c]
  cx<T>* work;          // npass planes, transposed like `in`
  cx<T>* spec_out;      // full spectrum F{e} (N, 2) row-major, or null
  int ny, nx, cols;
  int* status;          // k_cols_step_bulk: set to 1 when a bulk copy does not complete in time
};

// y transform of a tile of `cols` columns, then per pass: W = M·Ŝ (2×2), inverse y transform,
// store to work plane j. The x-transformed field, the work planes and the operator tables of a
// 3D solve are stored transposed (x-major), so every column is one contiguous run in memory.
// smem: spectrum tile [y][col][2] and, for several passes, a work tile.
template <typename T>
__global__ void __launch_bounds__(kPlaneThreads, kPlaneMinBlocks<T>) k_cols_step(ColStep<T> a, const PassRec* __restrict__ ps, int npass, const __grid_constant__ FftPlan plan,
                            const Tw<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* sbuf = reinterpret_cast<cx<T>*>(smem_raw);
  const int ny = a.ny, nx = a.nx, cols = a.cols;
  const long long n = static_cast<long long>(ny) * nx;
  const int tile = ny * cols * 2;
  const int run = 2 * ny;  // one column, both components
  cx<T>* wbuf = npass > 1 ? sbuf + tile : sbuf;
  const int x0 = blockIdx.x * cols;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int idx = tid; idx < tile; idx += nt) {
    const int xc = idx / run, rem = idx - xc * run;
    const int x = x0 + xc;
    sbuf[((rem >> 1) * cols + xc) * 2 + (rem & 1)] =
        x < nx ? a.in[static_cast<long long>(x) * run + rem] : cx<T>{0, 0};
  }
  __syncthreads();
  fft_smem_inline<-1>(sbuf, plan, tw, 2 * cols, tid, nt);
  if (a.spec_out)
    for (int idx = tid; idx < tile; idx += nt) {
      const int y = idx / (2 * cols), rem = idx - y * 2 * cols;
      const int x = x0 + (rem >> 1);
      if (x < nx) a.spec_out[(static_cast<long long>(y) * nx + x) * 2 + (rem & 1)] = sbuf[idx];
    }
  constexpr int kB = table_blocks<T>();  // table values per point (3 entries, FP32: + lo parts)
  constexpr int U = 4;                   // points per thread whose table values load together
  for (int j = 0; j < npass; ++j) {
    const cx<T>* m = static_cast<const cx<T>*>(ps[j].tab);
    if constexpr (sizeof(T) != sizeof(double)) {
      if (ps[j].scalar) {  // propagator only: two table values per point
        for (int base = tid; base < ny * cols; base += U * nt) {
          cx<T> tv[U][2];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int idx = base + u * nt;
            const int xc = idx / ny, y = idx - xc * ny;
            if (idx < ny * cols && x0 + xc < nx) {
              const long long q = static_cast<long long>(x0 + xc) * ny + y;
              tv[u][0] = m[q];
              tv[u][1] = m[n + q];
            }
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int idx = base + u * nt;
            if (idx >= ny * cols) break;
            const int xc = idx / ny, y = idx - xc * ny;
            const int sidx = y * cols + xc;
            if (x0 + xc >= nx) {
              wbuf[2 * sidx] = cx<T>{0, 0};
              wbuf[2 * sidx + 1] = cx<T>{0, 0};
              continue;
            }
            wbuf[2 * sidx] = pmul(sbuf[2 * sidx], tv[u][0], tv[u][1]);
            wbuf[2 * sidx + 1] = pmul(sbuf[2 * sidx + 1], tv[u][0], tv[u][1]);
          }
        }
        __syncthreads();
        fft_smem_inline<+1>(wbuf, plan, tw, 2 * cols, tid, nt);
        cx<T>* w = a.work + static_cast<long long>(j) * 2 * n;
        for (int idx = tid; idx < tile; idx += nt) {
          const int xc = idx / run, rem = idx - xc * run;
          const int x = x0 + xc;
          if (x < nx) w[static_cast<long long>(x) * run + rem] = wbuf[((rem >> 1) * cols + xc) * 2 + (rem & 1)];
        }
        __syncthreads();
        continue;
      }
    }
    for (int base = tid; base < ny * cols; base += U * nt) {
      cx<T> tv[U][kB];
#pragma unroll
      for (int u = 0; u < U; ++u) {  // every table value of U points in flight at once
        const int idx = base + u * nt;
        const int xc = idx / ny, y = idx - xc * ny;
        const int x = x0 + xc;
        if (idx < ny * cols && x < nx) {
          const long long q = static_cast<long long>(x) * ny + y;  // transposed table index
#pragma unroll
          for (int b = 0; b < kB; ++b) tv[u][b] = m[b * n + q];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int idx = base + u * nt;
        if (idx >= ny * cols) break;
        const int xc = idx / ny, y = idx - xc * ny;
        const int x = x0 + xc;
        const int sidx = y * cols + xc;
        if (x >= nx) {
          wbuf[2 * sidx] = cx<T>{0, 0};
          wbuf[2 * sidx + 1] = cx<T>{0, 0};
          continue;
        }
        const cx<T> s0 = sbuf[2 * sidx], s1 = sbuf[2 * sidx + 1];
        wbuf[2 * sidx] = tmul_v(s0, tv[u], 0) + tmul_v(s1, tv[u], 1);
        wbuf[2 * sidx + 1] = tmul_v(s0, tv[u], 1) + tmul_v(s1, tv[u], 2);
      }
    }
    __syncthreads();
    fft_smem_inline<+1>(wbuf, plan, tw, 2 * cols, tid, nt);
    cx<T>* w = a.work + static_cast<long long>(j) * 2 * n;
    for (int idx = tid; idx < tile; idx += nt) {
      const int xc = idx / run, rem = idx - xc * run;
      const int x = x0 + xc;
      if (x < nx) w[static_cast<long long>(x) * run + rem] = wbuf[((rem >> 1) * cols + xc) * 2 + (rem & 1)];
    }
    __syncthreads();
  }
}

// k_cols_step for one column per CTA: the column is brought into shared memory by one bulk copy
// (cp.async.bulk on an mbarrier, bounded wait), and the passes go in groups of G whose spectral
// products share one inverse transform (smem [y][g][c], 2·G lanes), each thread loading the
// table values of several points at once. The tables stay in global memory (L2): staging them in
// shared memory as well took the kernel to one CTA per SM and made it slower. Needs an even ny
// (16-byte runs) and 16-byte aligned planes (the host checks).
// smem: column [y][c] (2·ny), work tile (2·G·ny), one mbarrier.
template <typename T>
__global__ void __launch_bounds__(kPlaneThreads, kPlaneMinBlocks<T>) k_cols_step_bulk(ColStep<T> a, const PassRec* __restrict__ ps, int npass,
                                 const __grid_constant__ FftPlan plan, const Tw<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int kB = table_blocks<T>();
  constexpr int U = 4;  // points per thread whose table values load together
  const int ny = a.ny, G = a.cols;  // a.cols carries the group size for this kernel
  const long long n = static_cast<long long>(ny) * a.nx;
  cx<T>* sbuf = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* wbuf = sbuf + 2 * ny;
  std::uint64_t* mbar = reinterpret_cast<std::uint64_t*>(wbuf + 2 * G * ny);
  const int x = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const unsigned run_bytes = 2u * ny * sizeof(cx<T>);
  if (tid == 0) {
    bulk_mbar_init(mbar, 1);
    bulk_fence_init();
  }
  __syncthreads();
  if (tid == 0) {
    bulk_expect(mbar, run_bytes);
    bulk_load(sbuf, a.in + static_cast<long long>(x) * 2 * ny, run_bytes, mbar);
  }
  bulk_wait(mbar, 0, a.status);
  fft_smem_inline<-1>(sbuf, plan, tw, 2, tid, nt);
  if (a.spec_out)
    for (int i = tid; i < 2 * ny; i += nt)
      a.spec_out[(static_cast<long long>(i >> 1) * a.nx + x) * 2 + (i & 1)] = sbuf[i];
  for (int j0 = 0; j0 < npass; j0 += G) {
    const int g = min(G, npass - j0);
    for (int base = tid; base < g * ny; base += U * nt) {
      cx<T> tv[U][kB];
      bool sc[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {  // the table values of U points in flight at once
        const int idx = base + u * nt;
        const int gi = idx / ny, y = idx - gi * ny;
        sc[u] = false;
        if (idx < g * ny) {
          const PassRec pr = ps[j0 + gi];
          const cx<T>* m = static_cast<const cx<T>*>(pr.tab);
          const long long q = static_cast<long long>(x) * ny + y;
          sc[u] = sizeof(T) != sizeof(double) && pr.scalar;
          if (sc[u]) {
            tv[u][0] = m[q];
            tv[u][1] = m[n + q];
          } else {
#pragma unroll
            for (int b = 0; b < kB; ++b) tv[u][b] = m[b * n + q];
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int idx = base + u * nt;
        if (idx >= g * ny) break;
        const int gi = idx / ny, y = idx - gi * ny;
        cx<T> w0{0, 0}, w1{0, 0};
        {
          const cx<T> s0 = sbuf[2 * y], s1 = sbuf[2 * y + 1];
          bool done = false;
          if constexpr (sizeof(T) != sizeof(double)) {
            if (sc[u]) {
              w0 = pmul(s0, tv[u][0], tv[u][1]);
              w1 = pmul(s1, tv[u][0], tv[u][1]);
              done = true;
            }
          }
          if (!done) {
            w0 = tmul_v(s0, tv[u], 0) + tmul_v(s1, tv[u], 1);
            w1 = tmul_v(s0, tv[u], 1) + tmul_v(s1, tv[u], 2);
          }
        }
        wbuf[(y * g + gi) * 2] = w0;
        wbuf[(y * g + gi) * 2 + 1] = w1;
      }
    }
    __syncthreads();
    fft_smem_inline<+1>(wbuf, plan, tw, 2 * g, tid, nt);
    for (int idx = tid; idx < g * ny; idx += nt) {  // per pass one contiguous column, by pixel
      const int gi = idx / ny, y = idx - gi * ny;
      st_px(a.work + static_cast<long long>(j0 + gi) * 2 * n + (static_cast<long long>(x) * ny + y) * 2,
            wbuf[(y * g + gi) * 2], wbuf[(y * g + gi) * 2 + 1]);
    }
    __syncthreads();
  }
}

// shared memory of k_cols_step_bulk with passes in groups of g
template <typename T>
constexpr std::size_t cols_bulk_smem(int ny, int g) {
  return static_cast<std::size_t>(2 + 2 * g) * ny * sizeof(cx<T>) + sizeof(std::uint64_t);
}

// Both components of one pixel (two adjacent complex values, 16-byte aligned in complex64).
template <typename T>
__device__ __forceinline__ void ld_px(const cx<T>* p, cx<T>& a, cx<T>& b) {
  if constexpr (sizeof(T) == sizeof(float)) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    a = cx<T>{v.x, v.y};
    b = cx<T>{v.z, v.w};
  } else {
    a = p[0];
    b = p[1];
  }
}
template <typename T>
__device__ __forceinline__ void st_px(cx<T>* p, cx<T> a, cx<T> b) {
  if constexpr (sizeof(T) == sizeof(float)) {
    *reinterpret_cast<float4*>(p) = make_float4(a.re, a.im, b.re, b.im);
  } else {
    p[0] = a;
    p[1] = b;
  }
}

template <typename T>
struct RowSelect {
  const cx<T>* work;        // npass planes after the inverse y transform, transposed (x-major)
  cx<T>* out;               // (N, 2)
  const uint8_t* pid;       // or null
  const T* mask;            // or null
  const int* iface;         // interface pixels of the step (sorted), or null
  const int* rowoff;        // (ny + 1) offsets into iface per row
  cx<T>* refl_out;          // (niface, 2) or null
  const cx<T>* add;         // (niface, 2) or null
  cx<T>* xnext;             // or null: also the x transform of the output rows (the next step's
                            // first transform, fused here), stored transposed
  int ny, nx, rows;
  int group;                // passes per inverse transform (shared memory holds group planes' rows)
  int store_out;            // with xnext on a single-pass step: 0 when nothing reads `out` later
  T inv_n;
};

// inverse x transform of each pass for `rows` rows, then select/mask/gather/add.
template <typename T>
__global__ void __launch_bounds__(kPlaneThreads, kPlaneMinBlocks<T>) k_rows_select(RowSelect<T> a, const PassRec* __restrict__ ps, int npass, const __grid_constant__ FftPlan plan,
                              const Tw<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* buf = reinterpret_cast<cx<T>*>(smem_raw);
  const int ny = a.ny, nx = a.nx, rows = a.rows;
  const long long n = static_cast<long long>(ny) * nx;
  const int y0 = blockIdx.x * rows;
  const int here = min(rows, ny - y0);
  const int tid = threadIdx.x, nt = blockDim.x;
  const int k0 = a.iface ? a.rowoff[y0] : 0, k1 = a.iface ? a.rowoff[y0 + here] : 0;
  // passes in groups of G: the G work planes' rows share one inverse transform, smem
  // [x][row][g][c] (G·2·rows lanes), so a multi-pass step pays the transform's latency per group
  const int G = a.group;
  // a single-pass step that feeds the next one: its selected rows stay in shared memory, where
  // the sources are added and the next x transform runs (no round trip through `out`)
  const bool fast = npass == 1 && !ps[0].refl && !a.pid && a.xnext;
  for (int j0 = 0; j0 < npass && !fast; j0 += G) {
    const int g = min(G, npass - j0);  // passes in this group: the transform has 2·rows·g lanes
    // per (pass, x) a run of `rows` pixels (transposed planes); four pixels in flight per thread
    const int npix = g * rows * nx;
    for (int base = tid; base < npix; base += 4 * nt) {
      cx<T> va[4], vb[4];
      int dst[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int idx = base + u * nt;
        dst[u] = -1;
        va[u] = vb[u] = cx<T>{0, 0};
        if (idx < npix) {
          const int gi = idx / (rows * nx), r = idx - gi * rows * nx;
          const int x = r / rows, row = r - x * rows;
          if (row < here)
            ld_px(a.work + static_cast<long long>(j0 + gi) * 2 * n +
                      (static_cast<long long>(x) * ny + y0 + row) * 2, va[u], vb[u]);
          dst[u] = (x * rows + row) * 2 * g + gi * 2;
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (dst[u] >= 0) {
          buf[dst[u]] = va[u];
          buf[dst[u] + 1] = vb[u];
        }
    }
    __syncthreads();
    fft_smem_inline<+1>(buf, plan, tw, 2 * rows * g, tid, nt);
    for (int gi = 0; gi < g; ++gi) {
      const int j = j0 + gi;
      const int pair = ps[j].pair;
      if (!ps[j].refl) {
        for (int idx = tid; idx < here * nx; idx += nt) {  // per pixel both components
          const int row = idx / nx, x = idx - row * nx;
          const long long q = static_cast<long long>(y0 + row) * nx + x;
          if (!a.pid || a.pid[q] == pair) {
            const int b = (x * rows + row) * 2 * g + gi * 2;
            cx<T> v0 = buf[b] * a.inv_n, v1 = buf[b + 1] * a.inv_n;
            if (a.mask) {
              v0 = mmul(v0, a.mask, q, n);
              v1 = mmul(v1, a.mask, q, n);
            }
            st_px(a.out + 2 * q, v0, v1);
          }
        }
      } else {
        for (int k = k0 + tid; k < k1; k += nt) {
          const int q = a.iface[k];
          if (a.pid && a.pid[q] != pair) continue;
          const int row = q / nx - y0, x = q - (q / nx) * nx;
          a.refl_out[2 * k] = buf[(x * rows + row) * 2 * g + gi * 2] * a.inv_n;
          a.refl_out[2 * k + 1] = buf[(x * rows + row) * 2 * g + gi * 2 + 1] * a.inv_n;
        }
      }
    }
    __syncthreads();
  }
  if (fast) {
    for (int idx = tid; idx < rows * nx; idx += nt) {
      const int row = idx / nx, x = idx - row * nx;
      cx<T> v0{0, 0}, v1{0, 0};
      if (row < here)
        ld_px(a.work + (static_cast<long long>(x) * ny + y0 + row) * 2, v0, v1);
      buf[(x * rows + row) * 2] = v0;
      buf[(x * rows + row) * 2 + 1] = v1;
    }
    __syncthreads();
    fft_smem_inline<+1>(buf, plan, tw, 2 * rows, tid, nt);
    for (int idx = tid; idx < here * nx; idx += nt) {  // scale, mask (and store) in place
      const int row = idx / nx, x = idx - row * nx;
      const long long q = static_cast<long long>(y0 + row) * nx + x;
      const int b = (x * rows + row) * 2;
      cx<T> v0 = buf[b] * a.inv_n, v1 = buf[b + 1] * a.inv_n;
      if (a.mask) {
        v0 = mmul(v0, a.mask, q, n);
        v1 = mmul(v1, a.mask, q, n);
      }
      buf[b] = v0;
      buf[b + 1] = v1;
      if (a.store_out && !a.add) st_px(a.out + 2 * q, v0, v1);
    }
    __syncthreads();
    if (a.add) {
      for (int k = k0 + tid; k < k1; k += nt) {  // interface pixels are distinct
        const int q = a.iface[k];
        const int b = ((q - (q / nx) * nx) * rows + (q / nx - y0)) * 2;
        buf[b] = buf[b] + a.add[2 * k];
        buf[b + 1] = buf[b + 1] + a.add[2 * k + 1];
      }
      __syncthreads();
      if (a.store_out)
        for (int idx = tid; idx < here * nx; idx += nt) {
          const int row = idx / nx, x = idx - row * nx;
          const int b = (x * rows + row) * 2;
          st_px(a.out + 2 * (static_cast<long long>(y0 + row) * nx + x), buf[b], buf[b + 1]);
        }
    }
    fft_smem_inline<-1>(buf, plan, tw, 2 * rows, tid, nt);
    for (int idx = tid; idx < nx * here; idx += nt) {
      const int x = idx / here, row = idx - x * here;
      st_px(a.xnext + (static_cast<long long>(x) * ny + y0 + row) * 2, buf[(x * rows + row) * 2],
            buf[(x * rows + row) * 2 + 1]);
    }
    return;
  }
  if (a.add)
    for (int k = k0 + tid; k < k1; k += nt) {
      const int q = a.iface[k];
      a.out[2 * q] = a.out[2 * q] + a.add[2 * k];
      a.out[2 * q + 1] = a.out[2 * q + 1] + a.add[2 * k + 1];
    }
  if (a.xnext) {  // forward x transform of this CTA's output rows (written by this CTA above)
    __syncthreads();
    for (int idx = tid; idx < rows * nx; idx += nt) {  // per pixel both components
      const int row = idx / nx, x = idx - row * nx;
      cx<T> v0{0, 0}, v1{0, 0};
      if (row < here) ld_px(a.out + (static_cast<long long>(y0 + row) * nx + x) * 2, v0, v1);
      buf[(x * rows + row) * 2] = v0;
      buf[(x * rows + row) * 2 + 1] = v1;
    }
    __syncthreads();
    fft_smem_inline<-1>(buf, plan, tw, 2 * rows, tid, nt);
    for (int idx = tid; idx < nx * here; idx += nt) {  // transposed: per x a run of `here` pixels
      const int x = idx / here, row = idx - x * here;
      st_px(a.xnext + (static_cast<long long>(x) * ny + y0 + row) * 2, buf[(x * rows + row) * 2],
            buf[(x * rows + row) * 2 + 1]);
    }
  }
}

// ---- small helpers ------------------------------------------------------------------------

template <typename T>
__global__ void k_add_plane(cx<T>* dst, const cx<T>* src, const T* mask, T scale, long long n2) {
  // dst += src·scale (· mask per pixel when given); n2 = complex entries of an (N, 2) plane
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i >= n2) return;
  const cx<T> s = mask ? mmul(src[i] * scale, mask, i >> 1, n2 >> 1) : src[i] * scale;
  dst[i] = dst[i] + s;
}

template <typename To, typename From>
__global__ void k_convert(cx<To>* dst, const cx<From>* src, long long count) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i < count) dst[i] = cast<To>(src[i]);
}

// Operator table of one (kind, ñ_r, ñ_s): entry q is mode (x, y) = (q mod nx, q div nx), or with
// `transposed` (3D solves, read column by column) (q div ny, q mod ny).
// `scalar` (complex64, equal indices): only m00 = e^{i k_z dz}/N, hi block then lo block.
template <typename T>
__global__ void k_build_table(cx<T>* out, int kind, cd nr, cd ns, int ny, int nx, double dy,
                              double dx, double k0, double dz, int transposed, int scalar) {
  const long long n = static_cast<long long>(ny) * nx;
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q >= n) return;
  const long long xi = transposed ? q / ny : q % nx;
  const long long yi = transposed ? q % ny : q / nx;
  const double kx = fftfreq(xi, nx, dx);
  const double ky = fftfreq(yi, ny, dy);
  cd m[3];
  operator_matrix(kind, kx, ky, nr, ns, k0, dz, m);
  if constexpr (sizeof(T) != sizeof(double)) {
    if (scalar) {
      const cd v = m[0] / static_cast<double>(n);
      const cf hi = cast<float>(v);
      out[q] = hi;
      out[n + q] = cf{static_cast<float>(v.re - hi.re), static_cast<float>(v.im - hi.im)};
      return;
    }
  }
  for (int e = 0; e < 3; ++e) {
    if constexpr (sizeof(T) == sizeof(double)) {
      out[e * n + q] = m[e];
    } else {  // FP32 fields: M/N as hi + lo (the inverse transform's 1/N folded in)
      const cd v = m[e] / static_cast<double>(n);
      const cf hi = cast<float>(v);
      out[e * n + q] = hi;
      out[(3 + e) * n + q] = cf{static_cast<float>(v.re - hi.re), static_cast<float>(v.im - hi.im)};
    }
  }
}

}  // namespace bwpm
