// GMRES(30) of the Born step with its scalar work on the device.
//
// The algorithm is the reference's restarted GMRES (cpp/src/solver.cpp:130-207: modified
// Gram-Schmidt Arnoldi, Givens rotations, back substitution; tolerance on the rotated residual,
// start from the right-hand side). The reference's CUDA core returns every inner product to the
// host (cpp/src/solver_cuda.cu:336-340, :474-477), one device round trip per dot. Here the
// inner products, the Hessenberg matrix, the rotations and the solution of the small triangular
// system stay in device memory: the dot kernels write h straight into the Hessenberg matrix, the
// vector updates read their coefficients from it, and one thread applies the rotations. The host
// learns of convergence from the flags: by default once per restart cycle, which runs as a CUDA
// graph whose Arnoldi steps sit under conditional nodes that the rotation kernel clears on
// convergence; or (host-driven form) one Arnoldi step behind, the step after a converged one
// computed speculatively and discarded (it touches no entry the solution uses).
#pragma once

#include "common.cuh"

namespace bwpm {

constexpr int kGmresRestart = 30;
constexpr int kDotBlocks = 256;

struct GmresState {
  cd h[(kGmresRestart + 1) * kGmresRestart];  // row-major, h[i·m + j]
  cd cs[kGmresRestart], sn[kGmresRestart];
  cd g[kGmresRestart + 1];
  cd y[kGmresRestart];
  cd dot;        // scratch inner product (norms)
  double nrm;    // last norm
  double hnext[kGmresRestart];
  double tolb;   // tolerance × ‖rhs‖ of the current solve (read by the cycle graph)
  int flag[kGmresRestart];
  unsigned counter;  // last-block ticket of the dot kernels (back at 0 after each dot)
};

// *out = Σ conj(u)·v in FP64; the last block to finish adds the block partials in block order
// (deterministic), then resets the ticket counter.
template <typename T>
__global__ void __launch_bounds__(256)
    k_dot_dev(const cx<T>* u, const cx<T>* v, long long m, cd* partial, unsigned* counter,
              cd* out) {
  __shared__ cd red[8];
  __shared__ bool last;
  cd acc{0.0, 0.0};
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < m;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    acc = acc + conj(cast<double>(u[i])) * cast<double>(v[i]);
  for (int o = 16; o > 0; o >>= 1) {
    acc.re += __shfl_down_sync(0xffffffffu, acc.re, o);
    acc.im += __shfl_down_sync(0xffffffffu, acc.im, o);
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    cd s{0.0, 0.0};
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s = s + red[w];
    partial[blockIdx.x] = s;
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    cd s{0.0, 0.0};
    for (unsigned b = 0; b < gridDim.x; ++b) s = s + partial[b];
    *out = s;
    *counter = 0u;
  }
}

// y = (sign·coef)·x + y, coef in device memory.
template <typename T>
__global__ void k_axpy_dev(cx<T>* y, const cx<T>* x, const cd* coef, double sign, long long m) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i >= m) return;
  const cd a = (*coef) * sign;
  y[i] = cast<T>(a * cast<double>(x[i]) + cd{1.0, 0.0} * cast<double>(y[i]));
}

// nrm = √Re(dot); out = in/nrm (when nrm > 0); nrm stored at *nrm_out by thread 0.
template <typename T>
__global__ void k_norm_scale(cx<T>* out, const cx<T>* in, const cd* dot, double* nrm_out,
                             long long m) {
  const double nrm = sqrt(dot->re);
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i == 0) *nrm_out = nrm;
  if (i >= m || !(nrm > 0.0)) return;
  const double inv = 1.0 / nrm;
  out[i] = cast<T>(cd{0.0, 0.0} + cast<double>(in[i]) * inv);
}

// g = (β, 0, …, 0) with β = √Re(dot); the cycle's flags cleared; tolb = tol·‖rhs‖.
__global__ void k_gmres_start(GmresState* s, double tol_bnorm) {
  const int i = threadIdx.x;
  if (i <= kGmresRestart) s->g[i] = cd{i == 0 ? sqrt(s->dot.re) : 0.0, 0.0};
  if (i < kGmresRestart) s->flag[i] = 0;
  if (i == 0) s->tolb = tol_bnorm;
}

// Column j of the Arnoldi step: earlier rotations, the new rotation from h[j][j] and
// hnext = √Re(dot) (cpp/src/solver.cpp:164-190); flag[j] = converged or breakdown.
__device__ __forceinline__ void gmres_givens(GmresState* s, int j, double tol_bnorm) {
  constexpr int m = kGmresRestart;
  const double hnext = sqrt(s->dot.re);
  s->hnext[j] = hnext;
  for (int i = 0; i < j; ++i) {
    const cd a = s->h[i * m + j], c = s->h[(i + 1) * m + j];
    s->h[i * m + j] = s->cs[i] * a + s->sn[i] * c;
    s->h[(i + 1) * m + j] = -(conj(s->sn[i]) * a) + s->cs[i] * c;
  }
  const cd a = s->h[j * m + j];
  const double aa = hypot(a.re, a.im);
  const double r = sqrt(aa * aa + hnext * hnext);
  if (aa == 0.0) {
    s->cs[j] = cd{0.0, 0.0};
    s->sn[j] = cd{1.0, 0.0};
  } else {
    s->cs[j] = cd{aa / r, 0.0};
    s->sn[j] = (a / aa) * (hnext / r);
  }
  s->h[j * m + j] = s->cs[j] * a + s->sn[j] * hnext;
  s->g[j + 1] = -(conj(s->sn[j]) * s->g[j]);
  s->g[j] = s->cs[j] * s->g[j];
  s->flag[j] = (hypot(s->g[j + 1].re, s->g[j + 1].im) <= tol_bnorm || hnext == 0.0) ? 1 : 0;
}

__global__ void k_gmres_givens(GmresState* s, int j, double tol_bnorm) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  gmres_givens(s, j, tol_bnorm);
}

// The same as the last node of Arnoldi step j in the cycle graph: the tolerance comes from the
// state, and the condition of step j + 1's node (`next`, when there is one) is set unless step j
// has converged.
__global__ void k_gmres_givens_cond(GmresState* s, int j, cudaGraphConditionalHandle next,
                                    int has_next) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  gmres_givens(s, j, s->tolb);
  if (has_next) cudaGraphSetConditional(next, s->flag[j] ? 0u : 1u);
}

// Back substitution for the first `used` unknowns (cpp/src/solver.cpp:193-199).
__global__ void k_gmres_backsolve(GmresState* s, int used) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  constexpr int m = kGmresRestart;
  for (int i = used - 1; i >= 0; --i) {
    cd acc = s->g[i];
    for (int k = i + 1; k < used; ++k) acc = acc - s->h[i * m + k] * s->y[k];
    s->y[i] = cdiv(acc, s->h[i * m + i]);
  }
}

}  // namespace bwpm
