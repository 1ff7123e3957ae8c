// GMRES(30) of the Born step with its scalar work on the device.
//
// The algorithm is the reference's restarted GMRES (cpp/src/solver.cpp:130-207: modified
// Gram-Schmidt Arnoldi, Givens rotations, back substitution; tolerance on the rotated residual,
// start from the right-hand side). The reference's CUDA core returns every inner product to the
// host (cpp/src/solver_cuda.cu:336-340, :474-477), one device round trip per dot. Here the
// inner products, the Hessenberg matrix, the rotations and the solution of the small triangular
// system stay in device memory: the dot kernels write h straight into the Hessenberg matrix, the
// vector updates read their coefficients from it, and one thread applies the rotations. By
// default the whole Born step runs as one CUDA graph (plane_solver.cu, build_born_graph) whose
// conditional nodes the one-thread kernels at the end of this file set: the decisions of the
// host loop (convergence, restart, true residual) are made on the device and the host waits for
// nothing. Host-driven (BWPM_GMRES=host), the host learns of convergence one Arnoldi step
// behind, the step after a converged one computed speculatively and discarded (it touches no
// entry the solution uses).
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
  double tolb;   // tolerance × ‖rhs‖ of the current solve (read by the graphs)
  int flag[kGmresRestart];
  unsigned counter;  // last-block ticket of the dot kernels (back at 0 after each dot)
  int used;          // Arnoldi steps of the last cycle (Born-step graph)
  int outer;         // restarts of the current solve (Born-step graph)
  int err;           // set when a solve ran out of restarts (Born-step graph)
  long long applies; // operator applications (Born-step graph)
};

// The conditions of the Born-step graph, one per conditional node: `active` (WHILE: another
// restart), `cycle` (IF: this restart's Arnoldi cycle runs), `done` (IF: the cycle converged,
// check the true residual), step[j] (IF: Arnoldi step j runs).
struct GmresConds {
  cudaGraphConditionalHandle active, cycle, done;
  cudaGraphConditionalHandle step[kGmresRestart];
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
  if (i == 0 && tol_bnorm >= 0.0) s->tolb = tol_bnorm;  // the Born-step graph set it already
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
__global__ void k_gmres_givens_cond(GmresState* s, int j, GmresConds c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  gmres_givens(s, j, s->tolb);
  if (j + 1 < kGmresRestart) cudaGraphSetConditional(c.step[j + 1], s->flag[j] ? 0u : 1u);
}

// Back substitution for the first `used` unknowns (cpp/src/solver.cpp:193-199); used < 0: the
// count the Born-step graph left in the state.
__global__ void k_gmres_backsolve(GmresState* s, int used) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (used < 0) used = s->used;
  constexpr int m = kGmresRestart;
  for (int i = used - 1; i >= 0; --i) {
    cd acc = s->g[i];
    for (int k = i + 1; k < used; ++k) acc = acc - s->h[i * m + k] * s->y[k];
    s->y[i] = cdiv(acc, s->h[i * m + i]);
  }
}

// ---- the decisions of the host loop (plane_solver.cu PlaneSolver::gmres), on the device ----
// Each kernel runs one thread and sets the conditions of the Born-step graph; every comparison
// is the host loop's, in the same FP64 operations.

// After ‖rhs‖²: ‖rhs‖ = 0 ends the solve at once (y = rhs = 0), else the restarts begin.
__global__ void k_gmres_init(GmresState* s, double tol, GmresConds c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double bnorm = sqrt(s->dot.re);
  s->tolb = tol * bnorm;
  s->outer = 0;
  cudaGraphSetConditional(c.active, bnorm == 0.0 ? 0u : 1u);
}

// After β² = ‖rhs − A·y‖²: β ≤ tol·‖rhs‖ ends the solve; else a cycle runs, unless the solve
// has used its 100 restarts (then `err`).
__global__ void k_gmres_restart(GmresState* s, GmresConds c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  s->applies += 1;
  const double beta = sqrt(s->dot.re);
  unsigned run = 1u;
  if (beta <= s->tolb) {
    run = 0u;
  } else if (s->outer >= 100) {
    s->err = 1;
    run = 0u;
  } else {
    s->outer += 1;
  }
  cudaGraphSetConditional(c.cycle, run);
  if (!run) cudaGraphSetConditional(c.active, 0u);
}

// Before a cycle: step 0 runs, the others wait for their predecessor.
__global__ void k_gmres_arm(GmresConds c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int j = 0; j < kGmresRestart; ++j) cudaGraphSetConditional(c.step[j], j == 0 ? 1u : 0u);
}

// After a cycle: used = steps up to the first converged one (all if none); `done` when one did.
__global__ void k_gmres_cycle_done(GmresState* s, GmresConds c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int used = kGmresRestart;
  unsigned done = 0u;
  for (int j = 0; j < kGmresRestart; ++j)
    if (s->flag[j]) {
      used = j + 1;
      done = 1u;
      break;
    }
  s->used = used;
  s->applies += used;
  cudaGraphSetConditional(c.done, done);
}

// After ‖rhs − A·y‖² of a converged cycle: within 10·tol·‖rhs‖ ends the solve, else restart.
__global__ void k_gmres_final(GmresState* s, GmresConds c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  s->applies += 1;
  if (sqrt(s->dot.re) <= s->tolb * 10.0) cudaGraphSetConditional(c.active, 0u);
}

// y += Σ_{i<used} y_i·v_i with `used` from the state, in the order and arithmetic of one
// k_axpy_dev per basis vector.
template <typename T>
__global__ void k_axpy_basis(cx<T>* y, cx<T>* const* basis, const GmresState* s, long long m) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i >= m) return;
  const int used = s->used;
  cx<T> v = y[i];
  for (int k = 0; k < used; ++k) {
    const cd a = s->y[k] * 1.0;
    v = cast<T>(a * cast<double>(basis[k][i]) + cd{1.0, 0.0} * cast<double>(v));
  }
  y[i] = v;
}

}  // namespace bwpm
