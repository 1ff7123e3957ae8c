// Resident 2D engine: many 2D solves in one persistent launch, complex64 fields.
//
// In 2D (nx = 1) the 2×2 operators are diagonal (k_x = 0 exactly), so E_x (TE, entry m00) and
// E_y (TM, entry m11) are independent scalar problems. A work item is one (solve, component)
// whose input is non-zero. One CTA owns one item for its whole sweep: the field line stays in
// shared memory across all slabs, passes and iterations (cpp/src/solver.cpp:444-528), and the
// CTA pulls the next item from a queue when done (items sorted by decreasing cost).
//
// Per step: forward transform of the line, then per pass (pair × kind) spectral multiply by a
// complex64 operator table (built once in FP64), inverse transform, and the epilogue: pixel
// selection by pair id, mask, gather of reflection sources at interface pixels; then the sparse
// add of the other pass's sources. Per iteration the transmitted/reflected power flux
// (src/bwpm/fpwpm.py:205-216) is accumulated in FP64 with compensated (Kahan) block sums.
#pragma once

#include "fft.cuh"

namespace bwpm {

constexpr int kR2Ept = 8;  // complex values a thread stages per FFT stage

struct R2Pass {
  long long tab;  // element offset of the scalar operator table: N hi values, then N lo values
  int pair;       // pair id selected by this pass
  int refl;       // 1: reflection (gathered at interface pixels), 0: transmission
};

struct R2Step {
  long long pid;      // element offset of the uint8 pair-id plane, −1: one pair
  long long iface;    // offset of the interface pixel list
  int niface;
  int fwd_off, fwd_t, fwd_r;  // passes of the forward step (transmission, reflection)
  int bwd_off, bwd_t, bwd_r;  // passes of the backward step
};

struct R2Item {
  const cf* input;        // (N) incident component
  const cf* tables;       // operator tables of this item's component (pass offsets added); each
                          // table holds M/N as N hi values then N lo values (M/N = hi + lo)
  cf* transmitted;        // (N)
  cf* reflected;          // (N)
  cf* src_fwd;            // sources for the forward pass (gathered by the backward pass)
  cf* src_bwd;            // sources for the backward pass
  const float* mask;      // (2N): hi values then lo values (mask = hi + lo), or null
  const R2Step* steps;    // nz records; offsets in them are relative to the bases below
  const R2Pass* passes;   // pass records of this solve
  const std::uint8_t* pids;  // pair-id planes of this solve
  const int* iface;       // interface pixel lists of this solve (also index the sources)
  const double* w_out;    // (N) flux weight of the transmitted medium
  const double* w_in;     // (N) flux weight of the incident medium
  double* energy;         // (iterations, 2) transmitted/reflected flux, then the incident flux
  long long* clock;       // (2): start and end global timer, ns
  int n, nz, iterations, plan;
};

struct R2Shared {
  const FftPlan* plans;   // twiddle offsets (twoff, rootoff) index the shared pool
  const Tw<float>* twiddles;  // (hi, lo) pairs
};

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Σ w[q]·|buf[q]|² over the line, FP64 with compensated block reduction; thread 0 returns it.
__device__ double r2_flux(const cf* buf, const double* w, int n, double* red) {
  double s = 0.0, c = 0.0;
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const double v = w[q] * (static_cast<double>(buf[q].re) * buf[q].re +
                             static_cast<double>(buf[q].im) * buf[q].im);
    const double y = v - c;
    const double t = s + y;
    c = (t - s) - y;
    s = t;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  double total = 0.0;
  if (threadIdx.x == 0) {
    double comp = 0.0;
    for (int i = 0; i < (blockDim.x >> 5); ++i) {
      const double y = red[i] - comp;
      const double t = total + y;
      comp = (t - total) - y;
      total = t;
    }
  }
  __syncthreads();
  return total;
}

// v·(hi + lo) for a real factor carried as a float pair.
__device__ __forceinline__ cf mask_mul(cf v, float hi, float lo) {
  return {fmaf(v.re, hi, v.re * lo), fmaf(v.im, hi, v.im * lo)};
}

// One step of an item: E holds the field, B and O are scratch lines (all length n, smem).
// backward selects the backward passes; `store` receives reflection sources, `add` the sources
// added after the step (both at this step's interface pixels).
__device__ __forceinline__ void r2_step(cf*& E, cf*& O, cf* B, const R2Item& it, const R2Shared& sh,
                                        const FftPlan& plan, const R2Step& st, bool backward,
                                        bool reflect, cf* store, const cf* add) {
  const int n = it.n, tid = threadIdx.x, nt = blockDim.x;
  const int off = backward ? st.bwd_off : st.fwd_off;
  const int nt_pass = backward ? st.bwd_t : st.fwd_t;
  const int nr_pass = reflect ? (backward ? st.bwd_r : st.fwd_r) : 0;
  const int npass = nt_pass + nr_pass;
  const std::uint8_t* pid = st.pid >= 0 ? it.pids + st.pid : nullptr;
  const int* iface = it.iface + st.iface;
  fft_smem<-1, kR2Ept>(E, plan, sh.twiddles, 1, tid, nt);
  if (npass == 1) {
    // a single transmission pass over all pixels: in place
    const R2Pass ps = it.passes[off];
    const cf* m = it.tables + ps.tab;
    for (int q = tid; q < n; q += nt) E[q] = pmul(E[q], m[q], m[n + q]);
    __syncthreads();
    fft_smem<+1, kR2Ept>(E, plan, sh.twiddles, 1, tid, nt);
    if (it.mask)
      for (int q = tid; q < n; q += nt) E[q] = mask_mul(E[q], it.mask[q], it.mask[n + q]);
  } else {
    for (int j = 0; j < npass; ++j) {
      const R2Pass ps = it.passes[off + j];
      const cf* m = it.tables + ps.tab;
      for (int q = tid; q < n; q += nt) B[q] = pmul(E[q], m[q], m[n + q]);
      __syncthreads();
      fft_smem<+1, kR2Ept>(B, plan, sh.twiddles, 1, tid, nt);
      if (!ps.refl) {
        for (int q = tid; q < n; q += nt)
          if (!pid || pid[q] == ps.pair) O[q] = it.mask ? mask_mul(B[q], it.mask[q], it.mask[n + q]) : B[q];
      } else {
        for (int k = tid; k < st.niface; k += nt) {
          const int q = iface[k];
          if (!pid || pid[q] == ps.pair) store[k] = B[q];
        }
      }
      __syncthreads();
    }
    cf* t = E;
    E = O;
    O = t;
  }
  __syncthreads();
  if (add) {
    for (int k = tid; k < st.niface; k += nt) {
      const int q = iface[k];
      E[q] = E[q] + add[k];
    }
    __syncthreads();
  }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_resident2d(const R2Item* __restrict__ items, int nitems,
                                                   int* queue, R2Shared sh) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_item;
  __shared__ double s_red[NT / 32];
  __shared__ FftPlan s_plan;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(queue, 1);
    __syncthreads();
    const int idx = s_item;
    if (idx >= nitems) return;
    const R2Item it = items[idx];
    if (tid == 0) {
      s_plan = sh.plans[it.plan];
      it.clock[0] = global_ns();
    }
    __syncthreads();
    const FftPlan& plan = s_plan;
    const int n = it.n;
    cf* lines = reinterpret_cast<cf*>(smem_raw);
    cf* E = lines;
    cf* O = lines + n;
    cf* B = lines + 2 * n;
    const int iters = it.iterations > 0 ? it.iterations : 1;
    {  // incident flux P_in in the medium before the volume
      for (int q = tid; q < n; q += NT) B[q] = it.input[q];
      __syncthreads();
      fft_smem<-1, kR2Ept>(B, plan, sh.twiddles, 1, tid, NT);
      const double pin = r2_flux(B, it.w_in, n, s_red);
      if (tid == 0) it.energy[2 * iters] = pin;
    }
    for (int iter = 0; iter < iters; ++iter) {
      for (int q = tid; q < n; q += NT) E[q] = it.input[q];
      __syncthreads();
      for (int p = 0; p < it.nz; ++p) {
        const R2Step st = it.steps[p];
        const bool reflect = it.iterations > 0 && st.niface > 0;
        const long long so = st.iface;
        r2_step(E, O, B, it, sh, plan, st, false, reflect, it.src_bwd + so,
                (iter > 0 && st.niface > 0) ? it.src_fwd + so : nullptr);
      }
      for (int q = tid; q < n; q += NT) it.transmitted[q] = E[q];
      if (it.iterations > 0) {
        for (int q = tid; q < n; q += NT) B[q] = E[q];
        __syncthreads();
        fft_smem<-1, kR2Ept>(B, plan, sh.twiddles, 1, tid, NT);
        const double pt = r2_flux(B, it.w_out, n, s_red);
        if (tid == 0) it.energy[2 * iter] = pt;
      }
      if (it.iterations == 0) break;
      for (int q = tid; q < n; q += NT) E[q] = cf{0.f, 0.f};
      __syncthreads();
      for (int p = it.nz; p > 0; --p) {
        const R2Step st = it.steps[p - 1];
        const long long so = st.iface;
        r2_step(E, O, B, it, sh, plan, st, true, st.niface > 0, it.src_fwd + so,
                st.niface > 0 ? it.src_bwd + so : nullptr);
      }
      for (int q = tid; q < n; q += NT) {
        it.reflected[q] = E[q];
        B[q] = E[q];
      }
      __syncthreads();
      fft_smem<-1, kR2Ept>(B, plan, sh.twiddles, 1, tid, NT);
      const double pr = r2_flux(B, it.w_in, n, s_red);
      if (tid == 0) it.energy[2 * iter + 1] = pr;
    }
    __syncthreads();
    if (tid == 0) it.clock[1] = global_ns();
    __syncthreads();
  }
}

}  // namespace bwpm
