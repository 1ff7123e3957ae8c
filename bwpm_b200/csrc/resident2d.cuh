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

constexpr int kR2Ept = 16;  // complex values a thread stages per FFT stage

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
  int* status;            // the batch's status word: set to 1 when a bounded wait gave up
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
__device__ inline double r2_flux(const cf* buf, const double* w, int n, double* red) {
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

// ---- specialised kernels for compile-time lengths (register-resident lines) -----------------
//
// Same work items and results as k_resident2d, for one length N per launch: the field, the
// spectrum of a multi-pass step and the output of the step stay in registers in the owned
// pattern of rf::fft (position t + m·NT in register m of thread t); shared memory holds only the
// two exchange buffers of the transform, which also serve the gather of reflection sources and
// the sparse add at interface pixels.

}  // namespace bwpm

#include "rfft.cuh"

namespace bwpm {

template <int N, int NT>
__device__ __forceinline__ void r2f_load(cf (&v)[N / NT], const cf* src, int t) {
#pragma unroll
  for (int m = 0; m < N / NT; ++m) v[m] = src[t + m * NT];
}

template <int N, int NT>
__device__ __forceinline__ void r2f_store(cf* dst, const cf (&v)[N / NT], int t) {
#pragma unroll
  for (int m = 0; m < N / NT; ++m) dst[t + m * NT] = v[m];
}

// Σ w[q]·|v|² over the owned values, compensated in FP64; thread 0 returns the block total.
template <int N, int NT>
__device__ __forceinline__ double r2f_flux(const cf (&v)[N / NT], const double* w, double* red, int t) {
  double s = 0.0, c = 0.0;
#pragma unroll
  for (int m = 0; m < N / NT; ++m) {
    const double a = w[t + m * NT] * (static_cast<double>(v[m].re) * v[m].re +
                                      static_cast<double>(v[m].im) * v[m].im);
    const double y = a - c;
    const double z = s + y;
    c = (z - s) - y;
    s = z;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((t & 31) == 0) red[t >> 5] = s;
  __syncthreads();
  double total = 0.0;
  if (t == 0) {
    double comp = 0.0;
    for (int i = 0; i < NT / 32; ++i) {
      const double y = red[i] - comp;
      const double z = total + y;
      comp = (z - total) - y;
      total = z;
    }
  }
  __syncthreads();
  return total;
}

// Bytes of `lines` padded lines of n points, rounded up to 16.
__host__ __device__ constexpr std::size_t lines_bytes(int n, int lines) {
  return (static_cast<std::size_t>(lines) * rf::padded(n) * sizeof(cf) + 15) / 16 * 16;
}

// Records of the next slab step, loaded while the current step computes: the step record first,
// its first pass record once the step record has arrived (mid-step). Hides the chain of
// dependent global loads (step record -> pass record -> table) behind the transforms.
struct R2Next {
  R2Step st;
  R2Pass p0;
  R2Pass p1;  // second pass record, loaded only when the step has more than one pass
};

// Reflection passes run on a step with interface pixels in a backward sweep, and in a forward
// sweep when the solve iterates (iterations > 0).
__device__ __forceinline__ bool r2_reflects(const R2Step& st, bool backward, int iterations) {
  return st.niface > 0 && (backward || iterations > 0);
}

// Passes of a step in one direction: its transmission passes, then its reflection passes.
__device__ __forceinline__ int r2_passes(const R2Step& st, bool backward, bool reflect) {
  return (backward ? st.bwd_t : st.fwd_t) + (reflect ? (backward ? st.bwd_r : st.fwd_r) : 0);
}

// The first pass record of the next step (nx.st has arrived), and its second when it has one.
__device__ __forceinline__ void r2_next_passes(R2Next& nx, const R2Item& it, bool next_backward) {
  const int off = next_backward ? nx.st.bwd_off : nx.st.fwd_off;
  nx.p0 = it.passes[off];
  if (r2_passes(nx.st, next_backward, r2_reflects(nx.st, next_backward, it.iterations)) > 1)
    nx.p1 = it.passes[off + 1];
}

// Brings the L1 line holding p in from L2; holds no register while in flight.
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Pair id of owned value k from ids packed four to a 32-bit word.
template <int E>
__device__ __forceinline__ int unpack_pid(const std::uint32_t (&pw)[(E + 3) / 4], int k) {
  return static_cast<int>((pw[k >> 2] >> (8 * (k & 3))) & 0xffu);
}

// The item's mask, (hi, lo) pairs, sits in shared memory beside the lines when it fits.
template <int N>
__host__ __device__ constexpr bool fixed_mask_in_smem() {
  return lines_bytes(N, 3) + 2 * static_cast<std::size_t>(N) * sizeof(float) <= 220 * 1024;
}
template <int N>
__host__ __device__ constexpr std::size_t fixed_smem_bytes() {
  return lines_bytes(N, 3) + (fixed_mask_in_smem<N>() ? 2 * static_cast<std::size_t>(N) * sizeof(float) : 0);
}

// One slab step. st/p0/p1: this step's record and first two pass records (prefetched; p1 is
// valid when the step has more than one pass); nx receives the records of step next_p (≥ 0) of
// direction next_backward. The spectrum of a multi-pass step is kept in the shared line S at the
// owned positions (each thread reads back only what it wrote, so S needs no barrier). mk: the
// item's mask (N hi values, then N lo values) or null.
//
// Latency of the multi-pass steps: the owned pixels' pair ids are loaded once per step (packed
// in registers), the operator values of pass j + 1 are prefetched into L1 while pass j computes
// (their record was loaded one pass earlier), and the first round of the interface loops (entry
// t: pixel, its pair id, its added source) is loaded before the forward transform.
template <int N, int NT, class RADS>
__device__ __forceinline__ void r2f_step(cf (&v)[N / NT], cf* S, cf (&out)[N / NT],
                                         cf* b0, cf* b1, int& phase, const R2Item& it,
                                         const R2Step& st, const R2Pass& p0, const R2Pass& p1,
                                         R2Next& nx, int next_p, bool next_backward, bool backward,
                                         bool reflect, cf* store, const cf* add, const float* mk,
                                         const Tw<float>* __restrict__ tw, int t) {
  constexpr int E = N / NT, EW = (E + 3) / 4;
  const int off = backward ? st.bwd_off : st.fwd_off;
  const int npass = r2_passes(st, backward, reflect);
  const std::uint8_t* pid = st.pid >= 0 ? it.pids + st.pid : nullptr;
  const int* iface = it.iface + st.iface;
  if (next_p >= 0) nx.st = it.steps[next_p];
  // interface entry t, the first round of the gather and add loops
  const bool own_if = t < st.niface;
  const int q0 = own_if ? iface[t] : 0;
  const cf a0 = (add && own_if) ? add[t] : cf{0.f, 0.f};
  if (npass == 1) {  // one transmission pass over every pixel
    // operator values first: their loads are in flight during the forward transform
    const cf* m = it.tables + p0.tab;
    cf th[E], tl[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
      th[k] = m[t + k * NT];
      tl[k] = m[N + t + k * NT];
    }
    rf::fft<-1, N, NT>(v, b0, b1, phase, tw, t, RADS{});
    if (next_p >= 0) r2_next_passes(nx, it, next_backward);
#pragma unroll
    for (int k = 0; k < E; ++k) v[k] = pmul(v[k], th[k], tl[k]);
    rf::fft<+1, N, NT>(v, b0, b1, phase, tw, t, RADS{});
    if (mk)
#pragma unroll
      for (int k = 0; k < E; ++k) {
        const int q = t + k * NT;
        v[k] = mask_mul(v[k], mk[q], mk[N + q]);
      }
  } else {
    std::uint32_t pw[EW];
    if (pid) {
#pragma unroll
      for (int w = 0; w < EW; ++w) pw[w] = 0;
#pragma unroll
      for (int k = 0; k < E; ++k) pw[k >> 2] |= static_cast<std::uint32_t>(pid[t + k * NT]) << (8 * (k & 3));
    }
    {
      const cf* m = it.tables + p0.tab;
#pragma unroll
      for (int k = 0; k < E; ++k) {
        prefetch_l1(m + t + k * NT);
        prefetch_l1(m + N + t + k * NT);
      }
    }
    rf::fft<-1, N, NT>(v, b0, b1, phase, tw, t, RADS{});
    if (next_p >= 0) r2_next_passes(nx, it, next_backward);
    const int pid0 = (pid && own_if) ? pid[q0] : 0;
#pragma unroll
    for (int k = 0; k < E; ++k) S[rf::pad(t + k * NT)] = v[k];
    R2Pass cur = p0, nxt = p1;
    for (int j = 0; j < npass; ++j) {
      R2Pass nn = cur;
      if (j + 2 < npass) nn = it.passes[off + j + 2];
      if (j + 1 < npass) {
        const cf* mn = it.tables + nxt.tab;
#pragma unroll
        for (int k = 0; k < E; ++k) {
          prefetch_l1(mn + t + k * NT);
          prefetch_l1(mn + N + t + k * NT);
        }
      }
      const cf* m = it.tables + cur.tab;
#pragma unroll
      for (int k = 0; k < E; ++k) {
        const int q = t + k * NT;
        v[k] = pmul(S[rf::pad(q)], m[q], m[N + q]);
        if ((k & 3) == 3) asm volatile("" ::: "memory");
      }
      rf::fft<+1, N, NT>(v, b0, b1, phase, tw, t, RADS{});
      if (!cur.refl) {
#pragma unroll
        for (int k = 0; k < E; ++k) {
          const int q = t + k * NT;
          if (!pid || unpack_pid<E>(pw, k) == cur.pair) out[k] = mk ? mask_mul(v[k], mk[q], mk[N + q]) : v[k];
          if ((k & 3) == 3) asm volatile("" ::: "memory");
        }
      } else {  // gather at the interface pixels through the free exchange buffer
        cf* buf = phase ? b1 : b0;
#pragma unroll
        for (int k = 0; k < E; ++k) buf[rf::pad(t + k * NT)] = v[k];
        __syncthreads();
        if (own_if && (!pid || pid0 == cur.pair)) store[t] = buf[rf::pad(q0)];
        for (int k = t + NT; k < st.niface; k += NT) {
          const int q = iface[k];
          if (!pid || pid[q] == cur.pair) store[k] = buf[rf::pad(q)];
        }
        phase ^= 1;
      }
      cur = nxt;
      nxt = nn;
    }
#pragma unroll
    for (int k = 0; k < E; ++k) v[k] = out[k];
  }
  if (add) {  // sparse sources of the other pass at this step's interface pixels
    cf* buf = phase ? b1 : b0;
#pragma unroll
    for (int k = 0; k < E; ++k) buf[rf::pad(t + k * NT)] = v[k];
    __syncthreads();
    if (own_if) {
      const int q = rf::pad(q0);
      buf[q] = buf[q] + a0;
    }
    for (int k = t + NT; k < st.niface; k += NT) {
      const int q = rf::pad(iface[k]);
      buf[q] = buf[q] + add[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < E; ++k) v[k] = buf[rf::pad(t + k * NT)];
    phase ^= 1;
  }
}

// The step after step p of a sweep: the next one of the sweep, else the first of the next
// sweep (−1: none).
__device__ __forceinline__ int next_step(int s, int p, int nz, int sw, int sweeps, bool backward,
                                         bool& next_backward) {
  next_backward = backward;
  if (s + 1 < nz) return backward ? p - 1 : p + 1;
  if (sw + 1 < sweeps) {
    next_backward = !backward;
    return next_backward ? nz - 1 : 0;
  }
  return -1;
}

// MINB: CTAs per SM the register budget is sized for (1: up to 255 registers a thread; 2: two
// items share an SM and hide each other's latencies, at the cost of registers).
template <int N, int NT, class RADS, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) k_resident2d_fixed(const R2Item* __restrict__ items,
                                                         int nitems, int* queue,
                                                         const Tw<float>* __restrict__ tw) {
  constexpr int E = N / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cf* b0 = reinterpret_cast<cf*>(smem_raw);
  cf* b1 = b0 + rf::padded(N);
  cf* S = b1 + rf::padded(N);
  float* mask_s = reinterpret_cast<float*>(smem_raw + lines_bytes(N, 3));
  __shared__ int s_item;
  __shared__ double s_red[NT / 32];
  const int t = threadIdx.x;
  int phase = 0;
  for (;;) {
    if (t == 0) s_item = atomicAdd(queue, 1);
    __syncthreads();
    const int idx = s_item;
    if (idx >= nitems) return;
    const R2Item it = items[idx];
    if (t == 0) it.clock[0] = global_ns();
    const float* mk = it.mask;
    if constexpr (fixed_mask_in_smem<N>()) {
      if (mk) {  // first read in the first step's epilogue, after the transforms' barriers
        for (int i = t; i < 2 * N; i += NT) mask_s[i] = it.mask[i];
        mk = mask_s;
      }
    }
    cf v[E], out[E];
    const int iters = it.iterations > 0 ? it.iterations : 1;
    r2f_load<N, NT>(v, it.input, t);
    rf::fft<-1, N, NT>(v, b0, b1, phase, tw, t, RADS{});
    {
      const double pin = r2f_flux<N, NT>(v, it.w_in, s_red, t);
      if (t == 0) it.energy[2 * iters] = pin;
    }
    // sweeps alternate forward (even) and backward (odd); iterations = 0: one forward sweep
    const int sweeps = it.iterations > 0 ? 2 * it.iterations : 1;
    R2Next nx;
    nx.st = it.steps[0];
    r2_next_passes(nx, it, false);
    for (int sw = 0; sw < sweeps; ++sw) {
      const bool backward = sw & 1;
      const int iter = sw >> 1;
      if (!backward) {
        r2f_load<N, NT>(v, it.input, t);
      } else {
#pragma unroll
        for (int k = 0; k < E; ++k) v[k] = cf{0.f, 0.f};
      }
      for (int s = 0; s < it.nz; ++s) {
        const int p = backward ? it.nz - 1 - s : s;  // step p: planes p and p + 1
        const R2Step st = nx.st;
        const R2Pass p0 = nx.p0, p1 = nx.p1;
        bool next_backward;
        const int next_p = next_step(s, p, it.nz, sw, sweeps, backward, next_backward);
        const bool reflect = r2_reflects(st, backward, it.iterations);
        const bool has_add = st.niface > 0 && (backward || iter > 0);
        cf* store = (backward ? it.src_fwd : it.src_bwd) + st.iface;
        const cf* add = has_add ? (backward ? it.src_bwd : it.src_fwd) + st.iface : nullptr;
        r2f_step<N, NT, RADS>(v, S, out, b0, b1, phase, it, st, p0, p1, nx, next_p,
                              next_backward, backward, reflect, store, add, mk, tw, t);
      }
      r2f_store<N, NT>(backward ? it.reflected : it.transmitted, v, t);
      if (it.iterations == 0) break;
#pragma unroll
      for (int k = 0; k < E; ++k) out[k] = v[k];
      rf::fft<-1, N, NT>(out, b0, b1, phase, tw, t, RADS{});
      const double flux = r2f_flux<N, NT>(out, backward ? it.w_in : it.w_out, s_red, t);
      if (t == 0) it.energy[2 * iter + (backward ? 1 : 0)] = flux;
    }
    __syncthreads();
    if (t == 0) it.clock[1] = global_ns();
    __syncthreads();
  }
}

}  // namespace bwpm
