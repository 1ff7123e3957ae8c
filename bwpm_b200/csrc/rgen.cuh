// Register-resident resident-2D kernels for run-time line lengths.
//
// The fixed-length kernels (rfft.cuh, k_resident2d_fixed) unroll everything for one N. This
// variant keeps the number of values per thread E a compile-time constant and takes the line
// length n = E·nt (nt ≤ blockDim threads own values) and the radix order (2, 3, 4, 5, 8) at
// run time, so one kernel serves many lengths. A stage whose radix divides E is the
// owned-pattern Stockham stage of rfft.cuh (one exchange); any other stage gathers whole
// butterflies from shared memory (two exchanges), so E need not contain every prime of n (the
// host picks E and the radix order per length). The run-time sub-length L costs one integer
// modulo per butterfly. Items of different lengths share a launch: threads t ≥ nt of an item
// own no values and only join the barriers.
#pragma once

#include "resident2d.cuh"

namespace bwpm {
namespace rg {

template <int DIR, int E, int R>
__device__ __forceinline__ void stage(cf (&v)[E], cf* buf, const Tw<float>* __restrict__ tw, int t,
                                      int nt, int L, int off, bool last) {
  constexpr int K = E / R;
  static_assert(E % R == 0, "radix must divide the values per thread");
  if (t < nt) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const int i = t + j * nt;
      const int k = i % L;
      cf u[R];
#pragma unroll
      for (int r = 0; r < R; ++r) u[r] = v[j + r * K];
      if (L > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) u[r] = twmul<DIR>(u[r], tw[off + (r - 1) * L + k]);
      }
      rf::dft<DIR, R>(u);
      if (last) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[j + r * K] = u[r];
      } else {
        const int base = (i - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[rf::pad(base + r * L)] = u[r];
      }
      asm volatile("" ::: "memory");
    }
  }
  if (!last) {
    __syncthreads();
    if (t < nt) {
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = buf[rf::pad(t + m * nt)];
    }
  }
}

// A stage whose radix does not divide E: the owned values go to shared memory, each thread
// gathers whole butterflies (i = t + j·nt < n/R, a run-time count), writes the outputs to the
// other buffer, and reads back its owned values. Two barriers instead of one; `phase` is left
// as it was (both buffers were used, the last reads were from the other one).
template <int DIR, int E, int R>
__device__ __forceinline__ void stage_gather(cf (&v)[E], cf* in_buf, cf* out_buf,
                                             const Tw<float>* __restrict__ tw, int t, int nt, int n,
                                             int L, int off) {
  if (t < nt) {
#pragma unroll
    for (int m = 0; m < E; ++m) in_buf[rf::pad(t + m * nt)] = v[m];
  }
  __syncthreads();
  const int nb = n / R;
  for (int i = t; i < nb; i += nt) {
    const int k = i % L;
    cf u[R];
#pragma unroll
    for (int r = 0; r < R; ++r) u[r] = in_buf[rf::pad(i + r * nb)];
    if (L > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) u[r] = twmul<DIR>(u[r], tw[off + (r - 1) * L + k]);
    }
    rf::dft<DIR, R>(u);
    const int base = (i - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) out_buf[rf::pad(base + r * L)] = u[r];
  }
  __syncthreads();
  if (t < nt) {
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = out_buf[rf::pad(t + m * nt)];
  }
}

// In-register transform (DIR −1 forward, +1 inverse unnormalised) of a line of E·nt points with
// the stages of `plan`; `phase` as in rf::fft. Every thread of the block must call it.
template <int DIR, int E, int R>
__device__ __forceinline__ void any_stage(cf (&v)[E], cf* b0, cf* b1, int& phase,
                                          const Tw<float>* __restrict__ tw, int t, int nt, int n,
                                          int L, int off, bool last) {
  if constexpr (E % R == 0) {
    stage<DIR, E, R>(v, phase ? b1 : b0, tw, t, nt, L, off, last);
    if (!last) phase ^= 1;
  } else {
    stage_gather<DIR, E, R>(v, phase ? b1 : b0, phase ? b0 : b1, tw, t, nt, n, L, off);
  }
}

template <int DIR, int E>
__device__ __forceinline__ void fft(cf (&v)[E], cf* b0, cf* b1, int& phase, const FftPlan& plan,
                                   const Tw<float>* __restrict__ tw, int t, int nt) {
  for (int s = 0; s < plan.nstages; ++s) {
    const bool last = s == plan.nstages - 1;
    const int L = plan.len[s], off = plan.twoff[s];
    switch (plan.radix[s]) {
      case 2: any_stage<DIR, E, 2>(v, b0, b1, phase, tw, t, nt, plan.n, L, off, last); break;
      case 3: any_stage<DIR, E, 3>(v, b0, b1, phase, tw, t, nt, plan.n, L, off, last); break;
      case 4: any_stage<DIR, E, 4>(v, b0, b1, phase, tw, t, nt, plan.n, L, off, last); break;
      case 5: any_stage<DIR, E, 5>(v, b0, b1, phase, tw, t, nt, plan.n, L, off, last); break;
      case 8: any_stage<DIR, E, 8>(v, b0, b1, phase, tw, t, nt, plan.n, L, off, last); break;
      default: break;  // the host plans radices 2, 3, 4, 5 and 8 only
    }
  }
}

// Σ w[q]·|v|² over the owned values of the first nt threads, FP64 (compensated per thread, tree
// over the block); thread 0 returns the total. red: blockDim doubles.
template <int E>
__device__ __forceinline__ double flux(const cf (&v)[E], const double* w, double* red, int t, int nt) {
  double s = 0.0, c = 0.0;
  if (t < nt) {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const double a = w[t + m * nt] * (static_cast<double>(v[m].re) * v[m].re +
                                        static_cast<double>(v[m].im) * v[m].im);
      const double y = a - c;
      const double z = s + y;
      c = (z - s) - y;
      s = z;
    }
  }
  red[t] = s;
  __syncthreads();
  for (int half = 1; half < static_cast<int>(blockDim.x); half <<= 1) {
    if ((t & (2 * half - 1)) == 0 && t + half < static_cast<int>(blockDim.x)) red[t] += red[t + half];
    __syncthreads();
  }
  const double total = red[0];
  __syncthreads();
  return total;
}

// One slab step (cf. r2f_step: prefetched records and operator values, pair ids of the owned
// pixels once per step, the next pass's operator values prefetched into L1, the first interface
// round loaded before the forward transform; mk: the item's mask in shared memory, n hi then n lo
// values, or null); every thread of the block calls it.
template <int E>
__device__ __forceinline__ void step(cf (&v)[E], cf* S, cf (&out)[E], cf* b0, cf* b1, int& phase,
                                     const R2Item& it, const R2Step& st, const R2Pass& p0,
                                     const R2Pass& p1, R2Next& nx, int next_p, bool next_backward,
                                     bool backward, bool reflect, cf* store, const cf* add,
                                     const float* mk, const FftPlan& plan,
                                     const Tw<float>* __restrict__ tw, int t, int nt) {
  constexpr int EW = (E + 3) / 4;
  const int n = it.n, nthr = static_cast<int>(blockDim.x);
  const bool own = t < nt;
  const int off = backward ? st.bwd_off : st.fwd_off;
  const int npass = r2_passes(st, backward, reflect);
  const std::uint8_t* pid = st.pid >= 0 ? it.pids + st.pid : nullptr;
  const int* iface = it.iface + st.iface;
  if (next_p >= 0) nx.st = it.steps[next_p];
  // interface entry t, the first round of the gather and add loops
  const bool own_if = t < st.niface;
  const int q0 = own_if ? iface[t] : 0;
  const cf a0 = (add && own_if) ? add[t] : cf{0.f, 0.f};
  if (npass == 1) {
    const cf* m = it.tables + p0.tab;
    cf th[E], tl[E];  // in flight during the forward transform
    if (own) {
#pragma unroll
      for (int k = 0; k < E; ++k) {
        th[k] = m[t + k * nt];
        tl[k] = m[n + t + k * nt];
      }
    }
    fft<-1, E>(v, b0, b1, phase, plan, tw, t, nt);
    if (next_p >= 0) r2_next_passes(nx, it, next_backward);
    if (own) {
#pragma unroll
      for (int k = 0; k < E; ++k) v[k] = pmul(v[k], th[k], tl[k]);
    }
    fft<+1, E>(v, b0, b1, phase, plan, tw, t, nt);
    if (own && mk) {
#pragma unroll
      for (int k = 0; k < E; ++k) {
        const int q = t + k * nt;
        v[k] = mask_mul(v[k], mk[q], mk[n + q]);
      }
    }
  } else {
    std::uint32_t pw[EW];
#pragma unroll
    for (int w = 0; w < EW; ++w) pw[w] = 0;
    if (pid && own) {
#pragma unroll
      for (int k = 0; k < E; ++k) pw[k >> 2] |= static_cast<std::uint32_t>(pid[t + k * nt]) << (8 * (k & 3));
    }
    if (own) {
      const cf* m = it.tables + p0.tab;
#pragma unroll
      for (int k = 0; k < E; ++k) {
        prefetch_l1(m + t + k * nt);
        prefetch_l1(m + n + t + k * nt);
      }
    }
    fft<-1, E>(v, b0, b1, phase, plan, tw, t, nt);
    if (next_p >= 0) r2_next_passes(nx, it, next_backward);
    const int pid0 = (pid && own_if) ? pid[q0] : 0;
    if (own) {
#pragma unroll
      for (int k = 0; k < E; ++k) S[rf::pad(t + k * nt)] = v[k];
    }
    R2Pass cur = p0, nxt = p1;
    for (int j = 0; j < npass; ++j) {
      R2Pass nn = cur;
      if (j + 2 < npass) nn = it.passes[off + j + 2];
      if (own && j + 1 < npass) {
        const cf* mn = it.tables + nxt.tab;
#pragma unroll
        for (int k = 0; k < E; ++k) {
          prefetch_l1(mn + t + k * nt);
          prefetch_l1(mn + n + t + k * nt);
        }
      }
      const cf* m = it.tables + cur.tab;
      if (own) {
#pragma unroll
        for (int k = 0; k < E; ++k) {
          const int q = t + k * nt;
          v[k] = pmul(S[rf::pad(q)], m[q], m[n + q]);
          if ((k & 3) == 3) asm volatile("" ::: "memory");
        }
      }
      fft<+1, E>(v, b0, b1, phase, plan, tw, t, nt);
      if (!cur.refl) {
        if (own) {
#pragma unroll
          for (int k = 0; k < E; ++k) {
            const int q = t + k * nt;
            if (!pid || unpack_pid<E>(pw, k) == cur.pair) out[k] = mk ? mask_mul(v[k], mk[q], mk[n + q]) : v[k];
            if ((k & 3) == 3) asm volatile("" ::: "memory");
          }
        }
      } else {  // gather at the interface pixels through the free exchange buffer
        cf* buf = phase ? b1 : b0;
        if (own) {
#pragma unroll
          for (int k = 0; k < E; ++k) buf[rf::pad(t + k * nt)] = v[k];
        }
        __syncthreads();
        if (own_if && (!pid || pid0 == cur.pair)) store[t] = buf[rf::pad(q0)];
        for (int k = t + nthr; k < st.niface; k += nthr) {
          const int q = iface[k];
          if (!pid || pid[q] == cur.pair) store[k] = buf[rf::pad(q)];
        }
        phase ^= 1;
      }
      cur = nxt;
      nxt = nn;
    }
    if (own) {
#pragma unroll
      for (int k = 0; k < E; ++k) v[k] = out[k];
    }
  }
  if (add) {  // sparse sources of the other pass at this step's interface pixels
    cf* buf = phase ? b1 : b0;
    if (own) {
#pragma unroll
      for (int k = 0; k < E; ++k) buf[rf::pad(t + k * nt)] = v[k];
    }
    __syncthreads();
    if (own_if) {
      const int q = rf::pad(q0);
      buf[q] = buf[q] + a0;
    }
    for (int k = t + nthr; k < st.niface; k += nthr) {
      const int q = rf::pad(iface[k]);
      buf[q] = buf[q] + add[k];
    }
    __syncthreads();
    if (own) {
#pragma unroll
      for (int k = 0; k < E; ++k) v[k] = buf[rf::pad(t + k * nt)];
    }
    phase ^= 1;
  }
}

// threads per CTA at most: 512 for E ≤ 8, else 256 (registers for the E values per thread)
__host__ __device__ constexpr int rt_max_threads(int e) { return e <= 8 ? 512 : 256; }

}  // namespace rg

// Shared memory of the run-time-length kernel for lines up to n points: three padded lines, the
// stage twiddles and the mask of the item in progress.
__host__ __device__ constexpr std::size_t rt_smem_bytes(int n) {
  return lines_bytes(n, 3) + static_cast<std::size_t>(n - 1) * sizeof(Tw<float>) +
         2 * static_cast<std::size_t>(n) * sizeof(float);  // + the mask
}

// Persistent kernel over items of any length n = E·nt (nt ≤ blockDim, plan per item). NTMAX:
// the thread limit (and so the register budget) of the instance; 512 for a small E is the wide
// form for lines whose n/E exceeds the default limit (128 registers: it spills, but a line of
// 4050 points then runs on 450 threads with E = 9 instead of 135 with E = 30: 57 → 36 µs a step).
template <int E, int NTMAX = rg::rt_max_threads(E)>
__global__ void __launch_bounds__(NTMAX, 1)
    k_resident2d_rt(const R2Item* __restrict__ items, int nitems, int* queue, R2Shared sh) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_item;
  __shared__ double s_red[512];
  __shared__ FftPlan s_plan;
  const int t = threadIdx.x;
  int phase = 0;
  for (;;) {
    if (t == 0) s_item = atomicAdd(queue, 1);
    __syncthreads();
    const int idx = s_item;
    if (idx >= nitems) return;
    const R2Item it = items[idx];
    const int n = it.n, nt = n / E;
    // the item's n − 1 stage twiddles, staged after the three lines (offsets rebased to 0)
    Tw<float>* tws = reinterpret_cast<Tw<float>*>(smem_raw + lines_bytes(n, 3));
    const int base = sh.plans[it.plan].twoff[0];
    if (t == 0) {
      s_plan = sh.plans[it.plan];
      for (int st = 0; st < s_plan.nstages; ++st) s_plan.twoff[st] -= base;
      it.clock[0] = global_ns();
    }
    for (int i = t; i < n - 1; i += static_cast<int>(blockDim.x)) tws[i] = sh.twiddles[base + i];
    float* mask_s = reinterpret_cast<float*>(tws + (n - 1));
    const float* mk = nullptr;
    if (it.mask) {
      for (int i = t; i < 2 * n; i += static_cast<int>(blockDim.x)) mask_s[i] = it.mask[i];
      mk = mask_s;
    }
    __syncthreads();
    const FftPlan& plan = s_plan;
    cf* b0 = reinterpret_cast<cf*>(smem_raw);
    cf* b1 = b0 + rf::padded(n);
    cf* S = b1 + rf::padded(n);
    const bool own = t < nt;
    cf v[E], out[E];
    const int iters = it.iterations > 0 ? it.iterations : 1;
    if (own) {
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = it.input[t + m * nt];
    }
    rg::fft<-1, E>(v, b0, b1, phase, plan, tws, t, nt);
    {
      const double pin = rg::flux<E>(v, it.w_in, s_red, t, nt);
      if (t == 0) it.energy[2 * iters] = pin;
    }
    const int sweeps = it.iterations > 0 ? 2 * it.iterations : 1;
    R2Next nx;
    nx.st = it.steps[0];
    r2_next_passes(nx, it, false);
    for (int sw = 0; sw < sweeps; ++sw) {
      const bool backward = sw & 1;
      const int iter = sw >> 1;
      if (own) {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = backward ? cf{0.f, 0.f} : it.input[t + m * nt];
      }
      for (int s = 0; s < it.nz; ++s) {
        const int p = backward ? it.nz - 1 - s : s;
        const R2Step st = nx.st;
        const R2Pass p0 = nx.p0, p1 = nx.p1;
        bool next_backward;
        const int next_p = next_step(s, p, it.nz, sw, sweeps, backward, next_backward);
        const bool reflect = r2_reflects(st, backward, it.iterations);
        const bool has_add = st.niface > 0 && (backward || iter > 0);
        cf* store = (backward ? it.src_fwd : it.src_bwd) + st.iface;
        const cf* add = has_add ? (backward ? it.src_bwd : it.src_fwd) + st.iface : nullptr;
        rg::step<E>(v, S, out, b0, b1, phase, it, st, p0, p1, nx, next_p, next_backward,
                    backward, reflect, store, add, mk, plan, tws, t, nt);
      }
      cf* dst = backward ? it.reflected : it.transmitted;
      if (own) {
#pragma unroll
        for (int m = 0; m < E; ++m) dst[t + m * nt] = v[m];
      }
      if (it.iterations == 0) break;
      if (own) {
#pragma unroll
        for (int m = 0; m < E; ++m) out[m] = v[m];
      }
      rg::fft<-1, E>(out, b0, b1, phase, plan, tws, t, nt);
      const double fl = rg::flux<E>(out, backward ? it.w_in : it.w_out, s_red, t, nt);
      if (t == 0) it.energy[2 * iter + (backward ? 1 : 0)] = fl;
    }
    __syncthreads();
    if (t == 0) it.clock[1] = global_ns();
    __syncthreads();
  }
}

}  // namespace bwpm
