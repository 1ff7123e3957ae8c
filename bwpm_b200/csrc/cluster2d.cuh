// Resident 2D engine, one line split over a cluster of C CTAs (thread-block cluster + DSMEM).
//
// For the longest lines one CTA per line makes the slab chain latency-bound (one SM's issue
// rate and register file). Here the C CTAs of a cluster, on C SMs, share one work item:
// N = C·M, CTA c holds the real-space points n = C·m + c (m < M) and the spectral points
// k = c·(M/C) + k1l + M·k2 (k1l < M/C, k2 < C). A length-N transform is
//   forward:  Y_c = DFT_M(x_c);  Y_c[k1] ·= w_N^{c·k1};  exchange;
//             X[k1 + M·k2] = Σ_c Y_c[k1]·w_C^{c·k2}   (C-point DFT over the cluster)
//   inverse:  Z_c[k1] = Σ_k2 X[k1 + M·k2]·w_C^{−c·k2}·w_N^{−c·k1};  exchange;
//             x_c = IDFT_M(Z_c)
// (a two-factor Cooley-Tukey split, N = M·C), each exchange one all-to-all through distributed
// shared memory: every CTA stores its values straight into the owners' buffers with st.async
// (no round trip) and waits on its own mbarrier for the bytes it expects (see "exchanges"
// below), then reads locally. The local M-point transforms are the register-resident transforms
// of rfft.cuh.
//
// Everything else (passes, selection by pair id, mask, interface sources, FP64 flux) follows
// k_resident2d_fixed; each CTA handles its own points. Cross twiddles w_N^{c·k1} (c < C,
// k1 < M) are (hi, lo) pairs from FP64, stored after the M-point plan's twiddles (which hold
// M − 1 entries for any radix order) and staged in the CTA's shared memory where they fit. The
// item index and the flux partial sums go through cluster barriers (once per item and sweep).
#pragma once

#include <cooperative_groups.h>

#include "resident2d.cuh"

namespace bwpm {
namespace r2c {

namespace cg = cooperative_groups;

template <int N, int C, int NT>
struct Shape {
  static constexpr int M = N / C;      // points per CTA
  static constexpr int E = M / NT;     // values per thread
  static constexpr int EB = E / C;     // spectral slots per thread and k2
  static constexpr int MB = M / C;     // spectral k1 block of one CTA
  static_assert(N % C == 0 && M % NT == 0 && E % C == 0, "cluster shape");
};

// Shared memory of a cluster kernel: three padded lines and two exchange buffers of G·M points
// (G: passes per exchange), then the mask of the CTA's points (M hi values, M lo values), then
// the CTA's cross twiddles (forward w_N^{c·k1}, k1 < M; inverse w_N^{−d·k1} of its spectral block,
// d < C) when they fit, loaded once per CTA.
template <int N, int C>
__host__ __device__ constexpr std::size_t cluster_base_bytes(int g) {
  return ((static_cast<std::size_t>(3 * rf::padded(N / C) + 2 * g * (N / C)) * sizeof(cf) + 15) / 16 * 16 +
          2 * static_cast<std::size_t>(N / C) * sizeof(float) + 15) / 16 * 16;
}
template <int N, int C>
__host__ __device__ constexpr std::size_t cluster_xtw_bytes() {
  return 2 * static_cast<std::size_t>(N / C) * sizeof(Tw<float>);
}
constexpr std::size_t kClusterSmemCap = 220 * 1024;
// Passes per inverse exchange: the largest G ≤ 4 that fits with the cross twiddles in shared
// memory, else the largest that fits without them.
template <int N, int C>
__host__ __device__ constexpr int cluster_group() {
  for (int g = 4; g >= 1; --g)
    if (cluster_base_bytes<N, C>(g) + cluster_xtw_bytes<N, C>() <= kClusterSmemCap) return g;
  for (int g = 4; g >= 1; --g)
    if (cluster_base_bytes<N, C>(g) <= kClusterSmemCap) return g;
  return 1;
}
// layout for a given G (the kernel's template parameter; the variant registry takes
// cluster_group's choice)
template <int N, int C, int G>
__host__ __device__ constexpr std::size_t cluster_lines_bytes() {
  return (static_cast<std::size_t>(3 * rf::padded(N / C) + 2 * G * (N / C)) * sizeof(cf) + 15) / 16 * 16;
}
template <int N, int C, int G>
__host__ __device__ constexpr std::size_t cluster_mask_end() {
  return cluster_base_bytes<N, C>(G);
}
template <int N, int C, int G>
__host__ __device__ constexpr bool cluster_xtw_in_smem() {
  return cluster_mask_end<N, C, G>() + cluster_xtw_bytes<N, C>() <= kClusterSmemCap;
}
template <int N, int C, int G>
__host__ __device__ constexpr std::size_t cluster_smem_bytes() {
  return cluster_mask_end<N, C, G>() + (cluster_xtw_in_smem<N, C, G>() ? cluster_xtw_bytes<N, C>() : 0);
}

// spectral index of slot s (= k2·EB + i) of thread t in CTA c
template <int N, int C, int NT>
__device__ __forceinline__ int kspec(int s, int t, int c) {
  using S = Shape<N, C, NT>;
  const int k2 = s / S::EB, i = s % S::EB;
  return c * S::MB + i * NT + t + S::M * k2;
}

// real-space index of owned value j of thread t in CTA c
template <int N, int C, int NT>
__device__ __forceinline__ int qreal(int j, int t, int c) {
  return C * (t + j * NT) + c;
}

// ---- exchanges through distributed shared memory -----------------------------------------------
//
// Each exchange is an all-to-all: every CTA sends values to every CTA of the cluster (itself
// included) with st.async, an asynchronous remote store that also counts its bytes on the
// receiver's mbarrier (complete_tx); the receiver has armed that mbarrier with the bytes it
// expects and waits for the phase to complete. No cluster-wide barrier is needed, and a buffer
// can be reused two exchanges later: a CTA sends exchange e + 2 only after receiving exchange
// e + 1 from every peer, which each peer sent after reading its exchange-e data. An exchange
// costs a DSMEM round of latency (≈ 0.5 µs), not bandwidth, so the inverse transforms of a
// multi-pass step share one: up to G passes go out into slots q·M of the receive buffer and the
// CTA waits once for g·M values.
struct Exchange {
  cf* buf[2];         // receive buffers (alternating)
  unsigned mbar[2];   // their mbarriers (shared-window addresses)
  unsigned parity;    // bit b: parity of the phase awaited on buffer b
  int cur;            // buffer of the next exchange
  int* status;        // set to 1 when a wait gives up
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// the same shared-memory offset in CTA `rank` of the cluster
__device__ __forceinline__ unsigned mapa(unsigned addr, int rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_async(unsigned raddr, cf v, unsigned rmbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];"
               :: "r"(raddr), "f"(v.re), "f"(v.im), "r"(rmbar) : "memory");
}
__device__ __forceinline__ void mbar_init(unsigned mbar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned mbar, unsigned bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}"
               :: "r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned mbar, unsigned parity) {
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
  return ok != 0;
}

// Opens the next exchange: thread 0 arms the receive mbarrier with the bytes to come.
__device__ __forceinline__ void xopen(Exchange& ex, int t, unsigned bytes) {
  if (t == 0) mbar_expect(ex.mbar[ex.cur], bytes);
}

// Waits for the current exchange's data, bounded: after 2 s the status word is set and the kernel
// goes on with whatever arrived. The status word is read only on the slow path (every 20 µs of
// waiting; a global load on the fast path would put an L2 round trip into every exchange): once
// it is set, a later wait gives up within 20 µs, so a fault in the protocol can neither hang the
// GPU nor stretch the run far (its results are then reported invalid).
__device__ __forceinline__ void xwait(Exchange& ex) {
  const unsigned mb = ex.mbar[ex.cur], par = (ex.parity >> ex.cur) & 1u;
  if (!mbar_try(mb, par)) {
    const long long t0 = global_ns();
    long long check = 20000;
    while (!mbar_try(mb, par)) {
      const long long dt = global_ns() - t0;
      if (dt > check) {
        if (*reinterpret_cast<volatile int*>(ex.status) != 0) break;
        if (dt > 2000000000LL) {
          atomicExch(ex.status, 1);
          break;
        }
        check = dt + 20000;
      }
    }
  }
  ex.parity ^= 1u << ex.cur;
  ex.cur ^= 1;
}

// Forward N-point transform: v holds the CTA's real-space values (owned pattern of the M-point
// transform) and receives its spectral slots.
template <int N, int C, int NT, class RADS>
__device__ __forceinline__ void forward(cf (&v)[Shape<N, C, NT>::E], cf* b0, cf* b1, int& phase,
                                        Exchange& ex, const Tw<float>* tw, const Tw<float>* xf,
                                        const Tw<float>* xi, int t, int c) {
  using S = Shape<N, C, NT>;
  rf::fft<-1, S::M, NT>(v, b0, b1, phase, tw, t, RADS{});
  cf* x = ex.buf[ex.cur];
  xopen(ex, t, S::M * sizeof(cf));
  const unsigned base = smem_u32(x), mb = ex.mbar[ex.cur];
  // Y_c[k1]·w_N^{c·k1} goes to the owner of k1's block (CTA j / EB, since
  // k1 = t + j·NT = (j / EB)·MB + (j mod EB)·NT + t), slot c·MB + (k1 mod MB) of its buffer
#pragma unroll
  for (int j = 0; j < S::E; ++j) {
    const int k1 = t + j * NT, dst = j / S::EB;
    const unsigned off = static_cast<unsigned>(c * S::MB + (j % S::EB) * NT + t) * sizeof(cf);
    st_async(mapa(base, dst) + off, c == 0 ? v[j] : twmul<-1>(v[j], xf[k1]), mapa(mb, dst));
  }
  xwait(ex);
#pragma unroll
  for (int i = 0; i < S::EB; ++i) {
    const int k1l = i * NT + t;
    cf u[C];
#pragma unroll
    for (int r = 0; r < C; ++r) u[r] = x[r * S::MB + k1l];
    rf::dft<-1, C>(u);
#pragma unroll
    for (int k2 = 0; k2 < C; ++k2) v[k2 * S::EB + i] = u[k2];
  }
}

// First half of an inverse (unnormalised) N-point transform: the C-point inverse DFTs of the
// spectral slots, the cross twiddles, and the values sent to group slot q (offset q·M) of every
// CTA's current receive buffer. The caller opens the exchange for all its slots and waits once.
template <int N, int C, int NT, int G>
__device__ __forceinline__ void inverse_send(const cf (&v)[Shape<N, C, NT>::E], const Exchange& ex,
                                             int q, const Tw<float>* xi, int t, int c) {
  using S = Shape<N, C, NT>;
  const unsigned base = smem_u32(ex.buf[ex.cur] + q * S::M), mb = ex.mbar[ex.cur];
#pragma unroll
  for (int i = 0; i < S::EB; ++i) {
    const int k1l = i * NT + t;
    cf u[C];
#pragma unroll
    for (int k2 = 0; k2 < C; ++k2) u[k2] = v[k2 * S::EB + i];
    rf::dft<+1, C>(u);
    // Z_d[k1]·w_N^{−d·k1} (k1 = c·MB + k1l; the twiddle is entry d·XS + k1l of xi: the CTA's
    // staged block in shared memory, else the global table from entry c·MB) goes to CTA d,
    // slot k1 of its buffer
    constexpr int XS = cluster_xtw_in_smem<N, C, G>() ? S::MB : S::M;
    const unsigned off = static_cast<unsigned>(c * S::MB + k1l) * sizeof(cf);
#pragma unroll
    for (int d = 0; d < C; ++d)
      st_async(mapa(base, d) + off, d == 0 ? u[d] : twmul<+1>(u[d], xi[d * XS + k1l]), mapa(mb, d));
  }
}

// Second half: the received slot x (M points) to the real-space owned values.
template <int N, int C, int NT, class RADS>
__device__ __forceinline__ void inverse_finish(cf (&v)[Shape<N, C, NT>::E], const cf* x, cf* b0,
                                               cf* b1, int& phase, const Tw<float>* tw, int t) {
  using S = Shape<N, C, NT>;
#pragma unroll
  for (int j = 0; j < S::E; ++j) v[j] = x[t + j * NT];
  rf::fft<+1, S::M, NT>(v, b0, b1, phase, tw, t, RADS{});
}

// Inverse (unnormalised) N-point transform: spectral slots in, real-space owned values out.
template <int N, int C, int NT, class RADS, int G>
__device__ __forceinline__ void inverse(cf (&v)[Shape<N, C, NT>::E], cf* b0, cf* b1, int& phase,
                                        Exchange& ex, const Tw<float>* tw, const Tw<float>* xi,
                                        int t, int c) {
  using S = Shape<N, C, NT>;
  const cf* x = ex.buf[ex.cur];
  xopen(ex, t, S::M * sizeof(cf));
  inverse_send<N, C, NT, G>(v, ex, 0, xi, t, c);
  xwait(ex);
  inverse_finish<N, C, NT, RADS>(v, x, b0, b1, phase, tw, t);
}

// Σ w[k]·|v|² over the CTA's spectral slots, compensated FP64; the cluster total is returned on
// rank 0 (others return 0). `part` is this CTA's shared slot for its partial sum.
template <int N, int C, int NT>
__device__ __forceinline__ double flux(const cf (&v)[Shape<N, C, NT>::E], const double* w,
                                       double* red, double* part, int t, int c,
                                       cg::cluster_group& cl) {
  using S = Shape<N, C, NT>;
  double s = 0.0, comp = 0.0;
#pragma unroll
  for (int j = 0; j < S::E; ++j) {
    const double a = w[kspec<N, C, NT>(j, t, c)] * (static_cast<double>(v[j].re) * v[j].re +
                                                     static_cast<double>(v[j].im) * v[j].im);
    const double y = a - comp;
    const double z = s + y;
    comp = (z - s) - y;
    s = z;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((t & 31) == 0) red[t >> 5] = s;
  __syncthreads();
  if (t == 0) {
    double total = 0.0, cc = 0.0;
    for (int i = 0; i < NT / 32; ++i) {
      const double y = red[i] - cc;
      const double z = total + y;
      cc = (z - total) - y;
      total = z;
    }
    *part = total;
  }
  cl.sync();
  double total = 0.0;
  if (c == 0 && t == 0) {
    double cc = 0.0;
    for (int r = 0; r < C; ++r) {
      const double y = *cl.map_shared_rank(part, r) - cc;
      const double z = total + y;
      cc = (z - total) - y;
      total = z;
    }
  }
  // the partials are rewritten at the next flux, after at least one more cluster barrier
  return total;
}

// Record q of a group held in registers (selects with constant indices, no local memory).
template <int G>
__device__ __forceinline__ R2Pass pick(const R2Pass (&r)[G], int q) {
  R2Pass x = r[0];
#pragma unroll
  for (int i = 1; i < G; ++i)
    if (q == i) x = r[i];
  return x;
}

// One slab step of the CTA's share of an item (cf. r2f_step: prefetched records and operator
// values, pair ids of the CTA's pixels loaded once per step, operator values of the next pass
// prefetched into L1, first interface round loaded early; mk: the mask of the CTA's points in
// shared memory, M hi then M lo values, or null).
template <int N, int C, int NT, class RADS, int G>
__device__ __forceinline__ void step(cf (&v)[Shape<N, C, NT>::E], cf* S, cf (&out)[Shape<N, C, NT>::E],
                                     cf* b0, cf* b1, int& phase, Exchange& ex,
                                     const R2Item& it, const R2Step& st, const R2Pass& p0,
                                     const R2Pass& p1, R2Next& nx, int next_p, bool next_backward,
                                     bool backward, bool reflect, cf* store, const cf* add,
                                     const float* mk, const Tw<float>* tw, const Tw<float>* xf,
                                     const Tw<float>* xi, int t, int c) {
  using Sh = Shape<N, C, NT>;
  constexpr int E = Sh::E, M = Sh::M, EW = (E + 3) / 4;
  const int off = backward ? st.bwd_off : st.fwd_off;
  const int npass = r2_passes(st, backward, reflect);
  const std::uint8_t* pid = st.pid >= 0 ? it.pids + st.pid : nullptr;
  const int* iface = it.iface + st.iface;
  if (next_p >= 0) nx.st = it.steps[next_p];
  const bool own_if = t < st.niface;
  const int q0 = own_if ? iface[t] : 0;
  const cf a0 = (add && own_if) ? add[t] : cf{0.f, 0.f};
  if (npass == 1) {
    const cf* m = it.tables + p0.tab;
    cf th[E], tl[E];  // in flight during the forward transform
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int k = kspec<N, C, NT>(j, t, c);
      th[j] = m[k];
      tl[j] = m[N + k];
    }
    forward<N, C, NT, RADS>(v, b0, b1, phase, ex, tw, xf, xi, t, c);
    if (next_p >= 0) r2_next_passes(nx, it, next_backward);
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = pmul(v[j], th[j], tl[j]);
    inverse<N, C, NT, RADS, G>(v, b0, b1, phase, ex, tw, xi, t, c);
    if (mk)
#pragma unroll
      for (int j = 0; j < E; ++j) {
        const int m = t + j * NT;
        v[j] = mask_mul(v[j], mk[m], mk[M + m]);
      }
  } else {
    // passes in groups of G: spectral multiply and send every pass of the group into its slot
    // of the receive buffer, wait once, then the local inverse transforms and epilogues
    std::uint32_t pw[EW];
    if (pid) {
#pragma unroll
      for (int w = 0; w < EW; ++w) pw[w] = 0;
#pragma unroll
      for (int j = 0; j < E; ++j)
        pw[j >> 2] |= static_cast<std::uint32_t>(pid[qreal<N, C, NT>(j, t, c)]) << (8 * (j & 3));
    }
    // the first group's records: p0 and p1 came with the step record, the others load now
    R2Pass rec[G];
#pragma unroll
    for (int q = 0; q < G; ++q) rec[q] = p0;
    if constexpr (G > 1) rec[1] = p1;
#pragma unroll
    for (int q = 2; q < G; ++q)
      if (q < npass) rec[q] = it.passes[off + q];
#pragma unroll
    for (int q = 0; q < (G < 2 ? G : 2); ++q) {
      const cf* m = it.tables + rec[q].tab;
#pragma unroll
      for (int j = 0; j < E; ++j) {
        const int k = kspec<N, C, NT>(j, t, c);
        prefetch_l1(m + k);
        prefetch_l1(m + N + k);
      }
    }
    forward<N, C, NT, RADS>(v, b0, b1, phase, ex, tw, xf, xi, t, c);
    if (next_p >= 0) r2_next_passes(nx, it, next_backward);
    const int pid0 = (pid && own_if) ? pid[q0] : 0;
#pragma unroll
    for (int q = 2; q < G; ++q)
      if (q < npass) {
        const cf* m = it.tables + rec[q].tab;
#pragma unroll
        for (int j = 0; j < E; ++j) {
          const int k = kspec<N, C, NT>(j, t, c);
          prefetch_l1(m + k);
          prefetch_l1(m + N + k);
        }
      }
#pragma unroll
    for (int j = 0; j < E; ++j) S[rf::pad(t + j * NT)] = v[j];
    for (int p = 0; p < npass; p += G) {
      const int g = npass - p < G ? npass - p : G;
      if (p > 0) {  // later groups (steps with more than G passes)
#pragma unroll
        for (int q = 0; q < G; ++q)
          if (q < g) rec[q] = it.passes[off + p + q];
      }
      const cf* x = ex.buf[ex.cur];
      xopen(ex, t, static_cast<unsigned>(g * M) * sizeof(cf));
#pragma unroll 1
      for (int q = 0; q < g; ++q) {
        const cf* m = it.tables + pick(rec, q).tab;
#pragma unroll
        for (int j = 0; j < E; ++j) {
          const int k = kspec<N, C, NT>(j, t, c);
          v[j] = pmul(S[rf::pad(t + j * NT)], m[k], m[N + k]);
        }
        inverse_send<N, C, NT, G>(v, ex, q, xi, t, c);
      }
      xwait(ex);
#pragma unroll 1
      for (int q = 0; q < g; ++q) {
        const R2Pass cur = pick(rec, q);
        inverse_finish<N, C, NT, RADS>(v, x + q * M, b0, b1, phase, tw, t);
        if (!cur.refl) {
#pragma unroll
          for (int j = 0; j < E; ++j) {
            const int ml = t + j * NT;
            if (!pid || unpack_pid<E>(pw, j) == cur.pair) out[j] = mk ? mask_mul(v[j], mk[ml], mk[M + ml]) : v[j];
          }
        } else {  // gather at this CTA's interface pixels through the free transform buffer
          cf* buf = phase ? b1 : b0;
#pragma unroll
          for (int j = 0; j < E; ++j) buf[rf::pad(t + j * NT)] = v[j];
          __syncthreads();
          if (own_if && q0 % C == c && (!pid || pid0 == cur.pair)) store[t] = buf[rf::pad(q0 / C)];
          for (int k = t + NT; k < st.niface; k += NT) {
            const int qq = iface[k];
            if (qq % C != c) continue;
            if (!pid || pid[qq] == cur.pair) store[k] = buf[rf::pad(qq / C)];
          }
          phase ^= 1;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = out[j];
  }
  if (add) {  // sparse sources of the other pass at this CTA's interface pixels
    cf* buf = phase ? b1 : b0;
#pragma unroll
    for (int j = 0; j < E; ++j) buf[rf::pad(t + j * NT)] = v[j];
    __syncthreads();
    if (own_if && q0 % C == c) {
      const int m = rf::pad(q0 / C);
      buf[m] = buf[m] + a0;
    }
    for (int k = t + NT; k < st.niface; k += NT) {
      const int q = iface[k];
      if (q % C != c) continue;
      const int m = rf::pad(q / C);
      buf[m] = buf[m] + add[k];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = buf[rf::pad(t + j * NT)];
    phase ^= 1;
  }
}

}  // namespace r2c

// Persistent cluster kernel: each cluster pulls work items from `queue` (rank 0 takes the next
// index and shares it through distributed shared memory).
template <int N, int C, int NT, class RADS, int G = r2c::cluster_group<N, C>()>
__global__ void __cluster_dims__(C, 1, 1) __launch_bounds__(NT, 1)
    k_resident2d_cluster(const R2Item* __restrict__ items, int nitems, int* queue,
                         const Tw<float>* __restrict__ tw_global) {
  using S = r2c::Shape<N, C, NT>;
  constexpr int E = S::E;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cf* b0 = reinterpret_cast<cf*>(smem_raw);
  cf* b1 = b0 + rf::padded(S::M);
  cf* Sl = b1 + rf::padded(S::M);
  __shared__ alignas(8) unsigned long long s_mbar[2];
  __shared__ int s_item;
  __shared__ double s_red[NT / 32];
  __shared__ double s_part;
  r2c::cg::cluster_group cl = r2c::cg::this_cluster();
  const int t = threadIdx.x;
  const int c = static_cast<int>(cl.block_rank());
  // global layout: M − 1 stage twiddles, then w_N^{c·k1} at (M − 1) + c·M + k1
  const Tw<float>* tw = tw_global;
  const Tw<float>* xg = tw_global + (S::M - 1);
  const Tw<float>* xf = xg + c * S::M;   // forward: this CTA's c, every k1
  const Tw<float>* xi = xg + c * S::MB;  // inverse: entry d·M + k1l for k1 = c·MB + k1l
  float* mask_s = reinterpret_cast<float*>(smem_raw + r2c::cluster_lines_bytes<N, C, G>());
  if constexpr (r2c::cluster_xtw_in_smem<N, C, G>()) {  // read first after the cluster barrier below
    Tw<float>* xfs = reinterpret_cast<Tw<float>*>(smem_raw + r2c::cluster_mask_end<N, C, G>());
    Tw<float>* xis = xfs + S::M;
    for (int i = t; i < S::M; i += NT) {
      xfs[i] = xf[i];
      xis[i] = xi[(i / S::MB) * S::M + i % S::MB];
    }
    xf = xfs;
    xi = xis;
  }
  r2c::Exchange ex;
  ex.buf[0] = Sl + rf::padded(S::M);
  ex.buf[1] = ex.buf[0] + G * S::M;
  ex.mbar[0] = r2c::smem_u32(&s_mbar[0]);
  ex.mbar[1] = r2c::smem_u32(&s_mbar[1]);
  ex.parity = 0;
  ex.cur = 0;
  ex.status = nullptr;
  if (t == 0) {  // one arrival (thread 0's) per phase; visible to the peers after the first
    r2c::mbar_init(ex.mbar[0], 1);  // cluster barrier below
    r2c::mbar_init(ex.mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  int phase = 0;
  for (;;) {
    if (c == 0 && t == 0) s_item = atomicAdd(queue, 1);
    cl.sync();
    const int idx = *cl.map_shared_rank(&s_item, 0);
    if (idx >= nitems) {  // every CTA of the cluster leaves together, after every CTA has read
      cl.sync();          // rank 0's index (no CTA exits while a peer reads its shared memory)
      return;
    }
    const R2Item it = items[idx];
    ex.status = it.status;
    if (c == 0 && t == 0) it.clock[0] = global_ns();
    const float* mk = nullptr;
    if (it.mask) {  // first read in the first step's epilogue, after the transforms' barriers
      for (int m = t; m < S::M; m += NT) {
        const int q = C * m + c;
        mask_s[m] = it.mask[q];
        mask_s[S::M + m] = it.mask[N + q];
      }
      mk = mask_s;
    }
    cf v[E], out[E];
    const int iters = it.iterations > 0 ? it.iterations : 1;
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = it.input[r2c::qreal<N, C, NT>(j, t, c)];
    r2c::forward<N, C, NT, RADS>(v, b0, b1, phase, ex, tw, xf, xi, t, c);
    {
      const double pin = r2c::flux<N, C, NT>(v, it.w_in, s_red, &s_part, t, c, cl);
      if (c == 0 && t == 0) it.energy[2 * iters] = pin;
    }
    const int sweeps = it.iterations > 0 ? 2 * it.iterations : 1;
    R2Next nx;
    nx.st = it.steps[0];
    r2_next_passes(nx, it, false);
    for (int sw = 0; sw < sweeps; ++sw) {
      const bool backward = sw & 1;
      const int iter = sw >> 1;
      if (!backward) {
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = it.input[r2c::qreal<N, C, NT>(j, t, c)];
      } else {
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = cf{0.f, 0.f};
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
        r2c::step<N, C, NT, RADS, G>(v, Sl, out, b0, b1, phase, ex, it, st, p0, p1, nx, next_p,
                                  next_backward, backward, reflect, store, add, mk, tw, xf, xi, t,
                                  c);
      }
      cf* dst = backward ? it.reflected : it.transmitted;
#pragma unroll
      for (int j = 0; j < E; ++j) dst[r2c::qreal<N, C, NT>(j, t, c)] = v[j];
      if (it.iterations == 0) break;
#pragma unroll
      for (int j = 0; j < E; ++j) out[j] = v[j];
      r2c::forward<N, C, NT, RADS>(out, b0, b1, phase, ex, tw, xf, xi, t, c);
      const double fl = r2c::flux<N, C, NT>(out, backward ? it.w_in : it.w_out, s_red, &s_part, t, c, cl);
      if (c == 0 && t == 0) it.energy[2 * iter + (backward ? 1 : 0)] = fl;
    }
    cl.sync();  // the whole cluster is done with the item
    if (c == 0 && t == 0) it.clock[1] = global_ns();
  }
}

}  // namespace bwpm
