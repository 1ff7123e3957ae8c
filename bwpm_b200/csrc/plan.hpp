// Host-side FFT planning: factorisation into radices, thread requirement and FP64 twiddles.
#pragma once

#include <cmath>
#include <string>
#include <vector>

#include "fft.cuh"

namespace bwpm {

struct HostPlan {
  FftPlan plan;
  std::vector<cd> twiddles;  // FP64, forward sign; rounded to the kernel's type on upload
};

// Radices for n: powers of two as 8s with a 4/4·4/2 remainder, then 3s, 5s, 7s and other odd
// primes up to kMaxGenericRadix. Throws invalid_argument for larger prime factors.
inline std::vector<int> factorize(int n) {
  if (n < 1) throw invalid_argument("FFT length must be positive");
  std::vector<int> r;
  int m = n, twos = 0;
  while (m % 2 == 0) {
    m /= 2;
    ++twos;
  }
  std::vector<int> p2;
  if (twos % 3 == 1 && twos >= 4) {
    for (int i = 0; i < (twos - 4) / 3; ++i) p2.push_back(8);
    p2.push_back(4);
    p2.push_back(4);
  } else {
    for (int i = 0; i < twos / 3; ++i) p2.push_back(8);
    if (twos % 3 == 2) p2.push_back(4);
    if (twos % 3 == 1) p2.push_back(2);
  }
  for (int p : {3, 5, 7})
    while (m % p == 0) {
      r.push_back(p);
      m /= p;
    }
  for (int p = 11; m > 1 && p <= kMaxGenericRadix; p += 2)
    while (m % p == 0) {
      r.push_back(p);
      m /= p;
    }
  if (m > 1)
    throw invalid_argument("FFT length " + std::to_string(n) + " has a prime factor above " +
                           std::to_string(kMaxGenericRadix));
  r.insert(r.end(), p2.begin(), p2.end());
  if (static_cast<int>(r.size()) > kMaxStages) throw invalid_argument("FFT length has too many factors");
  return r;
}

inline HostPlan make_plan_radices(int n, const std::vector<int>& radices);

inline HostPlan make_plan(int n) { return make_plan_radices(n, n > 1 ? factorize(n) : std::vector<int>{}); }

// Plan with a given radix order (the product must be n).
inline HostPlan make_plan_radices(int n, const std::vector<int>& radices) {
  HostPlan hp;
  FftPlan& p = hp.plan;
  p.n = n;
  long long prod = 1;
  for (int r : radices) prod *= r;
  if (prod != n || static_cast<int>(radices.size()) > kMaxStages)
    throw invalid_argument("radices do not factor the FFT length");
  p.nstages = static_cast<int>(radices.size());
  int len = 1, off = 0;
  const double two_pi = 6.283185307179586476925286766559;
  for (int s = 0; s < p.nstages; ++s) {
    const int r = radices[s];
    p.radix[s] = r;
    p.len[s] = len;
    p.twoff[s] = off;
    const long long lr = static_cast<long long>(len) * r;
    for (int j = 1; j < r; ++j)  // r-major: entry (j − 1)·L + k
      for (int k = 0; k < len; ++k) {
        const long long m = (static_cast<long long>(j) * k) % lr;
        const double a = -two_pi * static_cast<double>(m) / static_cast<double>(lr);
        hp.twiddles.push_back(cd{std::cos(a), std::sin(a)});
      }
    off += len * (r - 1);
    len *= r;
  }
  p.rootoff = off;
  bool generic = false;
  for (int s = 0; s < p.nstages; ++s) generic |= p.radix[s] > 8;
  if (generic)
    for (int m = 0; m < n; ++m) {
      const double a = -two_pi * static_cast<double>(m) / static_cast<double>(n);
      hp.twiddles.push_back(cd{std::cos(a), std::sin(a)});
    }
  if (hp.twiddles.empty()) hp.twiddles.push_back(cd{1.0, 0.0});
  p.ntw = static_cast<int>(hp.twiddles.size());
  return hp;
}

// Threads needed so that every stage fits its register staging of EPT values per thread
// (multiple of 32).
inline int threads_needed(const FftPlan& p, int batch, int ept = 16) {
  long long need = 32;
  for (int s = 0; s < p.nstages; ++s) {
    const int r = p.radix[s];
    const long long total = static_cast<long long>(p.n / r) * batch;
    const long long k = kmax_for(r, ept);
    const long long t = (total + k - 1) / k;
    need = std::max(need, t);
  }
  return static_cast<int>((need + 31) / 32 * 32);
}

// Twiddles in the kernel's storage: FP64 values, or FP32 (hi, lo) pairs rounded from FP64.
template <typename T>
inline std::vector<Tw<T>> twiddles_for(const HostPlan& hp) {
  std::vector<Tw<T>> out(hp.twiddles.size());
  for (std::size_t i = 0; i < out.size(); ++i) {
    const cd w = hp.twiddles[i];
    if constexpr (sizeof(T) == sizeof(double)) {
      out[i].hi = cx<T>{static_cast<T>(w.re), static_cast<T>(w.im)};
    } else {
      const cf h{static_cast<float>(w.re), static_cast<float>(w.im)};
      out[i].hi = h;
      out[i].lo = cf{static_cast<float>(w.re - h.re), static_cast<float>(w.im - h.im)};
    }
  }
  return out;
}

}  // namespace bwpm
