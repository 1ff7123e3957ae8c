// Interface formulas in FP64 on the device: k_z with the grazing rule, Fresnel coefficients in
// Convention A, the 2×2 transmission/reflection matrices and the table-1 propagation factors.
//
// They restate cpp/src/interface.cpp:8-52 (same operations in the same order, so the grazing
// rule sees the same rounding) and the kind/phase selection of cpp/src/solver.cpp:73-106.
// Used once per solve to build operator tables; never on the per-slab hot path.
#pragma once

#include "common.cuh"

namespace bwpm {

constexpr double kGrazingTolerance = 1e-12;  // cpp/include/bwpm/interface.hpp:17

enum Kind : int { kFwdT = 0, kFwdR = 1, kBwdT = 2, kBwdR = 3 };

// 2π·numpy.fft.fftfreq(n, d)[i] with the rounding 2π·(m·(1/(n·d))) (cpp/src/solver.cpp:17-24).
__host__ __device__ __forceinline__ double fftfreq(long long i, long long n, double d) {
  const long long m = i - (i < (n + 1) / 2 ? 0LL : n);
  const double val = 1.0 / (static_cast<double>(n) * d);
  return 2.0 * 3.141592653589793 * (static_cast<double>(m) * val);
}

// k_z = sqrt(ñ²k₀² − k⊥²), Im ≥ 0 (Re ≥ 0 if Im = 0); grazing rule (cpp/src/interface.cpp:8-18).
__device__ __forceinline__ cd kz_of(cd index, double k0, double kp2) {
  const cd n2k2 = (index * index) * (k0 * k0);
  cd q{n2k2.re - kp2, n2k2.im};
  if (cabs(q) <= kGrazingTolerance * cabs(n2k2)) q = {0.0, 0.0};
  cd kz = csqrt(q);
  if (kz.im < 0.0 || (kz.im == 0.0 && kz.re < 0.0)) kz = -kz;
  const double tiny = 1e-12 * k0;
  if (cabs(kz) < tiny) kz = {0.0, tiny};
  return kz;
}

struct Fresnel {
  cd r_s, r_p, t_s, t_p, kz_in, kz_out;
};

// Convention A with q_j = k_z,j/k₀ (cpp/src/interface.cpp:20-28).
__device__ __forceinline__ Fresnel fresnel(double kx, double ky, cd n1, cd n2, double k0) {
  const double kp2 = kx * kx + ky * ky;
  const cd kz1 = kz_of(n1, k0, kp2);
  const cd kz2 = kz_of(n2, k0, kp2);
  const cd q1 = kz1 / k0, q2 = kz2 / k0;
  const cd den_p = (n2 * n2) * q1 + (n1 * n1) * q2;
  Fresnel f;
  f.r_s = cdiv(q1 - q2, q1 + q2);
  f.r_p = cdiv((n2 * n2) * q1 - (n1 * n1) * q2, den_p);
  f.t_s = cdiv(2.0 * q1, q1 + q2);
  f.t_p = cdiv((2.0 * n1) * n2 * q1, den_p);
  f.kz_in = kz1;
  f.kz_out = kz2;
  return f;
}

// T (reflection = false, cpp/src/interface.cpp:30-40) or R (cpp/src/interface.cpp:42-52) as
// the symmetric triple (m00, m01 = m10, m11); k⊥ = 0 gives t_s·I or r_s·I.
__device__ __forceinline__ void interface_matrix(bool reflection, double kx, double ky, cd n1,
                                                 cd n2, double k0, cd m[3]) {
  const Fresnel c = fresnel(kx, ky, n1, n2, k0);
  const double kp2 = kx * kx + ky * ky;
  if (kp2 == 0.0) {
    const cd d = reflection ? c.r_s : c.t_s;
    m[0] = d;
    m[1] = {0.0, 0.0};
    m[2] = d;
    return;
  }
  if (!reflection) {
    const cd kr = n1 * k0, ks = n2 * k0;
    const cd gamma = c.kz_in * c.kz_out + cdiv(c.kz_out * kp2, c.kz_in);
    const cd scale = cdiv(cd{1.0, 0.0}, (kp2 * kr) * ks);
    m[1] = ((c.t_p * gamma - (c.t_s * kr) * ks) * kx) * ky * scale;
    m[0] = ((c.t_p * kx) * kx * gamma + ((c.t_s * ky) * ky * kr) * ks) * scale;
    m[2] = ((c.t_p * ky) * ky * gamma + ((c.t_s * kx) * kx * kr) * ks) * scale;
  } else {
    const cd kr = n1 * k0;
    const cd gamma = c.kz_in * c.kz_in + cd{kp2, 0.0};
    const cd scale = cdiv(cd{1.0, 0.0}, (kp2 * kr) * kr);
    m[1] = -(((c.r_p * gamma + (c.r_s * kr) * kr) * kx) * ky) * scale;
    m[0] = ((-c.r_p * kx) * kx * gamma + ((c.r_s * ky) * ky * kr) * kr) * scale;
    m[2] = ((-c.r_p * ky) * ky * gamma + ((c.r_s * kx) * kx * kr) * kr) * scale;
  }
}

// Operator of table 1 (wende2023): FwdT T·e^{i k_z,s dz}, FwdR R, BwdT T·e^{i k_z,r dz},
// BwdR R·e^{2i k_z,r dz} (cpp/src/solver.cpp:87-103).
__device__ __forceinline__ void operator_matrix(int kind, double kx, double ky, cd nr, cd ns,
                                                double k0, double dz, cd m[3]) {
  const bool refl = (kind == kFwdR || kind == kBwdR);
  interface_matrix(refl, kx, ky, nr, ns, k0, m);
  const double kp2 = kx * kx + ky * ky;
  cd phase{1.0, 0.0};
  const cd im{0.0, 1.0};
  if (kind == kFwdT) phase = cexp(im * kz_of(ns, k0, kp2) * dz);
  if (kind == kBwdT) phase = cexp(im * kz_of(nr, k0, kp2) * dz);
  if (kind == kBwdR) phase = cexp((2.0 * im) * kz_of(nr, k0, kp2) * dz);
  for (int j = 0; j < 3; ++j) m[j] = m[j] * phase;
}

// Propagating and non-grazing in the host medium (cpp/src/solver.cpp:233; src/bwpm/fluctuation.py:51-59).
__device__ __forceinline__ bool born_propagating(cd host2k2, double kp2) {
  const double kabs2 = cabs(host2k2);
  return kp2 < kabs2 && cabs(cd{host2k2.re - kp2, host2k2.im}) > kGrazingTolerance * kabs2;
}

}  // namespace bwpm
