// Material labels generated on the device from a geometry, at the pixel centres.
//
// The rule is the reference's labels_at_centres (src/bwpm/geometry.py:24-37): slab j covers
// z ∈ [j·dz, (j + 1)·dz] and takes the material at its centre z_j = (j + 0.5)·dz; the lateral
// grid is centred, y_i = (i − ny//2)·dy, x_k = (k − nx//2)·dx. The bodies are the seeded
// geometry families of the workloads (bwpm_b200/workloads.py), evaluated with the same FP64
// operations in the same order as the host generators there, so that the labels are identical:
// - kTiltedFacet: label 1 where z ≥ base + tan(tilt)·y (a fibre facet tilted about x);
// - kLensArray: label 1 where z ≥ base − h(x, y), h the height of a square array of spherical
//   caps (pitch, sag, radius) over the substrate at `base`, clipped at 0;
// - kMicrolens: label 1 where z ≥ the sag of one spherical cap (vertex, radius), label 2 where
//   z ≥ back + tan(tilt)·y (a tilted back face), else 0;
// - kTiltedSlab: label 1 where front + tan(tilt)·y ≤ z < back, else 0.
// Labels are uint8, (nz, ny, nx) row-major, written straight into device memory (no host copy
// of the volume).
#pragma once

#include <cstdint>

#include "common.cuh"

namespace bwpm {

enum GeometryKind : int { kTiltedFacet = 0, kLensArray = 1, kMicrolens = 2, kTiltedSlab = 3 };

struct GeometrySpec {
  int kind = kTiltedFacet;
  int nz = 1, ny = 1, nx = 1;
  double dz = 1.0, dy = 1.0, dx = 1.0;
  double base = 0.0;    // facet / lens array substrate / slab front (z, mm)
  double tan_tilt = 0;  // facet, slab front and microlens back face slope
  double pitch = 0, sag = 0, radius = 0;  // lens array (radius = (half² + sag²)/(2·sag))
  double vertex = 0;    // microlens: vertex z of the cap
  double back = 0;      // microlens back face z at y = 0; slab back face z
};

__device__ __forceinline__ double centred(int i, int n, double d) {
  return static_cast<double>(i - n / 2) * d;
}

// Python's float modulo (numpy.remainder): fmod with the sign of the divisor.
__device__ __forceinline__ double py_mod(double a, double b) {
  double r = fmod(a, b);
  if (r != 0.0 && ((b < 0.0) != (r < 0.0))) r += b;
  return r;
}

__device__ __forceinline__ std::uint8_t geometry_label(const GeometrySpec& g, int j, int i, int k) {
  const double z = (static_cast<double>(j) + 0.5) * g.dz;
  const double y = centred(i, g.ny, g.dy);
  switch (g.kind) {
    case kTiltedFacet:
      return z >= g.base + g.tan_tilt * y ? 1 : 0;
    case kLensArray: {
      const double half = g.pitch / 2;
      const double ly = py_mod(y + half, g.pitch) - half;
      double r2 = 0.0 + ly * ly;
      if (g.nx > 1) {
        const double lx = py_mod(centred(k, g.nx, g.dx) + half, g.pitch) - half;
        r2 = r2 + lx * lx;
      }
      double h = sqrt(fmax(g.radius * g.radius - r2, 0.0)) - (g.radius - g.sag);
      h = fmax(h, 0.0);
      return z >= g.base - h ? 1 : 0;
    }
    case kMicrolens: {
      const double x = centred(k, g.nx, g.dx);
      const double r2 = x * x + y * y;
      const double rr = g.radius * g.radius;
      std::uint8_t lab = 0;
      if (r2 < rr && z >= g.vertex + g.radius - sqrt(fmax(rr - r2, 0.0))) lab = 1;
      if (z >= g.back + g.tan_tilt * y) lab = 2;
      return lab;
    }
    default: {  // kTiltedSlab
      const double front = g.base + g.tan_tilt * y;
      return (z >= front && z < g.back) ? 1 : 0;
    }
  }
}

}  // namespace bwpm
