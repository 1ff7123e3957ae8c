// Post-processing of transverse fields on the device (see postproc.cu).
#pragma once

#include <cstddef>

#include "common.cuh"

namespace bwpm {

struct PlaneGeometry {
  int ny = 1, nx = 1;
  double dy = 1.0, dx = 1.0, k0 = 1.0;
};

// Unnormalised forward FP64 2D FFT of a device field (ny, nx, 2); tmp: a scratch plane (nx > 1).
void field_spectrum(const cd* field, cd* out, cd* tmp, int ny, int nx, cudaStream_t stream);

// `field`: (ny, nx, 2) complex128, host memory unless on_device.
double port_power(const PlaneGeometry& g, const cd* field, bool on_device, cd index, int direction,
                  cudaStream_t stream);
double plane_power(const PlaneGeometry& g, const cd* field, bool on_device, double index,
                   cudaStream_t stream);
void axial_focus(const PlaneGeometry& g, const cd* field, bool on_device, double index,
                 const double* offsets, std::size_t noff, double na, double* best, double* peak,
                 double* intensity_out, cudaStream_t stream);

}  // namespace bwpm
