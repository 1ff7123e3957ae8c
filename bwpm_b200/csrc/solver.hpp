// Host interface of the plane engine (the CudaSolver behind the C ABI).
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

#include "common.cuh"

namespace bwpm {

// Constructor arguments of the reference's bwpm._core.CudaSolver
// (cpp/include/bwpm/solver_cuda.hpp:20-35, cpp/python/bindings.cpp:159-173).
struct SolverInput {
  std::size_t ny = 0, nx = 0;
  double dy = 0, dx = 0, dz = 0, k0 = 0;
  std::vector<cd> indices;
  std::vector<std::int32_t> labels;  // (nz, ny, nx)
  // or, when set, the caller's labels read in place during set-up (nz·ny·nx values, valid until
  // the solver has been constructed; `labels` is then empty)
  const std::int32_t* labels_view = nullptr;
  // or, when set, uint8 labels in device memory (nz·ny·nx values on `device`, e.g. generated
  // there from a geometry), read during set-up only; at most 255 materials, no fluctuation
  const std::uint8_t* labels_device = nullptr;
  // or, when geometry_kind ≥ 0, labels generated on the device from that geometry during
  // set-up (see generate_labels): kGeometryParams values in geometry_params
  int geometry_kind = -1;
  std::vector<double> geometry_params;
  std::size_t nz = 0;
  cd index_before{1.0, 0.0};
  std::vector<double> mask;          // (ny, nx) or empty
  std::vector<cd> fluct;             // δn (nz, ny, nx) or empty
  int device = 0;
  double gmres_tol = 1e-12;          // cpp/src/solver.cpp:209
};

// Outputs of one run, caller-owned complex128 buffers of ny·nx·2 values each (may be null).
struct RunOutputs {
  cd* transmitted = nullptr;
  cd* reflected = nullptr;
  cd* transmitted_iter = nullptr;  // iterations planes
  cd* reflected_iter = nullptr;
  cd* forward = nullptr;           // nkeep planes, in keep order
  cd* backward = nullptr;          // nkeep planes (iterations > 0)
  std::int64_t stored_values = 0;
};

class Solver {
 public:
  virtual ~Solver() = default;
  // keep: sorted unique plane numbers ≤ nz.
  virtual void run(const cd* field, int iterations, const std::int64_t* keep, std::size_t nkeep,
                   RunOutputs& out) = 0;
  virtual std::size_t device_bytes() const = 0;
  virtual std::int64_t kernel_launches() const = 0;
  virtual std::int64_t gmres_applies() const = 0;
};

// precision: 64 (complex128 fields, the drop-in path) or 32 (complex64 fields, FP64 tables).
std::unique_ptr<Solver> make_plane_solver(SolverInput in, int precision);

// Geometry of a label volume generated on the device (geometry.cuh): kind (0 tilted facet,
// 1 lens array, 2 microlens, 3 tilted slab) and kGeometryParams parameters
// (base, tan_tilt, pitch, sag, radius, vertex, back).
constexpr std::size_t kGeometryParams = 7;
struct GeometrySpec;
GeometrySpec geometry_spec(int kind, const double* params, std::size_t nparams, std::size_t nz,
                           std::size_t ny, std::size_t nx, double dz, double dy, double dx);
// materials a geometry labels (labels 0 … n − 1)
int geometry_materials(int kind);
// uint8 labels (nz, ny, nx) into device memory `out`, on `stream`
void generate_labels(const GeometrySpec& g, std::uint8_t* out, cudaStream_t stream);

// Interface matrices on the device for n points (kind 0: T, 1: R), out (n, 2, 2) complex128.
void interface_matrices(int reflection, const double* kx, const double* ky, std::size_t n, cd n_in,
                        cd n_out, double k0, cd* out);
void longitudinal_wavenumbers(cd index, double k0, const double* kp2, std::size_t n, cd* out);
int device_count();

}  // namespace bwpm
