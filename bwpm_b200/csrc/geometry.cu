// Label volumes generated on the device from a geometry (see geometry.cuh).
#include <algorithm>
#include <string>

#include "devbuf.hpp"
#include "geometry.cuh"
#include "solver.hpp"

namespace bwpm {

namespace {
__global__ void k_geometry_labels(GeometrySpec g, std::uint8_t* out) {
  const long long plane = static_cast<long long>(g.ny) * g.nx;
  const long long total = plane * g.nz;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(idx / plane);
    const long long q = idx - j * plane;
    const int i = static_cast<int>(q / g.nx), k = static_cast<int>(q - static_cast<long long>(i) * g.nx);
    out[idx] = geometry_label(g, j, i, k);
  }
}

}  // namespace

GeometrySpec geometry_spec(int kind, const double* params, std::size_t nparams, std::size_t nz,
                           std::size_t ny, std::size_t nx, double dz, double dy, double dx) {
  if (kind < kTiltedFacet || kind > kTiltedSlab) throw invalid_argument("unknown geometry kind");
  if (!params || nparams < kGeometryParams)
    throw invalid_argument("geometry takes " + std::to_string(kGeometryParams) + " parameters");
  if (nz < 1 || ny < 1 || nx < 1 || nz > 65535 || ny > (1u << 20) || nx > (1u << 20))
    throw invalid_argument("nz, ny, nx out of range");
  if (!(dz > 0.0) || !(dy > 0.0) || !(dx > 0.0)) throw invalid_argument("steps must be positive");
  GeometrySpec g;
  g.kind = kind;
  g.nz = static_cast<int>(nz);
  g.ny = static_cast<int>(ny);
  g.nx = static_cast<int>(nx);
  g.dz = dz;
  g.dy = dy;
  g.dx = dx;
  g.base = params[0];
  g.tan_tilt = params[1];
  g.pitch = params[2];
  g.sag = params[3];
  g.radius = params[4];
  g.vertex = params[5];
  g.back = params[6];
  if (kind == kLensArray && !(g.pitch > 0.0)) throw invalid_argument("pitch must be positive");
  return g;
}

int geometry_materials(int kind) { return kind == kMicrolens ? 3 : 2; }

void generate_labels(const GeometrySpec& g, std::uint8_t* out, cudaStream_t stream) {
  const long long total = static_cast<long long>(g.nz) * g.ny * g.nx;
  const int blocks = static_cast<int>(std::min<long long>(ceil_div(total, 256), 148LL * 16));
  k_geometry_labels<<<blocks, 256, 0, stream>>>(g, out);
  check_cuda(cudaGetLastError(), "k_geometry_labels");
}

}  // namespace bwpm
