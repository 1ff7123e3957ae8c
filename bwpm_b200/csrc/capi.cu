// extern "C" entry points of libbwpm_b200.so (declared in include/bwpm_b200.h).
#include <cstring>
#include <exception>
#include <memory>
#include <string>

#include "../../include/bwpm_b200.h"
#include "batch2d.hpp"
#include "devbuf.hpp"
#include "geometry.cuh"
#include "noalloc.hpp"
#include "postproc.hpp"
#include "server.hpp"
#include "solver.hpp"
#include "variants.hpp"

struct bwpm_solver {
  std::unique_ptr<bwpm::Solver> impl;
};

struct bwpm_batch {
  std::unique_ptr<bwpm::Batch2D> impl;
};

struct bwpm_server {
  std::unique_ptr<bwpm::Server> impl;
};

namespace {

thread_local std::string g_last_error;

template <class F>
int guarded(F&& f) {
  try {
    f();
    return BWPM_OK;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return BWPM_EINVAL;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return BWPM_ERUNTIME;
  } catch (...) {
    g_last_error = "unknown error";
    return BWPM_ERUNTIME;
  }
}

const bwpm::cd* as_cd(const double* p) { return reinterpret_cast<const bwpm::cd*>(p); }

// a stream of the call's own on `device`
struct CallStream {
  bwpm::OwnedStream s;
  explicit CallStream(int device) {
    bwpm::check_cuda(cudaSetDevice(device), "cudaSetDevice");
    s.create();
  }
};
bwpm::cd* as_cd(double* p) { return reinterpret_cast<bwpm::cd*>(p); }

}  // namespace

namespace {
// borrow: the labels stay caller-owned and are copied by a preparation worker of the server
int server_submit_2d(bwpm_server* s, size_t ny, double dy, double dz, double k0,
                     const double* indices, size_t m, const int32_t* labels, size_t nz,
                     double ib_re, double ib_im, const double* mask, const double* field,
                     int iterations, int64_t* ticket, bool borrow) {
  return guarded([&] {
    if (!s || !s->impl) throw bwpm::invalid_argument("null server");
    if (!indices || !labels || !field) throw bwpm::invalid_argument("null array");
    bwpm::Solve2D p;
    p.ny = static_cast<int>(ny);
    p.nz = static_cast<int>(nz);
    p.dy = dy;
    p.dz = dz;
    p.k0 = k0;
    p.indices.assign(as_cd(indices), as_cd(indices) + m);
    if (!borrow) p.labels.assign(labels, labels + nz * ny);
    p.index_before = bwpm::cd{ib_re, ib_im};
    if (mask) p.mask.assign(mask, mask + ny);
    p.field.assign(as_cd(field), as_cd(field) + 2 * ny);
    p.iterations = iterations;
    const int64_t k = s->impl->submit2d(std::move(p), borrow ? labels : nullptr);
    if (ticket) *ticket = k;
  });
}

int server_submit_3d(bwpm_server* s, size_t ny, size_t nx, double dy, double dx, double dz,
                     double k0, const double* indices, size_t m, const int32_t* labels,
                     size_t nz, double ib_re, double ib_im, const double* mask,
                     const double* field, int iterations, int64_t* ticket, bool borrow) {
  return guarded([&] {
    if (!s || !s->impl) throw bwpm::invalid_argument("null server");
    if (!indices || !labels || !field) throw bwpm::invalid_argument("null array");
    bwpm::SolverInput in;
    in.ny = ny;
    in.nx = nx;
    in.dy = dy;
    in.dx = dx;
    in.dz = dz;
    in.k0 = k0;
    in.indices.assign(as_cd(indices), as_cd(indices) + m);
    if (!borrow) in.labels.assign(labels, labels + nz * ny * nx);
    in.nz = nz;
    in.index_before = bwpm::cd{ib_re, ib_im};
    if (mask) in.mask.assign(mask, mask + ny * nx);
    std::vector<bwpm::cd> f(as_cd(field), as_cd(field) + 2 * ny * nx);
    const int64_t k = s->impl->submit3d(std::move(in), std::move(f), iterations, borrow ? labels : nullptr);
    if (ticket) *ticket = k;
  });
}
}  // namespace

extern "C" {

size_t bwpm_last_error(char* buf, size_t len) {
  if (buf && len) {
    const size_t k = std::min(len - 1, g_last_error.size());
    std::memcpy(buf, g_last_error.data(), k);
    buf[k] = '\0';
  }
  return g_last_error.size();
}

const char* bwpm_version(void) { return "bwpm_b200 0.1 sm_100a"; }

int bwpm_cuda_device_count(void) { return bwpm::device_count(); }

int bwpm_interface_matrices(int reflection, const double* k_x, const double* k_y, size_t n,
                            double in_re, double in_im, double out_re, double out_im, double k0,
                            double* out) {
  return guarded([&] {
    if (n && (!k_x || !k_y || !out)) throw bwpm::invalid_argument("null array");
    bwpm::interface_matrices(reflection, k_x, k_y, n, bwpm::cd{in_re, in_im},
                             bwpm::cd{out_re, out_im}, k0, as_cd(out));
  });
}

int bwpm_longitudinal_wavenumber(double index_re, double index_im, double k0,
                                 const double* k_perp_sq, size_t n, double* out) {
  return guarded([&] {
    if (n && (!k_perp_sq || !out)) throw bwpm::invalid_argument("null array");
    bwpm::longitudinal_wavenumbers(bwpm::cd{index_re, index_im}, k0, k_perp_sq, n, as_cd(out));
  });
}

int bwpm_solver_create(size_t ny, size_t nx, double dy, double dx, double dz, double k0,
                       const double* indices, size_t m, const int32_t* labels, size_t nz,
                       double ib_re, double ib_im, const double* mask, int device,
                       const double* fluctuation, int precision, double gmres_tol,
                       bwpm_solver** out) {
  return guarded([&] {
    if (!out) throw bwpm::invalid_argument("null output handle");
    *out = nullptr;
    bwpm::SolverInput in;
    in.ny = ny;
    in.nx = nx;
    in.dy = dy;
    in.dx = dx;
    in.dz = dz;
    in.k0 = k0;
    in.indices.assign(as_cd(indices), as_cd(indices) + m);
    in.labels.assign(labels, labels + nz * ny * nx);
    in.nz = nz;
    in.index_before = bwpm::cd{ib_re, ib_im};
    if (mask) in.mask.assign(mask, mask + ny * nx);
    if (fluctuation) in.fluct.assign(as_cd(fluctuation), as_cd(fluctuation) + nz * ny * nx);
    in.device = device;
    in.gmres_tol = gmres_tol;
    auto s = std::make_unique<bwpm_solver>();
    s->impl = bwpm::make_plane_solver(std::move(in), precision);
    *out = s.release();
  });
}

int bwpm_solver_create_geometry(size_t ny, size_t nx, double dy, double dx, double dz, double k0,
                                const double* indices, size_t m, int kind, const double* params,
                                size_t nparams, size_t nz, double ib_re, double ib_im,
                                const double* mask, int device, int precision, bwpm_solver** out) {
  return guarded([&] {
    if (!out) throw bwpm::invalid_argument("null output handle");
    *out = nullptr;
    if (!indices || !params) throw bwpm::invalid_argument("null array");
    bwpm::SolverInput in;
    in.ny = ny;
    in.nx = nx;
    in.dy = dy;
    in.dx = dx;
    in.dz = dz;
    in.k0 = k0;
    in.indices.assign(as_cd(indices), as_cd(indices) + m);
    in.geometry_kind = kind;
    in.geometry_params.assign(params, params + nparams);
    in.nz = nz;
    in.index_before = bwpm::cd{ib_re, ib_im};
    if (mask) in.mask.assign(mask, mask + ny * nx);
    in.device = device;
    auto s = std::make_unique<bwpm_solver>();
    s->impl = bwpm::make_plane_solver(std::move(in), precision);
    *out = s.release();
  });
}

int bwpm_geometry_labels(int device, int kind, const double* params, size_t nparams, size_t nz,
                         size_t ny, size_t nx, double dz, double dy, double dx, uint8_t* labels) {
  return guarded([&] {
    if (!labels) throw bwpm::invalid_argument("null array");
    const bwpm::GeometrySpec g = bwpm::geometry_spec(kind, params, nparams, nz, ny, nx, dz, dy, dx);
    CallStream cs(device);
    bwpm::DevBuf<uint8_t> d(nz * ny * nx, cs.s);
    bwpm::generate_labels(g, d.ptr, cs.s);
    bwpm::check_cuda(cudaMemcpyAsync(labels, d.ptr, d.bytes(), cudaMemcpyDeviceToHost, cs.s), "download");
    bwpm::check_cuda(cudaStreamSynchronize(cs.s), "synchronize");
  });
}

int bwpm_solver_run(bwpm_solver* s, const double* field, int iterations, const int64_t* keep,
                    size_t nkeep, double* transmitted, double* reflected, double* t_iter,
                    double* r_iter, double* forward, double* backward, int64_t* stored_values) {
  return guarded([&] {
    if (!s || !s->impl) throw bwpm::invalid_argument("null solver");
    if (!field) throw bwpm::invalid_argument("field must have shape (ny, nx, 2)");
    if (iterations < 0) throw bwpm::invalid_argument("iterations must be >= 0");
    bwpm::RunOutputs o;
    o.transmitted = as_cd(transmitted);
    o.reflected = as_cd(reflected);
    o.transmitted_iter = as_cd(t_iter);
    o.reflected_iter = as_cd(r_iter);
    o.forward = as_cd(forward);
    o.backward = as_cd(backward);
    s->impl->run(as_cd(field), iterations, keep, nkeep, o);
    if (stored_values) *stored_values = o.stored_values;
  });
}

int bwpm_solver_stats(const bwpm_solver* s, int64_t* device_bytes, int64_t* kernel_launches,
                      int64_t* gmres_applies) {
  return guarded([&] {
    if (!s || !s->impl) throw bwpm::invalid_argument("null solver");
    if (device_bytes) *device_bytes = static_cast<int64_t>(s->impl->device_bytes());
    if (kernel_launches) *kernel_launches = s->impl->kernel_launches();
    if (gmres_applies) *gmres_applies = s->impl->gmres_applies();
  });
}

void bwpm_solver_destroy(bwpm_solver* s) { delete s; }

int bwpm_batch_create(int device, bwpm_batch** out) {
  return guarded([&] {
    if (!out) throw bwpm::invalid_argument("null output handle");
    auto b = std::make_unique<bwpm_batch>();
    b->impl = bwpm::make_batch2d(device);
    *out = b.release();
  });
}

int bwpm_batch_add(bwpm_batch* b, size_t ny, double dy, double dz, double k0,
                   const double* indices, size_t m, const int32_t* labels, size_t nz,
                   double ib_re, double ib_im, const double* mask, const double* field,
                   int iterations, int64_t* id) {
  return guarded([&] {
    if (!b || !b->impl) throw bwpm::invalid_argument("null batch");
    if (!indices || !labels || !field) throw bwpm::invalid_argument("null array");
    bwpm::Solve2D s;
    s.ny = static_cast<int>(ny);
    s.nz = static_cast<int>(nz);
    s.dy = dy;
    s.dz = dz;
    s.k0 = k0;
    s.indices.assign(as_cd(indices), as_cd(indices) + m);
    s.labels.assign(labels, labels + nz * ny);
    s.index_before = bwpm::cd{ib_re, ib_im};
    if (mask) s.mask.assign(mask, mask + ny);
    s.field.assign(as_cd(field), as_cd(field) + 2 * ny);
    s.iterations = iterations;
    const int64_t k = b->impl->add(std::move(s));
    if (id) *id = k;
  });
}

int bwpm_batch_set_autotune(bwpm_batch* b, int on) {
  return guarded([&] {
    if (!b || !b->impl) throw bwpm::invalid_argument("null batch");
    b->impl->set_autotune(on != 0);
  });
}

int bwpm_batch_set_variant(bwpm_batch* b, size_t ny, int variant) {
  return guarded([&] {
    if (!b || !b->impl) throw bwpm::invalid_argument("null batch");
    b->impl->set_variant(static_cast<int>(ny), variant);
  });
}

int bwpm_batch_class_info(const bwpm_batch* b, int64_t k, int64_t* ny, int64_t* threads,
                          int64_t* cluster, int64_t* variant, int64_t* items, float* tuned_ms) {
  return guarded([&] {
    if (!b || !b->impl) throw bwpm::invalid_argument("null batch");
    int n = 0, t = 0, c = 0, v = 0;
    float ms = 0;
    const int count = b->impl->class_info(static_cast<int>(k), n, t, c, v, ms);
    if (ny) *ny = n;
    if (threads) *threads = t;
    if (cluster) *cluster = c;
    if (variant) *variant = v;
    if (items) *items = count;
    if (tuned_ms) *tuned_ms = ms;
  });
}

int bwpm_variant_count(size_t ny) {
  int k = 0;
  for (const auto& v : bwpm::fixed_variants()) k += v.n == static_cast<int>(ny);
  return k;
}

int bwpm_batch_prepare(bwpm_batch* b) {
  return guarded([&] {
    if (!b || !b->impl) throw bwpm::invalid_argument("null batch");
    b->impl->prepare();
  });
}

int bwpm_batch_run(bwpm_batch* b, float* device_ms) {
  return guarded([&] {
    if (!b || !b->impl) throw bwpm::invalid_argument("null batch");
    const float ms = b->impl->run();
    if (device_ms) *device_ms = ms;
  });
}

int bwpm_batch_solve_packed(bwpm_batch* b, const double* fields, double* out, float* device_ms) {
  return guarded([&] {
    if (!b || !b->impl) throw bwpm::invalid_argument("null batch");
    if (!fields || !out) throw bwpm::invalid_argument("null array");
    const float ms = b->impl->solve_packed(as_cd(fields), as_cd(out));
    if (device_ms) *device_ms = ms;
  });
}

int bwpm_batch_result(bwpm_batch* b, int64_t id, double* transmitted, double* reflected,
                      double* flux_t, double* flux_r, double* flux_in, double* latency_ms) {
  return guarded([&] {
    if (!b || !b->impl) throw bwpm::invalid_argument("null batch");
    bwpm::Solve2DResult r;
    b->impl->result(id, r);
    if (transmitted) std::memcpy(transmitted, r.transmitted.data(), r.transmitted.size() * sizeof(bwpm::cd));
    if (reflected) std::memcpy(reflected, r.reflected.data(), r.reflected.size() * sizeof(bwpm::cd));
    if (flux_t) std::memcpy(flux_t, r.flux_t.data(), r.flux_t.size() * sizeof(double));
    if (flux_r) std::memcpy(flux_r, r.flux_r.data(), r.flux_r.size() * sizeof(double));
    if (flux_in) *flux_in = r.flux_in;
    if (latency_ms) *latency_ms = r.latency_ms;
  });
}

int bwpm_batch_stats(const bwpm_batch* b, int64_t* device_bytes, int64_t* kernel_launches,
                     int64_t* work_items, int64_t* classes, int64_t* packed_inputs) {
  return guarded([&] {
    if (!b || !b->impl) throw bwpm::invalid_argument("null batch");
    if (device_bytes) *device_bytes = static_cast<int64_t>(b->impl->device_bytes());
    if (kernel_launches) *kernel_launches = b->impl->kernel_launches();
    if (work_items) *work_items = b->impl->work_items();
    if (classes) *classes = b->impl->classes();
    if (packed_inputs) *packed_inputs = static_cast<int64_t>(b->impl->packed_inputs());
  });
}

int bwpm_batch_work(const bwpm_batch* b, double* transforms, double* flops, double* bytes) {
  return guarded([&] {
    if (!b || !b->impl) throw bwpm::invalid_argument("null batch");
    double t = 0, f = 0, y = 0;
    b->impl->work(t, f, y);
    if (transforms) *transforms = t;
    if (flops) *flops = f;
    if (bytes) *bytes = y;
  });
}

void bwpm_batch_destroy(bwpm_batch* b) { delete b; }

int bwpm_server_create(int device, uint64_t budget_bytes, int max_groups, int max_group_solves,
                       int max_3d, bwpm_server** out) {
  return guarded([&] {
    if (!out) throw bwpm::invalid_argument("null output");
    bwpm::ServerOptions o;
    o.device = device;
    o.budget_bytes = static_cast<std::size_t>(budget_bytes);
    if (max_groups > 0) o.max_groups = max_groups;
    if (max_group_solves > 0) o.max_group_solves = max_group_solves;
    if (max_3d > 0) o.max_3d = max_3d;
    auto* s = new bwpm_server;
    try {
      s->impl = bwpm::make_server(o);
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
  });
}


int bwpm_server_submit_2d(bwpm_server* s, size_t ny, double dy, double dz, double k0,
                          const double* indices, size_t m, const int32_t* labels, size_t nz,
                          double ib_re, double ib_im, const double* mask, const double* field,
                          int iterations, int64_t* ticket) {
  return server_submit_2d(s, ny, dy, dz, k0, indices, m, labels, nz, ib_re, ib_im, mask, field,
                          iterations, ticket, false);
}

int bwpm_server_submit_2d_borrowed(bwpm_server* s, size_t ny, double dy, double dz, double k0,
                                   const double* indices, size_t m, const int32_t* labels,
                                   size_t nz, double ib_re, double ib_im, const double* mask,
                                   const double* field, int iterations, int64_t* ticket) {
  return server_submit_2d(s, ny, dy, dz, k0, indices, m, labels, nz, ib_re, ib_im, mask, field,
                          iterations, ticket, true);
}

int bwpm_server_submit_3d(bwpm_server* s, size_t ny, size_t nx, double dy, double dx, double dz,
                          double k0, const double* indices, size_t m, const int32_t* labels,
                          size_t nz, double ib_re, double ib_im, const double* mask,
                          const double* field, int iterations, int64_t* ticket) {
  return server_submit_3d(s, ny, nx, dy, dx, dz, k0, indices, m, labels, nz, ib_re, ib_im, mask,
                          field, iterations, ticket, false);
}

int bwpm_server_submit_3d_borrowed(bwpm_server* s, size_t ny, size_t nx, double dy, double dx,
                                   double dz, double k0, const double* indices, size_t m,
                                   const int32_t* labels, size_t nz, double ib_re, double ib_im,
                                   const double* mask, const double* field, int iterations,
                                   int64_t* ticket) {
  return server_submit_3d(s, ny, nx, dy, dx, dz, k0, indices, m, labels, nz, ib_re, ib_im, mask,
                          field, iterations, ticket, true);
}

int bwpm_server_submit_3d_geometry(bwpm_server* s, size_t ny, size_t nx, double dy, double dx,
                                   double dz, double k0, const double* indices, size_t m, int kind,
                                   const double* params, size_t nparams, size_t nz, double ib_re,
                                   double ib_im, const double* mask, const double* field,
                                   int iterations, int64_t* ticket) {
  return guarded([&] {
    if (!s || !s->impl) throw bwpm::invalid_argument("null server");
    if (!indices || !params || !field) throw bwpm::invalid_argument("null array");
    // validated here, so that a bad geometry fails the call rather than the request
    (void)bwpm::geometry_spec(kind, params, nparams, nz, ny, nx, dz, dy, dx);
    bwpm::SolverInput in;
    in.ny = ny;
    in.nx = nx;
    in.dy = dy;
    in.dx = dx;
    in.dz = dz;
    in.k0 = k0;
    in.indices.assign(as_cd(indices), as_cd(indices) + m);
    in.geometry_kind = kind;
    in.geometry_params.assign(params, params + nparams);
    in.nz = nz;
    in.index_before = bwpm::cd{ib_re, ib_im};
    if (mask) in.mask.assign(mask, mask + ny * nx);
    std::vector<bwpm::cd> f(as_cd(field), as_cd(field) + 2 * ny * nx);
    const int64_t k = s->impl->submit3d(std::move(in), std::move(f), iterations, nullptr);
    if (ticket) *ticket = k;
  });
}

int bwpm_server_wait(bwpm_server* s, int64_t ticket, double timeout_s, int* done) {
  return guarded([&] {
    if (!s || !s->impl) throw bwpm::invalid_argument("null server");
    const bool d = s->impl->wait(ticket, timeout_s);
    if (done) *done = d ? 1 : 0;
  });
}

int bwpm_server_result(bwpm_server* s, int64_t ticket, double* transmitted, double* reflected,
                       double* flux_t, double* flux_r, double* flux_in, double* latency_ms,
                       double* queue_ms, double* device_ms) {
  return guarded([&] {
    if (!s || !s->impl) throw bwpm::invalid_argument("null server");
    bwpm::ServedResult r;
    s->impl->result(ticket, r);
    if (transmitted) std::memcpy(transmitted, r.transmitted.data(), r.transmitted.size() * sizeof(bwpm::cd));
    if (reflected) std::memcpy(reflected, r.reflected.data(), r.reflected.size() * sizeof(bwpm::cd));
    if (flux_t) std::memcpy(flux_t, r.flux_t.data(), r.flux_t.size() * sizeof(double));
    if (flux_r) std::memcpy(flux_r, r.flux_r.data(), r.flux_r.size() * sizeof(double));
    if (flux_in) *flux_in = r.flux_in;
    if (latency_ms) *latency_ms = r.latency_ms;
    if (queue_ms) *queue_ms = r.queue_ms;
    if (device_ms) *device_ms = r.device_ms;
  });
}

int bwpm_server_stats(bwpm_server* s, int64_t* submitted, int64_t* completed, int64_t* failed,
                      int64_t* groups, int64_t* bytes_in_flight, int64_t* peak_bytes,
                      int64_t* kernel_launches, int64_t* max_concurrent) {
  return guarded([&] {
    if (!s || !s->impl) throw bwpm::invalid_argument("null server");
    bwpm::ServerStats st;
    s->impl->stats(st);
    if (submitted) *submitted = st.submitted;
    if (completed) *completed = st.completed;
    if (failed) *failed = st.failed;
    if (groups) *groups = st.groups;
    if (bytes_in_flight) *bytes_in_flight = st.bytes_in_flight;
    if (peak_bytes) *peak_bytes = st.peak_bytes;
    if (kernel_launches) *kernel_launches = st.kernel_launches;
    if (max_concurrent) *max_concurrent = st.max_concurrent;
  });
}

void bwpm_server_destroy(bwpm_server* s) { delete s; }

namespace {
bwpm::PlaneGeometry plane_geometry(size_t ny, size_t nx, double dy, double dx, double k0) {
  if (ny < 1 || nx < 1 || ny > (1u << 20) || nx > (1u << 20))
    throw bwpm::invalid_argument("ny and nx must be in [1, 2^20]");
  bwpm::PlaneGeometry g;
  g.ny = static_cast<int>(ny);
  g.nx = static_cast<int>(nx);
  g.dy = dy;
  g.dx = dx;
  g.k0 = k0;
  return g;
}

}  // namespace

int bwpm_port_power(int device, size_t ny, size_t nx, double dy, double dx, double k0,
                    double index_re, double index_im, int direction, const double* field,
                    double* power) {
  return guarded([&] {
    if (!field || !power) throw bwpm::invalid_argument("null array");
    const bwpm::PlaneGeometry g = plane_geometry(ny, nx, dy, dx, k0);
    CallStream cs(device);
    *power = bwpm::port_power(g, as_cd(field), false, bwpm::cd{index_re, index_im}, direction,
                              cs.s);
  });
}

int bwpm_plane_power(int device, size_t ny, size_t nx, double dy, double dx, double k0,
                     double index, const double* field, double* power) {
  return guarded([&] {
    if (!field || !power) throw bwpm::invalid_argument("null array");
    const bwpm::PlaneGeometry g = plane_geometry(ny, nx, dy, dx, k0);
    CallStream cs(device);
    *power = bwpm::plane_power(g, as_cd(field), false, index, cs.s);
  });
}

int bwpm_axial_focus(int device, size_t ny, size_t nx, double dy, double dx, double k0,
                     double index, const double* offsets, size_t noffsets, double na,
                     const double* field, double* best, double* peak, double* intensity) {
  return guarded([&] {
    if (!field || !offsets || !best || !peak) throw bwpm::invalid_argument("null array");
    const bwpm::PlaneGeometry g = plane_geometry(ny, nx, dy, dx, k0);
    CallStream cs(device);
    bwpm::axial_focus(g, as_cd(field), false, index, offsets, noffsets, na, best, peak, intensity,
                      cs.s);
  });
}

int bwpm_flush_l2(int device, size_t bytes) {
  return guarded([&] {
    static void* scratch[64] = {};
    static size_t size[64] = {};
    if (device < 0 || device >= 64) throw bwpm::invalid_argument("bad device");
    bwpm::check_cuda(cudaSetDevice(device), "cudaSetDevice");
    if (size[device] < bytes) {
      if (scratch[device]) cudaFree(scratch[device]);
      scratch[device] = nullptr;
      bwpm::check_cuda(cudaMalloc(&scratch[device], bytes), "cudaMalloc");
      size[device] = bytes;
    }
    bwpm::check_cuda(cudaMemset(scratch[device], size[device] & 0xff, bytes), "cudaMemset");
    bwpm::check_cuda(cudaDeviceSynchronize(), "flush");
  });
}

static_assert(BWPM_NOALLOC_MAX_N == bwpm::kNoAllocMaxN, "header and library disagree");
static_assert(BWPM_NOALLOC_SCRATCH_BYTES == bwpm::kNoAllocScratchBytes, "header and library disagree");

int bwpm_step2d_noalloc(int device, size_t ny, double dy, double dz, double k0,
                        const double* indices, size_t m, const int32_t* labels_before,
                        const int32_t* labels_after, double ib_re, double ib_im,
                        const double* mask, const double* field_in, double* field_out,
                        void* stream) {
  return guarded([&] {
    bwpm::step2d_noalloc(device, ny, dy, dz, k0, as_cd(indices), m, labels_before, labels_after,
                         bwpm::cd{ib_re, ib_im}, mask, as_cd(field_in), as_cd(field_out),
                         static_cast<cudaStream_t>(stream));
  });
}

int bwpm_host_register(void* ptr, size_t bytes) {
  return guarded([&] {
    bwpm::check_cuda(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault), "cudaHostRegister");
  });
}

int bwpm_host_unregister(void* ptr) {
  return guarded([&] { bwpm::check_cuda(cudaHostUnregister(ptr), "cudaHostUnregister"); });
}

}  // extern "C"
