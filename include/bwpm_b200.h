/* C ABI of bwpm_b200: the B200-native slab-stepping core of BWPM (libbwpm_b200.so).
 *
 * Drop-in boundary for the reference's compiled module `bwpm._core` (pybind11,
 * cpp/python/bindings.cpp:122-180). Every entry point takes plain pointers and sizes; complex
 * values are interleaved (re, im) doubles (numpy complex128 memory). All entry points return a
 * status: BWPM_OK, BWPM_EINVAL (the reference raises std::invalid_argument -> ValueError) or
 * BWPM_ERUNTIME (std::runtime_error -> RuntimeError: CUDA failure, GMRES non-convergence).
 * bwpm_last_error() gives the message of the last failure on the calling thread.
 */
#ifndef BWPM_B200_H
#define BWPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BWPM_OK 0
#define BWPM_EINVAL 1
#define BWPM_ERUNTIME 2

typedef struct bwpm_solver bwpm_solver;

/* Message of the last failed call on this thread; returns its full length. */
size_t bwpm_last_error(char* buf, size_t len);

/* Library version string. */
const char* bwpm_version(void);

/* Number of usable CUDA devices, 0 without a driver.
 * Replaces bwpm._core.cuda_device_count (cpp/python/bindings.cpp:157, cpp/src/solver_cuda.cu:357-364). */
int bwpm_cuda_device_count(void);

/* Transmission (reflection = 0) or reflection (reflection = 1) matrices of a plane interface
 * without propagation factor at n points (k_x[i], k_y[i]); out: n·2·2 complex (row-major 2×2).
 * Replaces bwpm._core.transmission_matrix / reflection_matrix
 * (cpp/python/bindings.cpp:124-137, cpp/src/interface.cpp:30-52). Computed in FP64 on device 0. */
int bwpm_interface_matrices(int reflection, const double* k_x, const double* k_y, size_t n,
                            double index_in_re, double index_in_im, double index_out_re,
                            double index_out_im, double k0, double* out);

/* k_z = sqrt(ñ²k₀² − k⊥²) with the grazing rule at n values of k⊥²; out: n complex.
 * Replaces bwpm._core.longitudinal_wavenumber (cpp/python/bindings.cpp:178-179,
 * cpp/src/interface.cpp:8-18). */
int bwpm_longitudinal_wavenumber(double index_re, double index_im, double k0,
                                 const double* k_perp_sq, size_t n, double* out);

/* Creates a solver on `device`. indices: m complex; labels: nz·ny·nx int32 (C order);
 * mask: ny·nx doubles or NULL; fluctuation: nz·ny·nx complex or NULL. precision: 64 for the
 * complex128 drop-in path, 32 for complex64 fields with FP64 operator tables. gmres_tol: GMRES
 * tolerance of the Born step (the reference uses 1e-12).
 * Replaces bwpm._core.CudaSolver(ny, nx, dy, dx, dz, k0, indices, labels, index_before, mask,
 * device, fluctuation) (cpp/python/bindings.cpp:158-171, cpp/src/solver_cuda.cu:643-719). */
int bwpm_solver_create(size_t ny, size_t nx, double dy, double dx, double dz, double k0,
                       const double* indices, size_t m, const int32_t* labels, size_t nz,
                       double index_before_re, double index_before_im, const double* mask,
                       int device, const double* fluctuation, int precision, double gmres_tol,
                       bwpm_solver** out);

/* Runs `iterations` bidirectional iterations (0: forward FPWPM only) on field (ny·nx·2 complex).
 * keep: nkeep sorted unique plane numbers ≤ nz. Outputs (complex, caller-allocated, may be
 * NULL): transmitted and reflected (ny·nx·2 each), transmitted_iter/reflected_iter
 * (iterations planes), forward/backward (nkeep planes; backward only for iterations > 0).
 * Replaces CudaSolver.run(field, iterations, keep) -> dict
 * (cpp/python/bindings.cpp:61-86, cpp/src/solver_cuda.cu:729-853). */
int bwpm_solver_run(bwpm_solver* s, const double* field, int iterations, const int64_t* keep,
                    size_t nkeep, double* transmitted, double* reflected,
                    double* transmitted_iter, double* reflected_iter, double* forward,
                    double* backward, int64_t* stored_values);

/* Device memory held by the solver, kernels it launched so far, GMRES operator applications. */
int bwpm_solver_stats(const bwpm_solver* s, int64_t* device_bytes, int64_t* kernel_launches,
                      int64_t* gmres_applies);

/* Releases the solver (CudaSolver destructor, cpp/src/solver_cuda.cu:721-727). */
void bwpm_solver_destroy(bwpm_solver* s);

/* ---- batched 2D solves (complex64 fields; no counterpart in the reference, which solves one
 * problem per CudaSolver.run call: cpp/src/solver_cuda.cu:729). Each solve is a 2D problem in the
 * reference's 2D convention (src/bwpm/fast.py:120-142: nx = 1, lateral axis y). All solves of a
 * batch run in one launch of persistent kernels; see bwpm_b200/csrc/resident2d.cuh. */
typedef struct bwpm_batch bwpm_batch;

int bwpm_batch_create(int device, bwpm_batch** out);

/* Adds one solve: labels nz·ny int32, mask ny doubles or NULL, field ny·2 complex; *id gets its
 * index. Same validation and messages as bwpm_solver_create. */
int bwpm_batch_add(bwpm_batch* b, size_t ny, double dy, double dz, double k0,
                   const double* indices, size_t m, const int32_t* labels, size_t nz,
                   double index_before_re, double index_before_im, const double* mask,
                   const double* field, int iterations, int64_t* id);

/* Kernel choice per line length (before prepare). Lengths with compiled register-resident
 * kernels (bwpm_variant_count(ny) > 0) have one or more variants (threads per CTA, FFT radices,
 * CTAs per line). on = 1: prepare picks them by timing the batch itself with every chain scaled
 * down to 1/4 of its slabs and one iteration (all lengths concurrently, as in a run),
 * coordinate descent from the first variants and from the variants with the most CTAs per line,
 * the better end kept (a variant wins on a clearly faster batch, or on an equal batch with
 * clearly less SM time for its length). Default: the first variant. set_variant forces
 * variant `variant` (0-based) for length ny. */
int bwpm_batch_set_autotune(bwpm_batch* b, int on);
int bwpm_batch_set_variant(bwpm_batch* b, size_t ny, int variant);
int bwpm_variant_count(size_t ny);

/* Class k of a prepared batch (k < classes of bwpm_batch_stats): line length (the largest of a
 * generic class), threads per CTA, CTAs per line, variant (−1: generic kernel), work items and
 * the scaled-batch time in ms of the autotuned choice (0: not tuned). */
int bwpm_batch_class_info(const bwpm_batch* b, int64_t k, int64_t* ny, int64_t* threads,
                          int64_t* cluster, int64_t* variant, int64_t* items, float* tuned_ms);

/* Builds the device pools, operator tables and launch shapes (once, after the last add). */
int bwpm_batch_prepare(bwpm_batch* b);

/* Solves every added problem once with the inputs already on the device; device_ms gets the
 * CUDA-event time of the launch. */
int bwpm_batch_run(bwpm_batch* b, float* device_ms);

/* End to end: copies new incident fields (packed: Σ ny·2 complex in add order) to the device,
 * solves, and copies (transmitted ny·2, reflected ny·2) per solve back into out (packed);
 * device_ms covers copies and kernels. */
int bwpm_batch_solve_packed(bwpm_batch* b, const double* fields, double* out, float* device_ms);

/* Results of solve `id` after a run: transmitted/reflected ny·2 complex; flux_t/flux_r
 * (iterations values, power flux per iteration as src/bwpm/fpwpm.py:205-216); flux_in; device
 * latency of the solve in ms. Any pointer may be NULL. */
int bwpm_batch_result(bwpm_batch* b, int64_t id, double* transmitted, double* reflected,
                      double* flux_t, double* flux_r, double* flux_in, double* latency_ms);

int bwpm_batch_stats(const bwpm_batch* b, int64_t* device_bytes, int64_t* kernel_launches,
                     int64_t* work_items, int64_t* classes, int64_t* packed_inputs);

/* Algorithmic work of one run: transforms, FLOPs (5·N·log2 N per transform, 6·N per spectral
 * multiply) and minimal DRAM bytes (pair ids, sparse sources, incident and output fields). */
int bwpm_batch_work(const bwpm_batch* b, double* transforms, double* flops, double* bytes);

void bwpm_batch_destroy(bwpm_batch* b);

/* ---- served request loop (continuous batching; no counterpart in the reference, which solves
 * one problem per CudaSolver.run call: cpp/src/solver_cuda.cu:729-853) ----------------------
 * Requests are submitted at any time and return a ticket at once. 2D requests (the reference's
 * 2D convention, src/bwpm/fast.py:120-142) are prepared on host worker threads, admitted
 * longest estimated chain first (then in arrival order) while the device-memory budget holds,
 * and launched in groups on the batched
 * resident engine; groups launched while others run share the GPU. 3D requests run through the
 * complex64 plane engine on their own streams. budget_bytes 0: 80 % of the free device memory;
 * max_groups / max_group_solves / max_3d ≤ 0: defaults (8, 64, 16). Destroying the server waits
 * for every submitted request. */
typedef struct bwpm_server bwpm_server;

int bwpm_server_create(int device, uint64_t budget_bytes, int max_groups, int max_group_solves,
                       int max_3d, bwpm_server** out);

/* Same arguments as bwpm_batch_add; *ticket identifies the request. */
int bwpm_server_submit_2d(bwpm_server* s, size_t ny, double dy, double dz, double k0,
                          const double* indices, size_t m, const int32_t* labels, size_t nz,
                          double index_before_re, double index_before_im, const double* mask,
                          const double* field, int iterations, int64_t* ticket);

/* Same arguments as bwpm_solver_create (precision 32) plus the field (ny·nx·2 complex) and the
 * iteration count of bwpm_solver_run. */
int bwpm_server_submit_3d(bwpm_server* s, size_t ny, size_t nx, double dy, double dx, double dz,
                          double k0, const double* indices, size_t m, const int32_t* labels,
                          size_t nz, double index_before_re, double index_before_im,
                          const double* mask, const double* field, int iterations,
                          int64_t* ticket);

/* The two submissions above with borrowed labels: the call copies only the small arrays and
 * returns; the server takes the labels later (2D: a preparation worker copies the nz·ny values;
 * 3D: the request's set-up reads the nz·ny·nx values in place), so the caller keeps `labels`
 * valid and unchanged until bwpm_server_wait reports the request finished. Submitting large 3D
 * requests then costs the submitting thread no copy. No reference counterpart (the served loop
 * is new). */
int bwpm_server_submit_2d_borrowed(bwpm_server* s, size_t ny, double dy, double dz, double k0,
                                   const double* indices, size_t m, const int32_t* labels,
                                   size_t nz, double index_before_re, double index_before_im,
                                   const double* mask, const double* field, int iterations,
                                   int64_t* ticket);
int bwpm_server_submit_3d_borrowed(bwpm_server* s, size_t ny, size_t nx, double dy, double dx,
                                   double dz, double k0, const double* indices, size_t m,
                                   const int32_t* labels, size_t nz, double index_before_re,
                                   double index_before_im, const double* mask,
                                   const double* field, int iterations, int64_t* ticket);

/* A 3D request whose labels are generated on the device from a geometry (see
 * bwpm_geometry_labels): no label volume is passed or held on the host. */
int bwpm_server_submit_3d_geometry(bwpm_server* s, size_t ny, size_t nx, double dy, double dx,
                                   double dz, double k0, const double* indices, size_t m, int kind,
                                   const double* params, size_t nparams, size_t nz,
                                   double index_before_re, double index_before_im,
                                   const double* mask, const double* field, int iterations,
                                   int64_t* ticket);

/* Waits up to timeout_s seconds (< 0: without limit); *done = 1 when the request finished. */
int bwpm_server_wait(bwpm_server* s, int64_t ticket, double timeout_s, int* done);

/* Results of a finished request, then releases it: transmitted/reflected (ny·nx·2 complex),
 * 2D only: flux_t/flux_r (iterations values) and flux_in; latency (submit → result), queueing
 * (submit → launch) and device time in ms. A failed request returns its error. Pointers may be
 * NULL. */
int bwpm_server_result(bwpm_server* s, int64_t ticket, double* transmitted, double* reflected,
                       double* flux_t, double* flux_r, double* flux_in, double* latency_ms,
                       double* queue_ms, double* device_ms);

int bwpm_server_stats(bwpm_server* s, int64_t* submitted, int64_t* completed, int64_t* failed,
                      int64_t* groups, int64_t* bytes_in_flight, int64_t* peak_bytes,
                      int64_t* kernel_launches, int64_t* max_concurrent);

void bwpm_server_destroy(bwpm_server* s);

/* ---- label volumes generated on the device from a geometry -----------------------------------
 * The labelling rule of the reference's bwpm.geometry.labels_at_centres
 * (src/bwpm/geometry.py:24-37): slab j takes the material at its centre z = (j + 0.5)·dz, on the
 * centred lateral grid y_i = (i − ny//2)·dy, x_k = (k − nx//2)·dx. The reference takes a Python
 * predicate for the body; these entry points take one of four parametrised bodies and write
 * uint8 labels straight into device memory, so a large volume never exists on the host.
 * params (BWPM_GEOMETRY_PARAMS doubles, mm): base, tan_tilt, pitch, sag, radius, vertex, back.
 *   TILTED_FACET: 1 where z ≥ base + tan_tilt·y, else 0.
 *   LENS_ARRAY:   1 where z ≥ base − h(x, y), h = max(√(radius² − r²) − (radius − sag), 0) with
 *                 r the distance to the nearest lenslet centre of a square array of `pitch`.
 *   MICROLENS:    1 where r² < radius² and z ≥ vertex + radius − √(radius² − r²); 2 where
 *                 z ≥ back + tan_tilt·y (takes precedence); else 0.
 *   TILTED_SLAB:  1 where base + tan_tilt·y ≤ z < back, else 0. */
#define BWPM_GEOMETRY_TILTED_FACET 0
#define BWPM_GEOMETRY_LENS_ARRAY 1
#define BWPM_GEOMETRY_MICROLENS 2
#define BWPM_GEOMETRY_TILTED_SLAB 3
#define BWPM_GEOMETRY_PARAMS 7

/* Generates the labels (nz·ny·nx uint8) on `device` and copies them to host `labels`. */
int bwpm_geometry_labels(int device, int kind, const double* params, size_t nparams, size_t nz,
                         size_t ny, size_t nx, double dz, double dy, double dx, uint8_t* labels);

/* bwpm_solver_create with the labels generated on the device from a geometry (no label volume
 * on the host; the per-step tables are built on the device too). No fluctuation. */
int bwpm_solver_create_geometry(size_t ny, size_t nx, double dy, double dx, double dz, double k0,
                                const double* indices, size_t m, int kind, const double* params,
                                size_t nparams, size_t nz, double index_before_re,
                                double index_before_im, const double* mask, int device,
                                int precision, bwpm_solver** out);

/* ---- post-processing of fields on the device (FP64, compensated sums) ----------------------
 * `field`: host complex128 (ny, nx, 2) (E_x, E_y) on the centred grid; k grids of
 * numpy.fft.fftfreq; the angular spectrum is this library's FP64 FFT.
 *
 * Replaces bwpm.adapter.port_power (src/bwpm/adapter.py:267-284): the Poynting flux through a
 * port, Σ Re k_z (|Ê_x|² + |Ê_y|² + |Ê_z|²)·dx·dy/(nx·ny), Ê_z = −direction·k⊥·Ê⊥/k_z, in a
 * homogeneous medium of complex index (index_re, index_im); direction ±1. With nx = 1 and
 * dx = 1 this is bwpm.fpwpm.power_flux (src/bwpm/fpwpm.py:205-216), the flux of the facade's
 * energy residual (src/bwpm/fast.py:148-155). */
int bwpm_port_power(int device, size_t ny, size_t nx, double dy, double dx, double k0,
                    double index_re, double index_im, int direction, const double* field,
                    double* power);

/* Replaces bwpm.pilot_imc3d.plane_power (src/bwpm/pilot_imc3d.py:55-67): n Σ cos θ (|E_s|² +
 * |E_p|²) over the propagating modes of a medium of real index n. */
int bwpm_plane_power(int device, size_t ny, size_t nx, double dy, double dx, double k0,
                     double index, const double* field, double* power);

/* Replaces bwpm.pilot_imc3d.axial_focus (src/bwpm/pilot_imc3d.py:96-131): the on-axis
 * intensity at each of `noffsets` distances (mm, along the direction of travel) of the
 * propagating modes (with na > 0 only those with k⊥ ≤ na·k0); returns the first offset of the
 * largest intensity (*best) and that intensity (*peak); `intensity` (noffsets doubles, or NULL)
 * receives every value. */
int bwpm_axial_focus(int device, size_t ny, size_t nx, double dy, double dx, double k0,
                     double index, const double* offsets, size_t noffsets, double na,
                     const double* field, double* best, double* peak, double* intensity);

/* Writes `bytes` of scratch memory on `device` (evicts the 126 MB L2 between timed runs). */
int bwpm_flush_l2(int device, size_t bytes);

/* ---- allocation-free slab step (no counterpart in the reference) ----------------------------
 * One FP64 forward transmission step of a 2D field (the reference's 2D convention: nx = 1,
 * lateral axis y), the same operation as one slab of bwpm_solver_run with iterations = 0:
 * out = mask · Σ_(r,s) I_r,s F⁻¹{T_r,s e^{i k_z,s dz} F{in}}. For callers that cannot allocate
 * device memory when they need the step (a host framework that owns all device memory through
 * its own arena, a real-time loop that must not allocate after start-up, a plugin with a fixed
 * memory budget): it calls no cudaMalloc or cudaFree. Its scratch (the spectrum of `field_in`
 * and the FFT twiddles) is one fixed device array of BWPM_NOALLOC_SCRATCH_BYTES bytes that every
 * GPU loading this library holds until exit; the array keeps the last call's contents and all
 * calls on a device share it, so calls that overlap on the GPU (other threads or streams) race.
 * The first call on a device looks up the array's address; make that first call before any
 * stream capture. Every call copies a status word back to the host and waits for its stream
 * before returning. The call makes `device` current and restores the caller's current device
 * before it returns.
 * Device pointers: field_in/field_out ny·2 complex, labels_before/labels_after ny int32
 * (labels_before NULL: the medium before the volume, index_before), mask ny doubles or NULL.
 * indices: host array of m ≤ 32 complex. Limits: 2 ≤ ny ≤ BWPM_NOALLOC_MAX_N, ny a product of
 * 2, 3, 5 and 7 (every such length is accepted); anything else returns BWPM_EINVAL with a
 * message, and so does a label outside [0, m) (found on the device). stream: a cudaStream_t or
 * NULL for the default stream. */
#define BWPM_NOALLOC_MAX_N 8192
#define BWPM_NOALLOC_SCRATCH_BYTES 393472
int bwpm_step2d_noalloc(int device, size_t ny, double dy, double dz, double k0,
                        const double* indices, size_t m, const int32_t* labels_before,
                        const int32_t* labels_after, double index_before_re,
                        double index_before_im, const double* mask, const double* field_in,
                        double* field_out, void* stream);

/* Page-locks host memory for fast copies (cudaHostRegister) and releases it. */
int bwpm_host_register(void* ptr, size_t bytes);
int bwpm_host_unregister(void* ptr);

#ifdef __cplusplus
}
#endif

#endif /* BWPM_B200_H */
