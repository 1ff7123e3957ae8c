// Plane engine: the drop-in CudaSolver (FP64) and its complex64 twin, general ny × nx planes.
//
// Same algorithm, inputs and outputs as the reference's bwpm::CudaSolver / bwpm::Solver
// (cpp/src/solver_cuda.cu:643-853, cpp/src/solver.cpp:27-528), re-designed for the device:
// - labels become per-step uint8 pair-id planes (deduplicated), resident on the device;
// - operator tables T/R × propagator are built once per (kind, ñ_r, ñ_s) in FP64 on the device
//   (the reference recomputes them in every kernel call) and stored in the field precision;
// - one forward transform per step feeds both the reflection and the transmission;
// - selection, mask, reflection gather and sparse source add are fused into the inverse
//   transform's epilogue; interface pixel lists and source stores are allocated once.
#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <tuple>
#include <unordered_map>

#include "born_kernels.cuh"
#include "devbuf.hpp"
#include "geometry.cuh"
#include "gmres_kernels.cuh"
#include "plan.hpp"
#include "plane_kernels.cuh"
#include "plane_rf.cuh"
#include "plane_setup.cuh"
#include "solver.hpp"

namespace bwpm {
namespace {

constexpr int kThreads = 256;

struct StepInfo {
  std::vector<std::pair<int, int>> pairs;  // (label at plane p, label at plane p + 1), sorted
  long long pid_off = -1;                  // offset into the pair-id pool, −1: a single pair
  long long iface_off = 0;
  int niface = 0;
  long long rowoff_off = -1;               // 3D: offsets of each row into the interface list
  int host_slot = -1;                      // Born slab: index into the host/potential arrays
};

struct LaunchShape {
  int rows = 1, threads = 32;
  std::size_t smem = 0;
  int group = 1;  // passes per inverse transform (row kernel of a 3D step)
};

template <typename T>
class PlaneSolver final : public Solver {
 public:
  explicit PlaneSolver(SolverInput in) : in_(std::move(in)) { setup(); }
  ~PlaneSolver() override = default;

  void run(const cd* field, int iterations, const std::int64_t* keep, std::size_t nkeep,
           RunOutputs& out) override;
  std::size_t device_bytes() const override;
  std::int64_t kernel_launches() const override { return launches_; }
  std::int64_t gmres_applies() const override { return gmres_applies_; }

 private:
  using C = cx<T>;
  void setup();
  // per-step pairs, pair-id planes and interface lists from uint8 labels on the device
  void device_steps(const std::uint8_t* labels_u8, const std::vector<int>& host_of);
  // operator table of (kind, ñ_r, ñ_s); scalar: the complex64 propagator-only table
  const C* table(int kind, cd nr, cd ns, bool scalar = false);
  // pass records of all steps on the device (forward, and backward when with_backward)
  void ensure_passes(bool with_backward);
  // x_ready: xbuf_ already holds the x transform of `in` (3D, fused into the previous step);
  // x_next: also leave the x transform of `out` in xbuf_ for the next step
  // need_out: the output plane is read after the step (with x_next the next step reads only its
  // x transform; `out` is still needed for keep planes and a sweep's last plane)
  void step(int s, bool backward, bool reflect, const C* in, C* out, C* refl_out, const C* add,
            bool want_spec, bool x_ready = false, bool x_next = false, bool need_out = true);
  void fft_plane(const C* in, C* out, int ncomp, int dir);
  // out = G·in (combine 0) or in − G·in/2 (combine 1)
  void born_operator(const C* in, C* out, int combine = 0);
  void born_step(const C* spec, C* inc, int slot, int dir);
  void born_sources(const C* spec, int slot, int dir);
  void born_emission(int slot, int dir, C* plane);
  void gmres();
  void arnoldi_step(int j, bool in_graph, double tol_bnorm);
  void gmres_alloc();
  void build_born_graph();
  // the forward/backward sweeps of a run (device work only, unless Born slabs need GMRES)
  void sweeps(int iterations, const std::vector<int>& keep_slot, DevBuf<C>& kept_f, DevBuf<C>& kept_b,
              DevBuf<C>& t_iter, DevBuf<C>& r_iter);
  void axpby(C* y, const C* x, cd a, cd b, long long m);
  void add_plane_scaled(C* dst, const C* src, const T* mask);
  LaunchShape rows_shape(int ncomp, int rows_max) const;
  LaunchShape cols_shape(int ncomp, int tiles) const;
  LaunchShape step_rows_shape() const;
  std::size_t n() const { return in_.ny * in_.nx; }
  bool is2d() const { return in_.nx == 1; }
  cd index_of(int label) const {
    return label < 0 ? in_.index_before : in_.indices[static_cast<std::size_t>(label)];
  }
  BornGrid born_grid(int slot) const {
    return BornGrid{hosts_[slot], in_.k0, in_.dz, in_.dy, in_.dx, static_cast<int>(in_.ny),
                    static_cast<int>(in_.nx)};
  }
  template <typename K, typename... A>
  void launch(K kernel, dim3 grid, dim3 block, std::size_t smem, A... args) {
    kernel<<<grid, block, smem, stream_>>>(args...);
    check_cuda(cudaGetLastError(), "kernel launch");
    ++launches_;
  }

  SolverInput in_;
  OwnedStream stream_;  // first: outlives the stream-ordered buffers below
  HostPlan hy_, hx_;
  DevBuf<Tw<T>> tw_y_, tw_x_;
  std::vector<StepInfo> steps_;
  DevBuf<std::uint8_t> pid_pool_;
  DevBuf<int> iface_pool_, rowoff_pool_;
  long long iface_total_ = 0;
  DevBuf<T> mask_;
  std::map<std::tuple<int, double, double, double, double>, DevBuf<C>> tables_;
  // fields
  DevBuf<C> input_, e_, next_, spec_, xbuf_, work_, src_fwd_, src_bwd_;
  DevBuf<cd> stage_;
  C* last_e_ = nullptr;  // plane holding the last sweep's result (set by sweeps)
  int max_pass_ = 1;
  // Born
  std::vector<cd> hosts_;
  DevBuf<C> pot_, born_fwd_, born_bwd_, w3_, t3_, sources_, g_x_, g_rhs_, g_y_, g_w_, g_tmp_,
      inc_;
  std::vector<DevBuf<C>> basis_;
  DevBuf<GmresState> gst_;
  DevBuf<BornCur<T>> born_cur_;  // the Born slab of the current step (set per step)
  OwnedGraph born_graph_;        // one Born step: P_½, right-hand side, GMRES, P_½^{±}, F⁻¹
  GmresConds conds_{};           // its conditional nodes' handles
  DevBuf<C*> basis_ptrs_;        // the Krylov basis vectors' addresses (device)
  bool born_graph_used_ = false; // a run launched it: its error flag and counts are read at the end
  int gm_vblocks_ = 0, gm_dblocks_ = 0;
  DevBuf<cd> dot_partial_;
  PinnedBuf<int> flags_host_;
  OwnedEvent gmres_events_[kGmresRestart];
  // launch shapes
  int thr2d_ = 32, thr_line3_ = 32;
  bool line_ept8_ = false;  // 2D line transforms with 8 values per thread (k_line_fft)
  int sms_ = 148;
  LaunchShape rows2_, rows3_, sel_, cols1_, cols2_, cols3_;
  std::int64_t launches_ = 0, gmres_applies_ = 0;
  // complex64 3D: the fixed-length step kernels (plane_rf.cuh) when both lateral sizes have one
  RfKernels rf_y_, rf_x_;
  DevBuf<Tw<float>> tw_rf_y_, tw_rf_x_;
  bool cols_bulk_ = false;  // 3D column kernel with bulk copies (k_cols_step_bulk)
  int cols_bulk_threads_ = 256, cols_bulk_group_ = 1;
  DevBuf<int> status_;      // set by a kernel whose bounded wait gave up
  DevBuf<PassRec> pass_pool_;
  std::vector<long long> pass_off_[2];
  std::vector<int> pass_nt_[2], pass_nr_[2];
  int pool_dirs_ = 0;  // directions in the pool: 0 none, 1 forward, 2 forward and backward
};

template <typename T>
LaunchShape PlaneSolver<T>::rows_shape(int ncomp, int rows_max) const {
  LaunchShape s;
  const std::size_t row_bytes = in_.nx * ncomp * sizeof(C);
  // at most rows_max rows per CTA, and few enough for two CTAs per SM over the plane's rows
  rows_max = std::min<int>(rows_max, std::max<int>(1, static_cast<int>(in_.ny) / (2 * sms_)));
  s.rows = static_cast<int>(std::max<std::size_t>(1, std::min<std::size_t>(rows_max, 49152 / row_bytes)));
  while (s.rows > 1 && threads_needed(hx_.plan, s.rows * ncomp) > kPlaneThreads) --s.rows;
  s.threads = std::max(64, threads_needed(hx_.plan, s.rows * ncomp));
  if (s.threads > kPlaneThreads) throw invalid_argument("nx too large for the row transform");
  s.smem = s.rows * row_bytes;
  return s;
}

// Rows per CTA of the slab-step row kernels (2 components): 4 when that still gives a CTA per
// SM, else 2, so that every transposed run (rows × 16 B in complex64) fills whole 32-byte sectors.
// Launch-shape override of the 3D step kernels for tuning measurements: BWPM_3D_SHAPE =
// "rows,row_group,col_group,col_threads,row_threads" (0 keeps a field's default choice).
inline void shape_override(int (&v)[5]) {
  for (int& x : v) x = 0;
  if (const char* e = std::getenv("BWPM_3D_SHAPE"))
    std::sscanf(e, "%d,%d,%d,%d,%d", &v[0], &v[1], &v[2], &v[3], &v[4]);
}

template <typename T>
LaunchShape PlaneSolver<T>::step_rows_shape() const {
  LaunchShape s;
  int ov[5];
  shape_override(ov);
  const std::size_t row_bytes = in_.nx * 2 * sizeof(C);
  int rows = static_cast<int>(in_.ny) / 4 >= sms_ ? 4 : 2;
  if (ov[0] > 0) rows = ov[0];
  rows = std::min<int>(rows, static_cast<int>(in_.ny));
  while (rows > 1 && (rows * row_bytes > 98304 || threads_needed(hx_.plan, rows * 2) > kPlaneThreads)) --rows;
  s.rows = rows;
  if (threads_needed(hx_.plan, rows * 2) > kPlaneThreads || rows * row_bytes > 227 * 1024)
    throw invalid_argument("nx too large for the row transform");
  // passes per inverse transform: up to 4, while the threads allow it and the shared memory
  // leaves room for at least 3 CTAs per SM (these kernels are latency-bound)
  int g = std::min(ov[1] > 0 ? ov[1] : 4, std::max(1, max_pass_));
  while (g > 1 && (threads_needed(hx_.plan, rows * 2 * g) > kPlaneThreads ||
                   static_cast<std::size_t>(g) * rows * row_bytes > (ov[1] > 0 ? 200 : 64) * 1024))
    g = g > 2 ? 2 : 1;
  s.group = g;
  s.threads = std::min(kPlaneThreads,
                       std::max(ov[4] > 0 ? ov[4] : 256, threads_needed(hx_.plan, rows * 2 * g)));
  s.smem = static_cast<std::size_t>(g) * rows * row_bytes;
  return s;
}

template <typename T>
LaunchShape PlaneSolver<T>::cols_shape(int ncomp, int tiles) const {
  LaunchShape s;
  const std::size_t col_bytes = in_.ny * ncomp * sizeof(C);
  int cols = std::max(1, static_cast<int>(64 / (ncomp * sizeof(C))));
  cols = std::min(cols, std::max(1, static_cast<int>(in_.nx) / (2 * sms_)));  // two CTAs per SM
  while (cols > 1 && (col_bytes * cols * tiles > 98304 ||
                      threads_needed(hy_.plan, cols * ncomp) > kPlaneThreads))
    --cols;
  s.rows = cols;
  // at least 256 threads: a column's loads and stores are spread over more warps than its
  // transform needs (the kernels are latency-bound otherwise: one column per CTA at 512²)
  s.threads = std::min(kPlaneThreads, std::max(256, threads_needed(hy_.plan, cols * ncomp)));
  s.smem = col_bytes * cols * tiles;
  if (s.threads > kPlaneThreads || s.smem > 227 * 1024)
    throw invalid_argument("ny too large for the column transform");
  return s;
}

template <typename T>
void PlaneSolver<T>::setup() {
  const std::size_t nn = n();
  if (in_.ny < 1 || in_.nx < 1) throw invalid_argument("ny and nx must be positive");
  const std::int32_t* labels = in_.labels_view ? in_.labels_view : in_.labels.data();
  if (in_.labels_device || in_.geometry_kind >= 0) {  // uint8 labels on the device (in range)
    if (in_.indices.size() > 255) throw invalid_argument("device labels take at most 255 materials");
    if (!in_.fluct.empty()) throw invalid_argument("fluctuation needs host labels");
    if (in_.geometry_kind >= 0 &&
        in_.indices.size() < static_cast<std::size_t>(geometry_materials(in_.geometry_kind)))
      throw invalid_argument("labels must index into `indices`");
    labels = nullptr;
  } else if (!in_.labels_view && in_.labels.size() != in_.nz * nn) {
    throw invalid_argument("labels must have shape (nz, ny, nx)");
  }
  if (!in_.mask.empty() && in_.mask.size() != nn) throw invalid_argument("mask must have shape (ny, nx)");
  if (labels) {  // range check as a min/max reduction (vectorises; one pass over the labels)
    std::int32_t lo = 0, hi = 0;
    const std::size_t nl = in_.nz * nn;
    if (nl > 0) lo = hi = labels[0];
    for (std::size_t i = 0; i < nl; ++i) {
      lo = std::min(lo, labels[i]);
      hi = std::max(hi, labels[i]);
    }
    if (lo < 0 || static_cast<std::size_t>(hi) >= in_.indices.size())
      throw invalid_argument("labels must index into `indices`");
  }
  if (nn > (1u << 30)) throw invalid_argument("plane too large");
  if (in_.indices.size() > 4096) throw invalid_argument("at most 4096 materials");
  // Born hosts per slab (cpp/src/solver.cpp:49-62)
  std::vector<int> host_of(in_.nz, -1);
  if (!in_.fluct.empty()) {
    if (in_.fluct.size() != in_.nz * nn)
      throw invalid_argument("fluctuation must have the shape of labels (nz, ny, nx)");
    for (std::size_t j = 0; j < in_.nz; ++j) {
      bool has = false;
      cd host{0.0, 0.0};
      for (std::size_t q = 0; q < nn; ++q) {
        const cd d = in_.fluct[j * nn + q];
        if (d.re == 0.0 && d.im == 0.0) continue;
        const cd idx = in_.indices[static_cast<std::size_t>(labels[j * nn + q])];
        if (has && (host.re != idx.re || host.im != idx.im))
          throw invalid_argument("slab " + std::to_string(j) + ": fluctuation must lie in one host index");
        has = true;
        host = idx;
      }
      if (has) {
        host_of[j] = static_cast<int>(hosts_.size());
        hosts_.push_back(host);
      }
    }
  }
  check_cuda(cudaSetDevice(in_.device), "cudaSetDevice");
  stream_.create();
  keep_pool_memory(in_.device);
  check_cuda(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, in_.device), "SM count");
  hy_ = make_plan(static_cast<int>(in_.ny));
  hx_ = make_plan(static_cast<int>(in_.nx));
  auto upload_tw = [&](const HostPlan& hp, DevBuf<Tw<T>>& d) {
    const std::vector<Tw<T>> t = twiddles_for<T>(hp);
    d.alloc(t.size(), stream_);
    d.upload(t.data(), t.size());
  };
  upload_tw(hy_, tw_y_);
  upload_tw(hx_, tw_x_);

  DevBuf<std::uint8_t> generated;  // labels generated from a geometry, freed after set-up
  if (in_.geometry_kind >= 0) {
    const GeometrySpec g = geometry_spec(in_.geometry_kind, in_.geometry_params.data(),
                                         in_.geometry_params.size(), in_.nz, in_.ny, in_.nx,
                                         in_.dz, in_.dy, in_.dx);
    generated.alloc(std::max<std::size_t>(1, in_.nz * nn), stream_);
    generate_labels(g, generated.ptr, stream_);
    in_.labels_device = generated.ptr;
  }
  // per-step pairs, pair-id planes and interface lists: on the device for large volumes (or
  // labels already on the device), else on the host (pair-id planes deduplicated); the
  // environment variable BWPM_SETUP=host|device overrides the choice where both can run
  bool on_device = in_.labels_device != nullptr ||
                   (in_.indices.size() <= 255 && in_.nz * nn >= (std::size_t{1} << 22));
  if (const char* e = std::getenv("BWPM_SETUP"); e && !in_.labels_device) {
    if (std::strcmp(e, "host") == 0) on_device = false;
    if (std::strcmp(e, "device") == 0) on_device = in_.indices.size() <= 255;
  }
  if (in_.nz > 65535) {
    if (in_.labels_device) throw invalid_argument("device labels take at most 65535 slabs");
    on_device = false;
  }
  if (on_device) {
    DevBuf<std::uint8_t> u8;
    const std::uint8_t* lab8 = in_.labels_device;
    if (!lab8) {  // upload the caller's int32 labels in chunks of planes, as uint8
      u8.alloc(std::max<std::size_t>(1, in_.nz * nn), stream_);
      const std::size_t per = std::max<std::size_t>(1, (std::size_t{64} << 20) / (4 * nn));
      DevBuf<std::int32_t> stage(std::min(per, in_.nz) * nn, stream_);
      DevBuf<int> bad(1, stream_);
      check_cuda(cudaMemsetAsync(bad.ptr, 0, sizeof(int), stream_), "memset");
      for (std::size_t p0 = 0; p0 < in_.nz; p0 += per) {
        const std::size_t cnt = std::min(per, in_.nz - p0) * nn;
        check_cuda(cudaMemcpyAsync(stage.ptr, labels + p0 * nn, cnt * sizeof(std::int32_t),
                                   cudaMemcpyHostToDevice, stream_), "labels upload");
        k_labels_to_u8<<<std::min<long long>(ceil_div(static_cast<long long>(cnt), 256), 4 * sms_), 256, 0,
                         stream_>>>(stage.ptr, u8.ptr + p0 * nn, static_cast<long long>(cnt), static_cast<int>(in_.indices.size()),
                                    bad.ptr);
        check_cuda(cudaGetLastError(), "k_labels_to_u8");
      }
      lab8 = u8.ptr;
      device_steps(lab8, host_of);
      // on the solver's (non-blocking) stream, after the kernels that set it
      int flag = 0;
      check_cuda(cudaMemcpyAsync(&flag, bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, stream_),
                 "labels check");
      check_cuda(cudaStreamSynchronize(stream_), "labels check");
      if (flag) throw invalid_argument("labels must index into `indices`");
    } else {
      device_steps(lab8, host_of);
    }
    in_.labels_device = nullptr;  // not read after set-up
  } else {
    // per-step pairs, pair-id planes (deduplicated), interface lists
    std::vector<std::uint8_t> pid_host;
    std::unordered_map<std::uint64_t, std::vector<long long>> pid_seen;
    std::vector<int> iface_host, rowoff_host;
    std::vector<std::int32_t> before(nn, -1);
    steps_.resize(in_.nz);
    std::vector<std::uint8_t> pid(nn);
    // a label pair (r, s), r ∈ [−1, m), s ∈ [0, m), as one code (r + 1)·m + s: codes sort like the
    // pairs, so a presence scan lists a step's pairs in the reference's std::set order
    // (cpp/src/solver.cpp:389-390); per code: whether the indices differ (an interface)
    const int m = static_cast<int>(in_.indices.size());
    const std::size_t ncode = static_cast<std::size_t>(m + 1) * m;
    std::vector<std::uint8_t> code_iface(ncode);
    for (int r = -1; r < m; ++r)
      for (int q = 0; q < m; ++q) {
        const cd x = index_of(r), y = index_of(q);
        code_iface[static_cast<std::size_t>(r + 1) * m + q] = x.re != y.re || x.im != y.im;
      }
    std::vector<std::uint32_t> code(nn), stamp(ncode, 0);
    std::vector<int> code_id(ncode, -1);
    for (std::size_t p = 0; p < in_.nz; ++p) {
      const std::int32_t* a = p == 0 ? before.data() : labels + (p - 1) * nn;
      const std::int32_t* b = labels + p * nn;
      const std::uint32_t mark = static_cast<std::uint32_t>(p) + 1;
      std::vector<std::uint32_t> present;
      for (std::size_t q = 0; q < nn; ++q) {
        const std::uint32_t k = static_cast<std::uint32_t>(a[q] + 1) * m + b[q];
        code[q] = k;
        if (stamp[k] != mark) {
          stamp[k] = mark;
          present.push_back(k);
        }
      }
      std::sort(present.begin(), present.end());
      StepInfo& st = steps_[p];
      st.pairs.clear();
      for (auto k : present) st.pairs.emplace_back(static_cast<int>(k / m) - 1, static_cast<int>(k % m));
      if (st.pairs.size() > 255) throw invalid_argument("more than 255 label pairs in one step");
      if (2 * st.pairs.size() > static_cast<std::size_t>(kMaxPasses))
        throw invalid_argument("too many label pairs in one step");
      if (st.pairs.size() > 1) {
        for (std::size_t i = 0; i < present.size(); ++i) code_id[present[i]] = static_cast<int>(i);
        std::uint64_t h = 1469598103934665603ULL;
        for (std::size_t q = 0; q < nn; ++q) {
          pid[q] = static_cast<std::uint8_t>(code_id[code[q]]);
          h = (h ^ pid[q]) * 1099511628211ULL;
        }
        long long found = -1;
        for (long long off : pid_seen[h])
          if (std::memcmp(pid_host.data() + off, pid.data(), nn) == 0) {
            found = off;
            break;
          }
        if (found < 0) {
          found = static_cast<long long>(pid_host.size());
          pid_host.insert(pid_host.end(), pid.begin(), pid.end());
          pid_seen[h].push_back(found);
        }
        st.pid_off = found;
      }
      st.iface_off = static_cast<long long>(iface_host.size());
      bool any_iface = false;
      for (auto k : present) any_iface |= code_iface[k] != 0;
      if (any_iface)
        for (std::size_t q = 0; q < nn; ++q)
          if (code_iface[code[q]]) iface_host.push_back(static_cast<int>(q));
      st.niface = static_cast<int>(iface_host.size() - st.iface_off);
      if (st.niface > 0 && !is2d()) {
        st.rowoff_off = static_cast<long long>(rowoff_host.size());
        const int* first = iface_host.data() + st.iface_off;
        for (std::size_t y = 0; y <= in_.ny; ++y)
          rowoff_host.push_back(static_cast<int>(
              std::lower_bound(first, first + st.niface, static_cast<int>(y * in_.nx)) - first));
      }
      st.host_slot = host_of[p];
      int npass = static_cast<int>(st.pairs.size());
      for (auto& pr : st.pairs) {
        const cd x = index_of(pr.first), y = index_of(pr.second);
        if (x.re != y.re || x.im != y.im) ++npass;
      }
      max_pass_ = std::max(max_pass_, npass);
    }
    in_.labels_view = nullptr;  // the caller's labels are not read after set-up
    iface_total_ = static_cast<long long>(iface_host.size());
    if (!pid_host.empty()) {
      pid_pool_.alloc(pid_host.size(), stream_);
      pid_pool_.upload(pid_host.data(), pid_host.size());
    }
    if (!iface_host.empty()) {
      iface_pool_.alloc(iface_host.size(), stream_);
      iface_pool_.upload(iface_host.data(), iface_host.size());
      src_fwd_.alloc(2 * iface_host.size(), stream_);
      src_bwd_.alloc(2 * iface_host.size(), stream_);
    }
    if (!rowoff_host.empty()) {
      rowoff_pool_.alloc(rowoff_host.size(), stream_);
      rowoff_pool_.upload(rowoff_host.data(), rowoff_host.size());
    }
  }
  if (!in_.mask.empty()) {  // FP32: hi values then lo values (mask = hi + lo)
    const bool pair = sizeof(T) != sizeof(double);
    std::vector<T> m((pair ? 2 : 1) * nn);
    for (std::size_t q = 0; q < nn; ++q) {
      m[q] = static_cast<T>(in_.mask[q]);
      if (pair) m[nn + q] = static_cast<T>(in_.mask[q] - static_cast<double>(m[q]));
    }
    mask_.alloc(m.size(), stream_);
    mask_.upload(m.data(), m.size());
  }
  input_.alloc(2 * nn, stream_);
  e_.alloc(2 * nn, stream_);
  next_.alloc(2 * nn, stream_);
  spec_.alloc(2 * nn, stream_);
  stage_.alloc(2 * nn, stream_);
  // launch shapes and shared-memory opt-in
  if (is2d()) {
    thr2d_ = std::max(64, threads_needed(hy_.plan, 1));
    if (thr2d_ > kPlaneThreads || nn * sizeof(C) > 227 * 1024)
      throw invalid_argument("ny too large for the single-CTA line transform");
    thr_line3_ = thr2d_;
    line_ept8_ = threads_needed(hy_.plan, 1, 8) <= kPlaneThreads;
    if (line_ept8_) thr_line3_ = std::max(64, threads_needed(hy_.plan, 1, 8));
    check_cuda(cudaFuncSetAttribute(k_step2d<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), "smem");
    check_cuda(cudaFuncSetAttribute(k_step2d<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), "smem");
    if (line_ept8_) thr2d_ = thr_line3_;
    for (auto k : {(const void*)k_line_fft<-1, T>, (const void*)k_line_fft<1, T>,
                   (const void*)k_line_fft<-1, T, 8>, (const void*)k_line_fft<1, T, 8>})
      check_cuda(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), "smem");
  } else {
    rows2_ = rows_shape(2, 8);
    rows3_ = rows_shape(3, 8);
    sel_ = step_rows_shape();
    cols1_ = cols_shape(2, 1);
    cols2_ = cols_shape(2, 2);
    cols3_ = cols_shape(3, 1);
    // the bulk-copy column kernel needs 16-byte runs (even ny) and its buffers in shared memory;
    // BWPM_COLS=plain selects the plain-load kernel
    const char* ck = std::getenv("BWPM_COLS");
    const int nyi = static_cast<int>(in_.ny);
    // group size: up to 4 passes, keeping shared memory for 4 CTAs per SM (occupancy matters
    // more than grouping: these kernels are latency-bound)
    int ov[5];
    shape_override(ov);
    cols_bulk_group_ = std::min(ov[2] > 0 ? ov[2] : 4, std::max(1, max_pass_));
    while (cols_bulk_group_ > 1 &&
           (cols_bulk_smem<T>(nyi, cols_bulk_group_) > (ov[2] > 0 ? 200 : 56) * 1024 ||
            threads_needed(hy_.plan, 2 * cols_bulk_group_) > kPlaneThreads))
      cols_bulk_group_ = cols_bulk_group_ > 2 ? 2 : 1;
    cols_bulk_ = in_.ny % 2 == 0 && cols_bulk_smem<T>(nyi, cols_bulk_group_) <= 200 * 1024 &&
                 threads_needed(hy_.plan, 2 * cols_bulk_group_) <= kPlaneThreads &&
                 !(ck && std::strcmp(ck, "plain") == 0);
    cols_bulk_threads_ = std::min(
        kPlaneThreads, std::max(ov[3] > 0 ? ov[3] : 256, threads_needed(hy_.plan, 2 * cols_bulk_group_)));
    status_.alloc(1, stream_);
    check_cuda(cudaMemsetAsync(status_.ptr, 0, sizeof(int), stream_), "memset");
    xbuf_.alloc(2 * nn, stream_);
    work_.alloc(static_cast<std::size_t>(max_pass_) * 2 * nn, stream_);
    for (auto k : {(const void*)k_rows_fft<-1, T>, (const void*)k_rows_fft<1, T>,
                   (const void*)k_rows_fft<-1, T, true>,
                   (const void*)k_cols_step<T>, (const void*)k_cols_step_bulk<T>,
                   (const void*)k_rows_select<T>,
                   (const void*)k_cols_fft<-1, T>, (const void*)k_cols_fft<1, T>})
      check_cuda(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), "smem");
    // complex64: fixed-length kernels where ny and nx have them (whole CTAs of lines);
    // BWPM_3D_KERNELS=general selects the general kernels
    const char* kk = std::getenv("BWPM_3D_KERNELS");
    if (sizeof(T) == sizeof(float) && !(kk && std::strcmp(kk, "general") == 0)) {
      RfKernels ky = rf_kernels(nyi), kx = rf_kernels(static_cast<int>(in_.nx));
      if (ky.cols && kx.rows && in_.nx % ky.lines == 0 && in_.ny % kx.lines == 0) {
        rf_y_ = ky;
        rf_x_ = kx;
        auto upload_rf = [&](const RfKernels& k, int len, DevBuf<Tw<float>>& d) {
          const std::vector<Tw<float>> t = twiddles_for<float>(make_plan_radices(len, k.radices));
          d.alloc(t.size(), stream_);
          d.upload(t.data(), t.size());
        };
        upload_rf(rf_y_, nyi, tw_rf_y_);
        upload_rf(rf_x_, static_cast<int>(in_.nx), tw_rf_x_);
        check_cuda(cudaFuncSetAttribute((const void*)rf_y_.cols,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(rf_y_.smem)), "smem");
        check_cuda(cudaFuncSetAttribute((const void*)rf_x_.rows,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(rf_x_.smem)), "smem");
      }
    }
  }
  // operator tables of the forward transmission (all runs need them)
  for (std::size_t p = 0; p < in_.nz; ++p)
    for (auto& pr : steps_[p].pairs) {
      const cd nr = index_of(pr.first), ns = index_of(pr.second);
      const bool same = nr.re == ns.re && nr.im == ns.im;
      table(kFwdT, nr, ns, sizeof(T) != sizeof(double) && !is2d() && same);
    }
  // Born: potential V = 2ñ₀k₀²δn per host slab, full-plane source stores
  if (!hosts_.empty()) {
    born_cur_.alloc(1, stream_);
    pot_.alloc(hosts_.size() * nn, stream_);
    std::vector<C> vt(hosts_.size() * nn);
    for (std::size_t p = 0; p < in_.nz; ++p) {
      const int slot = host_of[p];
      if (slot < 0) continue;
      const cd scale = ((2.0 * hosts_[slot]) * in_.k0) * in_.k0;  // cpp/src/solver.cpp:241
      for (std::size_t q = 0; q < nn; ++q) vt[slot * nn + q] = cast<T>(scale * in_.fluct[p * nn + q]);
    }
    pot_.upload(vt.data(), vt.size());
    born_fwd_.alloc(hosts_.size() * 2 * nn, stream_);
    born_bwd_.alloc(hosts_.size() * 2 * nn, stream_);
    w3_.alloc(3 * nn, stream_);
    t3_.alloc(3 * nn, stream_);
    sources_.alloc(6 * nn, stream_);
    for (auto* b : {&g_x_, &g_rhs_, &g_y_, &g_w_, &g_tmp_, &inc_}) b->alloc(2 * nn, stream_);
  }
  check_cuda(cudaStreamSynchronize(stream_), "setup");  // this solver's stream only
}

template <typename T>
void PlaneSolver<T>::device_steps(const std::uint8_t* labels_u8, const std::vector<int>& host_of) {
  const std::size_t nn = n();
  const int nz = static_cast<int>(in_.nz);
  const int m = static_cast<int>(in_.indices.size());
  const int ncode = (m + 1) * m;
  const int words = (ncode + 31) / 32;
  std::vector<std::uint8_t> code_iface(ncode);
  for (int r = -1; r < m; ++r)
    for (int q = 0; q < m; ++q) {
      const cd x = index_of(r), y = index_of(q);
      code_iface[static_cast<std::size_t>(r + 1) * m + q] = x.re != y.re || x.im != y.im;
    }
  SetupVolume v{labels_u8, static_cast<long long>(nn), nz, static_cast<int>(in_.ny),
                static_cast<int>(in_.nx), m, words};
  DevBuf<std::uint8_t> d_iface(ncode, stream_);
  d_iface.upload(code_iface.data(), code_iface.size());
  DevBuf<unsigned> bits(static_cast<std::size_t>(nz) * words, stream_);
  DevBuf<unsigned long long> counts(nz, stream_);
  check_cuda(cudaMemsetAsync(bits.ptr, 0, bits.bytes(), stream_), "memset");
  check_cuda(cudaMemsetAsync(counts.ptr, 0, counts.bytes(), stream_), "memset");
  const int per_step = static_cast<int>(std::max<long long>(
      1, std::min<long long>(ceil_div(static_cast<long long>(nn), 256LL * 8), 64)));
  k_setup_presence<<<dim3(per_step, nz), 256, words * sizeof(unsigned), stream_>>>(v, d_iface.ptr,
                                                                                 bits.ptr, counts.ptr);
  check_cuda(cudaGetLastError(), "k_setup_presence");
  std::vector<unsigned> h_bits(bits.n);
  std::vector<unsigned long long> h_counts(nz);
  check_cuda(cudaMemcpyAsync(h_bits.data(), bits.ptr, bits.bytes(), cudaMemcpyDeviceToHost, stream_), "bits");
  check_cuda(cudaMemcpyAsync(h_counts.data(), counts.ptr, counts.bytes(), cudaMemcpyDeviceToHost, stream_),
             "counts");
  check_cuda(cudaStreamSynchronize(stream_), "setup presence");
  // pairs per step in code order (the reference's std::set order), offsets of the pools
  std::vector<int> multi, with_iface;
  std::vector<long long> pid_off, iface_off, rowoff_off;
  std::vector<std::uint8_t> code_id;
  long long pid_total = 0, iface_total = 0, rowoff_total = 0;
  steps_.assign(in_.nz, StepInfo{});
  for (int p = 0; p < nz; ++p) {
    StepInfo& st = steps_[p];
    const unsigned* b = h_bits.data() + static_cast<std::size_t>(p) * words;
    std::vector<int> present;
    for (int c = 0; c < ncode; ++c)
      if (b[c >> 5] & (1u << (c & 31))) present.push_back(c);
    for (int c : present) st.pairs.emplace_back(c / m - 1, c % m);
    if (st.pairs.size() > 255) throw invalid_argument("more than 255 label pairs in one step");
    if (2 * st.pairs.size() > static_cast<std::size_t>(kMaxPasses))
      throw invalid_argument("too many label pairs in one step");
    if (st.pairs.size() > 1) {
      st.pid_off = pid_total;
      multi.push_back(p);
      pid_off.push_back(pid_total);
      pid_total += static_cast<long long>(nn);
      const std::size_t row = code_id.size();
      code_id.resize(row + ncode, 0);
      for (std::size_t i = 0; i < present.size(); ++i) code_id[row + present[i]] = static_cast<std::uint8_t>(i);
    }
    st.iface_off = iface_total;
    st.niface = static_cast<int>(h_counts[p]);
    if (st.niface > 0) {
      with_iface.push_back(p);
      iface_off.push_back(iface_total);
      iface_total += st.niface;
      if (!is2d()) {
        st.rowoff_off = rowoff_total;
        rowoff_off.push_back(rowoff_total);
        rowoff_total += static_cast<long long>(in_.ny) + 1;
      } else {
        rowoff_off.push_back(-1);
      }
    }
    st.host_slot = host_of[p];  // Born slab (δn) or −1
    int npass = static_cast<int>(st.pairs.size());
    for (auto& pr : st.pairs) {
      const cd x = index_of(pr.first), y = index_of(pr.second);
      if (x.re != y.re || x.im != y.im) ++npass;
    }
    max_pass_ = std::max(max_pass_, npass);
  }
  iface_total_ = iface_total;
  if (!multi.empty()) {
    pid_pool_.alloc(static_cast<std::size_t>(pid_total), stream_);
    DevBuf<int> d_steps(multi.size(), stream_);
    DevBuf<long long> d_off(pid_off.size(), stream_);
    DevBuf<std::uint8_t> d_code(code_id.size(), stream_);
    d_steps.upload(multi.data(), multi.size());
    d_off.upload(pid_off.data(), pid_off.size());
    d_code.upload(code_id.data(), code_id.size());
    k_setup_pid<<<dim3(static_cast<unsigned>(std::min<long long>(ceil_div(static_cast<long long>(nn), 256), 64)),
                       static_cast<unsigned>(multi.size())), 256, 0, stream_>>>(
        v, d_steps.ptr, d_off.ptr, d_code.ptr, ncode, pid_pool_.ptr);
    check_cuda(cudaGetLastError(), "k_setup_pid");
    check_cuda(cudaStreamSynchronize(stream_), "setup pid");
  }
  if (!with_iface.empty()) {
    iface_pool_.alloc(static_cast<std::size_t>(iface_total), stream_);
    src_fwd_.alloc(2 * static_cast<std::size_t>(iface_total), stream_);
    src_bwd_.alloc(2 * static_cast<std::size_t>(iface_total), stream_);
    if (rowoff_total > 0) rowoff_pool_.alloc(static_cast<std::size_t>(rowoff_total), stream_);
    DevBuf<int> d_steps(with_iface.size(), stream_);
    DevBuf<long long> d_ioff(iface_off.size(), stream_), d_roff(rowoff_off.size(), stream_);
    d_steps.upload(with_iface.data(), with_iface.size());
    d_ioff.upload(iface_off.data(), iface_off.size());
    d_roff.upload(rowoff_off.data(), rowoff_off.size());
    k_setup_iface<<<static_cast<unsigned>(with_iface.size()), kSetupThreads, 0, stream_>>>(
        v, d_steps.ptr, d_ioff.ptr, d_roff.ptr, d_iface.ptr, iface_pool_.ptr, rowoff_pool_.ptr);
    check_cuda(cudaGetLastError(), "k_setup_iface");
    check_cuda(cudaStreamSynchronize(stream_), "setup iface");
  }
}

template <typename T>
const cx<T>* PlaneSolver<T>::table(int kind, cd nr, cd ns, bool scalar) {
  auto key = std::make_tuple(kind + (scalar ? 8 : 0), nr.re, nr.im, ns.re, ns.im);
  auto it = tables_.find(key);
  if (it != tables_.end()) return it->second.ptr;
  DevBuf<C> t((scalar ? 2 : table_blocks<T>()) * n(), stream_);
  launch(k_build_table<T>, dim3(ceil_div(n(), kThreads)), dim3(kThreads), 0, t.ptr, kind, nr, ns,
         static_cast<int>(in_.ny), static_cast<int>(in_.nx), in_.dy, in_.dx, in_.k0, in_.dz,
         is2d() ? 0 : 1, scalar ? 1 : 0);
  const C* ptr = t.ptr;
  tables_.emplace(key, std::move(t));
  return ptr;
}

// Pass records of every step in one device pool, built before the first run that needs them:
// per step and direction the transmissions (all pairs), then the reflections (pairs whose
// indices differ); a step without reflection uses the first part only. Forward step s:
// (r, s) = (plane s, plane s + 1); the backward step from plane s + 1 to plane s swaps the
// roles (cpp/src/solver_cuda.cu:615-624).
template <typename T>
void PlaneSolver<T>::ensure_passes(bool with_backward) {
  if (pool_dirs_ >= (with_backward ? 2 : 1)) return;
  const int dirs = with_backward ? 2 : 1;
  std::vector<PassRec> host;
  for (int d = 0; d < 2; ++d) {
    pass_off_[d].assign(in_.nz, 0);
    pass_nt_[d].assign(in_.nz, 0);
    pass_nr_[d].assign(in_.nz, 0);
  }
  for (int d = 0; d < dirs; ++d) {
    const bool backward = d == 1;
    for (std::size_t s = 0; s < in_.nz; ++s) {
      const StepInfo& st = steps_[s];
      pass_off_[d][s] = static_cast<long long>(host.size());
      for (int pass = 0; pass < 2; ++pass) {
        for (std::size_t i = 0; i < st.pairs.size(); ++i) {
          const int lr = backward ? st.pairs[i].second : st.pairs[i].first;
          const int ls = backward ? st.pairs[i].first : st.pairs[i].second;
          const cd nr = index_of(lr), ns = index_of(ls);
          const bool same = nr.re == ns.re && nr.im == ns.im;
          if (pass == 1 && same) continue;
          const int kind = pass == 0 ? (backward ? kBwdT : kFwdT) : (backward ? kBwdR : kFwdR);
          // complex64 3D transmissions between equal indices: T = 1, the propagator alone
          const bool scalar = sizeof(T) != sizeof(double) && !is2d() && pass == 0 && same;
          host.push_back(PassRec{table(kind, nr, ns, scalar), static_cast<int>(i), pass,
                                 scalar ? 1 : 0});
          ++(pass == 0 ? pass_nt_[d][s] : pass_nr_[d][s]);
        }
      }
    }
  }
  pass_pool_.alloc(host.size(), stream_);
  pass_pool_.upload(host.data(), host.size());
  pool_dirs_ = dirs;
}

template <typename T>
void PlaneSolver<T>::step(int s, bool backward, bool reflect, const C* in, C* out, C* refl_out,
                          const C* add, bool want_spec, bool x_ready, bool x_next, bool need_out) {
  const StepInfo& st = steps_[s];
  const int dir = backward ? 1 : 0;
  const PassRec* ps = pass_pool_.ptr + pass_off_[dir][s];
  const int npass = pass_nt_[dir][s] + (reflect ? pass_nr_[dir][s] : 0);
  const std::uint8_t* pid = st.pid_off >= 0 ? pid_pool_.ptr + st.pid_off : nullptr;
  const int* iface = st.niface > 0 ? iface_pool_.ptr + st.iface_off : nullptr;
  // FP32 tables carry the inverse transform's 1/N already
  const T inv_n = sizeof(T) == sizeof(double) ? static_cast<T>(1.0 / static_cast<double>(n())) : T(1);
  if (is2d()) {
    Step2D<T> a;
    a.in = in;
    a.out = out;
    a.spec = spec_.ptr;
    a.pid = pid;
    a.mask = mask_.ptr;
    a.iface = iface;
    a.niface = st.niface;
    a.refl_out = refl_out;
    a.add = add;
    a.n = static_cast<int>(n());
    a.store_spec = want_spec ? 1 : 0;
    a.inv_n = inv_n;
    if (line_ept8_)
      launch(k_step2d<T, 8>, dim3(2), dim3(thr2d_), n() * sizeof(C), a, ps, npass, hy_.plan, tw_y_.ptr);
    else
      launch(k_step2d<T>, dim3(2), dim3(thr2d_), n() * sizeof(C), a, ps, npass, hy_.plan, tw_y_.ptr);
    return;
  }
  const int ny = static_cast<int>(in_.ny), nx = static_cast<int>(in_.nx);
  if (!x_ready)  // the x transform of the step's input, stored transposed for the column kernel
    launch(k_rows_fft<-1, T, true>, dim3(ceil_div(ny, sel_.rows)), dim3(sel_.threads), sel_.smem, in,
           xbuf_.ptr, ny, nx, 2, sel_.rows, hx_.plan, tw_x_.ptr);
  if constexpr (sizeof(T) == sizeof(float)) {
    if (rf_y_.cols) {
      ColStep<float> c{xbuf_.ptr, work_.ptr, want_spec ? spec_.ptr : nullptr, ny, nx, 0,
                       status_.ptr};
      launch(rf_y_.cols, dim3(nx / rf_y_.lines), dim3(kRfThreads), rf_y_.smem, c, ps, npass,
             (const Tw<float>*)tw_rf_y_.ptr);
      RowSelect<float> r;
      r.work = work_.ptr;
      r.out = out;
      r.pid = pid;
      r.mask = mask_.ptr;
      r.iface = iface;
      r.rowoff = st.rowoff_off >= 0 ? rowoff_pool_.ptr + st.rowoff_off : nullptr;
      r.refl_out = refl_out;
      r.add = add;
      r.xnext = x_next ? xbuf_.ptr : nullptr;
      r.ny = ny;
      r.nx = nx;
      r.rows = rf_x_.lines;
      r.group = 1;
      r.store_out = need_out ? 1 : 0;
      r.inv_n = inv_n;
      launch(rf_x_.rows, dim3(ny / rf_x_.lines), dim3(kRfThreads), rf_x_.smem, r, ps, npass,
             (const Tw<float>*)tw_rf_x_.ptr);
      return;
    }
  }
  if (cols_bulk_) {
    ColStep<T> c{xbuf_.ptr, work_.ptr, want_spec ? spec_.ptr : nullptr, ny, nx, cols_bulk_group_,
                 status_.ptr};
    launch(k_cols_step_bulk<T>, dim3(nx), dim3(cols_bulk_threads_),
           cols_bulk_smem<T>(ny, cols_bulk_group_), c, ps, npass, hy_.plan, tw_y_.ptr);
  } else {
    const LaunchShape& cs = npass > 1 ? cols2_ : cols1_;
    ColStep<T> c{xbuf_.ptr, work_.ptr, want_spec ? spec_.ptr : nullptr, ny, nx, cs.rows, nullptr};
    launch(k_cols_step<T>, dim3(ceil_div(nx, cs.rows)), dim3(cs.threads), cs.smem, c, ps, npass,
           hy_.plan, tw_y_.ptr);
  }
  RowSelect<T> r;
  r.work = work_.ptr;
  r.out = out;
  r.pid = pid;
  r.mask = mask_.ptr;
  r.iface = iface;
  r.rowoff = st.rowoff_off >= 0 ? rowoff_pool_.ptr + st.rowoff_off : nullptr;
  r.refl_out = refl_out;
  r.add = add;
  r.xnext = x_next ? xbuf_.ptr : nullptr;
  r.ny = ny;
  r.nx = nx;
  r.rows = sel_.rows;
  r.group = sel_.group;
  r.store_out = need_out ? 1 : 0;
  r.inv_n = inv_n;
  launch(k_rows_select<T>, dim3(ceil_div(ny, sel_.rows)), dim3(sel_.threads), sel_.smem, r, ps, npass,
         hx_.plan, tw_x_.ptr);
}

template <typename T>
void PlaneSolver<T>::fft_plane(const C* in, C* out, int ncomp, int dir) {
  const int ny = static_cast<int>(in_.ny), nx = static_cast<int>(in_.nx);
  if (is2d()) {
    const std::size_t sm = n() * sizeof(C);
    if (line_ept8_) {
      if (dir < 0)
        launch(k_line_fft<-1, T, 8>, dim3(ncomp), dim3(thr_line3_), sm, in, out, ny, ncomp, hy_.plan, tw_y_.ptr);
      else
        launch(k_line_fft<1, T, 8>, dim3(ncomp), dim3(thr_line3_), sm, in, out, ny, ncomp, hy_.plan, tw_y_.ptr);
    } else {
      if (dir < 0)
        launch(k_line_fft<-1, T>, dim3(ncomp), dim3(thr_line3_), sm, in, out, ny, ncomp, hy_.plan, tw_y_.ptr);
      else
        launch(k_line_fft<1, T>, dim3(ncomp), dim3(thr_line3_), sm, in, out, ny, ncomp, hy_.plan, tw_y_.ptr);
    }
    return;
  }
  const LaunchShape& rs = ncomp == 3 ? rows3_ : rows2_;
  const LaunchShape& cs = ncomp == 3 ? cols3_ : cols1_;
  C* tmp = ncomp == 3 ? t3_.ptr : xbuf_.ptr;
  if (dir < 0) {
    launch(k_rows_fft<-1, T>, dim3(ceil_div(ny, rs.rows)), dim3(rs.threads), rs.smem, in, tmp, ny,
           nx, ncomp, rs.rows, hx_.plan, tw_x_.ptr);
    launch(k_cols_fft<-1, T>, dim3(ceil_div(nx, cs.rows)), dim3(cs.threads), cs.smem,
           (const C*)tmp, out, ny, nx, ncomp, cs.rows, hy_.plan, tw_y_.ptr);
  } else {
    launch(k_rows_fft<1, T>, dim3(ceil_div(ny, rs.rows)), dim3(rs.threads), rs.smem, in, tmp, ny,
           nx, ncomp, rs.rows, hx_.plan, tw_x_.ptr);
    launch(k_cols_fft<1, T>, dim3(ceil_div(nx, cs.rows)), dim3(cs.threads), cs.smem,
           (const C*)tmp, out, ny, nx, ncomp, cs.rows, hy_.plan, tw_y_.ptr);
  }
}

template <typename T>
void PlaneSolver<T>::born_operator(const C* in, C* out, int combine) {
  // cpp/src/solver.cpp:262-311, for the slab in born_cur_ (set by born_step)
  const long long nn = static_cast<long long>(n());
  const BornCur<T>* cur = born_cur_.ptr;
  launch(k_born_prepare_cur<T>, dim3(ceil_div(nn, kThreads)), dim3(kThreads), 0, in, w3_.ptr, cur);
  fft_plane(w3_.ptr, w3_.ptr, 3, +1);
  launch(k_born_potential_cur<T>, dim3(ceil_div(nn, kThreads)), dim3(kThreads), 0, w3_.ptr, cur,
         nn, static_cast<T>(1.0 / static_cast<double>(nn)));
  fft_plane(w3_.ptr, w3_.ptr, 3, -1);
  // combine: out = in − G·in/2 in the same kernel
  launch(k_born_finish_cur<T>, dim3(ceil_div(nn, kThreads)), dim3(kThreads), 0,
         (const C*)w3_.ptr, out, cur, combine ? in : (const C*)nullptr);
}

template <typename T>
void PlaneSolver<T>::axpby(C* y, const C* x, cd a, cd b, long long m) {
  launch(k_axpby<T>, dim3(ceil_div(m, kThreads)), dim3(kThreads), 0, y, x, a, b, m);
}

// dst += src/N (· mask): Born increments and emitted planes are kept unnormalised.
template <typename T>
void PlaneSolver<T>::add_plane_scaled(C* dst, const C* src, const T* mask) {
  const long long n2 = 2 * static_cast<long long>(n());
  launch(k_add_plane<T>, dim3(ceil_div(n2, kThreads)), dim3(kThreads), 0, dst, src, mask,
         static_cast<T>(1.0 / static_cast<double>(n())), n2);
}

// Arnoldi step j of GMRES(30) (modified Gram-Schmidt, cpp/src/solver.cpp:150-190): w = A·v_j,
// h[i][j] = ⟨v_i, w⟩ and w −= h[i][j]·v_i for i ≤ j, v_{j+1} = w/‖w‖, the rotations. In the cycle
// graph the rotation kernel also sets the graph's condition for step j + 1; host-driven, the
// flag goes to pinned memory behind an event.
template <typename T>
void PlaneSolver<T>::arnoldi_step(int j, bool in_graph, double tol_bnorm) {
  constexpr int m = kGmresRestart;
  const long long m2 = 2 * static_cast<long long>(n());
  GmresState* st = gst_.ptr;
  born_operator(basis_[j].ptr, g_w_.ptr, 1);  // w = v_j − G v_j/2
  for (int i = 0; i <= j; ++i) {
    launch(k_dot_dev<T>, dim3(gm_dblocks_), dim3(256), 0, (const C*)basis_[i].ptr,
           (const C*)g_w_.ptr, m2, dot_partial_.ptr, &st->counter, &st->h[i * m + j]);
    launch(k_axpy_dev<T>, dim3(gm_vblocks_), dim3(kThreads), 0, g_w_.ptr, (const C*)basis_[i].ptr,
           (const cd*)&st->h[i * m + j], -1.0, m2);
  }
  launch(k_dot_dev<T>, dim3(gm_dblocks_), dim3(256), 0, (const C*)g_w_.ptr, (const C*)g_w_.ptr,
         m2, dot_partial_.ptr, &st->counter, &st->dot);
  launch(k_norm_scale<T>, dim3(gm_vblocks_), dim3(kThreads), 0, basis_[j + 1].ptr,
         (const C*)g_w_.ptr, (const cd*)&st->dot, &st->nrm, m2);
  if (in_graph) {
    launch(k_gmres_givens_cond, dim3(1), dim3(32), 0, st, j, conds_);
  } else {
    launch(k_gmres_givens, dim3(1), dim3(32), 0, st, j, tol_bnorm);
    check_cuda(cudaMemcpyAsync(flags_host_.ptr + j, &st->flag[j], sizeof(int), cudaMemcpyDeviceToHost,
                               stream_), "flag");
    check_cuda(cudaEventRecord(gmres_events_[j], stream_), "event");
  }
}

template <typename T>
void PlaneSolver<T>::gmres_alloc() {
  if (!basis_.empty()) return;
  const long long m2 = 2 * static_cast<long long>(n());
  constexpr int m = kGmresRestart;
  for (int i = 0; i <= m; ++i) basis_.emplace_back(static_cast<std::size_t>(m2), stream_);
  std::vector<C*> ptrs;
  for (auto& b : basis_) ptrs.push_back(b.ptr);
  basis_ptrs_.alloc(ptrs.size(), stream_);
  basis_ptrs_.upload(ptrs.data(), ptrs.size());
  gst_.alloc(1, stream_);
  check_cuda(cudaMemsetAsync(gst_.ptr, 0, sizeof(GmresState), stream_), "memset");
  dot_partial_.alloc(kDotBlocks, stream_);
  flags_host_.alloc(m + 2);
  for (auto& e : gmres_events_) e.create();
  gm_vblocks_ = static_cast<int>(ceil_div(m2, static_cast<long long>(kThreads)));
  gm_dblocks_ = static_cast<int>(std::min<long long>(kDotBlocks, ceil_div(m2, 256LL)));
}

// The Born step of born_step (P_½, right-hand side, GMRES(30), P_½^{±}, inverse transform) as
// one CUDA graph, built once per solver: the buffers it names are fixed, the slab comes from
// born_cur_ and the tolerance from the state, so one graph serves every Born slab and both
// directions. The host loop's decisions become conditional nodes (a handle per node) set by
// one-thread kernels (gmres_kernels.cuh) with the same FP64 comparisons:
//   P_½, G·x, y = rhs, ‖rhs‖ → init
//   WHILE active:  A·y, β → restart
//     IF cycle:    v_0 = r/β, g; arm; IF step_0 {Arnoldi 0} … IF step_29 {Arnoldi 29};
//                  cycle_done; back substitution; y += Σ y_i v_i
//       IF done:   A·y, ‖rhs − A·y‖ → final
//   P_½^{±}, F⁻¹
// The host launches it after writing the slab record and waits for nothing.
template <typename T>
void PlaneSolver<T>::build_born_graph() {
  if (born_graph_.exec) return;
  const std::int64_t launches = launches_;
  const long long nn = static_cast<long long>(n());
  const long long m2 = 2 * nn;
  GmresState* st = gst_.ptr;
  cudaGraph_t top = nullptr;
  check_cuda(cudaGraphCreate(&top, 0), "graph create");
  born_graph_.g = top;
  auto handle = [&](cudaGraphConditionalHandle& h) {
    check_cuda(cudaGraphConditionalHandleCreate(&h, top, 0u, cudaGraphCondAssignDefault),
               "conditional handle");
  };
  handle(conds_.active);
  handle(conds_.cycle);
  handle(conds_.done);
  for (auto& h : conds_.step) handle(h);
  // captures what `f` enqueues into graph g after `deps`; returns the capture's last nodes
  auto capture = [&](cudaGraph_t g, std::vector<cudaGraphNode_t> deps, auto&& f) {
    check_cuda(cudaStreamBeginCaptureToGraph(stream_, g, deps.empty() ? nullptr : deps.data(),
                                             nullptr, deps.size(),
                                             cudaStreamCaptureModeThreadLocal),
               "capture");
    f();
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* last = nullptr;
    std::size_t nlast = 0;
    check_cuda(cudaStreamGetCaptureInfo(stream_, &cs, nullptr, nullptr, &last, &nlast), "capture");
    std::vector<cudaGraphNode_t> out(last, last + nlast);
    cudaGraph_t g2;
    check_cuda(cudaStreamEndCapture(stream_, &g2), "capture");
    return out;
  };
  // adds a conditional node after `deps`; returns it and its body
  auto conditional = [&](cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps,
                         cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                         cudaGraph_t& body) {
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    check_cuda(cudaGraphAddNode(&node, g, deps.empty() ? nullptr : deps.data(), deps.size(), &p),
               "conditional node");
    body = p.conditional.phGraph_out[0];
    return std::vector<cudaGraphNode_t>{node};
  };
  const BornCur<T>* cur = born_cur_.ptr;
  const dim3 pts(ceil_div(nn, kThreads)), vec(gm_vblocks_), blk(kThreads);
  auto dot = [&](const C* u, const C* v, cd* out) {
    launch(k_dot_dev<T>, dim3(gm_dblocks_), dim3(256), 0, u, v, m2, dot_partial_.ptr, &st->counter,
           out);
  };
  auto copy = [&](C* dst, const C* src) {
    check_cuda(cudaMemcpyAsync(dst, src, m2 * sizeof(C), cudaMemcpyDeviceToDevice, stream_), "copy");
  };
  std::vector<cudaGraphNode_t> d = capture(top, {}, [&] {
    launch(k_born_half_cur<T>, pts, blk, 0, (const C*)spec_.ptr, g_x_.ptr, cur, 0);
    born_operator(g_x_.ptr, g_rhs_.ptr);
    copy(g_y_.ptr, g_rhs_.ptr);
    dot(g_rhs_.ptr, g_rhs_.ptr, &st->dot);
    launch(k_gmres_init, dim3(1), dim3(32), 0, st, in_.gmres_tol, conds_);
  });
  cudaGraph_t wbody, cbody, dbody;
  d = conditional(top, d, conds_.active, cudaGraphCondTypeWhile, wbody);
  std::vector<cudaGraphNode_t> w = capture(wbody, {}, [&] {
    born_operator(g_y_.ptr, g_w_.ptr, 1);
    copy(basis_[0].ptr, g_rhs_.ptr);
    axpby(basis_[0].ptr, g_w_.ptr, cd{-1.0, 0.0}, cd{1.0, 0.0}, m2);
    dot(basis_[0].ptr, basis_[0].ptr, &st->dot);
    launch(k_gmres_restart, dim3(1), dim3(32), 0, st, conds_);
  });
  conditional(wbody, w, conds_.cycle, cudaGraphCondTypeIf, cbody);
  std::vector<cudaGraphNode_t> c = capture(cbody, {}, [&] {
    launch(k_norm_scale<T>, vec, blk, 0, basis_[0].ptr, (const C*)basis_[0].ptr,
           (const cd*)&st->dot, &st->nrm, m2);
    launch(k_gmres_start, dim3(1), dim3(64), 0, st, -1.0);
    launch(k_gmres_arm, dim3(1), dim3(32), 0, conds_);
  });
  for (int j = 0; j < kGmresRestart; ++j) {
    cudaGraph_t sbody;
    c = conditional(cbody, c, conds_.step[j], cudaGraphCondTypeIf, sbody);
    capture(sbody, {}, [&] { arnoldi_step(j, true, 0.0); });
  }
  c = capture(cbody, c, [&] {
    launch(k_gmres_cycle_done, dim3(1), dim3(32), 0, st, conds_);
    launch(k_gmres_backsolve, dim3(1), dim3(32), 0, st, -1);
    launch(k_axpy_basis<T>, vec, blk, 0, g_y_.ptr, (C* const*)basis_ptrs_.ptr, (const GmresState*)st,
           m2);
  });
  conditional(cbody, c, conds_.done, cudaGraphCondTypeIf, dbody);
  capture(dbody, {}, [&] {
    born_operator(g_y_.ptr, g_w_.ptr, 1);
    copy(g_tmp_.ptr, g_rhs_.ptr);
    axpby(g_tmp_.ptr, g_w_.ptr, cd{-1.0, 0.0}, cd{1.0, 0.0}, m2);
    dot(g_tmp_.ptr, g_tmp_.ptr, &st->dot);
    launch(k_gmres_final, dim3(1), dim3(32), 0, st, conds_);
  });
  capture(top, d, [&] {
    launch(k_born_half_cur<T>, pts, blk, 0, (const C*)g_y_.ptr, g_y_.ptr, cur, 1);
    fft_plane(g_y_.ptr, inc_.ptr, 2, +1);
  });
  check_cuda(cudaGraphInstantiate(&born_graph_.exec, top, 0), "instantiate");
  launches_ = launches;
}

// GMRES(30) for (1 − G/2)·y = rhs with start y = rhs (cpp/src/solver.cpp:130-207, :336-342),
// driven from the host (BWPM_GMRES=host; the default runs the whole Born step as the graph of
// build_born_graph): scalar work on the device (gmres_kernels.cuh), the host waiting for ‖rhs‖,
// per restart for β and the final residual, and per Arnoldi step for the previous step's flag
// while the next one runs.
template <typename T>
void PlaneSolver<T>::gmres() {
  const long long m2 = 2 * static_cast<long long>(n());
  constexpr int m = kGmresRestart;
  const double tol = in_.gmres_tol;
  gmres_alloc();
  GmresState* st = gst_.ptr;
  auto host_norm = [&](const C* u) {  // ‖u‖ read back on the host
    launch(k_dot_dev<T>, dim3(gm_dblocks_), dim3(256), 0, u, u, m2, dot_partial_.ptr, &st->counter,
           &st->dot);
    cd d;
    check_cuda(cudaMemcpyAsync(&d, &st->dot, sizeof(cd), cudaMemcpyDeviceToHost, stream_), "dot");
    check_cuda(cudaStreamSynchronize(stream_), "dot");
    return std::sqrt(d.re);
  };
  check_cuda(cudaMemcpyAsync(g_y_.ptr, g_rhs_.ptr, m2 * sizeof(C), cudaMemcpyDeviceToDevice, stream_), "copy");
  const double bnorm = host_norm(g_rhs_.ptr);
  if (bnorm == 0.0) return;
  for (int outer = 0; outer < 100; ++outer) {
    born_operator(g_y_.ptr, g_w_.ptr, 1);
    ++gmres_applies_;
    check_cuda(cudaMemcpyAsync(basis_[0].ptr, g_rhs_.ptr, m2 * sizeof(C), cudaMemcpyDeviceToDevice, stream_), "copy");
    axpby(basis_[0].ptr, g_w_.ptr, cd{-1.0, 0.0}, cd{1.0, 0.0}, m2);
    const double beta = host_norm(basis_[0].ptr);  // leaves the dot in st->dot
    if (beta <= tol * bnorm) return;
    launch(k_norm_scale<T>, dim3(gm_vblocks_), dim3(kThreads), 0, basis_[0].ptr,
           (const C*)basis_[0].ptr, (const cd*)&st->dot, &st->nrm, m2);
    launch(k_gmres_start, dim3(1), dim3(64), 0, st, tol * bnorm);
    int used = 0;
    bool done = false;
    auto converged = [&](int j) {  // waits for the flag of Arnoldi step j
      check_cuda(cudaEventSynchronize(gmres_events_[j]), "gmres flag");
      return flags_host_.ptr[j] != 0;
    };
    for (int j = 0; j < m; ++j) {
      arnoldi_step(j, false, tol * bnorm);
      ++gmres_applies_;
      // step j is queued; the previous step's flag decides whether it counts
      if (j > 0 && converged(j - 1)) {
        used = j;
        done = true;
        break;
      }
      used = j + 1;
    }
    if (!done && converged(used - 1)) done = true;
    launch(k_gmres_backsolve, dim3(1), dim3(32), 0, st, used);
    for (int i = 0; i < used; ++i)
      launch(k_axpy_dev<T>, dim3(gm_vblocks_), dim3(kThreads), 0, g_y_.ptr, (const C*)basis_[i].ptr,
             (const cd*)&st->y[i], 1.0, m2);
    if (done) {
      born_operator(g_y_.ptr, g_w_.ptr, 1);
      ++gmres_applies_;
      check_cuda(cudaMemcpyAsync(g_tmp_.ptr, g_rhs_.ptr, m2 * sizeof(C), cudaMemcpyDeviceToDevice, stream_), "copy");
      axpby(g_tmp_.ptr, g_w_.ptr, cd{-1.0, 0.0}, cd{1.0, 0.0}, m2);
      if (host_norm(g_tmp_.ptr) <= tol * bnorm * 10.0) return;
    }
  }
  throw std::runtime_error("GMRES did not converge in the Born step (CUDA)");
}

// inc = F⁻¹{P_½^{±}·y}·N, (1 − G/2)y = G·P_½·F{e} (cpp/src/solver.cpp:313-350); the caller adds
// inc/N (scaled in the add).
template <typename T>
void PlaneSolver<T>::born_step(const C* spec, C* inc, int slot, int dir) {
  const BornGrid g = born_grid(slot);
  const long long nn = static_cast<long long>(n());
  launch(k_set_born_cur<T>, dim3(1), dim3(32), 0, born_cur_.ptr,
         BornCur<T>{g, dir, pot_.ptr + slot * nn});
  const char* gm = std::getenv("BWPM_GMRES");
  if (!(gm && std::strcmp(gm, "host") == 0) && spec == spec_.ptr && inc == inc_.ptr) {
    gmres_alloc();
    build_born_graph();
    check_cuda(cudaGraphLaunch(born_graph_.exec, stream_), "graph launch");
    ++launches_;
    born_graph_used_ = true;
    return;
  }
  launch(k_born_half<T>, dim3(ceil_div(nn, kThreads)), dim3(kThreads), 0, spec, g_x_.ptr, g, 1.0);
  born_operator(g_x_.ptr, g_rhs_.ptr);
  gmres();
  launch(k_born_half<T>, dim3(ceil_div(nn, kThreads)), dim3(kThreads), 0, (const C*)g_y_.ptr,
         g_y_.ptr, g, dir > 0 ? 1.0 : -1.0);
  fft_plane(g_y_.ptr, inc, 2, +1);
}

// Ŝ_m = F{V·F⁻¹{e^{i k_z s_m}(Ê⊥, Ê_z)}} into sources_ (cpp/src/solver.cpp:215-260).
template <typename T>
void PlaneSolver<T>::born_sources(const C* spec, int slot, int dir) {
  const BornGrid g = born_grid(slot);
  const long long nn = static_cast<long long>(n());
  const double r3 = 0.57735026918962576451;
  const double gauss[2] = {(1.0 - r3) / 2.0, (1.0 + r3) / 2.0};
  for (int m = 0; m < 2; ++m) {
    const double dist = (dir > 0 ? gauss[m] : 1.0 - gauss[m]) * in_.dz;
    launch(k_born_prepare<T>, dim3(ceil_div(nn, kThreads)), dim3(kThreads), 0, spec, w3_.ptr, g, dir, dist);
    fft_plane(w3_.ptr, w3_.ptr, 3, +1);
    launch(k_born_potential<T>, dim3(ceil_div(nn, kThreads)), dim3(kThreads), 0, w3_.ptr,
           (const C*)(pot_.ptr + slot * nn), nn, static_cast<T>(1.0 / static_cast<double>(nn)));
    fft_plane(w3_.ptr, sources_.ptr + 3 * nn * m, 3, -1);
  }
}

// Field radiated by sources_ in direction `dir` at the right slab edge, real space, times N
// (cpp/src/solver.cpp:352-382); the caller scales by 1/N when adding.
template <typename T>
void PlaneSolver<T>::born_emission(int slot, int dir, C* plane) {
  const BornGrid g = born_grid(slot);
  const long long nn = static_cast<long long>(n());
  launch(k_born_emit<T>, dim3(ceil_div(nn, kThreads)), dim3(kThreads), 0, (const C*)sources_.ptr,
         inc_.ptr, g, dir);
  fft_plane(inc_.ptr, plane, 2, +1);
}

template <typename T>
void PlaneSolver<T>::sweeps(int iterations, const std::vector<int>& keep_slot, DevBuf<C>& kept_f,
                            DevBuf<C>& kept_b, DevBuf<C>& t_iter, DevBuf<C>& r_iter) {
  const std::size_t nn = n();
  const long long n2 = 2 * static_cast<long long>(nn);
  const int nz = static_cast<int>(in_.nz);
  const int iters = std::max(iterations, 1);
  auto copy = [&](C* dst, const C* src) {
    check_cuda(cudaMemcpyAsync(dst, src, n2 * sizeof(C), cudaMemcpyDeviceToDevice, stream_), "copy");
  };
  C* e = e_.ptr;
  C* next = next_.ptr;
  const bool born = !hosts_.empty();
  for (int it = 0; it < iters; ++it) {
    const bool last = it == iters - 1;
    copy(e, input_.ptr);
    if (last && keep_slot[0] >= 0) copy(kept_f.ptr + keep_slot[0] * n2, e);
    for (int p = 0; p < nz; ++p) {
      const StepInfo& st = steps_[p];
      const bool reflect = iterations > 0 && st.niface > 0;
      const C* add = (it > 0 && st.niface > 0) ? src_fwd_.ptr + 2 * st.iface_off : nullptr;
      const bool host = born && st.host_slot >= 0;
      // 3D without Born slabs: each step leaves the next one's x transform (nothing else
      // touches the plane between two steps of a sweep)
      const bool fuse = !is2d() && !born;
      step(p, false, reflect, e, next, reflect ? src_bwd_.ptr + 2 * st.iface_off : nullptr, add, host,
           fuse && p > 0, fuse && p + 1 < nz,
           !(fuse && p + 1 < nz) || (last && keep_slot[p + 1] >= 0));
      if (host) {
        born_step(spec_.ptr, inc_.ptr, st.host_slot, +1);
        add_plane_scaled(next, inc_.ptr, mask_.ptr);
        if (iterations > 0) {
          born_sources(spec_.ptr, st.host_slot, +1);
          born_emission(st.host_slot, -1, born_bwd_.ptr + st.host_slot * n2);  // born_bwd[p + 1]
        }
      }
      std::swap(e, next);
      if (it > 0 && host) add_plane_scaled(e, born_fwd_.ptr + st.host_slot * n2, nullptr);  // born_fwd[p + 1]
      if (last && keep_slot[p + 1] >= 0) copy(kept_f.ptr + keep_slot[p + 1] * n2, e);
    }
    if (iterations > 0) copy(t_iter.ptr + it * n2, e);
    if (iterations == 0) break;
    check_cuda(cudaMemsetAsync(e, 0, n2 * sizeof(C), stream_), "memset");
    if (born && steps_[nz - 1].host_slot >= 0)
      add_plane_scaled(e, born_bwd_.ptr + steps_[nz - 1].host_slot * n2, nullptr);  // born_bwd[nz]
    if (last && keep_slot[nz] >= 0) copy(kept_b.ptr + keep_slot[nz] * n2, e);
    for (int p = nz; p > 0; --p) {
      const StepInfo& st = steps_[p - 1];
      if (born && st.host_slot >= 0) {
        fft_plane(e, spec_.ptr, 2, -1);
        born_sources(spec_.ptr, st.host_slot, -1);
        born_emission(st.host_slot, +1, born_fwd_.ptr + st.host_slot * n2);  // born_fwd[p]
        born_step(spec_.ptr, inc_.ptr, st.host_slot, -1);
        add_plane_scaled(e, inc_.ptr, nullptr);  // R2 at plane p
      }
      const bool reflect = st.niface > 0;
      const C* add = st.niface > 0 ? src_bwd_.ptr + 2 * st.iface_off : nullptr;
      const bool fuse = !is2d() && !born;
      step(p - 1, true, reflect, e, next, reflect ? src_fwd_.ptr + 2 * st.iface_off : nullptr, add, false,
           fuse && p < nz, fuse && p > 1, !(fuse && p > 1) || (last && keep_slot[p - 1] >= 0));
      std::swap(e, next);
      if (born && p >= 2 && steps_[p - 2].host_slot >= 0)
        add_plane_scaled(e, born_bwd_.ptr + steps_[p - 2].host_slot * n2, nullptr);  // born_bwd[p − 1]
      if (last && keep_slot[p - 1] >= 0) copy(kept_b.ptr + keep_slot[p - 1] * n2, e);
    }
    copy(r_iter.ptr + it * n2, e);
  }
  last_e_ = e;
}

template <typename T>
void PlaneSolver<T>::run(const cd* field, int iterations, const std::int64_t* keep,
                         std::size_t nkeep, RunOutputs& out) {
  check_cuda(cudaSetDevice(in_.device), "cudaSetDevice");
  const std::size_t nn = n();
  const long long n2 = 2 * static_cast<long long>(nn);
  const int nz = static_cast<int>(in_.nz);
  const int iters = std::max(iterations, 1);
  // keep planes: device slots
  std::vector<int> keep_slot(nz + 1, -1);
  for (std::size_t i = 0; i < nkeep; ++i)
    if (keep[i] >= 0 && keep[i] <= nz) keep_slot[keep[i]] = static_cast<int>(i);
  DevBuf<C> kept_f(nkeep * 2 * nn, stream_), kept_b(nkeep * 2 * nn, stream_), t_iter, r_iter;
  if (iterations > 0) {
    t_iter.alloc(iterations * 2 * nn, stream_);
    r_iter.alloc(iterations * 2 * nn, stream_);
  }
  ensure_passes(iterations > 0);
  check_cuda(cudaMemcpyAsync(stage_.ptr, field, n2 * sizeof(cd), cudaMemcpyHostToDevice, stream_), "field upload");
  launch(k_convert<T, double>, dim3(ceil_div(n2, kThreads)), dim3(kThreads), 0, input_.ptr,
         (const cd*)stage_.ptr, n2);
  sweeps(iterations, keep_slot, kept_f, kept_b, t_iter, r_iter);
  C* e = last_e_;
  // outputs
  auto download = [&](const C* src, cd* dst) {
    if (!dst) return;
    launch(k_convert<double, T>, dim3(ceil_div(n2, kThreads)), dim3(kThreads), 0, stage_.ptr, src, n2);
    check_cuda(cudaMemcpyAsync(dst, stage_.ptr, n2 * sizeof(cd), cudaMemcpyDeviceToHost, stream_), "download");
    check_cuda(cudaStreamSynchronize(stream_), "download");
  };
  download(iterations > 0 ? t_iter.ptr + (iterations - 1) * n2 : e, out.transmitted);
  if (out.reflected) {
    if (iterations > 0)
      download(r_iter.ptr + (iterations - 1) * n2, out.reflected);
    else
      std::memset(static_cast<void*>(out.reflected), 0, n2 * sizeof(cd));
  }
  for (int it = 0; it < iterations; ++it) {
    if (out.transmitted_iter) download(t_iter.ptr + it * n2, out.transmitted_iter + it * n2);
    if (out.reflected_iter) download(r_iter.ptr + it * n2, out.reflected_iter + it * n2);
  }
  for (std::size_t i = 0; i < nkeep; ++i) {
    if (out.forward) download(kept_f.ptr + i * n2, out.forward + i * n2);
    if (out.backward && iterations > 0) download(kept_b.ptr + i * n2, out.backward + i * n2);
  }
  out.stored_values = iterations > 0 ? 2 * iface_total_ : 0;
  check_cuda(cudaStreamSynchronize(stream_), "synchronize");
  if (born_graph_used_) {
    born_graph_used_ = false;
    GmresState hs;
    check_cuda(cudaMemcpy(&hs, gst_.ptr, sizeof(GmresState), cudaMemcpyDeviceToHost), "gmres state");
    gmres_applies_ += hs.applies;
    char* base = reinterpret_cast<char*>(gst_.ptr);
    check_cuda(cudaMemsetAsync(base + offsetof(GmresState, err), 0, sizeof(int), stream_),
               "gmres state");
    check_cuda(cudaMemsetAsync(base + offsetof(GmresState, applies), 0, sizeof(long long), stream_),
               "gmres state");
    if (hs.err) throw std::runtime_error("GMRES did not converge in the Born step (CUDA)");
  }
  if (status_.ptr) {
    int st = 0;
    check_cuda(cudaMemcpy(&st, status_.ptr, sizeof(int), cudaMemcpyDeviceToHost), "status");
    if (st) {
      check_cuda(cudaMemsetAsync(status_.ptr, 0, sizeof(int), stream_), "status");
      throw std::runtime_error("a bulk copy of the 3D slab step did not complete in time");
    }
  }
}

template <typename T>
std::size_t PlaneSolver<T>::device_bytes() const {
  std::size_t b = 0;
  for (auto& kv : tables_) b += kv.second.bytes();
  for (const auto* d : {&input_, &e_, &next_, &spec_, &xbuf_, &work_, &src_fwd_, &src_bwd_, &pot_,
                        &born_fwd_, &born_bwd_, &w3_, &t3_, &sources_})
    b += d->bytes();
  return b + pid_pool_.bytes() + iface_pool_.bytes() + rowoff_pool_.bytes() + mask_.bytes();
}

}  // namespace

std::unique_ptr<Solver> make_plane_solver(SolverInput in, int precision) {
  if (precision == 64) return std::make_unique<PlaneSolver<double>>(std::move(in));
  if (precision == 32) return std::make_unique<PlaneSolver<float>>(std::move(in));
  throw invalid_argument("precision must be 64 or 32");
}

namespace {
__global__ void k_interface(int reflection, const double* kx, const double* ky, long long n,
                            cd n_in, cd n_out, double k0, cd* out) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  cd m[3];
  interface_matrix(reflection != 0, kx[i], ky[i], n_in, n_out, k0, m);
  out[4 * i] = m[0];
  out[4 * i + 1] = m[1];
  out[4 * i + 2] = m[1];
  out[4 * i + 3] = m[2];
}

__global__ void k_kz(cd index, double k0, const double* kp2, long long n, cd* out) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i < n) out[i] = kz_of(index, k0, kp2[i]);
}
}  // namespace

void interface_matrices(int reflection, const double* kx, const double* ky, std::size_t n,
                        cd n_in, cd n_out, double k0, cd* out) {
  if (n == 0) return;
  DevBuf<double> dkx(n), dky(n);
  DevBuf<cd> dout(4 * n);
  check_cuda(cudaMemcpy(dkx.ptr, kx, n * sizeof(double), cudaMemcpyHostToDevice), "upload");
  check_cuda(cudaMemcpy(dky.ptr, ky, n * sizeof(double), cudaMemcpyHostToDevice), "upload");
  k_interface<<<ceil_div(n, kThreads), kThreads>>>(reflection, dkx.ptr, dky.ptr,
                                                    static_cast<long long>(n), n_in, n_out, k0, dout.ptr);
  check_cuda(cudaGetLastError(), "k_interface");
  check_cuda(cudaMemcpy(out, dout.ptr, 4 * n * sizeof(cd), cudaMemcpyDeviceToHost), "download");
}

void longitudinal_wavenumbers(cd index, double k0, const double* kp2, std::size_t n, cd* out) {
  if (n == 0) return;
  DevBuf<double> d(n);
  DevBuf<cd> o(n);
  check_cuda(cudaMemcpy(d.ptr, kp2, n * sizeof(double), cudaMemcpyHostToDevice), "upload");
  k_kz<<<ceil_div(n, kThreads), kThreads>>>(index, k0, d.ptr, static_cast<long long>(n), o.ptr);
  check_cuda(cudaGetLastError(), "k_kz");
  check_cuda(cudaMemcpy(out, o.ptr, n * sizeof(cd), cudaMemcpyDeviceToHost), "download");
}

int device_count() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

}  // namespace bwpm
