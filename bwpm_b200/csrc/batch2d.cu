// Batched resident 2D engine: host preparation, size classes and launches.
//
// Preparation turns each solve's int32 labels (nz, ny) into per-step records (pairs, uint8
// pair-id planes deduplicated within the solve, interface pixel lists, pass lists of the four
// table-1 kinds; cpp/src/solver.cpp:384-417, :444-460) and registers one operator table per
// (kind, ñ_r, ñ_s) and solve, built on the device in FP64 and stored as complex64 for E_x (m00)
// and E_y (m11). Work items (solve, component) are grouped into size classes by CTA width; each
// class is one persistent kernel on its own stream, all launched together.
#include <algorithm>
#include <cstdlib>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <thread>
#include <tuple>
#include <unordered_map>

#include "batch2d.hpp"
#include "devbuf.hpp"
#include "interface.cuh"
#include "plan.hpp"
#include "resident2d.cuh"
#include "rgen.cuh"
#include "variants.hpp"

namespace bwpm {
namespace {

constexpr int kClassThreads[] = {64, 128, 256, 512};
constexpr int kGenericClasses = 4;
constexpr int kMaxFixedLengths = 28;
constexpr int kMaxRt = 12;
constexpr int kRtBase = kGenericClasses + kMaxFixedLengths;  // classes of the run-time-length kernels
constexpr int kNumClasses = kRtBase + kMaxRt;  // [4, kRtBase): fixed lengths, then E values
constexpr int kTuneScale = 4;     // autotuning runs keep 1/kTuneScale of every chain
constexpr int kTuneMinSlabs = 8;

// distinct lengths with compiled variants, increasing; class kGenericClasses + i serves entry i
const std::vector<int>& fixed_lengths() {
  static const std::vector<int> lengths = [] {
    std::vector<int> v;
    for (auto& f : fixed_variants())
      if (v.empty() || v.back() != f.n) v.push_back(f.n);
    if (static_cast<int>(v.size()) > kMaxFixedLengths) throw std::logic_error("too many fixed lengths");
    return v;
  }();
  return lengths;
}

int fixed_length_index(int n) {
  const auto& l = fixed_lengths();
  auto it = std::lower_bound(l.begin(), l.end(), n);
  return it != l.end() && *it == n ? static_cast<int>(it - l.begin()) : -1;
}

// Radices of a length n for a run-time-length kernel with E values per thread: the powers of two
// as 8s (4s, 2s) when E allows, then 3s and 5s; empty if n has another prime factor. Stages
// whose radix does not divide E run as gather stages (rgen.cuh).
std::vector<int> rt_radices(int n, int e) {
  std::vector<int> r;
  int m = n, twos = 0;
  while (m % 2 == 0) {
    m /= 2;
    ++twos;
  }
  const int big = e % 8 == 0 ? 8 : e % 4 == 0 ? 4 : e % 2 == 0 ? 2 : 4;
  const int lb = big == 8 ? 3 : big == 4 ? 2 : 1;
  while (twos >= lb) {
    r.push_back(big);
    twos -= lb;
  }
  if (twos == 2) r.push_back(4);
  if (twos == 1) r.push_back(2);
  for (int p : {3, 5})
    while (m % p == 0) {
      r.push_back(p);
      m /= p;
    }
  if (m != 1) return {};
  return r;
}

// Position in rt_variants() of the run-time-length kernel for length n, or −1: among the E
// that divide n within the kernel's thread limit, the smallest estimated per-thread work over
// the stages (measured: more threads with fewer values each beat fewer stages). A wide form
// counts only where its default form cannot run n, and at 1.2× its estimate (its 128 registers
// spill: 3645 points run faster with E = 15 on 243 threads than with wide E = 9 on 405).
// BWPM_RT_E=<E> (tuning measurements) takes the kernel with that E where it can run n.
int rt_choice(int n) {
  const auto& rv = rt_variants();
  if (rt_smem_bytes(n) > 220 * 1024) return -1;
  int best = -1;
  double best_score = 1e30;
  const char* force = std::getenv("BWPM_RT_E");
  const int forced_e = force ? std::atoi(force) : 0;
  for (std::size_t i = 0; i < rv.size(); ++i) {
    const int e = rv[i].e;
    const bool wide = rv[i].max_threads > rg::rt_max_threads(e);
    if (n % e || n / e > rv[i].max_threads || (wide && n / e <= rg::rt_max_threads(e))) continue;
    const std::vector<int> r = rt_radices(n, e);
    if (r.empty()) continue;
    if (e == forced_e) return static_cast<int>(i);
    // a stage costs about (8 + E) value-times per thread (E values plus fixed overhead), twice
    // for a gather stage
    double score = 0;
    for (int x : r) score += (e % x == 0 ? 1.0 : 2.0) * (8.0 + e);
    if (wide) score *= 1.2;
    if (score < best_score - 1e-9) {
      best_score = score;
      best = static_cast<int>(i);
    }
  }
  return best;
}

// indices into fixed_variants() of the variants of length n (first: the default)
std::vector<int> variants_of(int n) {
  std::vector<int> v;
  const auto& all = fixed_variants();
  for (std::size_t i = 0; i < all.size(); ++i)
    if (all[i].n == n) v.push_back(static_cast<int>(i));
  return v;
}


// Twiddles of a variant: the stage twiddles of its per-CTA transform (N/C points); for a line
// split over C CTAs followed by the cross twiddles w_N^{c·k1} (c < C, k1 < N/C), all (hi, lo).
std::vector<Tw<float>> variant_twiddles(const FixedVariant& f) {
  const int m = f.n / f.cluster;
  const HostPlan hp = make_plan_radices(m, f.radices);
  std::vector<Tw<float>> t = twiddles_for<float>(hp);
  if (f.cluster == 1) return t;
  t.resize(static_cast<std::size_t>(hp.plan.rootoff));  // the M − 1 stage twiddles
  const double two_pi = 6.283185307179586476925286766559;
  for (int c = 0; c < f.cluster; ++c)
    for (int k = 0; k < m; ++k) {
      const long long e = (static_cast<long long>(c) * k) % f.n;
      const double a = -two_pi * static_cast<double>(e) / static_cast<double>(f.n);
      const cd w{std::cos(a), std::sin(a)};
      const cf h{static_cast<float>(w.re), static_cast<float>(w.im)};
      t.push_back(Tw<float>{h, cf{static_cast<float>(w.re - h.re), static_cast<float>(w.im - h.im)}});
    }
  return t;
}

// Operator table job: M/N of `kind` for (ñ_r, ñ_s), entry m00 (E_x) at out[0..2N) and m11 (E_y)
// at out[2N..4N), each as N hi values then N lo values with M/N = hi + lo (built in FP64; the
// inverse transform's 1/N is folded in).
struct TableJob {
  cf* out;
  cd nr, ns;
  double dy, k0, dz;
  int n, kind;
};

__global__ void k_table_jobs(const TableJob* jobs) {
  const TableJob j = jobs[blockIdx.y];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= j.n) return;
  const double ky = fftfreq(q, j.n, j.dy);
  cd m[3];
  operator_matrix(j.kind, 0.0, ky, j.nr, j.ns, j.k0, j.dz, m);
  const double inv_n = 1.0 / static_cast<double>(j.n);
  for (int c = 0; c < 2; ++c) {
    const cd v = m[2 * c] * inv_n;
    const cf hi = cast<float>(v);
    j.out[2 * c * j.n + q] = hi;
    j.out[(2 * c + 1) * j.n + q] = cf{static_cast<float>(v.re - hi.re), static_cast<float>(v.im - hi.im)};
  }
}

// Flux weights Re k_z·(1 + [E_y] k_y²/|k_z|²)·dy/ny of a medium (src/bwpm/fpwpm.py:205-216).
struct WeightJob {
  double* out;
  cd index;
  double dy, k0;
  int n, comp;
};

__global__ void k_weight_jobs(const WeightJob* jobs) {
  const WeightJob j = jobs[blockIdx.y];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= j.n) return;
  const double ky = fftfreq(q, j.n, j.dy);
  const cd kz = kz_of(j.index, j.k0, ky * ky);
  double w = kz.re * j.dy / j.n;
  if (j.comp == 1) w *= 1.0 + ky * ky / (kz.re * kz.re + kz.im * kz.im);
  j.out[q] = w;
}

// Scatter packed complex128 inputs (ny, 2) per solve into the per-item complex64 lines.
struct ItemIo {
  long long packed;  // offset of the solve's (ny, 2) block in the packed arrays
  cf* line_in;
  const cf* line_t;
  const cf* line_r;
  int n, comp;
};

__global__ void k_unpack_inputs(const ItemIo* io, const cd* packed) {
  const ItemIo j = io[blockIdx.y];
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < j.n; q += gridDim.x * blockDim.x)
    j.line_in[q] = cast<float>(packed[j.packed + 2 * q + j.comp]);
}

__global__ void k_pack_outputs(const ItemIo* io, cd* out) {
  // out: per solve (transmitted (ny, 2), reflected (ny, 2)); components without an item stay 0
  const ItemIo j = io[blockIdx.y];
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < j.n; q += gridDim.x * blockDim.x) {
    out[2 * j.packed + 2 * q + j.comp] = cast<double>(j.line_t[q]);
    out[2 * j.packed + 2 * j.n + 2 * q + j.comp] = cast<double>(j.line_r[q]);
  }
}

}  // namespace

// One solve with its host-side records (validated, pairs, pair ids, interface lists, passes);
// built by prepare_solve() off the launch path, added to a batch by add_prepared().
struct PreparedSolve {
  Solve2D in;
  // offsets into the pools
  long long step_base = 0, pass_base = 0, pid_base = 0, iface_base = 0, table_base = 0;
  long long iface_count = 0;
  long long packed = 0;
  std::vector<R2Step> steps;
  std::vector<R2Pass> passes;
  std::vector<std::uint8_t> pids;
  std::vector<int> iface;
  std::vector<std::tuple<int, cd, cd>> tables;  // (kind, ñ_r, ñ_s) per table slot
  int items[2] = {-1, -1};
  bool built = false;  // host records built
};

namespace {
using HostSolve = PreparedSolve;

struct Item {
  int solve, comp, cls, n;
  double cost;
};

void validate2d(const Solve2D& s) {
  if (s.ny < 2) throw invalid_argument("ny must be >= 2");
  if (s.nz < 1) throw invalid_argument("nz must be >= 1");
  if (s.labels.size() != static_cast<std::size_t>(s.nz) * s.ny)
    throw invalid_argument("labels must have shape (nz, ny)");
  if (!s.mask.empty() && s.mask.size() != static_cast<std::size_t>(s.ny))
    throw invalid_argument("mask must have shape (ny,)");
  if (s.field.size() != static_cast<std::size_t>(2 * s.ny)) throw invalid_argument("field must have shape (ny, 2)");
  if (s.iterations < 0) throw invalid_argument("iterations must be >= 0");
  for (auto l : s.labels)
    if (l < 0 || static_cast<std::size_t>(l) >= s.indices.size())
      throw invalid_argument("labels must index into `indices`");
  if (s.indices.size() > 255) throw invalid_argument("at most 255 materials per 2D solve");
  if (3 * static_cast<std::size_t>(s.ny) * sizeof(cf) > 220 * 1024)
    throw invalid_argument("ny too large for the resident 2D engine (max 9216)");
}

class Batch2DImpl final : public Batch2D {
 public:
  explicit Batch2DImpl(int device) : device_(device) {
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    keep_pool_memory(device);
    for (auto& s : streams_) check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    main_.create();
    check_cuda(cudaEventCreateWithFlags(&ev0_, cudaEventDisableTiming), "event");
    check_cuda(cudaEventCreate(&ev_start_), "event");
    check_cuda(cudaEventCreate(&ev_stop_), "event");
    check_cuda(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming), "event");
    for (auto& e : class_done_) check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    cudaDeviceProp prop{};
    check_cuda(cudaGetDeviceProperties(&prop, device), "props");
    sms_ = prop.multiProcessorCount;
    check_cuda(cudaDeviceGetStreamPriorityRange(&prio_least_, &prio_greatest_), "priorities");
  }
  ~Batch2DImpl() override {
    if (exec_) cudaGraphExecDestroy(exec_);
    if (exec_packed_) cudaGraphExecDestroy(exec_packed_);
    cudaStreamSynchronize(main_);
    for (auto& s : streams_) cudaStreamDestroy(s);
    cudaEventDestroy(ev0_);
    cudaEventDestroy(ev_start_);
    cudaEventDestroy(ev_stop_);
    cudaEventDestroy(done_);
    for (auto& e : class_done_) cudaEventDestroy(e);
  }

  std::int64_t add(Solve2D s) override {
    if (prepared_) throw invalid_argument("batch already prepared");
    validate2d(s);
    HostSolve h;
    h.in = std::move(s);
    solves_.push_back(std::move(h));
    return static_cast<std::int64_t>(solves_.size()) - 1;
  }
  std::int64_t add_prepared(std::shared_ptr<PreparedSolve> p) override {
    if (prepared_) throw invalid_argument("batch already prepared");
    if (!p || !p->built) throw invalid_argument("solve not prepared");
    solves_.push_back(std::move(*p));
    return static_cast<std::int64_t>(solves_.size()) - 1;
  }

  void prepare() override;
  void set_graphs(bool on) override { use_graphs_ = on; }
  void set_autotune(bool on) override { autotune_ = on; }
  void set_variant(int n, int k) override {
    if (prepared_) throw invalid_argument("batch already prepared");
    if (k == -1) {  // the run-time-length kernel instead of the compiled ones
      if (rt_choice(n) < 0) throw invalid_argument("ny = " + std::to_string(n) + " has no run-time-length kernel");
    } else if (fixed_length_index(n) < 0) {
      throw invalid_argument("ny = " + std::to_string(n) + " has no fixed variants");
    }
    forced_[n] = k;
  }
  int class_info(int k, int& n, int& threads, int& cluster, int& variant, float& tuned_ms) const override {
    int seen = 0;
    for (int c = 0; c < kNumClasses; ++c) {
      if (!class_count_[c]) continue;
      if (seen++ != k) continue;
      const bool fixed = c >= kGenericClasses && c < kRtBase;
      n = fixed ? fixed_lengths()[c - kGenericClasses] : class_maxn_[c];
      threads = class_threads_[c];
      cluster = fixed ? fixed_variants()[class_variant_[c]].cluster : 1;
      variant = c >= kRtBase ? -2 - (c - kRtBase) : -1;
      if (fixed) {
        const std::vector<int> vs = variants_of(n);
        variant = static_cast<int>(std::find(vs.begin(), vs.end(), class_variant_[c]) - vs.begin());
      }
      tuned_ms = class_tuned_ms_[c];
      return class_count_[c];
    }
    throw invalid_argument("no class " + std::to_string(k));
  }
  void enqueue() override;
  bool ready() override;
  float run() override;
  float solve_packed(const cd* fields, cd* out) override;
  void result(std::int64_t id, Solve2DResult& r) override;
  std::size_t device_bytes() const override { return bytes_; }
  std::int64_t kernel_launches() const override { return launches_; }
  int work_items() const override { return static_cast<int>(items_.size()); }
  int classes() const override {
    int c = 0;
    for (int k = 0; k < kNumClasses; ++k) c += class_count_[k] > 0;
    return c;
  }
  std::size_t packed_inputs() const override { return static_cast<std::size_t>(packed_total_); }
  void work(double& transforms, double& flops, double& bytes) const override {
    transforms = work_transforms_;
    flops = work_flops_;
    bytes = work_bytes_;
  }

 private:
  void launch_classes(cudaStream_t origin, const R2Item* base = nullptr);
  void capture_graphs();
  void download();
  void use_variant(int c, int v);
  void autotune();
  void check_status();
  // a compiled fixed-length kernel serves n (unless the run-time-length kernel was forced)
  bool uses_fixed(int n) const {
    auto f = forced_.find(n);
    return fixed_length_index(n) >= 0 && !(f != forced_.end() && f->second == -1);
  }
  template <typename K, typename... A>
  void launch(K kernel, dim3 grid, dim3 block, std::size_t smem, cudaStream_t s, A... args) {
    kernel<<<grid, block, smem, s>>>(args...);
    check_cuda(cudaGetLastError(), "kernel launch");
    ++launches_;
  }

  int device_;
  OwnedStream main_;  // first: the pools below are stream-ordered allocations on it
  int sms_ = 148;
  int prio_least_ = 0, prio_greatest_ = 0;  // launch priorities (greatest is numerically lowest)
  bool prepared_ = false;
  std::vector<HostSolve> solves_;
  std::vector<Item> items_;
  cudaStream_t streams_[kNumClasses] = {};
  cudaGraphExec_t exec_ = nullptr, exec_packed_ = nullptr;
  int graph_kernels_ = 0, graph_packed_kernels_ = 0;
  cudaEvent_t ev0_ = nullptr, ev_start_ = nullptr, ev_stop_ = nullptr, done_ = nullptr;
  cudaEvent_t class_done_[kNumClasses] = {};
  int class_count_[kNumClasses] = {};
  int class_first_[kNumClasses] = {};
  int class_maxn_[kNumClasses] = {};
  int class_grid_[kNumClasses] = {};
  int class_threads_[kNumClasses] = {};
  std::size_t class_smem_[kNumClasses] = {};
  const void* class_fn_[kNumClasses] = {};
  int class_variant_[kNumClasses] = {};
  float class_tuned_ms_[kNumClasses] = {};
  std::map<int, int> variant_twbase_;  // variant index -> twiddle pool offset
  std::map<int, int> forced_;          // length -> variant position among its variants
  bool autotune_ = false;
  // device pools
  DevBuf<R2Step> d_steps_;
  DevBuf<R2Pass> d_passes_;
  DevBuf<std::uint8_t> d_pids_;
  DevBuf<int> d_iface_;
  DevBuf<cf> d_tables_, d_lines_, d_src_;
  DevBuf<Tw<float>> d_twiddles_;
  DevBuf<FftPlan> d_plans_;
  DevBuf<float> d_mask_;
  DevBuf<double> d_weights_, d_energy_;
  DevBuf<long long> d_clock_;
  DevBuf<int> d_status_;
  DevBuf<R2Item> d_items_;
  DevBuf<int> d_queue_;
  DevBuf<ItemIo> d_io_;
  DevBuf<cd> d_packed_in_, d_packed_out_;
  std::vector<R2Item> h_items_;
  std::vector<cf> h_lines_;
  std::vector<double> h_energy_;
  std::vector<long long> h_clock_;
  bool downloaded_ = false;
  bool use_graphs_ = true;
  std::vector<long long> item_energy_off_;
  long long packed_total_ = 0;
  std::size_t bytes_ = 0;
  std::int64_t launches_ = 0;
  double work_transforms_ = 0, work_flops_ = 0, work_bytes_ = 0;
};

void build_host(HostSolve& h) {
  const Solve2D& s = h.in;
  const int n = s.ny;
  auto index_of = [&](int l) { return l < 0 ? s.index_before : s.indices[static_cast<std::size_t>(l)]; };
  auto same = [](cd a, cd b) { return a.re == b.re && a.im == b.im; };
  std::map<std::tuple<int, double, double, double, double>, int> slot;
  auto table = [&](int kind, cd nr, cd ns) -> long long {
    auto key = std::make_tuple(kind, nr.re, nr.im, ns.re, ns.im);
    auto it = slot.find(key);
    int id;
    if (it == slot.end()) {
      id = static_cast<int>(h.tables.size());
      slot.emplace(key, id);
      h.tables.emplace_back(kind, nr, ns);
    } else {
      id = it->second;
    }
    return static_cast<long long>(id) * 4 * n;
  };
  std::unordered_map<std::uint64_t, std::vector<long long>> seen;
  std::vector<std::int32_t> before(n, -1);
  std::vector<std::uint8_t> pid(n);
  std::vector<std::pair<int, int>> pairs;
  const bool refl = s.iterations > 0;
  h.steps.resize(s.nz);
  // a label pair (r, s), r ∈ [−1, m), s ∈ [0, m), as the code (r + 1)·m + s (< 2^16 for m ≤ 255):
  // codes sort like the pairs (the reference's std::set order, cpp/src/solver.cpp:389-390)
  const int m = static_cast<int>(s.indices.size());
  const std::size_t ncode = static_cast<std::size_t>(m + 1) * m;
  std::vector<std::uint8_t> code_iface(ncode);
  for (int r = -1; r < m; ++r)
    for (int q = 0; q < m; ++q)
      code_iface[static_cast<std::size_t>(r + 1) * m + q] = !same(index_of(r), index_of(q));
  std::vector<std::uint16_t> code(n);
  std::vector<std::uint32_t> stamp(ncode, 0), present;
  std::vector<int> code_id(ncode, 0);
  for (int p = 0; p < s.nz; ++p) {
    const std::int32_t* a = p == 0 ? before.data() : s.labels.data() + static_cast<std::size_t>(p - 1) * n;
    const std::int32_t* b = s.labels.data() + static_cast<std::size_t>(p) * n;
    const std::uint32_t mark = static_cast<std::uint32_t>(p) + 1;
    present.clear();
    for (int q = 0; q < n; ++q) {
      const std::uint32_t k = static_cast<std::uint32_t>(a[q] + 1) * m + b[q];
      code[q] = static_cast<std::uint16_t>(k);
      if (stamp[k] != mark) {
        stamp[k] = mark;
        present.push_back(k);
      }
    }
    std::sort(present.begin(), present.end());
    pairs.clear();
    for (auto k : present) pairs.emplace_back(static_cast<int>(k / m) - 1, static_cast<int>(k % m));
    R2Step st{};
    st.pid = -1;
    if (pairs.size() > 1) {
      for (std::size_t i = 0; i < present.size(); ++i) code_id[present[i]] = static_cast<int>(i);
      std::uint64_t hash = 1469598103934665603ULL;
      for (int q = 0; q < n; ++q) {
        pid[q] = static_cast<std::uint8_t>(code_id[code[q]]);
        hash = (hash ^ pid[q]) * 1099511628211ULL;
      }
      long long found = -1;
      for (long long off : seen[hash])
        if (std::memcmp(h.pids.data() + off, pid.data(), n) == 0) {
          found = off;
          break;
        }
      if (found < 0) {
        found = static_cast<long long>(h.pids.size());
        h.pids.insert(h.pids.end(), pid.begin(), pid.end());
        seen[hash].push_back(found);
      }
      st.pid = found;
    }
    st.iface = static_cast<long long>(h.iface.size());
    bool any_iface = false;
    for (auto k : present) any_iface |= code_iface[k] != 0;
    if (any_iface)
      for (int q = 0; q < n; ++q)
        if (code_iface[code[q]]) h.iface.push_back(q);
    st.niface = static_cast<int>(h.iface.size() - st.iface);
    // forward passes: T for every pair, then R where the indices differ (cpp/src/solver.cpp:396-397)
    st.fwd_off = static_cast<int>(h.passes.size());
    for (std::size_t i = 0; i < pairs.size(); ++i)
      h.passes.push_back({table(kFwdT, index_of(pairs[i].first), index_of(pairs[i].second)), static_cast<int>(i), 0});
    st.fwd_t = static_cast<int>(pairs.size());
    st.fwd_r = 0;
    if (refl)
      for (std::size_t i = 0; i < pairs.size(); ++i) {
        const cd nr = index_of(pairs[i].first), ns = index_of(pairs[i].second);
        if (same(nr, ns)) continue;
        h.passes.push_back({table(kFwdR, nr, ns), static_cast<int>(i), 1});
        ++st.fwd_r;
      }
    // backward step from plane p + 1 to plane p: roles swapped
    st.bwd_off = static_cast<int>(h.passes.size());
    st.bwd_t = st.bwd_r = 0;
    if (refl) {
      for (std::size_t i = 0; i < pairs.size(); ++i) {
        h.passes.push_back({table(kBwdT, index_of(pairs[i].second), index_of(pairs[i].first)), static_cast<int>(i), 0});
        ++st.bwd_t;
      }
      for (std::size_t i = 0; i < pairs.size(); ++i) {
        const cd nr = index_of(pairs[i].second), ns = index_of(pairs[i].first);
        if (same(nr, ns)) continue;
        h.passes.push_back({table(kBwdR, nr, ns), static_cast<int>(i), 1});
        ++st.bwd_r;
      }
    }
    h.steps[p] = st;
  }
  h.iface_count = static_cast<long long>(h.iface.size());
  h.built = true;
}

void Batch2DImpl::prepare() {
  if (prepared_) return;
  if (solves_.empty()) throw invalid_argument("empty batch");
  check_cuda(cudaSetDevice(device_), "cudaSetDevice");
  // host preparation, parallel over solves
  {
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    std::atomic<std::size_t> next{0};
    std::vector<std::exception_ptr> errs(hw);
    for (unsigned t = 0; t < hw; ++t)
      pool.emplace_back([&, t] {
        try {
          for (std::size_t i = next++; i < solves_.size(); i = next++) if (!solves_[i].built) build_host(solves_[i]);
        } catch (...) {
          errs[t] = std::current_exception();
        }
      });
    for (auto& th : pool) th.join();
    for (auto& e : errs)
      if (e) std::rethrow_exception(e);
  }
  // plans per distinct length (generic kernels) and twiddles of every variant of the fixed
  // lengths (autotuning may pick any of them)
  std::map<int, int> plan_of;
  std::vector<FftPlan> plans;
  std::vector<Tw<float>> tw;
  std::map<int, bool> seen_n;
  for (auto& h : solves_) {
    const int n = h.in.ny;
    if (seen_n.count(n)) continue;
    seen_n[n] = true;
    if (uses_fixed(n)) {
      for (int v : variants_of(n)) {
        variant_twbase_[v] = static_cast<int>(tw.size());
        for (auto& t : variant_twiddles(fixed_variants()[v])) tw.push_back(t);
      }
      continue;
    }
    const int rt = rt_choice(n);
    HostPlan hp = rt >= 0 ? make_plan_radices(n, rt_radices(n, rt_variants()[rt].e)) : make_plan(n);
    const int base = static_cast<int>(tw.size());
    for (auto& t : twiddles_for<float>(hp)) tw.push_back(t);
    for (int st = 0; st < hp.plan.nstages; ++st) hp.plan.twoff[st] += base;
    hp.plan.rootoff += base;
    plan_of[n] = static_cast<int>(plans.size());
    plans.push_back(hp.plan);
  }
  // pool offsets
  long long nsteps = 0, npass = 0, npid = 0, niface = 0, ntab = 0, nlines = 0, nsrc = 0, nmask = 0,
            nweights = 0, nenergy = 0;
  for (auto& h : solves_) {
    h.step_base = nsteps;
    h.pass_base = npass;
    h.pid_base = npid;
    h.iface_base = niface;
    h.table_base = ntab;
    h.packed = packed_total_;
    nsteps += h.in.nz;
    npass += static_cast<long long>(h.passes.size());
    npid += static_cast<long long>(h.pids.size());
    niface += h.iface_count;
    ntab += static_cast<long long>(h.tables.size()) * 4 * h.in.ny;
    packed_total_ += 2LL * h.in.ny;
    if (!h.in.mask.empty()) nmask += 2LL * h.in.ny;
  }
  // work items: (solve, component) with a non-zero input component
  for (std::size_t i = 0; i < solves_.size(); ++i) {
    HostSolve& h = solves_[i];
    const int n = h.in.ny;
    for (int c = 0; c < 2; ++c) {
      bool any = false;
      for (int q = 0; q < n && !any; ++q) any = h.in.field[2 * q + c].re != 0.0 || h.in.field[2 * q + c].im != 0.0;
      if (!any) continue;
      int cls = 0;
      if (uses_fixed(n)) {
        cls = kGenericClasses + fixed_length_index(n);
      } else if (rt_choice(n) >= 0) {
        cls = kRtBase + rt_choice(n);
      } else {
        const int want = threads_needed(plans[plan_of[n]], 1, kR2Ept);
        if (want > kClassThreads[kGenericClasses - 1])
          throw invalid_argument("ny = " + std::to_string(n) + " needs more than 512 threads in the resident 2D engine");
        while (cls < kGenericClasses - 1 && kClassThreads[cls] < want) ++cls;
      }
      double passes = 0;
      for (auto& st : h.steps) passes += 2 + st.fwd_t + st.fwd_r + st.bwd_t + st.bwd_r;
      const double cost = std::max(1, h.in.iterations) * passes * n * std::log2(std::max(2, n));
      h.items[c] = static_cast<int>(items_.size());
      items_.push_back({static_cast<int>(i), c, cls, n, cost});
    }
  }
  // algorithmic work of one run (what the resident kernel executes per item)
  for (auto& it : items_) {
    const HostSolve& h = solves_[it.solve];
    const int iters = std::max(1, h.in.iterations);
    const bool refl = h.in.iterations > 0;
    const double n = it.n, lg = std::log2(std::max(2.0, n));
    double ffts = 1, passes = 0, pid_bytes = 0, src_bytes = 0;
    for (int k = 0; k < iters; ++k) {
      for (auto& st : h.steps) {
        const int pf = st.fwd_t + (refl ? st.fwd_r : 0);
        ffts += 1 + pf;
        passes += pf;
        if (st.pid >= 0) pid_bytes += n;
        if (refl) src_bytes += 8.0 * st.niface + (k > 0 ? 12.0 * st.niface : 0.0);
        if (!refl) continue;
        ffts += 1 + st.bwd_t + st.bwd_r;
        passes += st.bwd_t + st.bwd_r;
        if (st.pid >= 0) pid_bytes += n;
        src_bytes += 8.0 * st.niface + 12.0 * st.niface;
      }
      ffts += refl ? 2 : 0;
    }
    work_transforms_ += ffts;
    work_flops_ += ffts * 5.0 * n * lg + passes * 6.0 * n;
    work_bytes_ += pid_bytes + src_bytes + 3.0 * 8.0 * n;  // + input, transmitted, reflected
  }
  // order items by class, then by decreasing cost (longest first)
  std::vector<int> order(items_.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    if (items_[a].cls != items_[b].cls) return items_[a].cls > items_[b].cls;
    return items_[a].cost > items_[b].cost;
  });
  std::vector<Item> sorted;
  for (int k : order) sorted.push_back(items_[k]);
  items_ = sorted;
  for (auto& h : solves_) h.items[0] = h.items[1] = -1;
  for (std::size_t k = 0; k < items_.size(); ++k) solves_[items_[k].solve].items[items_[k].comp] = static_cast<int>(k);
  for (int c = 0; c < kNumClasses; ++c) class_count_[c] = 0;
  for (std::size_t k = 0; k < items_.size(); ++k) {
    const int c = items_[k].cls;
    if (class_count_[c] == 0) class_first_[c] = static_cast<int>(k);
    ++class_count_[c];
    class_maxn_[c] = std::max(class_maxn_[c], items_[k].n);
  }
  for (auto& it : items_) {
    nlines += 3LL * it.n;  // input, transmitted, reflected
    nsrc += 2 * solves_[it.solve].iface_count;
    nweights += 2LL * it.n;
    nenergy += 2LL * std::max(1, solves_[it.solve].in.iterations) + 1;
  }
  // allocate and upload pools
  std::vector<R2Step> steps(nsteps);
  std::vector<R2Pass> passes(npass);
  std::vector<std::uint8_t> pids(npid);
  std::vector<int> iface(niface);
  std::vector<float> mask(nmask);
  long long moff = 0;
  std::vector<long long> mask_off(solves_.size(), -1);
  for (std::size_t i = 0; i < solves_.size(); ++i) {
    HostSolve& h = solves_[i];
    std::copy(h.steps.begin(), h.steps.end(), steps.begin() + h.step_base);
    std::copy(h.passes.begin(), h.passes.end(), passes.begin() + h.pass_base);
    std::copy(h.pids.begin(), h.pids.end(), pids.begin() + h.pid_base);
    std::copy(h.iface.begin(), h.iface.end(), iface.begin() + h.iface_base);
    if (!h.in.mask.empty()) {  // hi values, then lo values (mask = hi + lo)
      mask_off[i] = moff;
      for (int q = 0; q < h.in.ny; ++q) {
        const float hi = static_cast<float>(h.in.mask[q]);
        mask[moff + q] = hi;
        mask[moff + h.in.ny + q] = static_cast<float>(h.in.mask[q] - static_cast<double>(hi));
      }
      moff += 2LL * h.in.ny;
    }
  }
  d_steps_.alloc(nsteps, main_);
  d_steps_.upload(steps.data(), nsteps);
  d_passes_.alloc(std::max<long long>(npass, 1), main_);
  d_passes_.upload(passes.data(), npass);
  d_pids_.alloc(std::max<long long>(npid, 1), main_);
  d_pids_.upload(pids.data(), npid);
  d_iface_.alloc(std::max<long long>(niface, 1), main_);
  d_iface_.upload(iface.data(), niface);
  d_mask_.alloc(std::max<long long>(nmask, 1), main_);
  d_mask_.upload(mask.data(), nmask);
  d_tables_.alloc(std::max<long long>(ntab, 1), main_);
  d_twiddles_.alloc(tw.size(), main_);
  d_twiddles_.upload(tw.data(), tw.size());
  d_plans_.alloc(plans.size(), main_);
  d_plans_.upload(plans.data(), plans.size());
  d_lines_.alloc(nlines, main_);
  d_src_.alloc(std::max<long long>(nsrc, 1), main_);
  d_weights_.alloc(nweights, main_);
  d_energy_.alloc(nenergy, main_);
  d_clock_.alloc(2 * items_.size(), main_);
  d_status_.alloc(1, main_);
  d_status_.zero();
  d_items_.alloc(items_.size(), main_);
  d_queue_.alloc(kNumClasses, main_);
  d_io_.alloc(items_.size(), main_);
  d_packed_in_.alloc(packed_total_, main_);
  d_packed_out_.alloc(2 * packed_total_, main_);
  d_src_.zero();
  d_lines_.zero();
  // operator tables (FP64 on the device, stored as complex64)
  std::vector<TableJob> tjobs;
  for (auto& h : solves_)
    for (std::size_t t = 0; t < h.tables.size(); ++t) {
      const auto& [kind, nr, ns] = h.tables[t];
      tjobs.push_back({d_tables_.ptr + h.table_base + static_cast<long long>(t) * 4 * h.in.ny, nr, ns,
                       h.in.dy, h.in.k0, h.in.dz, h.in.ny, kind});
    }
  // item records, flux weights, packed-IO records
  std::vector<WeightJob> wjobs;
  std::vector<ItemIo> io(items_.size());
  h_items_.resize(items_.size());
  item_energy_off_.resize(items_.size());
  long long loff = 0, soff = 0, woff = 0, eoff = 0;
  for (std::size_t k = 0; k < items_.size(); ++k) {
    const Item& itm = items_[k];
    HostSolve& h = solves_[itm.solve];
    const int n = h.in.ny;
    R2Item r{};
    r.input = d_lines_.ptr + loff;
    r.transmitted = d_lines_.ptr + loff + n;
    r.reflected = d_lines_.ptr + loff + 2 * n;
    loff += 3LL * n;
    r.tables = d_tables_.ptr + h.table_base + static_cast<long long>(itm.comp) * 2 * n;
    r.src_fwd = d_src_.ptr + soff;
    r.src_bwd = d_src_.ptr + soff + h.iface_count;
    soff += 2 * h.iface_count;
    r.mask = mask_off[itm.solve] >= 0 ? d_mask_.ptr + mask_off[itm.solve] : nullptr;
    r.steps = d_steps_.ptr + h.step_base;
    r.passes = d_passes_.ptr + h.pass_base;
    r.pids = d_pids_.ptr + h.pid_base;
    r.iface = d_iface_.ptr + h.iface_base;
    r.w_out = d_weights_.ptr + woff;
    r.w_in = d_weights_.ptr + woff + n;
    // transmitted medium: label at the centre pixel of the last slab (src/bwpm/fast.py:148-151)
    const cd last = h.in.indices[static_cast<std::size_t>(h.in.labels[static_cast<std::size_t>(h.in.nz - 1) * n + n / 2])];
    wjobs.push_back({d_weights_.ptr + woff, last, h.in.dy, h.in.k0, n, itm.comp});
    wjobs.push_back({d_weights_.ptr + woff + n, h.in.index_before, h.in.dy, h.in.k0, n, itm.comp});
    woff += 2LL * n;
    r.energy = d_energy_.ptr + eoff;
    item_energy_off_[k] = eoff;
    eoff += 2LL * std::max(1, h.in.iterations) + 1;
    r.clock = d_clock_.ptr + 2 * k;
    r.status = d_status_.ptr;
    r.n = n;
    r.nz = h.in.nz;
    r.iterations = h.in.iterations;
    r.plan = plan_of.count(n) ? plan_of[n] : 0;  // fixed kernels carry their plan
    h_items_[k] = r;
    io[k] = {h.packed, const_cast<cf*>(r.input), r.transmitted, r.reflected, n, itm.comp};
  }
  d_items_.upload(h_items_.data(), h_items_.size());
  d_io_.upload(io.data(), io.size());
  if (!tjobs.empty()) {
    DevBuf<TableJob> dj(tjobs.size(), main_);
    dj.upload(tjobs.data(), tjobs.size());
    int maxn = 0;
    for (auto& j : tjobs) maxn = std::max(maxn, j.n);
    for (std::size_t b = 0; b < tjobs.size(); b += 60000) {
      const unsigned cnt = static_cast<unsigned>(std::min<std::size_t>(60000, tjobs.size() - b));
      launch(k_table_jobs, dim3(ceil_div(maxn, 256), cnt), dim3(256), 0, main_, (const TableJob*)(dj.ptr + b));
    }
    check_cuda(cudaStreamSynchronize(main_), "tables");
  }
  {
    DevBuf<WeightJob> dj(wjobs.size(), main_);
    dj.upload(wjobs.data(), wjobs.size());
    int maxn = 0;
    for (auto& j : wjobs) maxn = std::max(maxn, j.n);
    for (std::size_t b = 0; b < wjobs.size(); b += 60000) {
      const unsigned cnt = static_cast<unsigned>(std::min<std::size_t>(60000, wjobs.size() - b));
      launch(k_weight_jobs, dim3(ceil_div(maxn, 256), cnt), dim3(256), 0, main_, (const WeightJob*)(dj.ptr + b));
    }
    check_cuda(cudaStreamSynchronize(main_), "weights");
  }
  // inputs: packed complex128 of every solve -> per-item complex64 lines
  std::vector<cd> packed(packed_total_);
  for (auto& h : solves_) std::copy(h.in.field.begin(), h.in.field.end(), packed.begin() + h.packed);
  d_packed_in_.upload(packed.data(), packed.size());
  launch(k_unpack_inputs, dim3(8, static_cast<unsigned>(items_.size())), dim3(256), 0, main_,
         (const ItemIo*)d_io_.ptr, (const cd*)d_packed_in_.ptr);
  check_cuda(cudaStreamSynchronize(main_), "inputs");
  // launch shapes
  auto set_attr = [](const void* k) {
    check_cuda(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024), "smem");
  };
  set_attr((const void*)k_resident2d<64>);
  set_attr((const void*)k_resident2d<128>);
  set_attr((const void*)k_resident2d<256>);
  set_attr((const void*)k_resident2d<512>);
  for (int c = 0; c < kNumClasses; ++c) {
    if (!class_count_[c]) continue;
    if (c >= kGenericClasses && c < kRtBase) {
      const int n = fixed_lengths()[c - kGenericClasses];
      const std::vector<int> vs = variants_of(n);
      for (int v : vs) set_attr(fixed_variants()[v].fn);
      int pick = vs.front();
      auto f = forced_.find(n);
      if (f != forced_.end()) {
        if (f->second < 0 || f->second >= static_cast<int>(vs.size()))
          throw invalid_argument("no variant " + std::to_string(f->second) + " for ny = " + std::to_string(n));
        pick = vs[f->second];
      }
      use_variant(c, pick);
      continue;
    }
    const void* k;
    int threads;
    if (c >= kRtBase) {  // run-time-length kernel: threads of the class's longest line
      const RtVariant& r = rt_variants()[c - kRtBase];
      k = r.fn;
      threads = (class_maxn_[c] / r.e + 31) / 32 * 32;
      class_smem_[c] = rt_smem_bytes(class_maxn_[c]);
      set_attr(k);
    } else {
      k = c == 0 ? (const void*)k_resident2d<64> : c == 1 ? (const void*)k_resident2d<128>
          : c == 2 ? (const void*)k_resident2d<256> : (const void*)k_resident2d<512>;
      threads = kClassThreads[c];
      class_smem_[c] = 3 * static_cast<std::size_t>(class_maxn_[c]) * sizeof(cf);
    }
    int per_sm = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, class_smem_[c]), "occupancy");
    per_sm = std::max(1, per_sm);
    class_grid_[c] = std::min(class_count_[c], per_sm * sms_);
    class_threads_[c] = threads;
    class_fn_[c] = k;
  }
  if (autotune_) autotune();
  bytes_ = d_steps_.bytes() + d_passes_.bytes() + d_pids_.bytes() + d_iface_.bytes() +
           d_tables_.bytes() + d_twiddles_.bytes() + d_lines_.bytes() + d_src_.bytes() +
           d_mask_.bytes() + d_weights_.bytes() + d_energy_.bytes() + d_packed_in_.bytes() +
           d_packed_out_.bytes();
  for (auto& h : solves_) {  // label planes live on the device now (pair ids, lists)
    std::vector<std::int32_t>().swap(h.in.labels);
    std::vector<std::uint8_t>().swap(h.pids);
    std::vector<int>().swap(h.iface);
    std::vector<R2Pass>().swap(h.passes);
  }
  prepared_ = true;
  if (use_graphs_) capture_graphs();
}

void Batch2DImpl::launch_classes(cudaStream_t origin, const R2Item* base) {
  if (!base) base = d_items_.ptr;
  check_cuda(cudaMemsetAsync(d_queue_.ptr, 0, kNumClasses * sizeof(int), origin), "queue reset");
  check_cuda(cudaEventRecord(ev0_, origin), "event");
  // longest chains first: classes in decreasing order of their first item's cost
  std::vector<int> order;
  for (int c = 0; c < kNumClasses; ++c)
    if (class_count_[c]) order.push_back(c);
  // the longest item chain of a class: its first item's work over the CTAs that share a line
  auto chain = [&](int c) {
    const int cl = c >= kGenericClasses && c < kRtBase ? fixed_variants()[class_variant_[c]].cluster : 1;
    return items_[class_first_[c]].cost / cl;
  };
  std::sort(order.begin(), order.end(), [&](int a, int b) { return chain(a) > chain(b); });
  for (std::size_t rank = 0; rank < order.size(); ++rank) {
    const int c = order[rank];
    cudaStream_t s = streams_[c];
    check_cuda(cudaStreamWaitEvent(s, ev0_, 0), "wait");
    const R2Item* items = base + class_first_[c];
    int count = class_count_[c];
    int* q = d_queue_.ptr + c;
    // the longest chains first: their CTAs win free SMs over the other classes' CTAs
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = prio_greatest_ + std::min(static_cast<int>(rank), prio_least_ - prio_greatest_);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(class_grid_[c]);
    cfg.blockDim = dim3(class_threads_[c]);
    cfg.dynamicSmemBytes = class_smem_[c];
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (c >= kGenericClasses && c < kRtBase) {
      const Tw<float>* tw = d_twiddles_.ptr + variant_twbase_[class_variant_[c]];
      void* args[] = {&items, &count, &q, &tw};
      check_cuda(cudaLaunchKernelExC(&cfg, class_fn_[c], args), "launch");
    } else {
      R2Shared sh{d_plans_.ptr, d_twiddles_.ptr};
      void* args[] = {&items, &count, &q, &sh};
      check_cuda(cudaLaunchKernelExC(&cfg, class_fn_[c], args), "launch");
    }
    ++launches_;
    check_cuda(cudaEventRecord(class_done_[c], s), "event");
    check_cuda(cudaStreamWaitEvent(origin, class_done_[c], 0), "wait");
  }
}

void Batch2DImpl::use_variant(int c, int v) {
  const FixedVariant& f = fixed_variants()[v];
  class_variant_[c] = v;
  class_fn_[c] = f.fn;
  class_threads_[c] = f.nt;
  class_smem_[c] = f.smem;
  if (f.cluster == 1) {
    int per_sm = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f.fn, f.nt, f.smem), "occupancy");
    class_grid_[c] = std::min(class_count_[c], std::max(1, per_sm) * sms_);
    return;
  }
  // clusters of f.cluster CTAs (compile-time cluster size of the kernel)
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(static_cast<unsigned>(f.cluster * sms_));
  cfg.blockDim = dim3(static_cast<unsigned>(f.nt));
  cfg.dynamicSmemBytes = f.smem;
  int clusters = 0;
  check_cuda(cudaOccupancyMaxActiveClusters(&clusters, f.fn, &cfg), "cluster occupancy");
  class_grid_[c] = std::min(class_count_[c], std::max(1, clusters)) * f.cluster;
}

// Autotuning by measurement of the batch itself.
//
// The whole batch runs with every chain scaled down (kTuneScale of its slabs, at least
// kTuneMinSlabs, one iteration), all classes concurrently as in a real run, so SM sharing
// between classes and co-resident CTAs are part of what is measured. Coordinate descent over
// the fixed-length classes tries each alternative variant and keeps it when the scaled batch
// gets faster (two rounds at most), from two starts (see below). The scaled runs
// write only into this batch's own output and source buffers, which every full run rewrites
// before reading.
void Batch2DImpl::autotune() {
  std::vector<int> tunable;
  for (int c = kGenericClasses; c < kRtBase; ++c) {
    if (!class_count_[c]) continue;
    const int n = fixed_lengths()[c - kGenericClasses];
    if (variants_of(n).size() > 1 && !forced_.count(n)) tunable.push_back(c);
  }
  if (tunable.empty()) return;
  std::vector<R2Item> cut(h_items_);
  for (auto& it : cut) {
    it.nz = std::min(it.nz, std::max(kTuneMinSlabs, it.nz / kTuneScale));
    it.iterations = std::min(it.iterations, 1);
  }
  DevBuf<R2Item> d_cut(cut.size(), main_.s);
  d_cut.upload(cut.data(), cut.size());
  std::vector<long long> clk(2 * items_.size());
  // one measurement: the scaled batch's time (median of three runs after a warm run) and, per
  // class, its SM time in that run (Σ item latency × CTAs per item)
  struct Meas {
    float ms;
    std::vector<double> class_sm;
  };
  auto measure = [&] {
    std::vector<float> runs;
    for (int rep = 0; rep < 4; ++rep) {
      check_cuda(cudaEventRecord(ev_start_, main_), "event");
      launch_classes(main_, d_cut.ptr);
      check_cuda(cudaEventRecord(ev_stop_, main_), "event");
      check_cuda(cudaEventSynchronize(ev_stop_), "autotune");
      float ms = 0;
      check_cuda(cudaEventElapsedTime(&ms, ev_start_, ev_stop_), "elapsed");
      if (rep > 0) runs.push_back(ms);
    }
    std::sort(runs.begin(), runs.end());
    Meas m{runs[runs.size() / 2], std::vector<double>(kNumClasses, 0.0)};
    check_cuda(cudaMemcpyAsync(clk.data(), d_clock_.ptr, clk.size() * sizeof(long long),
                               cudaMemcpyDeviceToHost, main_), "clocks");
    check_cuda(cudaStreamSynchronize(main_), "clocks");
    for (std::size_t k = 0; k < items_.size(); ++k) {
      const int c = items_[k].cls;
      const int cl = c >= kGenericClasses && c < kRtBase ? fixed_variants()[class_variant_[c]].cluster : 1;
      m.class_sm[c] += static_cast<double>(clk[2 * k + 1] - clk[2 * k]) * 1e-6 * cl;
    }
    return m;
  };
  // coordinate descent from the current assignment; returns the batch time it ends at
  auto descend = [&] {
    Meas current = measure();
    for (int round = 0; round < 2; ++round) {
      bool changed = false;
      for (int c : tunable) {
        const int n = fixed_lengths()[c - kGenericClasses];
        const int keep = class_variant_[c];
        int best_v = keep;
        for (int v : variants_of(n)) {
          if (v == keep) continue;
          use_variant(c, v);
          const Meas t = measure();
          // clearly faster batch, or an equal batch (within the run-to-run spread) whose class
          // needs clearly less SM time (frees SMs for the other classes)
          const bool faster = t.ms < 0.98f * current.ms;
          const bool leaner = t.ms < 1.01f * current.ms && t.class_sm[c] < 0.8 * current.class_sm[c];
          if (faster || leaner) {
            current = t;
            best_v = v;
          }
        }
        use_variant(c, best_v);
        changed |= best_v != keep;
      }
      if (!changed) break;
    }
    return current.ms;
  };
  // Two starts: the first-listed variants, and for every class the one with the most CTAs per
  // line (the shortest chains). One class alone rarely moves the batch time when several classes
  // share the critical path (measured: 8192 and 6144 points together gain 20 %, each alone
  // nothing), so a descent from either start can stop short; the better end wins.
  std::vector<int> start_a, start_b;
  for (int c : tunable) {
    start_a.push_back(class_variant_[c]);
    const int n = fixed_lengths()[c - kGenericClasses];
    int wide = variants_of(n).front();
    for (int v : variants_of(n))
      if (fixed_variants()[v].cluster > fixed_variants()[wide].cluster) wide = v;
    start_b.push_back(wide);
  }
  const float ta = descend();
  std::vector<int> end_a;
  for (int c : tunable) end_a.push_back(class_variant_[c]);
  float best = ta;
  if (start_b != start_a) {
    for (std::size_t i = 0; i < tunable.size(); ++i) use_variant(tunable[i], start_b[i]);
    const float tb = descend();
    if (tb < ta) {
      best = tb;
    } else {
      for (std::size_t i = 0; i < tunable.size(); ++i) use_variant(tunable[i], end_a[i]);
    }
  }
  for (int c : tunable) class_tuned_ms_[c] = best;
}

void Batch2DImpl::capture_graphs() {
  // one graph per entry point: the persistent class kernels (forked onto their streams and
  // joined back), and for the packed end-to-end path unpack + classes + pack around them
  auto capture = [&](bool packed, cudaGraphExec_t& exec, int& kernels) {
    const std::int64_t before = launches_;
    cudaGraph_t g;
    check_cuda(cudaStreamBeginCapture(main_, cudaStreamCaptureModeThreadLocal), "capture");
    if (packed)
      launch(k_unpack_inputs, dim3(8, static_cast<unsigned>(items_.size())), dim3(256), 0, main_,
             (const ItemIo*)d_io_.ptr, (const cd*)d_packed_in_.ptr);
    launch_classes(main_);
    if (packed) {
      check_cuda(cudaMemsetAsync(d_packed_out_.ptr, 0, d_packed_out_.bytes(), main_), "memset");
      launch(k_pack_outputs, dim3(8, static_cast<unsigned>(items_.size())), dim3(256), 0, main_,
             (const ItemIo*)d_io_.ptr, d_packed_out_.ptr);
    }
    check_cuda(cudaStreamEndCapture(main_, &g), "capture");
    check_cuda(cudaGraphInstantiate(&exec, g, cudaGraphInstantiateFlagUseNodePriority), "instantiate");
    cudaGraphDestroy(g);
    kernels = static_cast<int>(launches_ - before);
    launches_ = before;
  };
  capture(false, exec_, graph_kernels_);
  capture(true, exec_packed_, graph_packed_kernels_);
}

void Batch2DImpl::enqueue() {
  if (!prepared_) prepare();
  check_cuda(cudaSetDevice(device_), "cudaSetDevice");
  if (exec_) {
    check_cuda(cudaGraphLaunch(exec_, main_), "graph launch");
    launches_ += graph_kernels_;
  } else {
    launch_classes(main_);
  }
  check_cuda(cudaEventRecord(done_, main_), "event");
  downloaded_ = false;
}

bool Batch2DImpl::ready() {
  const cudaError_t e = cudaEventQuery(done_);
  if (e == cudaErrorNotReady) return false;
  check_cuda(e, "batch");
  return true;
}

// A bounded wait inside a kernel gave up (a cluster exchange that never completed): the results
// of that run are not valid.
void Batch2DImpl::check_status() {
  int st = 0;
  check_cuda(cudaMemcpyAsync(&st, d_status_.ptr, sizeof(int), cudaMemcpyDeviceToHost, main_), "status");
  check_cuda(cudaStreamSynchronize(main_), "status");
  if (st != 0) throw std::runtime_error("resident 2D engine: a cluster exchange timed out");
}

float Batch2DImpl::run() {
  if (!prepared_) prepare();
  check_cuda(cudaSetDevice(device_), "cudaSetDevice");
  check_cuda(cudaEventRecord(ev_start_, main_), "event");
  enqueue();
  check_cuda(cudaEventRecord(ev_stop_, main_), "event");
  check_cuda(cudaEventSynchronize(ev_stop_), "run");
  float ms = 0;
  check_cuda(cudaEventElapsedTime(&ms, ev_start_, ev_stop_), "elapsed");
  check_status();
  return ms;
}

float Batch2DImpl::solve_packed(const cd* fields, cd* out) {
  if (!prepared_) prepare();
  check_cuda(cudaSetDevice(device_), "cudaSetDevice");
  check_cuda(cudaEventRecord(ev_start_, main_), "event");
  check_cuda(cudaMemcpyAsync(d_packed_in_.ptr, fields, packed_total_ * sizeof(cd), cudaMemcpyHostToDevice, main_), "h2d");
  if (exec_packed_) {
    check_cuda(cudaGraphLaunch(exec_packed_, main_), "graph launch");
    launches_ += graph_packed_kernels_;
  } else {
    launch(k_unpack_inputs, dim3(8, static_cast<unsigned>(items_.size())), dim3(256), 0, main_,
           (const ItemIo*)d_io_.ptr, (const cd*)d_packed_in_.ptr);
    launch_classes(main_);
    check_cuda(cudaMemsetAsync(d_packed_out_.ptr, 0, d_packed_out_.bytes(), main_), "memset");
    launch(k_pack_outputs, dim3(8, static_cast<unsigned>(items_.size())), dim3(256), 0, main_,
           (const ItemIo*)d_io_.ptr, d_packed_out_.ptr);
  }
  check_cuda(cudaMemcpyAsync(out, d_packed_out_.ptr, 2 * packed_total_ * sizeof(cd), cudaMemcpyDeviceToHost, main_), "d2h");
  check_cuda(cudaEventRecord(ev_stop_, main_), "event");
  check_cuda(cudaEventRecord(done_, main_), "event");
  check_cuda(cudaEventSynchronize(ev_stop_), "solve");
  downloaded_ = false;
  float ms = 0;
  check_cuda(cudaEventElapsedTime(&ms, ev_start_, ev_stop_), "elapsed");
  check_status();
  return ms;
}

void Batch2DImpl::download() {
  if (downloaded_) return;
  check_cuda(cudaSetDevice(device_), "cudaSetDevice");
  h_lines_.resize(d_lines_.n);
  h_energy_.resize(d_energy_.n);
  h_clock_.resize(d_clock_.n);
  check_cuda(cudaMemcpyAsync(h_lines_.data(), d_lines_.ptr, d_lines_.bytes(), cudaMemcpyDeviceToHost, main_), "d2h");
  check_cuda(cudaMemcpyAsync(h_energy_.data(), d_energy_.ptr, d_energy_.bytes(), cudaMemcpyDeviceToHost, main_), "d2h");
  check_cuda(cudaMemcpyAsync(h_clock_.data(), d_clock_.ptr, d_clock_.bytes(), cudaMemcpyDeviceToHost, main_), "d2h");
  check_cuda(cudaStreamSynchronize(main_), "d2h");
  check_status();
  downloaded_ = true;
}

void Batch2DImpl::result(std::int64_t id, Solve2DResult& r) {
  if (!prepared_) throw invalid_argument("batch not run");
  if (id < 0 || id >= static_cast<std::int64_t>(solves_.size())) throw invalid_argument("unknown solve id");
  download();
  const HostSolve& h = solves_[id];
  const int n = h.in.ny;
  const int iters = std::max(1, h.in.iterations);
  r.transmitted.assign(2 * n, cd{0.0, 0.0});
  r.reflected.assign(2 * n, cd{0.0, 0.0});
  r.flux_t.assign(h.in.iterations, 0.0);
  r.flux_r.assign(h.in.iterations, 0.0);
  r.flux_in = 0.0;
  long long t0 = -1, t1 = -1;
  for (int c = 0; c < 2; ++c) {
    const int k = h.items[c];
    if (k < 0) continue;
    const R2Item& it = h_items_[k];
    const cf* lt = h_lines_.data() + (it.transmitted - d_lines_.ptr);
    const cf* lr = h_lines_.data() + (it.reflected - d_lines_.ptr);
    for (int q = 0; q < n; ++q) r.transmitted[2 * q + c] = cast<double>(lt[q]);
    if (h.in.iterations > 0)
      for (int q = 0; q < n; ++q) r.reflected[2 * q + c] = cast<double>(lr[q]);
    const double* en = h_energy_.data() + item_energy_off_[k];
    for (int i = 0; i < h.in.iterations; ++i) {
      r.flux_t[i] += en[2 * i];
      r.flux_r[i] += en[2 * i + 1];
    }
    r.flux_in += en[2 * iters];
    const long long* clk = h_clock_.data() + 2 * k;
    t0 = t0 < 0 ? clk[0] : std::min(t0, clk[0]);
    t1 = std::max(t1, clk[1]);
  }
  r.latency_ms = t0 >= 0 ? static_cast<double>(t1 - t0) * 1e-6 : 0.0;
}

}  // namespace

std::unique_ptr<Batch2D> make_batch2d(int device) { return std::make_unique<Batch2DImpl>(device); }

std::shared_ptr<PreparedSolve> prepare_solve(Solve2D s) {
  validate2d(s);
  auto p = std::make_shared<PreparedSolve>();
  p->in = std::move(s);
  build_host(*p);
  return p;
}

std::size_t prepared_device_bytes(const PreparedSolve& p) {
  // the pools prepare() allocates for this solve (an upper bound: a batch shares the twiddles
  // of equal lengths)
  const Solve2D& s = p.in;
  const std::size_t n = static_cast<std::size_t>(s.ny);
  int items = 0;
  for (int c = 0; c < 2; ++c)
    for (std::size_t q = 0; q < n; ++q)
      if (s.field[2 * q + c].re != 0.0 || s.field[2 * q + c].im != 0.0) {
        ++items;
        break;
      }
  const std::size_t iters = static_cast<std::size_t>(std::max(1, s.iterations));
  std::size_t b = p.steps.size() * sizeof(R2Step) + p.passes.size() * sizeof(R2Pass) + p.pids.size() +
                  p.iface.size() * sizeof(int) + p.tables.size() * 4 * n * sizeof(cf) +
                  (s.mask.empty() ? 0 : 2 * n * sizeof(float)) + 6 * n * sizeof(cd) +
                  n * sizeof(Tw<float>) + 64;  // twiddles of the length (shared within a batch)
  b += static_cast<std::size_t>(items) *
       (3 * n * sizeof(cf) + 2 * p.iface.size() * sizeof(cf) + 2 * n * sizeof(double) +
        (2 * iters + 1) * sizeof(double) + 2 * sizeof(long long) + sizeof(R2Item) + sizeof(ItemIo));
  return b;
}

}  // namespace bwpm
