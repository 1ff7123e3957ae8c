// Served request loop: continuous batching on one GPU.
//
// Requests arrive at any time (submit2d/submit3d). Host preparation workers build each 2D
// request's step records (pairs, pair-id planes, interface lists) off the launch path and price
// its device memory exactly. Waiting requests are taken longest estimated chain first (slab
// steps × transform cost; ties in arrival order): the resident engine keeps each solve's SMs
// for its whole chain, so the wall time of a burst is set by its longest chain, which should
// start first (lengths without a compiled kernel run on the run-time-length kernels, ≈ 2.5×
// slower per step). A launcher admits prepared requests in that order while the
// device-memory budget holds (a request larger than the whole budget runs alone): the 2D
// requests admitted together form a launch group, one batched launch of the resident engine on
// its own streams (stream-ordered allocations, no device-wide synchronisation), so groups
// launched while others still run share the GPU: their CTAs start on the SMs that earlier items
// release. 3D requests run on runner threads through the complex64 plane engine, each on its own
// stream. A completer polls the groups' completion events, downloads their results, frees
// their memory and releases the budget, which admits the next requests. Each request's field
// state lives on the device from launch to completion (the resident engine keeps the forward
// and backward fields on chip across all iterations).
//
// The reference has no server: it solves one problem per CudaSolver.run call
// (cpp/src/solver_cuda.cu:729-853).
#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>

#include "devbuf.hpp"
#include "server.hpp"
#include "variants.hpp"

namespace bwpm {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
  std::int64_t id = 0;
  bool is3d = false;
  const std::int32_t* borrowed = nullptr;  // caller-owned labels (2D: copied in preparation; 3D:
                                           // read in place by the plane engine's set-up)
  Solve2D s2;
  std::shared_ptr<PreparedSolve> prep;
  SolverInput s3;
  std::vector<cd> field3;
  int iters3 = 0;
  std::size_t bytes = 0;
  double cost = 0;  // estimated device time of the chain (relative units)
  Clock::time_point arrival, launched, finished;
  enum State { kQueued, kReady, kRunning, kDone, kFailed } state = kQueued;
  std::string error;
  ServedResult res;
};
using Req = std::shared_ptr<Request>;

// Order of the waiting queues: longest estimated chain first, then arrival.
bool before(const Req& a, const Req& b) {
  return a->cost != b->cost ? a->cost > b->cost : a->id < b->id;
}

// Slab steps × transform work of a solve: steps × n·log2(n), the 2D lengths without a compiled
// kernel of the resident engine (run-time-length kernels) at 2.5× per step.
double chain_cost(double steps, double n, bool compiled) {
  return steps * n * std::log2(std::max(2.0, n)) * (compiled ? 1.0 : 2.5);
}

bool has_compiled_kernel(int n) {
  for (const auto& v : fixed_variants())
    if (v.n == n) return true;
  return false;
}

struct Group {
  std::unique_ptr<Batch2D> batch;
  std::vector<Req> reqs;
  std::vector<std::int64_t> ids;  // solve index of each request in the batch
  std::size_t bytes = 0;
};

// Device memory of a complex64 3D solve: field planes and work planes (≈ 10 planes of
// ny·nx·2 complex64), operator tables (48 B per point each, about 16 for two materials), and
// during set-up the uint8 label volume and pair-id planes (at most one byte per point and slab
// each).
std::size_t estimate_3d_bytes(const SolverInput& in) {
  const std::size_t n = in.ny * in.nx;
  return n * (16 * 10 + 48 * 16) + 2 * in.nz * n;
}

class ServerImpl final : public Server {
 public:
  explicit ServerImpl(const ServerOptions& o) : opt_(o) {
    check_cuda(cudaSetDevice(opt_.device), "cudaSetDevice");
    keep_pool_memory(opt_.device);
    if (opt_.budget_bytes == 0)  // free memory counts the pool's cached, unused memory
      opt_.budget_bytes = static_cast<std::size_t>(0.8 * static_cast<double>(free_device_bytes(opt_.device)));
    opt_.max_groups = std::max(1, opt_.max_groups);
    opt_.max_group_solves = std::max(1, opt_.max_group_solves);
    opt_.max_3d = std::max(1, opt_.max_3d);
    if (opt_.prep_threads <= 0)
      opt_.prep_threads = static_cast<int>(std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
    for (int i = 0; i < opt_.prep_threads; ++i) threads_.emplace_back([this] { prep_loop(); });
    threads_.emplace_back([this] { launch_loop(); });
    threads_.emplace_back([this] { complete_loop(); });
    for (int i = 0; i < opt_.max_3d; ++i) threads_.emplace_back([this] { run3d_loop(); });
  }

  ~ServerImpl() override {
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return unfinished_ == 0; });
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }

  std::int64_t submit2d(Solve2D s, const std::int32_t* labels) override {
    auto r = std::make_shared<Request>();
    r->cost = chain_cost(2.0 * std::max(1, s.iterations) * s.nz, s.ny, has_compiled_kernel(s.ny));
    r->s2 = std::move(s);
    r->borrowed = labels;
    return enqueue(std::move(r));
  }

  std::int64_t submit3d(SolverInput in, std::vector<cd> field, int iterations,
                        const std::int32_t* labels) override {
    if (in.ny * in.nx * 2 != field.size()) throw invalid_argument("field must have shape (ny, nx, 2)");
    if (iterations < 0) throw invalid_argument("iterations must be >= 0");
    auto r = std::make_shared<Request>();
    r->is3d = true;
    r->borrowed = labels;
    r->cost = chain_cost(2.0 * std::max(1, iterations) * static_cast<double>(in.nz),
                         static_cast<double>(in.ny * in.nx), true);
    in.device = opt_.device;
    r->s3 = std::move(in);
    r->field3 = std::move(field);
    r->iters3 = iterations;
    return enqueue(std::move(r));
  }

  bool wait(std::int64_t ticket, double timeout_s) override {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(ticket);
    if (it == reqs_.end()) throw invalid_argument("unknown ticket");
    Req r = it->second;
    auto finished = [&] { return r->state == Request::kDone || r->state == Request::kFailed; };
    if (timeout_s < 0) {
      cv_.wait(lk, finished);
      return true;
    }
    return cv_.wait_for(lk, std::chrono::duration<double>(timeout_s), finished);
  }

  void result(std::int64_t ticket, ServedResult& out) override {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(ticket);
    if (it == reqs_.end()) throw invalid_argument("unknown ticket");
    Req r = it->second;
    if (r->state == Request::kFailed) {
      reqs_.erase(it);
      throw std::runtime_error("request " + std::to_string(ticket) + " failed: " + r->error);
    }
    if (r->state != Request::kDone) throw invalid_argument("request not finished");
    out = std::move(r->res);
    reqs_.erase(it);
  }

  void stats(ServerStats& s) override {
    std::lock_guard<std::mutex> lk(mu_);
    s = stats_;
    s.bytes_in_flight = static_cast<std::int64_t>(in_flight_bytes_);
  }

 private:
  std::int64_t enqueue(Req r) {
    std::lock_guard<std::mutex> lk(mu_);
    r->id = next_id_++;
    r->arrival = Clock::now();
    reqs_[r->id] = r;
    incoming_.push_back(r);
    ++unfinished_;
    ++stats_.submitted;
    cv_.notify_all();
    return r->id;
  }

  void fail(const Req& r, const std::string& what) {  // caller holds mu_
    r->state = Request::kFailed;
    r->error = what;
    r->finished = Clock::now();
    --unfinished_;
    ++stats_.failed;
  }

  void prep_loop() {
    for (;;) {
      Req r;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || !incoming_.empty(); });
        if (incoming_.empty()) return;
        auto it = std::min_element(incoming_.begin(), incoming_.end(), before);
        r = *it;
        incoming_.erase(it);
      }
      std::string err;
      try {
        if (r->borrowed) {  // caller-owned labels: 2D copies them here, on the worker threads;
          if (r->is3d)      // the 3D set-up reads them in place on its runner thread
            r->s3.labels_view = r->borrowed;
          else
            r->s2.labels.assign(r->borrowed, r->borrowed + static_cast<std::size_t>(r->s2.nz) * r->s2.ny);
          r->borrowed = nullptr;
        }
        if (r->is3d) {
          r->bytes = estimate_3d_bytes(r->s3);
        } else {
          r->prep = prepare_solve(std::move(r->s2));
          r->bytes = prepared_device_bytes(*r->prep);
        }
      } catch (const std::exception& e) {
        err = e.what();
      }
      std::lock_guard<std::mutex> lk(mu_);
      if (!err.empty()) {
        fail(r, err);
      } else {
        r->state = Request::kReady;
        // keep the admission queue in its order (workers finish out of order)
        ready_.insert(std::upper_bound(ready_.begin(), ready_.end(), r, before), r);
      }
      cv_.notify_all();
    }
  }

  // Admits ready requests in queue order while memory allows; 2D requests form one group.
  // Caller holds mu_.
  void admit(std::vector<Req>& group, std::vector<Req>& runs3d) {
    std::size_t taken = 0;
    for (auto it = ready_.begin(); it != ready_.end();) {
      const Req& r = *it;
      if (!r->is3d && (groups_in_flight_ >= opt_.max_groups ||
                       static_cast<int>(group.size()) >= opt_.max_group_solves)) {
        ++it;  // 2D capacity is full: 3D requests behind it may still go
        continue;
      }
      if (r->is3d && threed_in_flight_ + static_cast<int>(runs3d.size()) >= opt_.max_3d) {
        ++it;
        continue;
      }
      const std::size_t used = in_flight_bytes_ + taken;
      if (used > 0 && used + r->bytes > opt_.budget_bytes) break;  // no overtaking on memory
      taken += r->bytes;
      (r->is3d ? runs3d : group).push_back(r);
      it = ready_.erase(it);
    }
    in_flight_bytes_ += taken;
    stats_.peak_bytes = std::max<std::int64_t>(stats_.peak_bytes, static_cast<std::int64_t>(in_flight_bytes_));
    for (auto& r : group) r->state = Request::kRunning;
    for (auto& r : runs3d) r->state = Request::kRunning;
  }

  void launch_loop() {
    check_cuda(cudaSetDevice(opt_.device), "cudaSetDevice");
    for (;;) {
      std::vector<Req> group, runs3d;
      {
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
          if (stop_ && ready_.empty()) return;
          admit(group, runs3d);
          if (!group.empty() || !runs3d.empty()) break;
          cv_.wait(lk);
        }
        for (auto& r : runs3d) queue3d_.push_back(r);
        threed_in_flight_ += static_cast<int>(runs3d.size());
        if (!group.empty()) ++groups_in_flight_;
        cv_.notify_all();
      }
      if (group.empty()) continue;
      Group g;
      std::size_t reserved = 0;
      for (auto& r : group) reserved += r->bytes;
      try {
        g.batch = make_batch2d(opt_.device);
        g.batch->set_graphs(false);
        for (auto& r : group) g.ids.push_back(g.batch->add_prepared(std::move(r->prep)));
        g.batch->prepare();
        const Clock::time_point now = Clock::now();
        for (auto& r : group) r->launched = now;
        g.batch->enqueue();
        g.reqs = group;
        g.bytes = g.batch->device_bytes();
      } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(mu_);
        for (auto& r : group) fail(r, e.what());
        in_flight_bytes_ -= reserved;
        --groups_in_flight_;
        cv_.notify_all();
        continue;
      }
      std::lock_guard<std::mutex> lk(mu_);
      // account the group at its allocated size from now on
      in_flight_bytes_ = in_flight_bytes_ - reserved + g.bytes;
      stats_.peak_bytes = std::max<std::int64_t>(stats_.peak_bytes, static_cast<std::int64_t>(in_flight_bytes_));
      ++stats_.groups;
      running_ += static_cast<std::int64_t>(g.reqs.size());
      stats_.max_concurrent = std::max(stats_.max_concurrent, running_);
      groups_.push_back(std::move(g));
      cv_.notify_all();
    }
  }

  void complete_loop() {
    check_cuda(cudaSetDevice(opt_.device), "cudaSetDevice");
    for (;;) {
      bool any = false;
      {
        std::unique_lock<std::mutex> lk(mu_);
        if (groups_.empty()) {
          if (stop_) return;
          cv_.wait(lk, [&] { return stop_ || !groups_.empty(); });
          continue;
        }
      }
      // groups_ is only appended to by the launcher; this thread alone removes entries
      for (std::size_t i = 0;; ++i) {
        Group* g = nullptr;
        {
          std::lock_guard<std::mutex> lk(mu_);
          if (i >= groups_.size()) break;
          g = &groups_[i];
        }
        bool ready = false;
        std::string err;
        try {
          ready = g->batch->ready();
          if (ready)
            for (std::size_t k = 0; k < g->reqs.size(); ++k) {
              Solve2DResult sr;
              g->batch->result(g->ids[k], sr);
              ServedResult& o = g->reqs[k]->res;
              o.transmitted = std::move(sr.transmitted);
              o.reflected = std::move(sr.reflected);
              o.flux_t = std::move(sr.flux_t);
              o.flux_r = std::move(sr.flux_r);
              o.flux_in = sr.flux_in;
              o.device_ms = sr.latency_ms;
            }
        } catch (const std::exception& e) {
          ready = true;
          err = e.what();
        }
        if (!ready) continue;
        any = true;
        const std::int64_t launches = g->batch->kernel_launches();
        std::unique_ptr<Batch2D> done_batch;
        {
          std::lock_guard<std::mutex> lk(mu_);
          Group& gg = groups_[i];
          const Clock::time_point now = Clock::now();
          for (auto& r : gg.reqs) {
            if (!err.empty()) {
              fail(r, err);
              continue;
            }
            r->finished = now;
            r->res.latency_ms = ms_between(r->arrival, now);
            r->res.queue_ms = ms_between(r->arrival, r->launched);
            r->state = Request::kDone;
            --unfinished_;
            ++stats_.completed;
          }
          stats_.kernel_launches += launches;
          running_ -= static_cast<std::int64_t>(gg.reqs.size());
          in_flight_bytes_ -= gg.bytes;
          --groups_in_flight_;
          done_batch = std::move(gg.batch);
          groups_.erase(groups_.begin() + static_cast<std::ptrdiff_t>(i));
          --i;
          cv_.notify_all();
        }
        done_batch.reset();  // frees the group's device memory (stream-ordered)
      }
      if (!any) std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
  }

  void run3d_loop() {
    check_cuda(cudaSetDevice(opt_.device), "cudaSetDevice");
    for (;;) {
      Req r;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || !queue3d_.empty(); });
        if (queue3d_.empty()) return;
        r = queue3d_.front();
        queue3d_.pop_front();
        ++running_;
        stats_.max_concurrent = std::max(stats_.max_concurrent, running_);
      }
      std::string err;
      std::int64_t launches = 0;
      const std::size_t n2 = r->s3.ny * r->s3.nx * 2;
      try {
        r->launched = Clock::now();
        auto solver = make_plane_solver(std::move(r->s3), 32);
        r->res.transmitted.assign(n2, cd{0.0, 0.0});
        r->res.reflected.assign(n2, cd{0.0, 0.0});
        RunOutputs out;
        out.transmitted = r->res.transmitted.data();
        out.reflected = r->res.reflected.data();
        const Clock::time_point t0 = Clock::now();
        solver->run(r->field3.data(), r->iters3, nullptr, 0, out);
        r->res.device_ms = ms_between(t0, Clock::now());
        launches = solver->kernel_launches();
      } catch (const std::exception& e) {
        err = e.what();
      }
      std::lock_guard<std::mutex> lk(mu_);
      std::vector<cd>().swap(r->field3);
      if (!err.empty()) {
        fail(r, err);
      } else {
        const Clock::time_point now = Clock::now();
        r->finished = now;
        r->res.latency_ms = ms_between(r->arrival, now);
        r->res.queue_ms = ms_between(r->arrival, r->launched);
        r->state = Request::kDone;
        --unfinished_;
        ++stats_.completed;
      }
      stats_.kernel_launches += launches;
      --running_;
      --threed_in_flight_;
      in_flight_bytes_ -= r->bytes;
      cv_.notify_all();
    }
  }

  ServerOptions opt_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::map<std::int64_t, Req> reqs_;
  std::deque<Req> incoming_, queue3d_;
  std::vector<Req> ready_;
  std::deque<Group> groups_;
  std::vector<std::thread> threads_;
  std::int64_t next_id_ = 0, unfinished_ = 0, running_ = 0;
  int groups_in_flight_ = 0, threed_in_flight_ = 0;
  std::size_t in_flight_bytes_ = 0;
  ServerStats stats_;
  bool stop_ = false;
};

}  // namespace

std::unique_ptr<Server> make_server(const ServerOptions& opt) { return std::make_unique<ServerImpl>(opt); }

}  // namespace bwpm
