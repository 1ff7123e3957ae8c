// Served request loop: continuous batching of 2D and 3D solves on one GPU.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

#include "batch2d.hpp"
#include "solver.hpp"

namespace bwpm {

struct ServerOptions {
  int device = 0;
  std::size_t budget_bytes = 0;  // device memory for requests in flight; 0: 80 % of free memory
  int max_groups = 8;            // 2D launch groups in flight
  int max_group_solves = 64;     // solves per 2D launch group
  int max_3d = 16;               // 3D solves in flight (each runner also does its host set-up)
  int prep_threads = 0;          // host preparation workers; 0: one per host core, at most 16
};

struct ServedResult {
  std::vector<cd> transmitted, reflected;  // (ny·nx·2)
  std::vector<double> flux_t, flux_r;      // 2D: power flux per iteration
  double flux_in = 0;                      // 2D: incident power flux
  double latency_ms = 0;                   // submit → result on the host
  double queue_ms = 0;                     // submit → launch
  double device_ms = 0;                    // 2D: device time of the solve's items; 3D: run time
};

struct ServerStats {
  std::int64_t submitted = 0, completed = 0, failed = 0, groups = 0;
  std::int64_t bytes_in_flight = 0, peak_bytes = 0, kernel_launches = 0;
  std::int64_t max_concurrent = 0;  // most requests on the GPU at once
};

class Server {
 public:
  virtual ~Server() = default;  // finishes every submitted request first
  // Thread-safe; return a ticket at once. A request that fails validation or on the device is
  // marked failed: wait() returns, result() throws its error. With `labels` non-null the
  // request's labels (nz·ny·nx int32) are taken from there instead of s.labels / in.labels (2D:
  // copied by a preparation worker; 3D: read in place by the set-up of its plane engine): the
  // caller keeps them valid and unchanged until wait() has reported the request finished.
  virtual std::int64_t submit2d(Solve2D s, const std::int32_t* labels = nullptr) = 0;
  virtual std::int64_t submit3d(SolverInput in, std::vector<cd> field, int iterations,
                                const std::int32_t* labels = nullptr) = 0;
  // true when the request has finished (done or failed) within timeout_s
  virtual bool wait(std::int64_t ticket, double timeout_s) = 0;
  // results of a finished request (the record is released); throws the request's error
  virtual void result(std::int64_t ticket, ServedResult& r) = 0;
  virtual void stats(ServerStats& s) = 0;
};

std::unique_ptr<Server> make_server(const ServerOptions& opt);

}  // namespace bwpm
