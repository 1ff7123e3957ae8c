// Host interface of the batched resident 2D engine (complex64 fields, FP64 tables/energy).
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

#include "common.cuh"

namespace bwpm {

// One 2D solve in the reference's call convention (nx = 1, lateral axis y).
struct Solve2D {
  int ny = 0, nz = 0, iterations = 0;
  double dy = 0, dz = 0, k0 = 0;
  std::vector<cd> indices;
  std::vector<std::int32_t> labels;  // (nz, ny)
  cd index_before{1.0, 0.0};
  std::vector<double> mask;          // (ny) or empty
  std::vector<cd> field;             // (ny, 2)
};

struct Solve2DResult {
  std::vector<cd> transmitted, reflected;  // (ny, 2)
  std::vector<double> flux_t, flux_r;      // per iteration
  double flux_in = 0;
  double latency_ms = 0;                   // device time from first CTA start to last CTA end
};

// One solve with its host-side records (validated; pairs, pair-id planes, interface lists and
// passes per step), built off the launch path by prepare_solve().
struct PreparedSolve;
std::shared_ptr<PreparedSolve> prepare_solve(Solve2D s);  // throws std::invalid_argument
// device memory a batch allocates for this solve
std::size_t prepared_device_bytes(const PreparedSolve& p);

class Batch2D {
 public:
  virtual ~Batch2D() = default;
  virtual std::int64_t add(Solve2D s) = 0;
  virtual std::int64_t add_prepared(std::shared_ptr<PreparedSolve> p) = 0;
  // builds pools, tables, plans and launch shapes; called once after the last add
  virtual void prepare() = 0;
  // off: no CUDA graphs are captured at prepare (single-use batches); default on
  virtual void set_graphs(bool on) = 0;
  // on: prepare() picks the kernel variant of each fixed length by timing the batch itself with
  // every chain scaled down (all classes concurrently, as in a run): coordinate descent from
  // the first listed variants. Default off (the first listed variant).
  virtual void set_autotune(bool on) = 0;
  // forces variant k (position among the variants of length n) for this batch
  virtual void set_variant(int n, int k) = 0;
  // class k (0 ≤ k < classes()): length (the largest for a generic class), threads, CTAs per
  // line, variant position (−1: generic kernel), scaled-batch time in ms of the autotuned
  // choice (0: not tuned); returns its items
  virtual int class_info(int k, int& n, int& threads, int& cluster, int& variant, float& tuned_ms) const = 0;
  // enqueues one batched solve on the batch's stream and returns at once; ready() tells whether
  // it has finished (results then come from result())
  virtual void enqueue() = 0;
  virtual bool ready() = 0;
  // one batched solve of every added problem with inputs resident; returns device ms
  virtual float run() = 0;
  // end-to-end: uploads packed complex128 inputs (Σ ny·2 values, add order), runs, downloads
  // packed complex128 (transmitted, reflected) per solve; returns device ms of the whole chain
  virtual float solve_packed(const cd* fields, cd* out) = 0;
  virtual void result(std::int64_t id, Solve2DResult& r) = 0;
  virtual std::size_t device_bytes() const = 0;
  virtual std::int64_t kernel_launches() const = 0;
  virtual int work_items() const = 0;
  virtual int classes() const = 0;
  virtual std::size_t packed_inputs() const = 0;  // complex values of the packed inputs
  // algorithmic work of one run: transforms, FLOPs (5·N·log2 N per transform + 6·N per
  // spectral multiply) and minimal DRAM bytes (pair ids, sparse sources, fields in/out)
  virtual void work(double& transforms, double& flops, double& bytes) const = 0;
};

std::unique_ptr<Batch2D> make_batch2d(int device);

}  // namespace bwpm
