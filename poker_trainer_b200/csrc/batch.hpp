// Batched river solves (batch.cu): many independent river spots solved
// together by one persistent kernel per block of iterations.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "../../include/dcfr.h"
#include "engine.hpp"
#include "game.hpp"
#include "plan.hpp"

namespace dcfr {

constexpr int BATCH_MAX_THREADS = 256;  // threads per block of the batched kernel
constexpr int BATCH_MAX_SLOTS = 4096;   // reach slots of one spot's traversal

class Batch {
 public:
  static Status create(const dcfr_config* cfgs, int count, std::unique_ptr<Batch>& out);
  ~Batch();

  int count() const;
  uint32_t iterations() const;
  double last_iterate_ms() const;
  uint64_t kernel_launches() const;
  dcfr_batch_tuning tuning() const;
  // Algorithmic bytes of one DCFR iteration of every spot (the single
  // solve's figure summed over spots).
  double iteration_bytes() const;

  Status iterate(uint32_t n);
  Status exploitability(double* out);
  Status storage_len(int spot, uint64_t& len) const;
  Status download(int spot, float* regrets, float* sums);
  Status set_tuning(const dcfr_batch_tuning& t);
  Status autotune(uint32_t trial_iterations, dcfr_batch_tuning& best);

 private:
  Batch();
  Status root_values(int mode, std::vector<double>& out);
  struct Impl;
  std::unique_ptr<Impl> impl_;
};

}  // namespace dcfr
