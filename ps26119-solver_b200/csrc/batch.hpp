// batch.hpp — host interface of the GPU batch engine: r²HPDHG in lockstep on K scenarios that
// share one constraint matrix (≙ ps26119::solve_batch, reference include/ps26119/batch.h:22-33,
// src/pdhg/batch.cpp:129-441).
#pragma once

#include <chrono>
#include <string>
#include <vector>

#include "engine.hpp"

namespace b200 {

// One scenario: host arrays of the base's sizes; nullptr keeps the base model's vector
// (an empty std::vector in the reference's Scenario).
struct BatchScenarioView {
  const double *c = nullptr, *col_lower = nullptr, *col_upper = nullptr, *row_lower = nullptr, *row_upper = nullptr;
};

struct BatchOutcome {
  Status status = Status::NotSolved;
  std::string message;
  std::vector<double> x, y, z;  // original space; y in the model's sense (z = c − Aᵀy)
  double objective = 0, dual_objective = 0, primal_residual = 0, dual_residual = 0, gap = 0;
  long long iterations = 0, iterations_to_fast = -1, kernel_launches = 0;
  double seconds = 0, setup_seconds = 0, seconds_to_fast = -1, primal_weight = 1;
  double spmm_kernel_ms = 0;     // the batch's SpMM kernels (CUDA events), whole batch
  long long spmm_launches = 0;
};

// Runs the scenarios listed in `slots` (indices into `scenarios`, all valid) on the device;
// outcomes are returned at the same indices (others untouched). `t0` is the start of the whole
// batch call (time limit and reported seconds count from it, batch.cpp:131-132).
std::vector<BatchOutcome> run_batch_host(const HostModelView& base, const std::vector<BatchScenarioView>& scenarios,
                                         const std::vector<int>& slots, const EngineOptions& opt,
                                         std::chrono::steady_clock::time_point t0);

}  // namespace b200
