// Kinetic orchestration (internal).
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "../../include/rcmps_b200.h"
#include "context.h"

namespace rcmps {

struct KineticJob {
  int n = 0;
  const int* dims = nullptr;            // host
  const double *R = nullptr, *K = nullptr, *rho = nullptr;   // device, packed
  rcmps_settings settings{};
  double* value = nullptr;              // device [n], optional
  double* covector = nullptr;           // device packed, optional
  double* environment = nullptr;        // device packed, optional
  rcmps_state_stats* stats = nullptr;   // host [n]
  bool accumulate = false;
  int slot = 1;
  double memory_share = 0.7;
};

void angular_grid(int nodes, std::vector<double>& shifts, std::vector<double>& weights);
int kinetic_run(rcmps_context* ctx, KineticJob& job, cudaStream_t stream);

}  // namespace rcmps
