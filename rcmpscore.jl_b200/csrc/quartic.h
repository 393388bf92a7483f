// Quartic term orchestration (internal).
#pragma once
#include <cuda_runtime.h>
#include <functional>
#include <vector>
#include "../../include/rcmps_b200.h"
#include "context.h"

namespace rcmps {

struct QuarticJob {
  int n = 0;
  const int* dims = nullptr;            // host
  const double* couplings = nullptr;    // host, NULL: 1
  const double *R = nullptr, *K = nullptr, *rho = nullptr;   // device, packed
  rcmps_settings settings{};
  const rcmps_state_controls* controls = nullptr;   // host [n], per-state tolerances, optional
  double* value = nullptr;              // device [n] (g * quartic density), optional
  double* covector = nullptr;           // device packed, optional
  double* environment = nullptr;        // device packed, optional
  double* samples_out = nullptr;        // device, single-state samples, optional
  rcmps_state_stats* stats = nullptr;   // host [n]
  bool accumulate = false;              // add into value/covector/environment instead of storing
  int slot = 0;                         // context slot (workspace, staging, events)
  double memory_share = 0.7;            // fraction of free device memory this job may hold
  int system = 0;                       // 0: the quartic term (reduced system); 1: all terms by ODEs
  // Early environment (system 0): when on_env is set, the environment is written to `environment`
  // right after each trajectory, before the pullback; after the last one env_ready is recorded on
  // the stream and on_env() is called (from the calling thread), so that a boundary solve can start
  // while the pullback runs.
  cudaEvent_t env_ready = nullptr;
  int pullback_ctas = 0;                // CTAs of the quartic pullback (0: one per work item)
  std::function<void()> on_env;
};

cudaError_t quartic_init();
int quartic_run(rcmps_context* ctx, QuarticJob& job, cudaStream_t stream);

void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);
void trajectory_points(double half_window, int n_quad, std::vector<double>& points, std::vector<double>& weights);
int check_settings(rcmps_context* ctx, const rcmps_settings* s);
int check_dims(rcmps_context* ctx, int n, const int* dims);

}  // namespace rcmps
