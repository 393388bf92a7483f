// Boundary/finish and stationary orchestration (internal).
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "../../include/rcmps_b200.h"
#include "context.h"

namespace rcmps {

struct FinishJob {
  int n = 0;
  const int* dims = nullptr;                  // host
  const double *R = nullptr, *K = nullptr, *rho = nullptr;   // device, packed
  const double *covector = nullptr, *environment = nullptr;  // device, packed
  rcmps_settings settings{};
  double* gradient = nullptr;                 // device, packed
  rcmps_state_stats* stats = nullptr;         // host [n]
  int slot = 2;
  // device, packed, optional: initial guesses of the boundary Poisson solutions (a warm start);
  // the stopping target stays tol max(1, |b|)
  const double* x0 = nullptr;
  // optional: a learned right preconditioner (flexible GMRES); every state has d with 2 d^2 = net->n
  const rcmps_gmres_network* net = nullptr;
  int max_restarts = 200;                     // restart cycles of the boundary GMRES
};

struct StationaryJob {
  int n = 0;
  const int* dims = nullptr;
  const double *R = nullptr, *K = nullptr;    // device, packed
  double tolerance = 1e-11;
  double* rho = nullptr;                      // device, packed
  // device, packed, optional: a nearby density to start from (the warm correction of
  // stationary_correction.py:19-96); the GMRES then solves for the correction to an absolute
  // residual of `tolerance`
  const double* rho_previous = nullptr;
  rcmps_state_stats* stats = nullptr;
  int slot = 2;
};

int finish_run(rcmps_context* ctx, FinishJob& job, cudaStream_t stream);

// finish_run in two halves: finish_solve needs R, K, rho and the environment (the boundary
// Poisson GMRES); finish_complete then needs the covector (finish kernel, metric solve, gradient).
// The plan keeps the workspace layout between the two; the slot's workspace must not be reused
// in between.
struct FinishPlan {
  struct Group;
  std::vector<Group> groups;
  std::vector<long long> off;
  bool prepared = false;   // finish_prepare ran
  bool nojump = false;     // the boundary GMRES takes the no-jump preconditioner
  int m = 64;              // its restart length
  FinishPlan();
  ~FinishPlan();
};
// finish_prepare needs only R, K and rho: the workspace, the per-state operators and the no-jump
// preconditioner's eigenbasis. A caller may run it before the environment exists (the composite
// entry does, on the solve stream, while the trajectory integrates); finish_solve runs it itself
// otherwise.
int finish_prepare(rcmps_context* ctx, FinishJob& job, cudaStream_t stream, FinishPlan& plan);
int finish_solve(rcmps_context* ctx, FinishJob& job, cudaStream_t stream, FinishPlan& plan);
int finish_complete(rcmps_context* ctx, FinishJob& job, cudaStream_t stream, FinishPlan& plan);
int stationary_run(rcmps_context* ctx, StationaryJob& job, cudaStream_t stream);
// The boundary Poisson solve alone: H (device, packed) and the per-state GMRES statistics.
int boundary_run(rcmps_context* ctx, FinishJob& job, double* H, cudaStream_t stream);

}  // namespace rcmps
