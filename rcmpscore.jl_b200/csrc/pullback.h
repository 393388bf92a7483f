// Quartic pullback kernels (internal).
#pragma once
#include <cuda_runtime.h>

namespace rcmps {

struct PullbackArgs {
  int dp, nstates, nodes, npoints, nodes_per_block;
  const double2* samples;      // [state][npoints][7 dp^2]
  long long samples_stride;
  const double2* ops;          // [state][8 dp^2] (Q, Qh, R, Rh, fixed0, fixed6, S, rho)
  long long ops_stride;
  const double* wj;            // [nodes][2]: weight 2|t|, weight source(t)
  const double* coupling;      // [state]
  const double* traj_value;    // [state] scalar channel at the endpoint
  double2* scratch;            // [CTAs][3 dp^2]
  double2* partial;            // [state][nblk][4][dp^2]
  double2* fin;                // [state][8 dp^2]
  double2* cov_out;            // [state][dp^2] (padded)
  double2* env_out;            // [state][dp^2] (padded)
  double* value_out;           // [state]
  int* error_flag;             // [state]
};

cudaError_t pullback_launch(const PullbackArgs& a, int nblk, cudaStream_t s);
int pullback_row_blocks(int dp);
size_t pullback_smem_bytes(int dp);

}  // namespace rcmps
