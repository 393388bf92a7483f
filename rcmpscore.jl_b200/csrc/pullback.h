// Quartic pullback kernels (internal).
#pragma once
#include <cuda_runtime.h>

namespace rcmps {

struct PullbackArgs {
  int dp, nstates, nodes, npoints, nodes_per_block;
  int nblk;                    // node blocks
  int ctas;                    // CTAs of the pullback kernel (0: one per work item)
  const double2* samples;      // [state][npoints][7 dp^2]
  long long samples_stride;
  const double2* ops;          // [state][8 dp^2] (Q, Qh, R, Rh, fixed0, fixed6, S, rho)
  long long ops_stride;
  const double* wj;            // [nodes][2]: weight 2|t|, weight source(t)
  const double* coupling;      // [state]
  const double* traj_value;    // [state] scalar channel at the endpoint
  double2* scratch;            // [CTAs][3 dp^2]
  double2* partial;            // [state][nblk][4][dp^2]: slots 0 (m) and 1 (P) are used
  double2* fin;                // [state][8 dp^2]
  double2* cov_out;            // [state][dp^2] (padded)
  double2* env_out;            // [state][dp^2] (padded)
  double* value_out;           // [state]
  int* error_flag;             // [state]
  // packed Z2 states (may be NULL): the trajectory's per-state route flag (int at byte offset
  // packed_offset of each packed_stride-byte record) and the physical dimensions; a packed state
  // with d = dp and d/2 a multiple of 16 skips the structural zeros of its products
  const char* packed = nullptr;
  int packed_stride = 0, packed_offset = 0;
  const int* dims = nullptr;
};

cudaError_t pullback_launch(const PullbackArgs& a, int nblk, cudaStream_t s);
// env_out = g Herm(b_0 at the endpoint) only (the finalize kernel writes the same values later)
cudaError_t quartic_env_launch(const PullbackArgs& a, cudaStream_t s);

// ---- the all-ODE route (pullback_full.cu)
constexpr int kMaxPullSpecs = 3;
constexpr int kMaxPullChannels = 5;
constexpr int kMaxPullEdges = 8;

// One channel spec of the all-ODE route: forward channels fwd0..fwd0+nch-1 and adjoint channels
// adj0..adj0+nch-1 of a sample row; edges (src -> dst, left or right insertion, coefficient).
struct FullPullSpec {
  int nch, fwd0, adj0, comm, nedge, coupling_scaled;
  int esrc[kMaxPullEdges], edst[kMaxPullEdges], eleft[kMaxPullEdges];
  double ecoef[kMaxPullEdges];
};

struct FullPullbackArgs {
  int dp, nstates, nodes, npoints, nodes_per_block, channels;
  const double2* samples;      // [state][npoints][channels dp^2]
  long long samples_stride;
  const double2* ops;          // [state][...] (Q, Qh, R, Rh first)
  long long ops_stride;
  const double* wj;            // [nodes][2]
  const double* coupling;      // [state]
  double2* scratch;            // [CTAs][kMaxPullChannels dp^2]
  double2* partial;            // [state][spec][nblk][6][dp^2]
  double2* fin;                // [state][10 dp^2]
  double2* cov_out;            // [state][dp^2] (padded)
  double2* env_out;            // [state][dp^2] (padded)
  double* value_out;           // [state]
  int* error_flag;             // [state]
};

cudaError_t pullback_full_set_specs(const FullPullSpec* specs, int nspec);
cudaError_t pullback_full_launch(const FullPullbackArgs& a, int nblk, int nspec, cudaStream_t s);
int pullback_full_row_blocks(int dp);
int pullback_row_blocks(int dp);
size_t pullback_smem_bytes(int dp);

}  // namespace rcmps
