// Host/device interface of the DOP853 trajectory kernel (internal to the library).
#pragma once
#include <cuda_runtime.h>

namespace rcmps {

// Outcome of one trajectory (written by CTA 0 of the state's cluster). Names follow the
// reference's diagnostics (device_control_backend.py:263-265 of rcmps_gpu).
struct TrajStats {
  int status;
  int packed;     // 1: the packed Z2 route was taken
  long long attempts, accepted, rejected, dense_steps, next_point;
  double t, h, min_h, max_h, last_error;
  double value;   // the scalar channel at the endpoint: the quartic density before g
};

// One state of a batch: device pointers of dp x dp complex matrices (zero padded beyond d)
// and its workspace. All matrices row-major double2.
struct TrajState {
  const double2 *Q, *Qh, *R, *Rh;     // Q, Q^dag, R, R^dag
  const double2 *fixed0, *fixed6;     // R rho + rho R^dag, 4 (R + R^dag) (quartic system)
  const double2* S;                   // conj(R) + R^T: weights of the scalar trace (quartic system)
  const double2 *C, *Ch;              // [Q, R] and its adjoint (all-ODE route)
  const double2* rho;                 // initial value of the rho channels (all-ODE route)
  double2 *y, *prop, *k, *z, *P;      // y, proposed [V]; k [16][V]; z [2][V]; P [V]; V = channels dp^2
  double2* L;                         // [V] commutator products O X (all-ODE route)
  double2* samples;                   // [npoints][V]
  TrajStats* stats;
  double atol, rtol;
  long long max_steps;
  int d;                              // physical bond dimension (d <= dp)
  int z2;                             // quartic system: 1 the packed Z2 error norm (10 (d/2)^2 + 1
                                      // entries), 0 the dense one, -1 refused (no exact Z2 structure)
  // split-precision engine (dp = 64): BF16 slices of the constant operands and their scales,
  // written by split_prep_launch (split_state_bytes() per state)
  const unsigned char* split_g1;      // [rank 4][direction 2][chunk 2] panel^T slices, 48 KB each
  const unsigned char* split_g2;      // [direction 2][chunk 4] [F1^T | F2^T] slices, 48 KB each
  const double* split_g1_scale;       // [rank][direction][32]
  const double* split_g2_scale;       // [direction][64]
};

struct TrajControls {
  double endpoint;          // sqrt(half_window)
  double initial_h;
  unsigned long long max_ns;  // device-clock watchdog in ns (0: none)
  int ring = 0;               // stages of the FP64 engine's operand ring on the quartic system (2, 3;
                              // anything else: the default 4)
  int groups = 0;             // CTAs per row block of a state, each for a group of channels: 1, 2 or 4
                              // (0: chosen by the launch, see trajectory_groups)
};

cudaError_t trajectory_set_tables();
// system: 0 the reduced quartic system (7 channels + scalar), 1 the all-ODE route (26 channels),
// 2 the first monomial of <phi> (4 channels). engine: 0 FP64 tensor cores (mma.sync), 1 the
// split-precision BF16 engine on tcgen05 (system 0 and dp = 64 only; needs split_prep_launch).
cudaError_t trajectory_launch(int system, int dp, const TrajState* d_states, int nstates, const double* d_points,
                              int npoints, const TrajControls& ctl, cudaStream_t stream, int engine = 0);
// Bytes of split-engine constants per state, and the kernel that writes them (dp = 64).
size_t split_state_bytes();
void split_state_pointers(unsigned char* block, TrajState& t);   // t.split_* inside `block`
cudaError_t split_prep_launch(const TrajState* d_states, int nstates, cudaStream_t stream);
int trajectory_channels(int system);
// The channel groups a launch of nstates states takes (requested 0: the most, up to 4, that keeps
// every state's cluster resident at once; 1, 2, 4: the largest supported count up to that one).
// A state's cluster has dp/16 x groups CTAs (at most 16). Only the FP64 engine on the quartic
// system groups; everything else takes 1.
int trajectory_groups(int system, int dp, int nstates, int requested, int engine = 0);
cudaError_t node_weights_launch(const double* d_points, const double* d_weights, int n, double* d_wj,
                                cudaStream_t stream);

}  // namespace rcmps
