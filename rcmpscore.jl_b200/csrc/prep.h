// Padding and per-state operator preparation (internal).
#pragma once
#include <cuda_runtime.h>

namespace rcmps {
// Number of dp x dp matrices in the operator block of one state (Q, Qh, R, Rh, fixed0, fixed6, S, rho).
constexpr int kOps = 8;
enum OpIndex { kQ = 0, kQh = 1, kR = 2, kRh = 3, kFixed0 = 4, kFixed6 = 5, kS = 6, kRho = 7, kC = 8, kCh = 9 };
// The all-ODE route adds the commutator C = QR - RQ and C^dag.
constexpr int kOpsFull = 10;

cudaError_t launch_pad(const double* src, const long long* d_src_off, const int* d_dims, double* dst, int dp,
                       long long stride, int nstates, cudaStream_t stream);
cudaError_t launch_unpad(const double* src, long long stride, int dp, const long long* d_dst_off,
                         const int* d_dims, double* dst, int nstates, cudaStream_t stream);
// dst (packed d_i^2 per state) (+)= src (padded dp^2 per state)
cudaError_t launch_unpad_acc(const double* src, long long stride, int dp, const long long* d_dst_off,
                             const int* d_dims, double* dst, int nstates, bool accumulate, cudaStream_t stream);
// dst[idx[i]] (+)= src[i]
cudaError_t launch_scatter_values(const double* src, int n, const int* d_idx, double* dst, bool accumulate,
                                  cudaStream_t stream);
// samples (padded [npoints][7][dp][dp]) -> out [npoints][7 d^2 + 1]; the scalar is `value` at the endpoint
cudaError_t launch_export_samples(const double2* samples, int dp, int d, int npoints, const double* value,
                                  double* out, cudaStream_t stream);
cudaError_t launch_commutator(double* ops, int dp, long long ops_stride, int nstates, cudaStream_t stream);
// out[s] = Re tr of the leading d_s x d_s block of the dp x dp matrix at samples + s stride + offset
cudaError_t launch_endpoint_trace(const double2* samples, long long stride, long long offset, int dp,
                                  const int* d_dims, double* out, int nstates, cudaStream_t stream);
// Exact Z2 block structure of each padded state (ode_backend.py:246-256): even d, R's diagonal
// blocks, K's and rho's off-diagonal blocks exactly zero, ||rho - rho^dag||_F <= 1e-13 max(1,
// ||rho||_F). Writes z2_flags[i] = 1 where the structure holds; mode 1 writes -1 elsewhere
// (refused), mode 2 writes 0 there.
cudaError_t launch_z2_check(const double* R, const double* K, const double* rho, const int* d_dims, int dp,
                            long long in_stride, int nstates, int mode, int* z2_flags, long long flag_stride,
                            cudaStream_t stream);
cudaError_t launch_prepare(const double* R, const double* K, const double* rho, double* ops, int dp,
                           long long in_stride, long long ops_stride, int nstates, cudaStream_t stream);
}  // namespace rcmps
