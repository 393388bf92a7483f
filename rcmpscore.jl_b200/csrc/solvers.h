// GMRES, boundary/finish and stationary kernels (internal).
#pragma once
#include <cuda_runtime.h>
#include "kinetic.h"

namespace rcmps {

struct FinishArgs {
  int dp;
  const int* dims;           // [n]
  const double2* ops;        // [n][8 dp^2]
  long long ops_stride;
  const double2* env;        // [n][dp^2] environment (padded)
  const double2* cov;        // [n][dp^2] covector (padded)
  double2* b;                // [n][dp^2] Poisson right-hand side
  const double2* x;          // [n][dp^2] Poisson solution H
  double2* tmp;              // [n][4 dp^2]; gradient at slot 3
  double metric_reg;
  int* status;               // [n]
};

struct StationaryArgs {
  int dp;
  const int* dims;
  const double2* x;          // [n][dp^2] GMRES solution
  double2* rho;              // [n][dp^2] output (padded)
  double2* tmp;              // [n][dp^2]
  double* herm;              // [n] |rho - rho^dag| before symmetrisation
  double* scale;             // [n] max(1, 2|Q| + |R|^2)
  const double2* ops;        // [n][8 dp^2]
  long long ops_stride;
  double tolerance;
  int* status;
};

cudaError_t gmres_residual_launch(ArnoldiProblem* d, int nprob, int n, cudaStream_t s);
cudaError_t gmres_bnorm_launch(ArnoldiProblem* d, int nprob, cudaStream_t s);
cudaError_t gmres_givens_launch(ArnoldiProblem* d, int nprob, int j, cudaStream_t s);
cudaError_t gmres_update_launch(ArnoldiProblem* d, int nprob, int n, int kmax, cudaStream_t s);
cudaError_t gmres_x_tasks_launch(const ArnoldiProblem* d, int nprob, LindbladTask* tasks, cudaStream_t s);
cudaError_t boundary_rhs_launch(const FinishArgs& a, int n, cudaStream_t s);
cudaError_t finish_launch(const FinishArgs& a, int n, cudaStream_t s);
cudaError_t stationary_finish_launch(const StationaryArgs& a, int n, cudaStream_t s);

}  // namespace rcmps
