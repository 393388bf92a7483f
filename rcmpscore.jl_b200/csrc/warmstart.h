// Kernels of the learned GMRES preconditioner and warm start shared with the solvers (internal).
#pragma once
#include <cuda_runtime.h>
#include "kinetic.h"

namespace rcmps {

// C = alpha op(A) op(B) + beta C, FP32, row-major.
cudaError_t warmstart_gemm(bool ta, bool tb, int M, int N, int K, float alpha, const float* A, int lda, const float* B,
                           int ldb, float beta, float* C, int ldc, cudaStream_t s);
// X32[(2 (r d + c) + part) NP + p] = (Re, Im) of V_j[r dp + c] of problem p (the network's input).
cudaError_t net_pack_launch(const ArnoldiProblem* probs, int NP, int j, int d, int dp, float* X32, cudaStream_t s);
// Z_j of problem p from column p of Y32 (the network's output) + identity V_j, zero padding.
cudaError_t net_unpack_launch(const ArnoldiProblem* probs, int NP, int j, int d, int dp, const float* Y32,
                              float identity, cudaStream_t s);

}  // namespace rcmps
