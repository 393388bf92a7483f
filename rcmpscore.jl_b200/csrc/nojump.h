// The no-jump preconditioner of the boundary Poisson GMRES (internal).
#pragma once
#include <cuda_runtime.h>
#include "kinetic.h"

namespace rcmps {

// One state's no-jump inverse in the eigenbasis of Q (dp x dp row-major device matrices, the
// physical d x d block followed by an identity/zero padding). Written by nojump_setup_launch.
struct NoJumpSet {
  const double2 *Q, *R, *rho;         // inputs (padded)
  double2 *V, *Vh, *Vinv, *Vinvh;     // eigenvectors of Q, V^dag, V^-1, V^-dag
  double2* nS;                        // -1 / (conj(l_i) + l_j - shift) on the physical block, else 0
  double2* z;                         // the no-jump inverse of the identity
  double2 *H, *U, *W, *M, *T;         // set-up scratch: Hessenberg/Schur form, Schur vectors,
                                      // eigenvectors of T, their inverse, a product
  double2* lambda;                    // [dp] eigenvalues of Q
  double2* den;                       // 1 + tr(rho z)
  double* shift;                      // the reference's shift (0 unless Q has an eigenvalue with
                                      // real part >= -100 eps scale)
  int* status;                        // 0 ready; 1 the QR iteration did not converge; 2 V is
                                      // ill-conditioned or a value is not finite (the state's
                                      // solve then runs unpreconditioned)
  int d, dp;
};

// Number of dp x dp matrices a NoJumpSet takes (outputs and scratch) and of dp-vectors.
constexpr int kNoJumpMats = 11;

cudaError_t nojump_setup_launch(const NoJumpSet* d_sets, int n, int dp, cudaStream_t stream);
// Z_j = P(V_j) for every problem still extending at Arnoldi step j: P(y) = N(y) - tr(rho N(y)) /
// den z with N the no-jump inverse (problem p uses d_sets[p]; a set whose status is not 0 gives
// Z_j = V_j). W: NP dp^2 scratch.
cudaError_t nojump_apply_launch(const ArnoldiProblem* d_probs, int NP, int j, const NoJumpSet* d_sets, double2* W,
                                int dp, cudaStream_t stream);

}  // namespace rcmps
