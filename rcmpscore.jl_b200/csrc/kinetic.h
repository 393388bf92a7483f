// Kinetic resolvent kernels (internal).
#pragma once
#include <cuda_runtime.h>

namespace rcmps {

// out = L(X) (mode 0) or res[rb] = |X - shift L(X) - rhs|^2 of row block rb (mode 1), with
// L(X) = A1 X + X A1h + A2 X A2h.
struct LindbladTask {
  const double2* X;          // NULL: skip
  double2* out;
  const double2 *A1, *A1h, *A2, *A2h;
  const double2* rhs;
  double* res;               // [dp/16]
  double shift;
  int* flag;                 // set when a bounded wait gave up
  const double2* trw;        // non-NULL: out = -L(X) + tr(trw X) I_d (the Poisson/stationary operators)
  int d;                     // physical dimension (I_d: identity on the physical block)
};

// One Krylov problem (I - c L) x = rhs with its Arnoldi basis.
struct ArnoldiProblem {
  double2* V;                // [kmax+1][ldv]
  long long ldv;
  double2* H;                // [(kmax+1)][kmax] row-major
  double2* W;                // work vector [n]
  const double2* rhs;        // [n]
  double2* partial;          // [nchunk][kmax1]
  double* norms;             // [2 nchunk]
  double2* Yt;               // [nshift][kmax] projected solutions
  double2* LV;               // [kmax][ldv] L(V_j), kept for the true residuals (kinetic problems; else NULL)
  double2* X;                // [nshift][n] solutions (adjoint problems: conjugate transposed)
  const double2 *A1, *A1h, *A2, *A2h;   // L = A1 X + X A1h + A2 X A2h
  const double2* trw;        // GMRES operators: -L(X) + tr(trw X) I
  int* flag;
  // restarted GMRES (solvers.cu)
  double2* x;                // [n] solution
  const double2* b;          // [n] right-hand side
  double2* g;                // [kmax + 1] rotated residual vector
  double2* cs;               // [kmax] Givens cosines (real part used) and sines
  double2* sn;
  double gtarget, gres, bnorm, gtol;
  int converged, restarts, d, iters;
  double beta, estimate, residual;
  int n, n_phys, dp, kmax, kmax1, target;
  int k, exhausted, nonfinite, active, solve, reconstruct, adjoint;
  int reorth;                // the current Arnoldi step runs its second Gram-Schmidt pass
  // flexible GMRES (solvers_host.cu): Z_j = M V_j, the basis passed through a preconditioner M;
  // the Lindblad action is applied to Z_j and the update is x += Z y. NULL: unpreconditioned.
  double2* Z;                // [kmax][ldv]
};

struct KineticSetup {
  int dp;
  const double2* ops;        // [state][8 dp^2]
  long long ops_stride;
  double2* comm;             // [state][2 dp^2]: C, C^dag
  double2* rhs;              // [state][4 dp^2]
};

struct ContractArgs {
  int dp, nstates, nodes, nodes_per_block;
  const double2* const* X;   // [2 nstates]: forward solutions of (state, op)
  const double2* const* A;   // [2 nstates]: adjoint solutions, conjugate transposed
  const double2* const* Q;   // [nstates]
  const double2* const* Qh;
  const double2* const* R;
  const double2* const* Rh;
  const double2* const* rho;
  const double* weights;     // [nodes]
  const double* shifts;      // [nodes]
  double2* partial;          // [2 nstates][nblk][4][dp^2]
  double2* fin;              // [nstates][12 dp^2]; covector at 9, environment at 10
  double* value_out;         // [nstates]
  int* error_flag;           // [nstates]
};

cudaError_t lindblad_launch(int dp, const LindbladTask* d_tasks, int ntasks, int mode, cudaStream_t s);
cudaError_t arnoldi_tasks_launch(const ArnoldiProblem* d_probs, int nprob, int j, LindbladTask* d_tasks,
                                cudaStream_t s);
cudaError_t arnoldi_start_launch(ArnoldiProblem* d_probs, int nprob, cudaStream_t s);
cudaError_t cgs_step_launch(ArnoldiProblem* d_probs, int nprob, int j, int n, cudaStream_t s);
// The same Gram-Schmidt step in one launch (a cluster per problem; no partial or norm arrays).
cudaError_t cgs_fused_launch(ArnoldiProblem* d_probs, int nprob, int j, int n, cudaStream_t s);
// The Gram-Schmidt step by whichever of the two forms suits the batch (sms: the device's SMs).
cudaError_t gram_schmidt_launch(ArnoldiProblem* d_probs, int nprob, int j, int n, int sms, cudaStream_t s);
// W = L(V_j) (or L(Z_j)) of step j of every problem still extending, the task built in the kernel.
cudaError_t lindblad_arnoldi_launch(int dp, const ArnoldiProblem* d_probs, int nprob, int j, cudaStream_t s);
cudaError_t hessenberg_launch(ArnoldiProblem* d_probs, int nprob, const double* d_shifts, int nshift,
                              double2* scratch, long long slot_elems, int nslots, int kmax, cudaStream_t s);
// X = V Y for every shift and the true residual |X - c L(X) - rhs|^2 = |(V - c LV) Y - rhs|^2 per
// (problem, shift, 64-column tile) into res[p][s][n/64]
cudaError_t reconstruct_residual_launch(ArnoldiProblem* d_probs, int nprob, const double* d_shifts, int nshift,
                                        int n, double* d_res, cudaStream_t s);
cudaError_t residual_reduce_launch(ArnoldiProblem* d_probs, int nprob, const double* d_res, int nshift, int rbs,
                                   cudaStream_t s);
cudaError_t kinetic_rhs_launch(const KineticSetup& a, int nstates, cudaStream_t s);
cudaError_t contract_launch(const ContractArgs& a, int nblk, cudaStream_t s);

}  // namespace rcmps
