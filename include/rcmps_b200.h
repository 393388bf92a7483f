/* C ABI of the B200 fg_phi4 library (librcmps_b200.so).
 *
 * The phi^4 energy density of a relativistic continuous matrix product state and its
 * Riemannian gradient, as the reference's GPU optimizer evaluates it (RcmpsCore.jl, package
 * rcmps_gpu). Matrices are complex128, row-major (the memory of a C-ordered NumPy array),
 * passed as `double*` pointing at interleaved (re, im) pairs. A batch packs its states one
 * after the other: state i occupies dims[i]^2 complex values at offset sum_{j<i} dims[j]^2.
 *
 * Every entry returns an rcmps status (0 = success). A per-state status in the stats records
 * which numerical requirement failed; rcmps_context_error() describes the last failure.
 * No entry falls back to host arithmetic.
 */
#ifndef RCMPS_B200_H
#define RCMPS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. 0-6 are the reference's device-controller codes
 * (gpu/src/rcmps_gpu/optimizer/runtime/device_control_backend.py:23-27 and the timeout 6 of
 * persistent_trajectory_backend.py:29). */
#define RCMPS_OK 0
#define RCMPS_MAX_STEPS 1
#define RCMPS_STEP_UNDERFLOW 2
#define RCMPS_NONFINITE_ERROR 3
#define RCMPS_SOURCE_DOMAIN 4
#define RCMPS_MISSING_SAMPLES 5
#define RCMPS_DEVICE_TIMEOUT 6
#define RCMPS_WAIT_LIMIT 7
#define RCMPS_KRYLOV_FAILURE 8
#define RCMPS_SOLVE_FAILURE 9
#define RCMPS_NONFINITE_RESULT 10
#define RCMPS_INVALID_ARGUMENT 20
#define RCMPS_CUDA_ERROR 21
#define RCMPS_OUT_OF_MEMORY 22

typedef struct rcmps_context rcmps_context;

/* Integration and solver controls. Defaults (rcmps_default_settings) are those of the
 * reference's optimizer command line (gpu/src/rcmps_gpu/optimizer/cli.py:39-42 and
 * runtime/sweep_driver.py:122-168). */
typedef struct rcmps_settings {
  double half_window;          /* W: the window is x in [-W, W], t in [-sqrt W, sqrt W]; 0 < W <= 40 */
  int n_quad;                  /* Gauss-Legendre nodes per half window */
  double atol, rtol;           /* DOP853 tolerances */
  double initial_step;         /* first trial step in t */
  long long max_steps;         /* attempted steps per trajectory */
  double max_device_seconds;   /* device-clock watchdog per trajectory launch (0: none) */
  int kinetic_nodes;           /* angular Gauss nodes of the kinetic resolvents */
  double krylov_tolerance;     /* true relative residual of every shifted solve */
  int krylov_initialdim;       /* first Arnoldi basis size (doubles until converged) */
  int krylov_maxdim;           /* largest basis */
  double metric_reg;           /* regulariser of the metric solve */
  double boundary_tolerance;   /* GMRES tolerance of the boundary Poisson solve */
  int symmetry;                /* quartic route: 0 the unpacked channels for every state (the
                                  reference's --reduced); 1 the packed Z2 route for every state,
                                  a state without the exact Z2 block structure fails with
                                  RCMPS_INVALID_ARGUMENT (--packed-z2, the default of
                                  evaluate_quartic_persistent_trajectory); 2 packed for the states
                                  with that structure, unpacked for the others */
  int precision;               /* quartic trajectory products: 0 FP64 tensor cores (DMMA); 1 split
                                  precision on the 5th-generation tensor cores (each FP64 operand cut
                                  into seven 7-bit BF16 slices, slice products accumulated in FP32 in
                                  tensor memory, recombined in FP64; error about 2^-48 of the row and
                                  column scales per term) for the states of padded dimension 64, FP64
                                  for the others. The DOP853 error estimate and step control, the
                                  stage sums and every solve stay FP64. */
  int trajectory_groups;       /* FP64 quartic trajectory: CTAs per 16-row block of a state, each for
                                  a group of channels (1, 2 or 4; a state's cluster has dp/16 times
                                  as many CTAs, at most 16). 0 (default): the most that keeps every
                                  state of the launch resident at once, so a lone state spreads over
                                  up to 16 SMs and a full batch keeps one CTA per row block. Results
                                  agree to rounding (the reductions' summation order changes). */
  int boundary_preconditioner; /* boundary Poisson GMRES: 1 (default) right-preconditioned by the
                                  no-jump inverse with the Sherman-Morrison correction, as the
                                  reference solves it (numerics.py:37-71, 103-117), restart
                                  min(40, d^2); the inverse is applied in the eigenbasis of Q
                                  (found once per state and call on the device); a state whose
                                  eigenbasis is ill-conditioned runs unpreconditioned. 0:
                                  unpreconditioned GMRES(64). */
} rcmps_settings;

/* Per-state diagnostics. */
typedef struct rcmps_state_stats {
  int status;                  /* first failure of this state, RCMPS_OK if none */
  int failed_component;        /* 0 none, 1 trajectory, 2 pullback, 3 kinetic, 4 boundary, 5 stationary */
  long long attempts, accepted, rejected, dense_steps, rhs_calls;
  double t_end, last_step, min_step, max_step;
  double quartic_value;        /* g * <phi^4> */
  double kinetic_value;        /* kinetic1 + kinetic2 */
  int krylov_basis[4];         /* R forward, R adjoint, [Q,R] forward, [Q,R] adjoint */
  double krylov_residual;      /* largest true relative residual of the shifted solves */
  int gmres_iterations;        /* boundary Poisson solve */
  double boundary_residual;
  int packed_z2;               /* 1: the quartic term took the packed Z2 route */
  int gmres_matvecs;           /* boundary Poisson solve: operator applications as the reference's
                                  GMRES counts them (Arnoldi steps plus one true residual per
                                  restart cycle) */
} rcmps_state_stats;

void rcmps_default_settings(rcmps_settings* settings);

/* Context of one device: streams, events and a device workspace that grows on demand.
 * Replaces the per-call solver objects of the reference (PersistentTrajectoryDOP853,
 * persistent_trajectory_backend.py:339-403; KineticContext, kinetic_backend.py:236-275).
 * A context serves one call at a time, as the reference's coordinator serves one state at a
 * time (overlap_sweep_driver.py:132-135): its workspace, streams and cached GMRES graphs are
 * shared by its calls. Use one context per host thread for concurrent calls. */
int rcmps_context_create(int device, rcmps_context** context);
int rcmps_context_destroy(rcmps_context* context);
const char* rcmps_context_error(const rcmps_context* context);
const char* rcmps_status_name(int status);
/* Device milliseconds of the phases of the last batched call: 0 trajectory, 1 pullback,
 * 2 kinetic, 3 boundary/finish (from the environment to the gradient), 4 whole call, 5 the
 * boundary solve's preparation (operators and the no-jump preconditioner's eigenbasis; it runs
 * on the solve stream beside the trajectory), 6 the boundary GMRES alone (from the environment
 * to the solution; phase 3 also waits for the pullback's covector). */
int rcmps_last_timings(const rcmps_context* context, float* milliseconds, int n);
/* Bytes of device workspace that rcmps_fg_phi4_batch needs for these dimensions. */
long long rcmps_workspace_bytes(const rcmps_context* context, int n_states, const int* dims,
                                const rcmps_settings* settings);

/* phi^4 energy density and finished gradient of a batch of states, on device memory.
 * Replaces the objective callable objective(r, k, rho, coupling, args, xp) ->
 * (energy, gradient, stats) (runtime/sweep_driver.py:78-119; GPU form
 * runtime/overlap_sweep_driver.py:132-212), for n_states states at once.
 *   dims, couplings, stats: host arrays of n_states
 *   R, K, rho: device, packed; K Hermitian, rho the stationary density of (Q, R)
 *   energy: device [n_states]; gradient: device, packed
 *   covector, environment: device, packed, or NULL (the raw summed components)
 * `stream` is a cudaStream_t (NULL: the context's stream); the call returns after the
 * results are complete. */
int rcmps_fg_phi4_batch(rcmps_context* context, int n_states, const int* dims, const double* couplings,
                        const double* R, const double* K, const double* rho, const rcmps_settings* settings,
                        double* energy, double* gradient, double* covector, double* environment,
                        rcmps_state_stats* stats, void* stream);

/* Per-state integration controls of rcmps_fg_phi4_batch_controls. A value <= 0 takes the
 * settings' value. No counterpart in the reference, whose objective integrates one state per
 * call with one (atol, rtol) pair (runtime/sweep_driver.py:78-119): here a batch of states with
 * mixed tolerance pairs shares one persistent trajectory launch. */
typedef struct rcmps_state_controls {
  double atol, rtol;           /* DOP853 tolerances of this state's quartic trajectory */
} rcmps_state_controls;

/* rcmps_fg_phi4_batch with per-state DOP853 tolerances: controls[i] (host, n_states entries)
 * replaces settings->atol / rtol for state i; the same checks apply (atol > 0,
 * rtol >= 100 eps). controls = NULL is rcmps_fg_phi4_batch. */
int rcmps_fg_phi4_batch_controls(rcmps_context* context, int n_states, const int* dims, const double* couplings,
                                 const double* R, const double* K, const double* rho,
                                 const rcmps_settings* settings, const rcmps_state_controls* controls,
                                 double* energy, double* gradient, double* covector, double* environment,
                                 rcmps_state_stats* stats, void* stream);

/* Same with every array in host memory (copies in and out inside the call, through a device
 * buffer the context keeps and grows on demand). */
int rcmps_fg_phi4_batch_host(rcmps_context* context, int n_states, const int* dims, const double* couplings,
                             const double* R, const double* K, const double* rho,
                             const rcmps_settings* settings, double* energy, double* gradient,
                             double* covector, double* environment, rcmps_state_stats* stats);

/* The g*phi^4 term: value, raw covector and environment, scaled by the coupling, on device memory.
 * Replaces evaluate_quartic_persistent_trajectory(R, Q, rho, g, ...) -> dict(value, covector,
 * environment, stats) (runtime/persistent_trajectory_backend.py:439-461). */
int rcmps_quartic_batch(rcmps_context* context, int n_states, const int* dims, const double* couplings,
                        const double* R, const double* K, const double* rho, const rcmps_settings* settings,
                        double* value, double* covector, double* environment, rcmps_state_stats* stats,
                        void* stream);

/* All three terms (kinetic1 + kinetic2 + g phi^4) by ODEs: value, raw covector and environment,
 * on device memory. The 26-channel system is integrated by the same DOP853 controller and
 * pulled back per channel spec. Replaces evaluate_phi4(R, Q, rho, g, ...) -> dict(value,
 * covector, environment, stats) (runtime/ode_backend.py:851-858), the objective's --mode ode
 * (runtime/sweep_driver.py:90-92) and Julia's default kinetic_backend=:ode
 * (src/observables.jl:131-159). stats[i].quartic_value holds the total value of state i and
 * kinetic_value stays 0. Follow with rcmps_finish_gradient_batch for the finished gradient. */
int rcmps_phi4_ode_batch(rcmps_context* context, int n_states, const int* dims, const double* couplings,
                         const double* R, const double* K, const double* rho, const rcmps_settings* settings,
                         double* value, double* covector, double* environment, rcmps_state_stats* stats,
                         void* stream);

/* The one-point function <phi> by the ODE of the first monomial: F0 = rho and
 * dF1 = 2|t| L(F1) dt + j(t) (R F0 + F0 R^dag) dt with their adjoint channels, integrated by the
 * same DOP853 controller; phi[i] = Re tr F1 at the endpoint (device, [n_states]). Replaces
 * validate_sweep.phi_by_ode(r, k, rho, controls, xp) (optimizer/validate_sweep.py:23-32),
 * RcmpsCore's phi_monomial(s, 1). stats[i].quartic_value holds the same value. */
int rcmps_phi_ode_batch(rcmps_context* context, int n_states, const int* dims, const double* R, const double* K,
                        const double* rho, const rcmps_settings* settings, double* phi, rcmps_state_stats* stats,
                        void* stream);

/* The trajectory alone, for one state: samples [2 n_quad + 1][7 d^2 + 1] complex (the seven
 * channels at every Gauss node and the endpoint, and the scalar channel, only filled at the
 * endpoint). Replaces PersistentTrajectoryDOP853.run() -> (samples, stats)
 * (runtime/persistent_trajectory_backend.py:405-432). Device memory. */
int rcmps_quartic_samples(rcmps_context* context, int d, const double* R, const double* K, const double* rho,
                          const rcmps_settings* settings, double* samples, rcmps_state_stats* stats,
                          void* stream);

/* The two kinetic terms (unit coefficients), raw covector and environment, on device memory.
 * Replaces kinetic_raw(q, r, rho, nodes, ...) -> dict(value, covector, environment, stats)
 * (runtime/kinetic_backend.py:499-592; runtime/cooperative_arnoldi.py:293-316). */
int rcmps_kinetic_batch(rcmps_context* context, int n_states, const int* dims, const double* R,
                        const double* K, const double* rho, const rcmps_settings* settings, double* value,
                        double* covector, double* environment, rcmps_state_stats* stats, void* stream);

/* Boundary Poisson correction and metric solve, on device memory. Replaces
 * finish_gradient(q, r, rho, covector, environment, metric_reg, tolerance) -> (gradient, stats)
 * (runtime/numerics.py:120-126). */
int rcmps_finish_gradient_batch(rcmps_context* context, int n_states, const int* dims, const double* R,
                                const double* K, const double* rho, const double* covector,
                                const double* environment, const rcmps_settings* settings, double* gradient,
                                rcmps_state_stats* stats, void* stream);

/* A learned approximate inverse of the boundary operator, used as the right preconditioner of a
 * flexible GMRES: M v = W2 (W1 v) + identity v on the n = 2 d^2 reals of a d x d matrix ((Re, Im)
 * interleaved, row-major), FP32 device weights W1 (rank x n) and W2 (n x rank) trained by
 * rcmps_warmstart_* (rcmps_b200.warmstart). No counterpart in the reference. */
typedef struct rcmps_gmres_network {
  const float* W1;
  const float* W2;
  int n, rank;
  float identity;
} rcmps_gmres_network;

/* The boundary Poisson solve alone: H with (-L*(H) + tr(rho H) I) = environment - tr(rho environment) I,
 * by restarted GMRES(64) to |r| <= boundary_tolerance max(1, |b|), on device memory. x0 (packed, or
 * NULL) is an initial guess of H for each state (a warm start, e.g. the learned one of
 * rcmps_b200.warmstart); network (or NULL) a learned right preconditioner, applied in flexible
 * GMRES (the basis passes through M in FP32, the Arnoldi relation and the update stay FP64, so
 * the attainable accuracy is that of the plain solve); every state then has the network's d.
 * Neither changes the stopping target or the acceptance test. Unpreconditioned GMRES is the
 * fallback: states that the preconditioned pass (at most 8 restart cycles) leaves unconverged are
 * solved again without the network, from where that pass left them (gmres_iterations counts both
 * passes). H is written packed;
 * stats[i].gmres_iterations and boundary_residual report the solve. Replaces
 * boundary_environment(q, r, rho, environment, tolerance) -> (H, stats) (runtime/numerics.py:103-117). */
int rcmps_boundary_environment_batch(rcmps_context* context, int n_states, const int* dims, const double* R,
                                     const double* K, const double* rho, const double* environment, const double* x0,
                                     const rcmps_gmres_network* network, const rcmps_settings* settings, double* H,
                                     rcmps_state_stats* stats, void* stream);

/* rcmps_finish_gradient_batch for ONE state, without allocating anything: no cudaMalloc, no
 * cudaFree, no pinned host buffer. No counterpart in the reference. It serves callers that may
 * not allocate at the moment they need the finished gradient: a host whose memory planner
 * reserves all device memory up front (a serving process, or a framework whose caching
 * allocator owns the device), a plugin callback that must not allocate, or a process near its
 * memory limit where an allocation in the middle of an optimizer step would fail or stall.
 * Its workspace is one fixed 2 MiB array in the library's device image, so it supports
 * 1 <= d <= 32 only; larger d returns RCMPS_INVALID_ARGUMENT with a message naming the limit.
 * The first call on each device looks up that array's device address (cudaGetSymbolAddress)
 * and keeps it for the life of the process, so do not use this entry on a device after a
 * cudaDeviceReset of it. Every call copies GMRES state back to the host and synchronizes the
 * stream once per GMRES restart and once at the end, so it must not be called on a capturing
 * stream. All calls share the one array:
 * calls that overlap on the GPU (different streams or host threads) race on it, and the
 * caller must order them. Each call clears what must start at zero (the Poisson solution and
 * the status words). Arguments are those of rcmps_finish_gradient_batch with n_states = 1:
 * R, K, rho, covector, environment and gradient are d x d device matrices. Its boundary solve
 * is unpreconditioned GMRES(64) whatever settings->boundary_preconditioner says (the no-jump
 * sets would not fit the fixed array); the result meets the same residual bound. */
int rcmps_finish_gradient_noalloc(rcmps_context* context, int d, const double* R, const double* K,
                                  const double* rho, const double* covector, const double* environment,
                                  const rcmps_settings* settings, double* gradient, rcmps_state_stats* stats,
                                  void* stream);

/* Stationary density rho of (Q, R) by GMRES on -L(X) + tr(X) I/D = I/D, on device memory.
 * Replaces stationary_state(q, r, tolerance) -> (rho, stats) (runtime/numerics.py:74-100). */
int rcmps_stationary_state_batch(rcmps_context* context, int n_states, const int* dims, const double* R,
                                 const double* K, double tolerance, double* rho, rcmps_state_stats* stats,
                                 void* stream);

/* The same density started from a nearby one (a normalized Hermitian density of the previous
 * state of an optimizer, device, packed): GMRES solves for the correction to an absolute
 * residual of `tolerance`, and the result passes the same normalization, Hermiticity and
 * stationarity checks. Replaces stationary_state_correction(q, r, rho_previous, tolerance)
 * -> (rho, stats) (runtime/stationary_correction.py:19-96). */
int rcmps_stationary_correction_batch(rcmps_context* context, int n_states, const int* dims, const double* R,
                                      const double* K, const double* rho_previous, double tolerance,
                                      double* rho, rcmps_state_stats* stats, void* stream);

/* C_b = A_b B_b for n_states pairs of d x d complex matrices (1 <= d <= 64; device, packed
 * row-major like every batch of this header) by the split-precision tensor-core engine of the
 * trajectory: FP64 values cut into six 7-bit BF16 slices per operand (per-row scales of A,
 * per-column scales of B), the slice products on tcgen05 with FP32 accumulation in TMEM,
 * recombined in FP64 (error about 2^-42 of row scale x column scale x d). No counterpart in
 * the reference; the engine's unit-level check. */
int rcmps_split_product_batch(rcmps_context* context, int n_states, int d, const double* A, const double* B,
                              double* C, void* stream);

/* Kernels of the learned GMRES warm start (rcmps_b200.warmstart), FP32, device memory, row-major.
 * No counterpart in the reference. The network maps n = 2 d^2 reals of a right-hand side of the
 * boundary solve to an approximate solution: H = W1 X (W1: rank x n, X: n x batch, one sample per
 * column), Y = W2 H (W2: n x rank). */
int rcmps_warmstart_forward(rcmps_context* context, int n, int rank, int batch, const float* W1, const float* W2,
                            const float* X, float* H, float* Y, void* stream);
/* Gradients of loss = sum (Y - T)^2 / batch: dY = 2 (Y - T) / batch, dW2 = dY H^T, dH = W2^T dY,
 * dW1 = dH X^T (dY: n x batch and dH: rank x batch are caller scratch); *loss (device double). */
int rcmps_warmstart_backward(rcmps_context* context, int n, int rank, int batch, const float* W2, const float* X,
                             const float* H, const float* Y, const float* T, float* dY, float* dH, float* dW1,
                             float* dW2, double* loss, void* stream);
/* One Adam step (step >= 1, bias-corrected) of `count` parameters with gradients and moments m, v. */
int rcmps_warmstart_adam(rcmps_context* context, long long count, float* param, const float* grad, float* m, float* v,
                         float lr, float beta1, float beta2, float eps, int step, void* stream);

/* The L-BFGS search direction of the optimizer on the device (one CTA; d <= 128), the algebra of
 * runtime/optimizer.py:73-107 with the metric <X, Y> = 2 Re tr(X^dag Y (rho + metric_reg I)) and
 * the preconditioner P(X) = ((rho + precond_reg I)^-1 (X (rho + metric_reg I))^dag)^dag:
 *   m > 0: the two-loop recursion over the pairs S[j], Y[j] (d x d each, oldest first) with
 *          inv_sy[j] = 1 / <S[j], Y[j]>, the middle preconditioner scaled by
 *          gamma = <s, y> / <y, P(y)> of the newest pair; direction = -H g;
 *   m = 0: the first direction -first_norm P(g) / |P(g)|.
 * scalars (device, 3 doubles): gamma (NaN for m = 0 or when gamma is not positive: then no
 * direction is written), the slope <g, direction>, and a status (1: rho + precond_reg I is not
 * positive definite). work: device scratch of 8 d^2 + m doubles. All device memory, row-major
 * complex128. No counterpart as an entry in the reference (its controller is host NumPy). */
int rcmps_lbfgs_direction(rcmps_context* context, int d, int m, const double* rho, const double* gradient,
                          const double* S, const double* Y, const double* inv_sy, double metric_reg,
                          double precond_reg, double first_norm, double* direction, double* work, double* scalars,
                          void* stream);
/* The canonical retraction on the device: R' = R + alpha X, K' = Herm(K + i alpha/2 (X^dag R - R^dag X))
 * (runtime/numerics.py:133-136). */
int rcmps_retract(rcmps_context* context, int d, const double* R, const double* K, const double* direction,
                  double alpha, double* R_out, double* K_out, void* stream);

/* The tile choice of the FP64 trajectory kernel's autotuner for (system: 0 quartic, 1 all-ODE,
 * 2 <phi>; padded dimension dp) at the channel-group count of the last launch of that pair: the
 * depth of the operand ring (2, 3 or 4 staged chunks; 0 while not yet decided). The quartic
 * system tunes on the caller's own launches: the first three of a pair and group count take the
 * depths 4, 2, 3 and each records its device ms per 1000 right-hand sides of the launch's longest
 * trajectory (ms[0..2] for the depths 2, 3, 4; ms may be NULL); the fastest is then kept, the
 * default 4 unless another is faster by more than 2%. The other systems use 4 (3 for the all-ODE
 * route at dp 128). The depth changes the schedule only; results are identical. No counterpart
 * in the reference (its tiles follow a fixed rule, runtime/generic_layout.py:21-52). */
int rcmps_trajectory_tuning(const rcmps_context* context, int system, int dp, int* ring, float* ms);
/* The channel groups of the last trajectory launch of (system, dp) in this context (1, 2 or 4
 * CTAs per 16-row block of a state, rcmps_settings.trajectory_groups; 0: no launch yet). No
 * counterpart in the reference (its cooperative grid takes a fixed CTA count per state,
 * persistent_trajectory_backend.py:207-283). */
int rcmps_trajectory_groups(const rcmps_context* context, int system, int dp, int* groups);

/* Number of kernel launches this library has issued in the process (all contexts). No
 * counterpart in the reference. */
long long rcmps_launch_count(void);

/* FP64 tensor-core throughput of this device (TFLOP/s), measured by a short in-register
 * mma.sync loop: the denominator of the FP64 roofline. No counterpart in the reference. */
double rcmps_fp64_peak_tflops(rcmps_context* context);

#ifdef __cplusplus
}
#endif
#endif /* RCMPS_B200_H */
