// Batched restarted GMRES for the transfer-operator solves, the boundary Poisson correction with
// the metric solve, and the stationary density.
//
// Reference: rcmps_gpu numerics.py:55-126 (GMRES _right_solve, stationary_state,
// boundary_environment, finish_gradient) and src/transfer.jl:33-153. The reference
// right-preconditions GMRES with a Schur/trsyl no-jump inverse on the host; this library runs
// unpreconditioned restarted GMRES(m) on the device for every state of a batch at once (the
// Arnoldi steps reuse the Lindblad and Gram-Schmidt kernels of the kinetic term), stops on
// |b - A x| <= tol max(1, |b|) and accepts with the reference's check |A x - b| <= 20 tol max(1, |b|).
#include <cuda_runtime.h>
#include <cfloat>
#include "common.cuh"
#include "kinetic.h"
#include "solvers.h"

namespace rcmps {

constexpr int GCH = 512;   // rows per chunk (the Gram-Schmidt kernels' CH)

// r = b - W (W = A x), V_0 = r (unnormalised), partial |r|^2
__global__ void gmres_residual(ArnoldiProblem* __restrict__ probs, int nprob, int nchunk) {
  const int p = blockIdx.y, ch = blockIdx.x;
  ArnoldiProblem& P = probs[p];
  if (P.converged) return;
  const int r0 = ch * GCH, r1 = min(P.n, r0 + GCH);
  double s = 0.0;
  for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const double2 v = zsub(P.b[r], P.W[r]);
    P.V[r] = v;
    s += zabs2(v);
  }
  __shared__ double red[32];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    P.norms[ch] = t;
  }
}

// bnorm = |b| of every problem (one CTA per problem): the stopping target of a warm-started solve
__global__ void gmres_bnorm(ArnoldiProblem* __restrict__ probs, int nprob) {
  ArnoldiProblem& P = probs[blockIdx.x];
  double s = 0.0;
  for (int r = threadIdx.x; r < P.n; r += blockDim.x) s += zabs2(P.b[r]);
  __shared__ double red[32];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    P.bnorm = sqrt(t);
  }
}

cudaError_t gmres_bnorm_launch(ArnoldiProblem* probs, int nprob, cudaStream_t stream) {
  note_launch();
  gmres_bnorm<<<nprob, 256, 0, stream>>>(probs, nprob);
  return cudaGetLastError();
}

// beta = |r|; converged if beta <= gtarget; V_0 /= beta; g = beta e1; H = 0
__global__ void gmres_start(ArnoldiProblem* __restrict__ probs, int nprob, int nchunk) {
  const int p = blockIdx.y, ch = blockIdx.x;
  ArnoldiProblem& P = probs[p];
  if (P.converged) return;
  double t = 0.0;
  for (int c = 0; c < nchunk; ++c) t += P.norms[c];
  const double beta = sqrt(t);
  // first residual (x = 0) is |b|: the stopping target is tol max(1, |b|) (scipy gmres with rtol = atol)
  const double bn = P.bnorm >= 0.0 ? P.bnorm : beta;
  const double target = P.gtol * fmax(1.0, bn);
  const bool conv = beta <= target || !isfinite(beta);
  const int r0 = ch * GCH, r1 = min(P.n, r0 + GCH);
  if (!conv) {
    const double inv = 1.0 / beta;
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) P.V[r] = zscale(inv, P.V[r]);
  }
  const int hsz = (P.kmax + 1) * P.kmax;
  for (int i = ch * blockDim.x + threadIdx.x; i < hsz; i += nchunk * blockDim.x) P.H[i] = make_double2(0, 0);
  if (ch == 0 && threadIdx.x == 0) {
    P.bnorm = bn;
    P.gtarget = target;
    P.gres = beta;
    P.residual = beta;
    if (!isfinite(beta)) P.nonfinite = 1;
    if (conv) {
      P.converged = 1;
      P.active = 0;
    } else {
      P.active = 1;
      P.k = 0;
      P.exhausted = 0;
      P.g[0] = make_double2(beta, 0.0);
      for (int i = 1; i <= P.kmax; ++i) P.g[i] = make_double2(0, 0);
    }
  }
}

// Givens update of column j: apply the previous rotations, form a new one, rotate g; stop the
// problem when |g_{j+1}| <= target or the basis broke down. One thread per problem.
__global__ void gmres_givens(ArnoldiProblem* __restrict__ probs, int nprob, int j) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nprob) return;
  ArnoldiProblem& P = probs[p];
  if (!P.active || P.k != j + 1) return;
  double2* h = P.H;   // column j: h[i * kmax + j]
  const int ld = P.kmax;
  // apply the previous rotations to column j; the running entry stays in registers and the
  // column, cosines and sines are read eight rows at a time (independent loads in flight)
  double2 a = h[j];   // h[0][j]
  for (int i0 = 0; i0 < j; i0 += 8) {
    const int m = min(8, j - i0);
    double2 b[8], sn[8];
    double cs[8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (u < m) {
        b[u] = h[(i0 + u + 1) * ld + j];
        cs[u] = P.cs[i0 + u].x;
        sn[u] = P.sn[i0 + u];
      }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (u < m) {
        h[(i0 + u) * ld + j] = zadd(zscale(cs[u], a), zmul(sn[u], b[u]));
        a = zsub(zscale(cs[u], b[u]), zmul(zconj(sn[u]), a));
      }
  }
  const double2 b = h[(j + 1) * ld + j];
  const double na = hypot(a.x, a.y), nb = hypot(b.x, b.y);
  double c;
  double2 s;
  if (na == 0.0) {
    c = 0.0;
    s = make_double2(1.0, 0.0);
  } else {
    const double r = hypot(na, nb);
    c = na / r;
    const double2 phase = make_double2(a.x / na, a.y / na);
    s = zscale(1.0 / r, zmul(phase, zconj(b)));
  }
  P.cs[j] = make_double2(c, 0.0);
  P.sn[j] = s;
  h[j * ld + j] = zadd(zscale(c, a), zmul(s, b));
  h[(j + 1) * ld + j] = make_double2(0, 0);
  const double2 gj = P.g[j];
  P.g[j + 1] = zscale(-1.0, zmul(zconj(s), gj));
  P.g[j] = zscale(c, gj);
  const double res = hypot(P.g[j + 1].x, P.g[j + 1].y);
  P.gres = res;
  P.iters += 1;
  if (!isfinite(res)) {
    P.nonfinite = 1;
    P.active = 0;
  } else if (res <= P.gtarget || P.exhausted || j + 1 >= P.target) {
    P.active = 0;
  }
}

// y = R^-1 g (k x k upper triangular), x += V y. Every chunk CTA solves the small system itself.
__global__ void gmres_update(ArnoldiProblem* __restrict__ probs, int nprob, int nchunk) {
  const int p = blockIdx.y, ch = blockIdx.x;
  ArnoldiProblem& P = probs[p];
  if (P.converged || P.k == 0) return;
  extern __shared__ double2 y[];
  const int k = P.k, ld = P.kmax;
  if (threadIdx.x == 0) {
    for (int i = k - 1; i >= 0; --i) {
      double2 s = P.g[i];
      for (int q = i + 1; q < k; ++q) s = zsub(s, zmul(P.H[i * ld + q], y[q]));
      const double2 d = P.H[i * ld + i];
      const double den = zabs2(d);
      y[i] = den > 0.0 ? zscale(1.0 / den, zmul(s, zconj(d))) : make_double2(0, 0);
    }
  }
  __syncthreads();
  const int r0 = ch * GCH, r1 = min(P.n, r0 + GCH);
  const double2* basis = P.Z ? P.Z : P.V;   // flexible GMRES: x += Z y
  for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    double2 acc = P.x[r];
    for (int i = 0; i < k; ++i) acc = zadd(acc, zmul(basis[(size_t)i * P.ldv + r], y[i]));
    P.x[r] = acc;
  }
  if (ch == 0 && threadIdx.x == 0) P.restarts += 1;
}

// matvec tasks W = A x of every unconverged problem
__global__ void gmres_x_tasks(const ArnoldiProblem* __restrict__ probs, int nprob, LindbladTask* tasks) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nprob) return;
  const ArnoldiProblem& P = probs[p];
  LindbladTask t;
  t.X = P.converged ? nullptr : P.x;
  t.out = P.W;
  t.A1 = P.A1;
  t.A1h = P.A1h;
  t.A2 = P.A2;
  t.A2h = P.A2h;
  t.rhs = nullptr;
  t.res = nullptr;
  t.shift = 0.0;
  t.flag = P.flag;
  t.trw = P.trw;
  t.d = P.d;
  tasks[p] = t;
}

cudaError_t gmres_residual_launch(ArnoldiProblem* d, int nprob, int n, cudaStream_t s) {
  const int nchunk = (n + GCH - 1) / GCH;
  note_launch();
  gmres_residual<<<dim3(nchunk, nprob), 256, 0, s>>>(d, nprob, nchunk);
  note_launch();
  gmres_start<<<dim3(nchunk, nprob), 256, 0, s>>>(d, nprob, nchunk);
  return cudaGetLastError();
}
cudaError_t gmres_givens_launch(ArnoldiProblem* d, int nprob, int j, cudaStream_t s) {
  note_launch();
  gmres_givens<<<(nprob + 127) / 128, 128, 0, s>>>(d, nprob, j);
  return cudaGetLastError();
}
cudaError_t gmres_update_launch(ArnoldiProblem* d, int nprob, int n, int kmax, cudaStream_t s) {
  const int nchunk = (n + GCH - 1) / GCH;
  note_launch();
  gmres_update<<<dim3(nchunk, nprob), 256, (size_t)kmax * sizeof(double2), s>>>(d, nprob, nchunk);
  return cudaGetLastError();
}
cudaError_t gmres_x_tasks_launch(const ArnoldiProblem* d, int nprob, LindbladTask* tasks, cudaStream_t s) {
  note_launch();
  gmres_x_tasks<<<(nprob + 127) / 128, 128, 0, s>>>(d, nprob, tasks);
  return cudaGetLastError();
}

// ----------------------------------------------------------------------- dense helpers (one CTA)
__device__ void smat_mul(double2* C, const double2* A, const double2* B, int dp, double alpha, bool add) {
  for (int e = threadIdx.x; e < dp * dp; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    double2 s = make_double2(0.0, 0.0);
    for (int l = 0; l < dp; ++l) s = zadd(s, zmul(A[i * dp + l], B[l * dp + j]));
    s = zscale(alpha, s);
    C[e] = add ? zadd(C[e], s) : s;
  }
  __syncthreads();
}

// In-place Cholesky A = L L^dag of a Hermitian positive definite dp x dp matrix (lower part).
// Returns false if a pivot is not positive.
__device__ bool cholesky(double2* A, int dp) {
  __shared__ int ok;
  if (threadIdx.x == 0) ok = 1;
  __syncthreads();
  for (int j = 0; j < dp; ++j) {
    if (threadIdx.x == 0) {
      double d = A[j * dp + j].x;
      for (int k = 0; k < j; ++k) d -= zabs2(A[j * dp + k]);
      if (!(d > 0.0) || !isfinite(d)) ok = 0;
      A[j * dp + j] = make_double2(d > 0.0 ? sqrt(d) : 1.0, 0.0);
    }
    __syncthreads();
    const double ljj = A[j * dp + j].x;
    for (int i = j + 1 + threadIdx.x; i < dp; i += blockDim.x) {
      double2 s = A[i * dp + j];
      for (int k = 0; k < j; ++k) s = zsub(s, zmul(A[i * dp + k], zconj(A[j * dp + k])));
      A[i * dp + j] = zscale(1.0 / ljj, s);
    }
    __syncthreads();
  }
  return ok != 0;
}

// Solve (L L^dag) Z = C column by column (one thread per column); Z overwrites C.
__device__ void cholesky_solve(const double2* L, double2* C, int dp) {
  for (int col = threadIdx.x; col < dp; col += blockDim.x) {
    for (int i = 0; i < dp; ++i) {   // L y = c
      double2 s = C[i * dp + col];
      for (int k = 0; k < i; ++k) s = zsub(s, zmul(L[i * dp + k], C[k * dp + col]));
      C[i * dp + col] = zscale(1.0 / L[i * dp + i].x, s);
    }
    for (int i = dp - 1; i >= 0; --i) {   // L^dag z = y
      double2 s = C[i * dp + col];
      for (int k = i + 1; k < dp; ++k) s = zsub(s, zmul(zconj(L[k * dp + i]), C[k * dp + col]));
      C[i * dp + col] = zscale(1.0 / L[i * dp + i].x, s);
    }
  }
  __syncthreads();
}

// b = A - tr(rho A) I_d (numerics.py:104)
__global__ void boundary_rhs_kernel(FinishArgs a) {
  const int s = blockIdx.x, dp = a.dp, MAT = dp * dp;
  const double2* env = a.env + (size_t)s * MAT;
  const double2* rho = a.ops + (size_t)s * a.ops_stride + 7 * MAT;
  double2* b = a.b + (size_t)s * MAT;
  __shared__ double2 tr;
  __shared__ double2 red[32];
  double2 t = make_double2(0, 0);
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    t = zadd(t, zmul(rho[e], env[j * dp + i]));
  }
  t.x = warp_sum(t.x);
  t.y = warp_sum(t.y);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 u = make_double2(0, 0);
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) u = zadd(u, red[w]);
    tr = u;
  }
  __syncthreads();
  const int d = a.dims[s];
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    double2 v = env[e];
    if (i == j && i < d) v = zsub(v, tr);
    b[e] = v;
  }
}

// c = covector + rho R^dag H - rho H R^dag; gradient = ((rho + reg I)^-1 c)^dag (numerics.py:120-126)
__global__ void finish_kernel(FinishArgs a) {
  const int s = blockIdx.x, dp = a.dp, MAT = dp * dp;
  const double2* ops = a.ops + (size_t)s * a.ops_stride;
  const double2 *Rh = ops + 3 * MAT, *rho = ops + 7 * MAT;
  const double2* Hm = a.x + (size_t)s * MAT;
  double2* t = a.tmp + (size_t)s * 4 * MAT;
  double2 *c = t, *T1 = t + MAT, *Lm = t + 2 * MAT, *g = t + 3 * MAT;
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) c[e] = a.cov[(size_t)s * MAT + e];
  __syncthreads();
  smat_mul(T1, Rh, Hm, dp, 1.0, false);   // R^dag H
  smat_mul(c, rho, T1, dp, 1.0, true);
  smat_mul(T1, Hm, Rh, dp, 1.0, false);   // H R^dag
  smat_mul(c, rho, T1, dp, -1.0, true);
  const int d = a.dims[s];
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    double2 v = rho[e];
    if (i == j) v.x += (i < d ? a.metric_reg : 1.0);   // the padded block is the identity
    Lm[e] = v;
  }
  __syncthreads();
  const bool ok = cholesky(Lm, dp);
  cholesky_solve(Lm, c, dp);
  bool finite = true;
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    const double2 v = zconj(c[j * dp + i]);
    g[e] = v;
    if (!isfinite(v.x) || !isfinite(v.y)) finite = false;
  }
  if (!finite) atomicExch(a.status + s, (int)kNonfiniteResult);
  if (!ok && threadIdx.x == 0) atomicExch(a.status + s, (int)kSolveFailure);
}

// rho = x / tr x, Hermiticity check, symmetrisation; residual |L(rho)| and positivity follow
// (numerics.py:88-99; src/transfer.jl:33-47).
__global__ void stationary_finish_kernel(StationaryArgs a) {
  const int s = blockIdx.x, dp = a.dp, MAT = dp * dp;
  const double2* x = a.x + (size_t)s * MAT;
  double2* rho = a.rho + (size_t)s * MAT;
  const int d = a.dims[s];
  __shared__ double2 tr;
  __shared__ double red[32];
  if (threadIdx.x == 0) {
    double2 u = make_double2(0, 0);
    for (int i = 0; i < d; ++i) u = zadd(u, x[i * dp + i]);
    tr = u;
  }
  __syncthreads();
  const double den = zabs2(tr);
  double herm = 0.0;
  // x / tr once per element (scratch), then (rho + rho^dag)/2 from that one copy: every pair
  // (i, j), (j, i) is formed from the same two values, so the result is exactly Hermitian
  double2* nx = a.tmp + (size_t)s * MAT;
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) nx[e] = zscale(1.0 / den, zmul(x[e], zconj(tr)));
  __syncthreads();
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    const double2 v = nx[e], w = nx[j * dp + i];
    herm += zabs2(zsub(v, zconj(w)));
    rho[e] = zscale(0.5, zadd(v, zconj(w)));
  }
  herm = warp_sum(herm);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = herm;
  __syncthreads();
  // scale = max(1, 2|Q| + |R|^2) with Frobenius norms (bounds of the spectral norms of the reference)
  double qn = 0.0, rn = 0.0;
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    qn += zabs2(a.ops[(size_t)s * a.ops_stride + e]);
    rn += zabs2(a.ops[(size_t)s * a.ops_stride + 2 * MAT + e]);
  }
  qn = warp_sum(qn);
  rn = warp_sum(rn);
  __shared__ double red2[2][32];
  if ((threadIdx.x & 31) == 0) {
    red2[0][threadIdx.x >> 5] = qn;
    red2[1][threadIdx.x >> 5] = rn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double h = 0.0, q = 0.0, r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      h += red[w];
      q += red2[0][w];
      r += red2[1][w];
    }
    a.scale[s] = fmax(1.0, 2.0 * sqrt(q) + r);
    a.herm[s] = sqrt(h);
    if (!(sqrt(h) <= 100.0 * a.tolerance)) atomicExch(a.status + s, (int)kSolveFailure);
    if (!(den > 0.0) || !isfinite(den)) atomicExch(a.status + s, (int)kNonfiniteResult);
  }
  // positivity: Cholesky of rho + 10 tol I on the physical block
  __syncthreads();
  double2* Lm = a.tmp + (size_t)s * MAT;
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    double2 v = rho[e];
    if (i == j) v.x += (i < d ? 10.0 * a.tolerance : 1.0);
    Lm[e] = v;
  }
  __syncthreads();
  if (!cholesky(Lm, dp) && threadIdx.x == 0) atomicExch(a.status + s, (int)kSolveFailure);
}

cudaError_t boundary_rhs_launch(const FinishArgs& a, int n, cudaStream_t s) {
  note_launch();
  boundary_rhs_kernel<<<n, 256, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t finish_launch(const FinishArgs& a, int n, cudaStream_t s) {
  note_launch();
  finish_kernel<<<n, 256, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t stationary_finish_launch(const StationaryArgs& a, int n, cudaStream_t s) {
  note_launch();
  stationary_finish_kernel<<<n, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace rcmps
