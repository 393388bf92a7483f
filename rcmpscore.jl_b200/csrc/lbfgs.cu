// L-BFGS algebra of the optimizer on the device (rcmps_b200.optimizer with device history).
//
// The controller of rcmps_gpu's optimizer (runtime/optimizer.py:73-107) forms its search direction
// from the gradient and the curvature history with D x D matrix algebra: the metric
// <X, Y> = 2 Re tr(X^dag Y M), M = rho + metric_reg I; the preconditioner
// P(X) = (N^-1 (X M)^dag)^dag, N = rho + precond_reg I; the two-loop recursion with the newest
// pair's scaling gamma = <s, y> / <y, P(y)>; and the canonical retraction of (R, K). Here all of
// it runs in one CTA per call on device-resident history (pairs s_j, y_j with 1/<s_j, y_j>), so
// the host only reads back the scalars the line search needs (gamma, the slope <g, direction>).
//   lbfgs_direction_kernel: -H g (or the first direction -c P(g)/|P(g)| without history)
//   retract_kernel:         R' = R + a X, K' = Herm(K + i a/2 (X^dag R - R^dag X))
// Products are plain FP64 FMA loops over global memory (d <= 128; the matrices stay in L1/L2),
// N is factored once per call by a Cholesky in shared memory.
#include <cuda_runtime.h>
#include <cmath>
#include <string>
#include "../../include/rcmps_b200.h"
#include "common.cuh"
#include "context.h"

namespace rcmps {
namespace {

constexpr int kThreads = 512;
constexpr int kMaxD = 128;

struct LbfgsArgs {
  int d, m;                        // dimension, history pairs in use
  const double2* rho;              // d x d
  const double2* g;                // gradient, d x d
  const double2* S;                // [m][d^2] normalized steps (oldest first)
  const double2* Y;                // [m][d^2] gradient changes
  const double* inv;               // [m] 1 / <s_j, y_j>
  double metric_reg, precond_reg, first_norm;
  double2* dir;                    // out: direction, d x d
  double2* work;                   // [4][d^2] scratch: q, t (X M), u, L (Cholesky factor)
  double* scalars;                 // out: [0] gamma (NaN: no direction), [1] slope, [2] status
  double* alphas;                  // [m] scratch
};

__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < kThreads / 32; ++w) t += red[w];
  return t;
}

// C = A (B + shift I) for d x d complex row-major; every thread a strided set of outputs.
__device__ void mul_shift(const double2* A, const double2* B, double shift, double2* C, int d) {
  for (int e = threadIdx.x; e < d * d; e += kThreads) {
    const int r = e / d, c = e % d;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < d; ++k) acc = zadd(acc, zmul(A[r * d + k], B[k * d + c]));
    acc = zaxpy(shift, A[r * d + c], acc);
    C[e] = acc;
  }
  __syncthreads();
}

// <X, Y> = 2 Re sum conj(X) (Y M) with M = rho + reg I, through scratch t = Y M.
__device__ double inner(const double2* X, const double2* Yv, const LbfgsArgs& a, double2* t, double* red) {
  mul_shift(Yv, a.rho, a.metric_reg, t, a.d);
  double s = 0.0;
  for (int e = threadIdx.x; e < a.d * a.d; e += kThreads) s += X[e].x * t[e].x + X[e].y * t[e].y;
  return 2.0 * block_sum(s, red);
}

// Cholesky N = L L^dag of N = rho + reg I (Hermitian positive definite) into L (lower, row-major).
__device__ bool cholesky(const double2* rho, double reg, double2* L, int d, double* red) {
  for (int e = threadIdx.x; e < d * d; e += kThreads) {
    const int r = e / d, c = e % d;
    double2 v = r >= c ? rho[e] : make_double2(0.0, 0.0);
    if (r == c) v.x += reg;
    L[e] = v;
  }
  __syncthreads();
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int j = 0; j < d; ++j) {
    if (threadIdx.x == 0) {
      double s = L[j * d + j].x;
      if (!(s > 0.0) || !isfinite(s)) bad = 1;
      L[j * d + j] = make_double2(sqrt(fmax(s, 1e-300)), 0.0);
    }
    __syncthreads();
    const double piv = L[j * d + j].x;
    for (int i = j + 1 + threadIdx.x; i < d; i += kThreads) L[i * d + j] = zscale(1.0 / piv, L[i * d + j]);
    __syncthreads();
    // trailing update: L[i][k] -= L[i][j] conj(L[k][j]) for j < k <= i
    for (int e = threadIdx.x; e < d * d; e += kThreads) {
      const int i = e / d, k = e % d;
      if (k > j && i >= k) L[e] = zsub(L[e], zmul(L[i * d + j], zconj(L[k * d + j])));
    }
    __syncthreads();
  }
  return bad == 0;
}

// out = P(X) = (N^-1 (X M)^dag)^dag: W = (X M)^dag, solve L L^dag Z = W column by column, out = Z^dag.
__device__ void precondition(const double2* X, const LbfgsArgs& a, const double2* L, double2* t, double2* out) {
  const int d = a.d;
  mul_shift(X, a.rho, a.metric_reg, t, d);   // t = X M
  // column c of W is conj of row c of t: W[r][c] = conj(t[c][r]); one thread per column
  for (int c = threadIdx.x; c < d; c += kThreads) {
    // forward: L z = w
    for (int r = 0; r < d; ++r) {
      double2 s = zconj(t[c * d + r]);
      for (int k = 0; k < r; ++k) s = zsub(s, zmul(L[r * d + k], out[k * d + c]));
      out[r * d + c] = zscale(1.0 / L[r * d + r].x, s);
    }
    // backward: L^dag z' = z
    for (int r = d - 1; r >= 0; --r) {
      double2 s = out[r * d + c];
      for (int k = r + 1; k < d; ++k) s = zsub(s, zmul(zconj(L[k * d + r]), out[k * d + c]));
      out[r * d + c] = zscale(1.0 / L[r * d + r].x, s);
    }
  }
  __syncthreads();
  // out <- out^dag (in place, pairs above the diagonal)
  for (int e = threadIdx.x; e < d * d; e += kThreads) {
    const int r = e / d, c = e % d;
    if (r < c) {
      const double2 u = out[r * d + c], v = out[c * d + r];
      out[r * d + c] = zconj(v);
      out[c * d + r] = zconj(u);
    } else if (r == c) {
      out[e] = zconj(out[e]);
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads, 1) lbfgs_direction_kernel(LbfgsArgs a) {
  __shared__ double red[kThreads / 32];
  const int d = a.d, dd = d * d;
  double2* q = a.work;
  double2* t = a.work + dd;
  double2* u = a.work + 2 * dd;
  double2* L = a.work + 3 * dd;
  if (!cholesky(a.rho, a.precond_reg, L, d, red)) {
    if (threadIdx.x == 0) a.scalars[2] = 1.0;   // the preconditioner matrix is not positive definite
    return;
  }
  double gamma = 0.0;
  if (a.m == 0) {
    // first direction: -c P(g) / |P(g)|
    precondition(a.g, a, L, t, u);
    const double n2 = inner(u, u, a, t, red);
    const double c = n2 > 0.0 ? -a.first_norm / sqrt(n2) : 0.0;
    for (int e = threadIdx.x; e < dd; e += kThreads) a.dir[e] = zscale(c, u[e]);
    __syncthreads();
    gamma = NAN;
  } else {
    for (int e = threadIdx.x; e < dd; e += kThreads) q[e] = a.g[e];
    __syncthreads();
    for (int j = a.m - 1; j >= 0; --j) {   // newest first
      const double2* s = a.S + (size_t)j * dd;
      const double2* y = a.Y + (size_t)j * dd;
      const double al = a.inv[j] * inner(s, q, a, t, red);
      if (threadIdx.x == 0) a.alphas[j] = al;
      for (int e = threadIdx.x; e < dd; e += kThreads) q[e] = zaxpy(-al, y[e], q[e]);
      __syncthreads();
    }
    const double2* sn = a.S + (size_t)(a.m - 1) * dd;
    const double2* yn = a.Y + (size_t)(a.m - 1) * dd;
    precondition(yn, a, L, t, u);          // u = P(y_newest)
    const double den = inner(yn, u, a, t, red);
    const double num = inner(sn, yn, a, t, red);
    gamma = den > 0.0 ? num / den : NAN;
    if (!(isfinite(gamma) && gamma > 0.0)) {
      if (threadIdx.x == 0) {
        a.scalars[0] = gamma;
        a.scalars[1] = NAN;
        a.scalars[2] = 0.0;
      }
      return;
    }
    precondition(q, a, L, t, u);           // u = P(q)
    for (int e = threadIdx.x; e < dd; e += kThreads) u[e] = zscale(gamma, u[e]);
    __syncthreads();
    for (int j = 0; j < a.m; ++j) {        // oldest first
      const double2* s = a.S + (size_t)j * dd;
      const double2* y = a.Y + (size_t)j * dd;
      const double b = a.inv[j] * inner(y, u, a, t, red);
      const double coef = a.alphas[j] - b;
      for (int e = threadIdx.x; e < dd; e += kThreads) u[e] = zaxpy(coef, s[e], u[e]);
      __syncthreads();
    }
    for (int e = threadIdx.x; e < dd; e += kThreads) a.dir[e] = zscale(-1.0, u[e]);
    __syncthreads();
  }
  const double slope = inner(a.g, a.dir, a, t, red);
  if (threadIdx.x == 0) {
    a.scalars[0] = gamma;
    a.scalars[1] = slope;
    a.scalars[2] = 0.0;
  }
}

// R' = R + a X; K' = Herm(K + i a/2 (X^dag R - R^dag X))
__global__ void retract_kernel(int d, const double2* R, const double2* K, const double2* X, double alpha, double2* Rn,
                               double2* Kn) {
  const int dd = d * d;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < dd; e += gridDim.x * blockDim.x) {
    const int r = e / d, c = e % d;
    auto kplus = [&](int i, int j) {   // K + i a/2 (X^dag R - R^dag X) at (i, j)
      double2 s = make_double2(0.0, 0.0);
      for (int k = 0; k < d; ++k)
        s = zadd(s, zsub(zmul(zconj(X[k * d + i]), R[k * d + j]), zmul(zconj(R[k * d + i]), X[k * d + j])));
      const double2 is = make_double2(-0.5 * alpha * s.y, 0.5 * alpha * s.x);   // i a/2 s
      return zadd(K[i * d + j], is);
    };
    const double2 a1 = kplus(r, c), a2 = kplus(c, r);
    Kn[e] = make_double2(0.5 * (a1.x + a2.x), 0.5 * (a1.y - a2.y));
    Rn[e] = zaxpy(alpha, X[e], R[e]);
  }
}

}  // namespace
}  // namespace rcmps

using namespace rcmps;

extern "C" int rcmps_lbfgs_direction(rcmps_context* ctx, int d, int m, const double* rho, const double* gradient,
                                     const double* S, const double* Y, const double* inv_sy, double metric_reg,
                                     double precond_reg, double first_norm, double* direction, double* work,
                                     double* scalars, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  if (d < 1 || d > kMaxD || m < 0 || m > 4096)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "rcmps_lbfgs_direction: 1 <= d <= 128, 0 <= m <= 4096");
  if (!rho || !gradient || !direction || !work || !scalars || (m > 0 && (!S || !Y || !inv_sy)))
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  if (!(metric_reg >= 0.0) || !(precond_reg > 0.0) || !(first_norm > 0.0))
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "metric_reg >= 0, precond_reg > 0, first_norm > 0");
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->slot[2].stream;
  LbfgsArgs a;
  const size_t dd = (size_t)d * d;
  a.d = d;
  a.m = m;
  a.rho = reinterpret_cast<const double2*>(rho);
  a.g = reinterpret_cast<const double2*>(gradient);
  a.S = reinterpret_cast<const double2*>(S);
  a.Y = reinterpret_cast<const double2*>(Y);
  a.inv = inv_sy;
  a.metric_reg = metric_reg;
  a.precond_reg = precond_reg;
  a.first_norm = first_norm;
  a.dir = reinterpret_cast<double2*>(direction);
  a.work = reinterpret_cast<double2*>(work);
  a.scalars = scalars;
  a.alphas = reinterpret_cast<double*>(a.work + 4 * dd);
  note_launch();
  lbfgs_direction_kernel<<<1, kThreads, 0, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("L-BFGS direction: ") + cudaGetErrorString(e));
  return RCMPS_OK;
}

extern "C" int rcmps_retract(rcmps_context* ctx, int d, const double* R, const double* K, const double* direction,
                             double alpha, double* R_out, double* K_out, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  if (d < 1 || !std::isfinite(alpha)) return fail(ctx, RCMPS_INVALID_ARGUMENT, "rcmps_retract: d >= 1, finite alpha");
  if (!R || !K || !direction || !R_out || !K_out) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->slot[2].stream;
  note_launch();
  retract_kernel<<<(d * d + 255) / 256, 256, 0, s>>>(d, reinterpret_cast<const double2*>(R),
                                                    reinterpret_cast<const double2*>(K),
                                                    reinterpret_cast<const double2*>(direction), alpha,
                                                    reinterpret_cast<double2*>(R_out), reinterpret_cast<double2*>(K_out));
  const cudaError_t e = cudaGetLastError();
  if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("retraction: ") + cudaGetErrorString(e));
  return RCMPS_OK;
}
