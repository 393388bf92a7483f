// Training and inference kernels of the learned GMRES warm start (rcmps_b200.warmstart).
//
// The network maps a right-hand side b of the boundary Poisson solve (a d x d complex matrix as
// n = 2 d^2 reals, scaled to unit norm) to an approximate solution: y = W2 (W1 b), W1 of
// rank x n and W2 of n x rank. The solution map b -> H is linear, so the network is a learned
// rank-r approximation of it: trained on (state, right-hand side, solution) triples of nearby
// states (those an optimizer run visits), it captures the slowly converging part of the inverse,
// which is where restarted GMRES spends its iterations. Everything here is FP32 (the warm start
// only needs to be close; the GMRES residual judges the answer in FP64):
//   * gemm_f32: C = alpha op(A) op(B) + beta C, 64 x 64 tiles through shared memory, 4 x 4 per
//     thread (every product of the forward and backward passes);
//   * mse_kernel: dY = 2 (Y - T) / batch and the summed squared error;
//   * adam_kernel: one Adam step of a parameter array.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <string>
#include "../../include/rcmps_b200.h"
#include "common.cuh"
#include "context.h"
#include "warmstart.h"

namespace rcmps {
namespace {

constexpr int kT = 64, kBK = 16;

// op(A)[m][k] = TA ? A[k lda + m] : A[m lda + k]; op(B)[k][n] = TB ? B[n ldb + k] : B[k ldb + n]
// Split K (gridDim.z > 1): CTA z covers the k-range [z kspan, (z + 1) kspan) and adds its partial
// product to C atomically (C was cleared by the caller; alpha applies per partial, beta = 0).
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) gemm_f32(int M, int N, int K, float alpha, const float* __restrict__ A,
                                                int lda, const float* __restrict__ B, int ldb, float beta,
                                                float* __restrict__ C, int ldc, int kspan) {
  __shared__ float As[kBK][kT + 4];
  __shared__ float Bs[kBK][kT + 4];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * kT, n0 = blockIdx.x * kT;
  const int kbeg = blockIdx.z * kspan, kend = min(K, kbeg + kspan);
  const bool split = gridDim.z > 1;
  float acc[4][4] = {};
  for (int k0 = kbeg; k0 < kend; k0 += kBK) {
    for (int i = threadIdx.x; i < kT * kBK; i += 256) {
      const int mm = TA ? i % kT : i / kBK, kk = TA ? i / kT : i % kBK;   // coalesced along the contiguous index
      const int gm = m0 + mm, gk = k0 + kk;
      As[kk][mm] = (gm < M && gk < kend) ? (TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk]) : 0.f;
    }
    for (int i = threadIdx.x; i < kT * kBK; i += 256) {
      const int nn = TB ? i / kBK : i % kT, kk = TB ? i % kBK : i / kT;
      const int gn = n0 + nn, gk = k0 + kk;
      Bs[kk][nn] = (gn < N && gk < kend) ? (TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = As[kk][ty * 4 + i];
        b[i] = Bs[kk][tx * 4 + i];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gm = m0 + ty * 4 + i, gn = n0 + tx * 4 + j;
      if (gm < M && gn < N) {
        float* c = C + (size_t)gm * ldc + gn;
        if (split) atomicAdd(c, alpha * acc[i][j]);
        else *c = beta == 0.f ? alpha * acc[i][j] : fmaf(beta, *c, alpha * acc[i][j]);
      }
    }
}

// Tiles of C below about four waves of the 148 SMs split K (atomically accumulated partials) so
// that thin products (the preconditioner's n x NP and rank x NP outputs) still fill the GPU.
cudaError_t gemm(bool ta, bool tb, int M, int N, int K, float alpha, const float* A, int lda, const float* B, int ldb,
                 float beta, float* C, int ldc, cudaStream_t s) {
  const int tiles = ((N + kT - 1) / kT) * ((M + kT - 1) / kT);
  int splits = 1;
  if (beta == 0.f)
    while (tiles * splits < 4 * 148 && K / (2 * splits) >= 256) splits *= 2;
  const int kspan = ((K + splits - 1) / splits + kBK - 1) / kBK * kBK;
  const dim3 grid((N + kT - 1) / kT, (M + kT - 1) / kT, splits);
  if (splits > 1) {
    for (int r = 0; r < M; ++r) {   // C rows may be strided (ldc >= N)
      if (ldc == N) {
        const cudaError_t e = cudaMemsetAsync(C, 0, (size_t)M * N * sizeof(float), s);
        if (e) return e;
        break;
      }
      const cudaError_t e = cudaMemsetAsync(C + (size_t)r * ldc, 0, (size_t)N * sizeof(float), s);
      if (e) return e;
    }
  }
  note_launch();
  if (!ta && !tb) gemm_f32<false, false><<<grid, 256, 0, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, kspan);
  else if (!ta && tb) gemm_f32<false, true><<<grid, 256, 0, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, kspan);
  else if (ta && !tb) gemm_f32<true, false><<<grid, 256, 0, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, kspan);
  else gemm_f32<true, true><<<grid, 256, 0, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, kspan);
  return cudaGetLastError();
}

// dY = 2 (Y - T) / batch over count entries; *loss += sum (Y - T)^2 / batch
__global__ void mse_kernel(long long count, float inv_batch, const float* __restrict__ Y, const float* __restrict__ T,
                           float* __restrict__ dY, double* __restrict__ loss) {
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x) {
    const float d = Y[i] - T[i];
    dY[i] = 2.f * inv_batch * d;
    s += (double)d * d;
  }
  __shared__ double red[8];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(loss, t * inv_batch);
  }
}

// one Adam step: m = b1 m + (1 - b1) g; v = b2 v + (1 - b2) g^2; p -= lr mhat / (sqrt(vhat) + eps)
__global__ void adam_kernel(long long count, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

// The network's input columns from the Arnoldi vectors V_j of NP problems (one column each).
__global__ void net_pack_kernel(const ArnoldiProblem* __restrict__ probs, int NP, int j, int d, int dp,
                                float* __restrict__ X32) {
  const int p = blockIdx.y;
  const ArnoldiProblem& P = probs[p];
  const double2* v = P.V + (size_t)j * P.ldv;
  const bool live = P.active && !P.exhausted && j < P.target;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < d * d; e += gridDim.x * blockDim.x) {
    const double2 x = live ? v[(e / d) * dp + (e % d)] : make_double2(0.0, 0.0);
    X32[(size_t)(2 * e) * NP + p] = (float)x.x;
    X32[(size_t)(2 * e + 1) * NP + p] = (float)x.y;
  }
}

// Z_j = M V_j + identity V_j of every problem still extending, from the network's output columns.
__global__ void net_unpack_kernel(const ArnoldiProblem* __restrict__ probs, int NP, int j, int d, int dp,
                                  const float* __restrict__ Y32, float identity) {
  const int p = blockIdx.y;
  const ArnoldiProblem& P = probs[p];
  if (!(P.active && !P.exhausted && j < P.target)) return;
  const double2* v = P.V + (size_t)j * P.ldv;
  double2* z = P.Z + (size_t)j * P.ldv;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < dp * dp; e += gridDim.x * blockDim.x) {
    const int r = e / dp, c = e % dp;
    double2 out = make_double2(0.0, 0.0);
    if (r < d && c < d) {
      const int i = r * d + c;
      out.x = (double)Y32[(size_t)(2 * i) * NP + p] + (double)identity * v[e].x;
      out.y = (double)Y32[(size_t)(2 * i + 1) * NP + p] + (double)identity * v[e].y;
    }
    z[e] = out;
  }
}

int check_shape(rcmps_context* ctx, int n, int rank, int batch) {
  if (n < 1 || rank < 1 || batch < 1 || n > (1 << 26) || rank > 32768)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "warm-start network: 1 <= n, 1 <= rank <= 32768, 1 <= batch");
  return RCMPS_OK;
}

}  // namespace

cudaError_t warmstart_gemm(bool ta, bool tb, int M, int N, int K, float alpha, const float* A, int lda, const float* B,
                           int ldb, float beta, float* C, int ldc, cudaStream_t s) {
  return gemm(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, s);
}

cudaError_t net_pack_launch(const ArnoldiProblem* probs, int NP, int j, int d, int dp, float* X32, cudaStream_t s) {
  note_launch();
  net_pack_kernel<<<dim3((d * d + 255) / 256, NP), 256, 0, s>>>(probs, NP, j, d, dp, X32);
  return cudaGetLastError();
}

cudaError_t net_unpack_launch(const ArnoldiProblem* probs, int NP, int j, int d, int dp, const float* Y32,
                              float identity, cudaStream_t s) {
  note_launch();
  net_unpack_kernel<<<dim3((dp * dp + 255) / 256, NP), 256, 0, s>>>(probs, NP, j, d, dp, Y32, identity);
  return cudaGetLastError();
}

}  // namespace rcmps

using namespace rcmps;

extern "C" int rcmps_warmstart_forward(rcmps_context* ctx, int n, int rank, int batch, const float* W1,
                                       const float* W2, const float* X, float* H, float* Y, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_shape(ctx, n, rank, batch);
  if (rc) return rc;
  if (!W1 || !W2 || !X || !H || !Y) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->slot[2].stream;
  cudaError_t e = gemm(false, false, rank, batch, n, 1.f, W1, n, X, batch, 0.f, H, batch, s);   // H = W1 X
  if (!e) e = gemm(false, false, n, batch, rank, 1.f, W2, rank, H, batch, 0.f, Y, batch, s);     // Y = W2 H
  if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("warm-start forward: ") + cudaGetErrorString(e));
  return RCMPS_OK;
}

extern "C" int rcmps_warmstart_backward(rcmps_context* ctx, int n, int rank, int batch, const float* W2, const float* X,
                                        const float* H, const float* Y, const float* T, float* dY, float* dH,
                                        float* dW1, float* dW2, double* loss, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_shape(ctx, n, rank, batch);
  if (rc) return rc;
  if (!W2 || !X || !H || !Y || !T || !dY || !dH || !dW1 || !dW2 || !loss)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->slot[2].stream;
  const long long count = (long long)n * batch;
  cudaError_t e = cudaMemsetAsync(loss, 0, sizeof(double), s);
  if (!e) {
    note_launch();
    const int blocks = (int)std::min<long long>(4096, (count + 255) / 256);
    mse_kernel<<<blocks, 256, 0, s>>>(count, 1.f / batch, Y, T, dY, loss);
    e = cudaGetLastError();
  }
  if (!e) e = gemm(false, true, n, rank, batch, 1.f, dY, batch, H, batch, 0.f, dW2, rank, s);   // dW2 = dY H^T
  if (!e) e = gemm(true, false, rank, batch, n, 1.f, W2, rank, dY, batch, 0.f, dH, batch, s);   // dH = W2^T dY
  if (!e) e = gemm(false, true, rank, n, batch, 1.f, dH, batch, X, batch, 0.f, dW1, n, s);      // dW1 = dH X^T
  if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("warm-start backward: ") + cudaGetErrorString(e));
  return RCMPS_OK;
}

extern "C" int rcmps_warmstart_adam(rcmps_context* ctx, long long count, float* param, const float* grad, float* m,
                                    float* v, float lr, float beta1, float beta2, float eps, int step, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  if (count < 1 || step < 1 || !(lr > 0.f) || !(beta1 >= 0.f && beta1 < 1.f) || !(beta2 >= 0.f && beta2 < 1.f))
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "Adam: count >= 1, step >= 1, lr > 0, 0 <= beta < 1");
  if (!param || !grad || !m || !v) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->slot[2].stream;
  const float c1 = 1.f / (1.f - powf(beta1, (float)step)), c2 = 1.f / (1.f - powf(beta2, (float)step));
  note_launch();
  const int blocks = (int)std::min<long long>(4096, (count + 255) / 256);
  adam_kernel<<<blocks, 256, 0, s>>>(count, param, grad, m, v, lr, beta1, beta2, eps, c1, c2);
  const cudaError_t e = cudaGetLastError();
  if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("Adam: ") + cudaGetErrorString(e));
  return RCMPS_OK;
}
