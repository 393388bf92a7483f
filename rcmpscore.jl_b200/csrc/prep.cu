// Per-state preparation kernels: padding of packed inputs and the constant operators.
#include <cuda_runtime.h>
#include "common.cuh"
#include "prep.h"

namespace rcmps {

// dst[state][dp][dp] <- src (packed d_i x d_i), zero outside the physical block.
__global__ void pad_kernel(const double2* __restrict__ src, const long long* __restrict__ src_off,
                           const int* __restrict__ dims, double2* __restrict__ dst, int dp, long long stride) {
  const int s = blockIdx.y;
  const int d = dims[s];
  const double2* in = src + src_off[s];
  double2* out = dst + (long long)s * stride;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < dp * dp; e += gridDim.x * blockDim.x) {
    const int r = e / dp, c = e % dp;
    out[e] = (r < d && c < d) ? in[r * d + c] : make_double2(0.0, 0.0);
  }
}

// packed d_i x d_i <- padded dp x dp
__global__ void unpad_kernel(const double2* __restrict__ src, long long stride, int dp,
                             const long long* __restrict__ dst_off, const int* __restrict__ dims,
                             double2* __restrict__ dst) {
  const int s = blockIdx.y;
  const int d = dims[s];
  const double2* in = src + (long long)s * stride;
  double2* out = dst + dst_off[s];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < d * d; e += gridDim.x * blockDim.x) {
    const int r = e / d, c = e % d;
    out[e] = in[r * dp + c];
  }
}

// Q = -iK - R^dag R / 2, and the derived operators of one padded state (one CTA per state).
// Layout of `ops` per state: Q, Qh, R, Rh, fixed0, fixed6, S, rho (8 matrices of dp^2).
__global__ void prepare_kernel(const double2* __restrict__ R, const double2* __restrict__ K,
                               const double2* __restrict__ rho, double2* __restrict__ ops, int dp,
                               long long in_stride, long long ops_stride) {
  const int s = blockIdx.x;
  const int n = dp * dp;
  const double2* r = R + s * in_stride;
  const double2* k = K + s * in_stride;
  const double2* p = rho + s * in_stride;
  double2* o = ops + s * ops_stride;
  double2 *Q = o, *Qh = o + n, *Ro = o + 2 * n, *Rh = o + 3 * n, *F0 = o + 4 * n, *F6 = o + 5 * n,
          *S = o + 6 * n, *P = o + 7 * n;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    double2 rr = make_double2(0.0, 0.0);   // (R^dag R)_ij = sum_l conj(R_li) R_lj
    double2 rp = make_double2(0.0, 0.0);   // (R rho)_ij
    double2 pr = make_double2(0.0, 0.0);   // (rho R^dag)_ij = sum_l rho_il conj(R_jl)
    for (int l = 0; l < dp; ++l) {
      rr = zadd(rr, zmul(zconj(r[l * dp + i]), r[l * dp + j]));
      rp = zadd(rp, zmul(r[i * dp + l], p[l * dp + j]));
      pr = zadd(pr, zmul(p[i * dp + l], zconj(r[j * dp + l])));
    }
    const double2 kij = k[e];
    Q[e] = make_double2(kij.y - 0.5 * rr.x, -kij.x - 0.5 * rr.y);   // -i K - R^dag R / 2
    Ro[e] = r[e];
    Rh[e] = zconj(r[j * dp + i]);
    F0[e] = zadd(rp, pr);
    F6[e] = zscale(4.0, zadd(r[e], zconj(r[j * dp + i])));
    S[e] = zadd(zconj(r[e]), r[j * dp + i]);
    P[e] = p[e];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    Qh[e] = zconj(Q[j * dp + i]);
  }
}

// Operators of the commutator channels of the all-ODE route: C = Q R - R Q at slot kC and
// C^dag at slot kCh of each state's operator block (needs kOpsFull slots).
__global__ void commutator_kernel(double2* __restrict__ ops, int dp, long long ops_stride) {
  const int n = dp * dp;
  double2* o = ops + blockIdx.x * ops_stride;
  const double2 *Q = o + kQ * n, *R = o + kR * n;
  double2 *Cm = o + kC * n, *Ch = o + kCh * n;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    double2 c = make_double2(0.0, 0.0);
    for (int l = 0; l < dp; ++l) c = zadd(c, zsub(zmul(Q[i * dp + l], R[l * dp + j]), zmul(R[i * dp + l], Q[l * dp + j])));
    Cm[e] = c;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    Ch[e] = zconj(Cm[j * dp + i]);
  }
}

cudaError_t launch_commutator(double* ops, int dp, long long ops_stride, int nstates, cudaStream_t stream) {
  if (nstates == 0) return cudaSuccess;
  note_launch();
  commutator_kernel<<<nstates, 256, 0, stream>>>(reinterpret_cast<double2*>(ops), dp, ops_stride);
  return cudaGetLastError();
}

cudaError_t launch_pad(const double* src, const long long* d_src_off, const int* d_dims, double* dst, int dp,
                       long long stride, int nstates, cudaStream_t stream) {
  if (nstates == 0) return cudaSuccess;
  dim3 grid((dp * dp + 255) / 256, nstates);
  note_launch();
  pad_kernel<<<grid, 256, 0, stream>>>(reinterpret_cast<const double2*>(src), d_src_off, d_dims,
                                       reinterpret_cast<double2*>(dst), dp, stride);
  return cudaGetLastError();
}

cudaError_t launch_unpad(const double* src, long long stride, int dp, const long long* d_dst_off,
                         const int* d_dims, double* dst, int nstates, cudaStream_t stream) {
  if (nstates == 0) return cudaSuccess;
  dim3 grid((dp * dp + 255) / 256, nstates);
  note_launch();
  unpad_kernel<<<grid, 256, 0, stream>>>(reinterpret_cast<const double2*>(src), stride, dp, d_dst_off, d_dims,
                                         reinterpret_cast<double2*>(dst));
  return cudaGetLastError();
}

__global__ void unpad_acc_kernel(const double2* __restrict__ src, long long stride, int dp,
                                 const long long* __restrict__ dst_off, const int* __restrict__ dims,
                                 double2* __restrict__ dst, int accumulate) {
  const int s = blockIdx.y;
  const int d = dims[s];
  const double2* in = src + (long long)s * stride;
  double2* out = dst + dst_off[s];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < d * d; e += gridDim.x * blockDim.x) {
    const int r = e / d, c = e % d;
    const double2 v = in[r * dp + c];
    out[e] = accumulate ? zadd(out[e], v) : v;
  }
}

__global__ void scatter_values_kernel(const double* src, int n, const int* idx, double* dst, int accumulate) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[idx[i]] = accumulate ? dst[idx[i]] + src[i] : src[i];
}

__global__ void export_samples_kernel(const double2* __restrict__ samples, int dp, int d, int npoints,
                                      const double* value, double2* __restrict__ out) {
  const long long per = 7ll * d * d + 1;
  const long long total = per * npoints;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long node = e / per, rem = e % per;
    if (rem == 7ll * d * d) {
      out[e] = make_double2(node == npoints - 1 ? value[0] : 0.0, 0.0);
    } else {
      const int c = (int)(rem / (d * d)), ij = (int)(rem % (d * d)), i = ij / d, j = ij % d;
      out[e] = samples[(node * 7 + c) * (long long)dp * dp + (long long)i * dp + j];
    }
  }
}

cudaError_t launch_unpad_acc(const double* src, long long stride, int dp, const long long* d_dst_off,
                             const int* d_dims, double* dst, int nstates, bool accumulate, cudaStream_t stream) {
  if (nstates == 0) return cudaSuccess;
  dim3 grid((dp * dp + 255) / 256, nstates);
  note_launch();
  unpad_acc_kernel<<<grid, 256, 0, stream>>>(reinterpret_cast<const double2*>(src), stride, dp, d_dst_off, d_dims,
                                             reinterpret_cast<double2*>(dst), accumulate ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_scatter_values(const double* src, int n, const int* d_idx, double* dst, bool accumulate,
                                  cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  note_launch();
  scatter_values_kernel<<<(n + 255) / 256, 256, 0, stream>>>(src, n, d_idx, dst, accumulate ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_export_samples(const double2* samples, int dp, int d, int npoints, const double* value,
                                  double* out, cudaStream_t stream) {
  note_launch();
  export_samples_kernel<<<1024, 256, 0, stream>>>(samples, dp, d, npoints, value, reinterpret_cast<double2*>(out));
  return cudaGetLastError();
}

cudaError_t launch_prepare(const double* R, const double* K, const double* rho, double* ops, int dp,
                           long long in_stride, long long ops_stride, int nstates, cudaStream_t stream) {
  if (nstates == 0) return cudaSuccess;
  note_launch();
  prepare_kernel<<<nstates, 256, 0, stream>>>(reinterpret_cast<const double2*>(R),
                                              reinterpret_cast<const double2*>(K),
                                              reinterpret_cast<const double2*>(rho),
                                              reinterpret_cast<double2*>(ops), dp, in_stride, ops_stride);
  return cudaGetLastError();
}

}  // namespace rcmps
