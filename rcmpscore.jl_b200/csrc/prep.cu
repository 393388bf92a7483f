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

// One warp per state: the real part of the trace of one sample matrix.
__global__ void endpoint_trace_kernel(const double2* __restrict__ samples, long long stride, long long offset,
                                      int dp, const int* __restrict__ dims, double* __restrict__ out) {
  const int s = blockIdx.x;
  const int d = dims[s];
  const double2* m = samples + (long long)s * stride + offset;
  double v = 0.0;
  for (int i = threadIdx.x; i < d; i += 32) v += m[(long long)i * dp + i].x;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (threadIdx.x == 0) out[s] = v;
}

cudaError_t launch_endpoint_trace(const double2* samples, long long stride, long long offset, int dp,
                                  const int* d_dims, double* out, int nstates, cudaStream_t stream) {
  if (nstates == 0) return cudaSuccess;
  note_launch();
  endpoint_trace_kernel<<<nstates, 32, 0, stream>>>(samples, stride, offset, dp, d_dims, out);
  return cudaGetLastError();
}

// One CTA per state: the exact Z2 block structure test of the packed route
// (ode_backend.py:246-256). K's off-diagonal blocks stand for Q's: with R's diagonal blocks zero,
// R^dag R is block diagonal, so Q = -iK - R^dag R/2 has zero off-diagonal blocks iff K has.
__global__ void z2_check_kernel(const double2* __restrict__ R, const double2* __restrict__ K,
                                const double2* __restrict__ rho, const int* __restrict__ dims, int dp,
                                long long stride, int mode, int* __restrict__ flags, long long flag_stride) {
  const int s = blockIdx.x;
  const int d = dims[s];
  const int n = d / 2;
  const double2* r = R + (long long)s * stride;
  const double2* k = K + (long long)s * stride;
  const double2* p = rho + (long long)s * stride;
  __shared__ int bad;
  __shared__ double red[2][32];
  if (threadIdx.x == 0) bad = (d % 2) ? 1 : 0;
  __syncthreads();
  double herm = 0.0, nrm = 0.0;
  int mine = 0;
  for (int e = threadIdx.x; e < d * d; e += blockDim.x) {
    const int i = e / d, j = e % d;
    const double2 rv = r[i * dp + j], kv = k[i * dp + j], pv = p[i * dp + j], pt = p[j * dp + i];
    if ((i < n) == (j < n)) {
      if (rv.x != 0.0 || rv.y != 0.0) mine = 1;
    } else if (kv.x != 0.0 || kv.y != 0.0 || pv.x != 0.0 || pv.y != 0.0) {
      mine = 1;
    }
    const double dx = pv.x - pt.x, dy = pv.y + pt.y;   // (rho - rho^dag)_ij
    herm += dx * dx + dy * dy;
    nrm += pv.x * pv.x + pv.y * pv.y;
  }
  if (mine) atomicOr(&bad, 1);
  for (int o = 16; o > 0; o >>= 1) {
    herm += __shfl_xor_sync(0xffffffffu, herm, o);
    nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    red[0][warp] = herm;
    red[1][warp] = nrm;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double h = 0.0, m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      h += red[0][w];
      m += red[1][w];
    }
    const bool ok = !bad && sqrt(h) <= 1e-13 * fmax(1.0, sqrt(m));
    flags[(long long)s * flag_stride] = ok ? 1 : (mode == 1 ? -1 : 0);
  }
}

cudaError_t launch_z2_check(const double* R, const double* K, const double* rho, const int* d_dims, int dp,
                            long long in_stride, int nstates, int mode, int* z2_flags, long long flag_stride,
                            cudaStream_t stream) {
  if (nstates == 0) return cudaSuccess;
  note_launch();
  z2_check_kernel<<<nstates, 256, 0, stream>>>(reinterpret_cast<const double2*>(R),
                                                reinterpret_cast<const double2*>(K),
                                                reinterpret_cast<const double2*>(rho), d_dims, dp, in_stride, mode,
                                                z2_flags, flag_stride);
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
