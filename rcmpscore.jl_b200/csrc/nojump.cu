// The no-jump preconditioner of the boundary Poisson GMRES on the device.
//
// Reference: rcmps_gpu numerics.py:37-71 (NoJumpInverse: the complex Schur form Q = U T U^dag,
// LAPACK trsyl on T_s^dag X + X T_s = U^dag y U for the adjoint map of the boundary solve, the
// result -U X U^dag; the Sherman-Morrison correction of the tr(rho x) I term in
// boundary_environment) and src/transfer.jl:50-72, 122-152. The reference solves a triangular
// Sylvester equation per application: a chain of D dependent triangular solves. Here the same map
// is applied in the eigenbasis of Q_s = Q - shift/2 I = V L V^-1,
//     N(y) = -X,  Q_s^dag X + X Q_s = y   =>   N(y) = V^-dag [(V^dag y V) * nS] V^-1,
//     nS_ij = -1 / (conj(l_i) + l_j - shift),
// four dense products and an elementwise product, which the FP64 tensor cores take in a few
// microseconds per state (nojump_apply_kernel, one cluster of dp/16 CTAs per state, 16 rows each).
// The set-up (nojump_setup_kernel, one CTA per state, once per call) finds V:
//   1. Householder reduction of Q to Hessenberg form H = U^dag Q U (the whole CTA);
//   2. the single-shift complex QR iteration on H: Wilkinson shifts, exceptional shifts after 10
//      and 20 iterations, the Ahues-Tisseur deflation test, Givens rotations applied to the whole
//      of H (Schur form) and accumulated into U. One warp runs it: a rotation touches two rows
//      and two columns, so the warp's own barrier orders the rotations;
//   3. the eigenvectors W of the triangular T (back substitution, one thread per column, each
//      column scaled to unit norm) and W^-1 (one thread per column); V = U W, V^-1 = W^-1 U^dag;
//   4. the check |V^-1 V - I|_max <= 1e-8, z = N(I) and den = 1 + tr(rho z).
// A state whose QR iteration needs more than 60 iterations for one eigenvalue, or whose V fails
// the check, gets status != 0 and its Arnoldi basis passes through unchanged (unpreconditioned).
#include <cuda_runtime.h>
#include <cfloat>
#include "common.cuh"
#include "gemm.cuh"
#include "kinetic.h"
#include "nojump.h"

namespace rcmps {
namespace {

constexpr int kSetupThreads = 256;
constexpr int kQrIterations = 60;    // per eigenvalue
constexpr int kMaxDp = 128;
constexpr double kInverseCheck = 1e-8;

__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }

// a / b by Smith's scaling.
__device__ __forceinline__ double2 zdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    const double r = b.y / b.x, den = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
  }
  const double r = b.x / b.y, den = b.y + b.x * r;
  return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
}

// Principal square root (branch cut on the negative real axis).
__device__ __forceinline__ double2 zsqrt(double2 z) {
  const double r = hypot(z.x, z.y);
  if (r == 0.0) return make_double2(0.0, 0.0);
  if (z.x >= 0.0) {
    const double s = sqrt(0.5 * (r + z.x));
    return make_double2(s, z.y / (2.0 * s));
  }
  const double t = sqrt(0.5 * (r - z.x));
  return make_double2(fabs(z.y) / (2.0 * t), copysign(t, z.y));
}

__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  return t;
}

__device__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, red[w]);
  return t;
}

// C = op(A) op(B) on the leading n x n blocks (leading dimension dp); op 1: conjugate transpose.
// C must not alias A or B. Ends with a barrier.
__device__ void block_product(double2* C, const double2* A, int opa, const double2* B, int opb, int n, int dp) {
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < n; ++k) {
      const double2 a = opa ? zconj(A[k * dp + i]) : A[i * dp + k];
      const double2 b = opb ? zconj(B[j * dp + k]) : B[k * dp + j];
      acc = zadd(acc, zmul(a, b));
    }
    C[i * dp + j] = acc;
  }
  __syncthreads();
}

// |A|_2 of the leading n x n block by power iteration on A^dag A (tmp: 2 dp scratch).
__device__ double spectral_norm(const double2* A, int n, int dp, double2* tmp, double* red) {
  double2* x = tmp;
  double2* y = tmp + dp;
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = make_double2(1.0 / sqrt((double)n), 0.0);
  __syncthreads();
  double nrm = 0.0;
  for (int it = 0; it < 200; ++it) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double2 s = make_double2(0.0, 0.0);
      for (int k = 0; k < n; ++k) s = zadd(s, zmul(A[i * dp + k], x[k]));
      y[i] = s;
    }
    __syncthreads();
    double part = 0.0;
    double2 xs[kMaxDp / 32 + 1];
    int c = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x, ++c) {
      double2 s = make_double2(0.0, 0.0);
      for (int k = 0; k < n; ++k) s = zadd(s, zmul(zconj(A[k * dp + i]), y[k]));
      xs[c] = s;
      part += zabs2(s);
    }
    const double nn = sqrt(block_sum(part, red));   // |A^dag A x|, x of unit norm
    c = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x, ++c) x[i] = nn > 0.0 ? zscale(1.0 / nn, xs[c]) : xs[c];
    __syncthreads();
    nrm = nn;
    if (nn == 0.0) break;
  }
  return sqrt(nrm);
}

// Shared-memory plan of the set-up: H (and U when it fits) with leading dimension dp + 1, so that
// both a row and a column of threads read conflict-free.
__host__ __device__ constexpr int setup_ld(int dp) { return dp + 1; }
__host__ __device__ constexpr bool setup_h_shared(int dp) { return dp <= 96; }
__host__ __device__ constexpr bool setup_u_shared(int dp) { return dp <= 64; }
__host__ __device__ constexpr size_t setup_smem(int dp) {
  return ((setup_h_shared(dp) ? 1 : 0) + (setup_u_shared(dp) ? 1 : 0)) * (size_t)dp * setup_ld(dp) * 16;
}

struct Rotation {   // G = [c s; -conj(s) c] on rows/columns k, k+1
  double2 s;
  double c;
  int k;
};

__global__ void __launch_bounds__(kSetupThreads) nojump_setup_kernel(const NoJumpSet* __restrict__ sets) {
  const NoJumpSet S = sets[blockIdx.x];
  const int n = S.d, dp = S.dp, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int lds = setup_ld(dp);
  double2* H = setup_h_shared(dp) ? reinterpret_cast<double2*>(smem_raw) : S.H;
  const int ldh = setup_h_shared(dp) ? lds : dp;
  double2* U = setup_u_shared(dp) ? reinterpret_cast<double2*>(smem_raw) + (size_t)dp * lds : S.U;
  const int ldu = setup_u_shared(dp) ? lds : dp;
  __shared__ double red[kSetupThreads / 32];
  __shared__ double2 v[kMaxDp];
  __shared__ double2 vtmp[2 * kMaxDp];
  __shared__ Rotation rot[kMaxDp];
  __shared__ int sh_l, sh_ihi, sh_nrot, sh_state;   // state: 0 sweep to apply, 1 done, 2 failed
  const double ulp = DBL_EPSILON, smlnum = DBL_MIN * ((double)n / ulp);
  for (int e = tid; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    H[i * ldh + j] = S.Q[i * dp + j];
    U[i * ldu + j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();

  // 1. Hessenberg reduction by Householder reflectors P = I - tau v v^dag
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;
    double part = 0.0;
    for (int i = 1 + tid; i < m; i += blockDim.x) part += zabs2(H[(k + 1 + i) * ldh + k]);
    const double tail = block_sum(part, red);
    if (tail == 0.0) continue;   // column k is already reduced (the sum is uniform)
    const double2 x0 = H[(k + 1) * ldh + k];
    const double ax0 = hypot(x0.x, x0.y);
    const double alpha = sqrt(ax0 * ax0 + tail);
    const double2 ph = ax0 > 0.0 ? zscale(1.0 / ax0, x0) : make_double2(1.0, 0.0);
    const double2 beta = zscale(-alpha, ph);
    const double tau = 2.0 / ((ax0 + alpha) * (ax0 + alpha) + tail);
    for (int i = tid; i < m; i += blockDim.x) v[i] = i == 0 ? zscale(ax0 + alpha, ph) : H[(k + 1 + i) * ldh + k];
    __syncthreads();
    // left: rows k+1.., columns k+1.. (column k becomes beta e1)
    for (int j = k + 1 + tid; j < n; j += blockDim.x) {
      double2 w = make_double2(0.0, 0.0);
      for (int i = 0; i < m; ++i) w = zadd(w, zmul(zconj(v[i]), H[(k + 1 + i) * ldh + j]));
      w = zscale(tau, w);
      for (int i = 0; i < m; ++i) H[(k + 1 + i) * ldh + j] = zsub(H[(k + 1 + i) * ldh + j], zmul(v[i], w));
    }
    for (int i = tid; i < m; i += blockDim.x) H[(k + 1 + i) * ldh + k] = i == 0 ? beta : make_double2(0.0, 0.0);
    __syncthreads();
    // right: every row, columns k+1.. of H, and U <- U P
    for (int r = tid; r < 2 * n; r += blockDim.x) {
      double2* row = r < n ? H + (size_t)r * ldh + k + 1 : U + (size_t)(r - n) * ldu + k + 1;
      double2 w = make_double2(0.0, 0.0);
      for (int q = 0; q < m; ++q) w = zadd(w, zmul(row[q], v[q]));
      w = zscale(tau, w);
      for (int q = 0; q < m; ++q) row[q] = zsub(row[q], zmul(w, zconj(v[q])));
    }
    __syncthreads();
  }

  // 2. complex QR iteration to the Schur form. Warp 0 sweeps the active block l..ihi and records
  // its rotations; then every thread applies them to one line outside the block: a row of U, a
  // row of H above the block or a column of H right of it.
  if (tid == 0) {
    sh_ihi = n - 1;
    sh_state = n > 1 ? 0 : 1;
  }
  __syncthreads();
  int its = 0;   // warp 0: iterations on the current eigenvalue
  for (;;) {
    // every thread reads the state before warp 0 may change it
    const int state_now = sh_state;
    __syncthreads();
    if (state_now != 0) break;
    if (warp == 0) {
      int ihi = sh_ihi, l = 0, state = 0, nrot = 0;
      for (;;) {
        for (l = ihi; l > 0; --l) {
          const double h = cabs1(H[l * ldh + l - 1]);
          if (h <= smlnum) break;
          const double2 hll = H[l * ldh + l], hpp = H[(l - 1) * ldh + l - 1];
          double tst = cabs1(hpp) + cabs1(hll);
          if (tst == 0.0) {
            if (l - 2 >= 0) tst += cabs1(H[(l - 1) * ldh + l - 2]);
            if (l + 1 <= ihi) tst += cabs1(H[(l + 1) * ldh + l]);
          }
          if (h <= ulp * tst) {
            const double hup = cabs1(H[(l - 1) * ldh + l]);
            const double ab = fmax(h, hup), ba = fmin(h, hup);
            const double dd = cabs1(zsub(hpp, hll));
            const double aa = fmax(cabs1(hll), dd), bb = fmin(cabs1(hll), dd);
            const double s = aa + ab;
            if (ba * (ab / s) <= fmax(smlnum, ulp * (bb * (aa / s)))) break;
          }
        }
        if (l > 0) {
          if (lane == 0) H[l * ldh + l - 1] = make_double2(0.0, 0.0);
          __syncwarp();
        }
        if (l < ihi) break;
        // the trailing 1 x 1 block converged
        ihi = l - 1;
        its = 0;
        if (ihi <= 0) {
          state = 1;
          break;
        }
      }
      if (state == 0 && its >= kQrIterations) state = 2;
      if (state == 0) {
        // shift
        double2 t;
        if (its == 10) {
          t = H[l * ldh + l];
          t.x += 0.75 * cabs1(H[(l + 1) * ldh + l]);
        } else if (its == 20) {
          t = H[ihi * ldh + ihi];
          t.x += 0.75 * cabs1(H[ihi * ldh + ihi - 1]);
        } else {
          t = H[ihi * ldh + ihi];
          const double2 u = zmul(zsqrt(H[(ihi - 1) * ldh + ihi]), zsqrt(H[ihi * ldh + ihi - 1]));
          const double su = cabs1(u);
          if (su != 0.0) {
            const double2 x = zscale(0.5, zsub(H[(ihi - 1) * ldh + ihi - 1], t));
            const double sx = cabs1(x);
            const double sm = fmax(su, sx);
            const double2 xs = zscale(1.0 / sm, x), us = zscale(1.0 / sm, u);
            double2 y = zscale(sm, zsqrt(zadd(zmul(xs, xs), zmul(us, us))));
            if (sx > 0.0 && (x.x / sx) * y.x + (x.y / sx) * y.y < 0.0) y = zscale(-1.0, y);
            t = zsub(t, zmul(u, zdiv(u, zadd(x, y))));
          }
        }
        // one implicit single-shift sweep inside the active block
        for (int k = l; k < ihi; ++k) {
          const double2 a = k == l ? zsub(H[l * ldh + l], t) : H[k * ldh + k - 1];
          const double2 b = k == l ? H[(l + 1) * ldh + l] : H[(k + 1) * ldh + k - 1];
          const double na = hypot(a.x, a.y), nb = hypot(b.x, b.y);
          double c;
          double2 s;
          if (nb == 0.0) {
            c = 1.0;
            s = make_double2(0.0, 0.0);
          } else if (na == 0.0) {
            c = 0.0;
            s = zscale(1.0 / nb, zconj(b));
          } else {
            const double nrm = hypot(na, nb);
            c = na / nrm;
            s = zscale(1.0 / (na * nrm), zmul(a, zconj(b)));
          }
          if (lane == 0) rot[nrot] = Rotation{s, c, k};
          ++nrot;
          __syncwarp();
          // rows k, k+1 <- G rows, columns of the block
          for (int j = (k == l ? l : k - 1) + lane; j <= ihi; j += 32) {
            const double2 x = H[k * ldh + j], y = H[(k + 1) * ldh + j];
            H[k * ldh + j] = zadd(zscale(c, x), zmul(s, y));
            H[(k + 1) * ldh + j] = zsub(zscale(c, y), zmul(zconj(s), x));
          }
          __syncwarp();
          if (k > l && lane == 0) H[(k + 1) * ldh + k - 1] = make_double2(0.0, 0.0);
          // columns k, k+1 <- columns G^dag, rows of the block
          for (int r = l + lane; r <= min(k + 2, ihi); r += 32) {
            const double2 x = H[r * ldh + k], y = H[r * ldh + k + 1];
            H[r * ldh + k] = zadd(zscale(c, x), zmul(y, zconj(s)));
            H[r * ldh + k + 1] = zsub(zscale(c, y), zmul(x, s));
          }
          __syncwarp();
        }
        ++its;
      }
      if (lane == 0) {
        sh_l = l;
        sh_ihi = ihi;
        sh_nrot = nrot;
        sh_state = state;
      }
    }
    __syncthreads();
    // the sweep's rotations outside the block (state 0: a sweep ran on l..ihi)
    if (sh_state == 0) {
      const int l = sh_l, ihi = sh_ihi, nrot = sh_nrot;
      const int ncol = n - 1 - ihi;   // columns right of the block
      for (int line = tid; line < n + l + ncol; line += blockDim.x) {
        if (line < n + l) {   // a row of U, or a row of H above the block: column rotations
          double2* row = line < n ? U + (size_t)line * ldu : H + (size_t)(line - n) * ldh;
          for (int q = 0; q < nrot; ++q) {
            const Rotation g = rot[q];
            const double2 x = row[g.k], y = row[g.k + 1];
            row[g.k] = zadd(zscale(g.c, x), zmul(y, zconj(g.s)));
            row[g.k + 1] = zsub(zscale(g.c, y), zmul(x, g.s));
          }
        } else {              // a column of H right of the block: row rotations
          const int j = ihi + 1 + (line - n - l);
          for (int q = 0; q < nrot; ++q) {
            const Rotation g = rot[q];
            const double2 x = H[g.k * ldh + j], y = H[(g.k + 1) * ldh + j];
            H[g.k * ldh + j] = zadd(zscale(g.c, x), zmul(g.s, y));
            H[(g.k + 1) * ldh + j] = zsub(zscale(g.c, y), zmul(zconj(g.s), x));
          }
        }
      }
    }
    __syncthreads();
  }
  if (sh_state == 2) {
    if (tid == 0) *S.status = 1;
    return;
  }
  // T and U to their global homes (leading dimension dp) for the rest of the set-up
  if (H != S.H || U != S.U) {
    for (int e = tid; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      if (H != S.H) S.H[i * dp + j] = H[i * ldh + j];
      if (U != S.U) S.U[i * dp + j] = U[i * ldu + j];
    }
    __syncthreads();
  }
  H = S.H;
  U = S.U;

  // 3. eigenvectors W of T = H (upper triangular) and W^-1
  double2* W = S.W;
  double2* M = S.M;
  for (int j = tid; j < n; j += blockDim.x) {
    const double2 lj = H[j * dp + j];
    const double smin = fmax(ulp * cabs1(lj), smlnum);
    for (int i = j + 1; i < n; ++i) W[i * dp + j] = make_double2(0.0, 0.0);
    W[j * dp + j] = make_double2(1.0, 0.0);
    double nrm = 1.0;
    for (int i = j - 1; i >= 0; --i) {
      double2 s = make_double2(0.0, 0.0);
      for (int k = i + 1; k <= j; ++k) s = zadd(s, zmul(H[i * dp + k], W[k * dp + j]));
      double2 den = zsub(H[i * dp + i], lj);
      if (cabs1(den) < smin) den = make_double2(smin, 0.0);
      const double2 w = zscale(-1.0, zdiv(s, den));
      W[i * dp + j] = w;
      nrm += zabs2(w);
    }
    const double inv = 1.0 / sqrt(nrm);
    for (int i = 0; i <= j; ++i) W[i * dp + j] = zscale(inv, W[i * dp + j]);
  }
  __syncthreads();
  for (int j = tid; j < n; j += blockDim.x) {
    for (int i = j + 1; i < n; ++i) M[i * dp + j] = make_double2(0.0, 0.0);
    M[j * dp + j] = zdiv(make_double2(1.0, 0.0), W[j * dp + j]);
    for (int i = j - 1; i >= 0; --i) {
      double2 s = make_double2(0.0, 0.0);
      for (int k = i + 1; k <= j; ++k) s = zadd(s, zmul(W[i * dp + k], M[k * dp + j]));
      M[i * dp + j] = zscale(-1.0, zdiv(s, W[i * dp + i]));
    }
  }
  __syncthreads();
  block_product(S.V, U, 0, W, 0, n, dp);       // V = U W
  block_product(S.Vinv, M, 0, U, 1, n, dp);    // V^-1 = W^-1 U^dag
  block_product(S.T, S.Vinv, 0, S.V, 0, n, dp);
  double err = 0.0;
  for (int e = tid; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    double2 t = S.T[i * dp + j];
    if (i == j) t.x -= 1.0;
    const double a = cabs1(t);
    err = fmax(err, isfinite(a) ? a : INFINITY);
  }
  err = block_max(err, red);

  // the shift: max(1, |Q|_2, |R|_2^2) when an eigenvalue has real part >= -100 eps scale
  double maxre = -INFINITY;
  for (int i = 0; i < n; ++i) maxre = fmax(maxre, H[i * dp + i].x);
  double fq = 0.0, fr = 0.0;
  for (int e = tid; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    fq += zabs2(S.Q[i * dp + j]);
    fr += zabs2(S.R[i * dp + j]);
  }
  fq = sqrt(block_sum(fq, red));
  fr = block_sum(fr, red);
  double shift = 0.0;
  if (maxre >= -100.0 * ulp * fmax(1.0, fmax(fq, fr))) {   // the Frobenius bound first; rare
    const double nq = spectral_norm(S.Q, n, dp, vtmp, red), nr = spectral_norm(S.R, n, dp, vtmp, red);
    const double scale = fmax(1.0, fmax(nq, nr * nr));
    if (maxre >= -100.0 * ulp * scale) shift = scale;
  }

  // outputs on the padded blocks: V, V^-1 (and their adjoints) the identity, nS and z zero
  bool bad = !(err <= kInverseCheck);
  for (int e = tid; e < dp * dp; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    const bool phys = i < n && j < n;
    const double2 id = make_double2(i == j ? 1.0 : 0.0, 0.0);
    if (!phys) {
      S.V[e] = id;
      S.Vinv[e] = id;
    }
    S.Vh[e] = phys ? zconj(S.V[j * dp + i]) : id;
    S.Vinvh[e] = phys ? zconj(S.Vinv[j * dp + i]) : id;
    double2 ns = make_double2(0.0, 0.0);
    if (phys) {
      const double2 li = H[i * dp + i], lj = H[j * dp + j];
      const double2 den = make_double2(li.x + lj.x - shift, lj.y - li.y);
      if (cabs1(den) > 0.0) ns = zscale(-1.0, zdiv(make_double2(1.0, 0.0), den));
      else bad = true;
    }
    S.nS[e] = ns;
  }
  for (int i = tid; i < dp; i += blockDim.x) S.lambda[i] = i < n ? H[i * dp + i] : make_double2(0.0, 0.0);
  __syncthreads();
  // z = N(I) = V^-dag [(V^dag V) * nS] V^-1
  block_product(S.T, S.V, 1, S.V, 0, n, dp);
  for (int e = tid; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    S.T[i * dp + j] = zmul(S.T[i * dp + j], S.nS[i * dp + j]);
  }
  __syncthreads();
  block_product(W, S.Vinvh, 0, S.T, 0, n, dp);
  for (int e = tid; e < dp * dp; e += blockDim.x) S.z[e] = make_double2(0.0, 0.0);
  __syncthreads();
  block_product(S.z, W, 0, S.Vinv, 0, n, dp);
  double tre = 0.0, tim = 0.0;
  for (int e = tid; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    const double2 t = zmul(S.rho[i * dp + j], S.z[j * dp + i]);
    tre += t.x;
    tim += t.y;
  }
  tre = block_sum(tre, red);
  tim = block_sum(tim, red);
  const int bad_any = __syncthreads_or(bad ? 1 : 0);
  if (tid == 0) {
    const double2 den = make_double2(1.0 + tre, tim);
    *S.den = den;
    *S.shift = shift;
    *S.status = (bad_any || !isfinite(den.x) || !isfinite(den.y) || cabs1(den) == 0.0) ? 2 : 0;
  }
}

// ----------------------------------------------------------------------- application
template <int DP>
struct NGeo {
  static constexpr int TN = DP / 8;
  static constexpr int NW = DP == 96 ? 12 : (TN > 8 ? 8 : TN);
  static constexpr int KC = DP <= 64 ? 16 : 8;
  static constexpr int NST = 4;
  static constexpr int LDP = DP + 4;
  static constexpr int NT = 32 * NW;
  static constexpr size_t RING = (size_t)NST * KC * (DP + kBPad);
  static constexpr size_t SMEM = ((size_t)2 * 16 * LDP + RING) * 16 + 256;
};

template <int DP>
__global__ void __launch_bounds__(NGeo<DP>::NT, 1)
nojump_apply_kernel(const ArnoldiProblem* __restrict__ probs, int NP, int j, const NoJumpSet* __restrict__ sets,
                    double2* __restrict__ Wall) {
  using NG = NGeo<DP>;
  using GR = RowGemmRing<DP, NG::NW, NG::KC, NG::NST>;
  constexpr int TPW = Tiling<DP, 16, NG::NW>::TPW;
  constexpr int G = DP / 16;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double2* panel = reinterpret_cast<double2*>(smem_raw);   // [16][LDP]
  double2* aprime = panel + 16 * NG::LDP;                    // [16][LDP]
  double2* ring = aprime + 16 * NG::LDP;
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + NG::RING);
  int* flag = reinterpret_cast<int*>(full + NG::NST);
  double* xch = reinterpret_cast<double*>(full + NG::NST + 1);   // [2]: this CTA's part of tr(rho X)
  __shared__ double red[2 * 16];
  const int p = (int)cluster_id_x(), rank = (int)cluster_rank(), tid = threadIdx.x;
  const int row0 = rank * 16;
  if (p >= NP) return;
  const ArnoldiProblem& P = probs[p];
  // uniform over the cluster: every CTA reads the same problem
  if (!(P.Z && P.active && !P.exhausted && j < P.target)) return;
  const NoJumpSet S = sets[p];
  const double2* y = P.V + (size_t)j * P.ldv;
  double2* zout = P.Z + (size_t)j * P.ldv;
  if (*S.status != 0) {   // no preconditioner for this state: Z_j = V_j
    for (int e = tid; e < 16 * DP; e += NG::NT) {
      const size_t off = (size_t)(row0 + e / DP) * DP + (e % DP);
      zout[off] = y[off];
    }
    return;
  }
  GR gr;
  gr.ring = ring;
  gr.full = full;
  gr.wait_flag = flag;
  if (tid == 0) *flag = 0;
  gr.init();
  typename GR::Segs sb;
  sb.n = 1;
  sb.rows[0] = DP;
  ZFrag acc[TPW];
  auto to_aprime = [&]() {
#pragma unroll
    for (int t = 0; t < TPW; ++t)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        int row, col;
        GR::template coord<16>(t, i, row, col);
        aprime[row * NG::LDP + col] = acc[t].value(i);
      }
    __syncthreads();
  };
  // phase 1: W rows = ((V^dag)[rows] y) V * nS[rows]
  for (int e = tid; e < 16 * DP; e += NG::NT) panel[(e / DP) * NG::LDP + (e % DP)] = S.Vh[(size_t)(row0 + e / DP) * DP + (e % DP)];
  __syncthreads();
#pragma unroll
  for (int t = 0; t < TPW; ++t) acc[t].zero();
  sb.ptr[0] = y;
  gr.template run<16>(acc, panel, NG::LDP, sb);
  to_aprime();
#pragma unroll
  for (int t = 0; t < TPW; ++t) acc[t].zero();
  sb.ptr[0] = S.V;
  gr.template run<16>(acc, aprime, NG::LDP, sb);
  double2* W = Wall + (size_t)p * DP * DP;
#pragma unroll
  for (int t = 0; t < TPW; ++t)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int row, col;
      GR::template coord<16>(t, i, row, col);
      const size_t off = (size_t)(row0 + row) * DP + col;
      W[off] = zmul(acc[t].value(i), S.nS[off]);
    }
  fence_proxy_async_global();   // W is read by bulk copies of the other CTAs
  cluster_sync();
  // phase 2: X rows = (V^-dag[rows] W) V^-1, then Z_j = X - tr(rho X) / den z
  for (int e = tid; e < 16 * DP; e += NG::NT)
    panel[(e / DP) * NG::LDP + (e % DP)] = S.Vinvh[(size_t)(row0 + e / DP) * DP + (e % DP)];
  __syncthreads();
#pragma unroll
  for (int t = 0; t < TPW; ++t) acc[t].zero();
  sb.ptr[0] = W;
  gr.template run<16>(acc, panel, NG::LDP, sb);
  to_aprime();
#pragma unroll
  for (int t = 0; t < TPW; ++t) acc[t].zero();
  sb.ptr[0] = S.Vinv;
  gr.template run<16>(acc, aprime, NG::LDP, sb);
  double tre = 0.0, tim = 0.0;
#pragma unroll
  for (int t = 0; t < TPW; ++t)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int row, col;
      GR::template coord<16>(t, i, row, col);
      const double2 v = zmul(S.rho[(size_t)col * DP + row0 + row], acc[t].value(i));
      tre += v.x;
      tim += v.y;
    }
  tre = warp_sum(tre);
  tim = warp_sum(tim);
  if ((tid & 31) == 0) {
    red[2 * (tid >> 5)] = tre;
    red[2 * (tid >> 5) + 1] = tim;
  }
  __syncthreads();
  if (tid == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < NG::NW; ++w) {
      a += red[2 * w];
      b += red[2 * w + 1];
    }
    xch[0] = a;
    xch[1] = b;
  }
  cluster_sync();
  double2 tr = make_double2(0.0, 0.0);
  for (int g = 0; g < G; ++g) {
    tr.x += dsmem_load(&xch[0], (uint32_t)g);
    tr.y += dsmem_load(&xch[1], (uint32_t)g);
  }
  const double2 coef = zdiv(tr, *S.den);
#pragma unroll
  for (int t = 0; t < TPW; ++t)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int row, col;
      GR::template coord<16>(t, i, row, col);
      const size_t off = (size_t)(row0 + row) * DP + col;
      zout[off] = zsub(acc[t].value(i), zmul(coef, S.z[off]));
    }
  gr.drain();
  cluster_sync();   // every CTA's partial trace stays readable until all have read it
}

template <int DP>
cudaError_t launch_apply(const ArnoldiProblem* probs, int NP, int j, const NoJumpSet* sets, double2* W,
                         cudaStream_t stream) {
  using NG = NGeo<DP>;
  auto kern = nojump_apply_kernel<DP>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)NG::SMEM);
  if (e != cudaSuccess) return e;
  if (NP == 0) return cudaSuccess;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(NP * (DP / 16), 1, 1);
  cfg.blockDim = dim3(NG::NT, 1, 1);
  cfg.dynamicSmemBytes = NG::SMEM;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = DP / 16;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  note_launch();
  return cudaLaunchKernelEx(&cfg, kern, probs, NP, j, sets, W);
}

}  // namespace

cudaError_t nojump_setup_launch(const NoJumpSet* d_sets, int n, int dp, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  if (dp > kMaxDp) return cudaErrorInvalidValue;
  const size_t smem = setup_smem(dp);
  cudaError_t e = cudaFuncSetAttribute(nojump_setup_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  note_launch();
  nojump_setup_kernel<<<n, kSetupThreads, smem, stream>>>(d_sets);
  return cudaGetLastError();
}

cudaError_t nojump_apply_launch(const ArnoldiProblem* d_probs, int NP, int j, const NoJumpSet* d_sets, double2* W,
                                int dp, cudaStream_t stream) {
  switch (dp) {
    case 16: return launch_apply<16>(d_probs, NP, j, d_sets, W, stream);
    case 32: return launch_apply<32>(d_probs, NP, j, d_sets, W, stream);
    case 48: return launch_apply<48>(d_probs, NP, j, d_sets, W, stream);
    case 64: return launch_apply<64>(d_probs, NP, j, d_sets, W, stream);
    case 96: return launch_apply<96>(d_probs, NP, j, d_sets, W, stream);
    case 128: return launch_apply<128>(d_probs, NP, j, d_sets, W, stream);
  }
  return cudaErrorInvalidValue;
}

}  // namespace rcmps
