// Quadrature pullback of the all-ODE route (kinetic1 + kinetic2 + g phi^4 as 26 channels).
//
// Reference: rcmps_gpu ode_backend.py:589-619 (_pullback over the channel specs) and
// src/observables.jl:161-199. Per spec, with forward samples f_k at node i, adjoint samples
// b_k at node n-1-i (k < nch), w = weight 2|t| and j = weight source(t):
//   m  = sum_i sum_k f_k (w R^dag b_k - w b_k R^dag) + u,   u = sum_{left edges} c sum_i j f_src b_dst
//   nn = sum_i sum_k (w b_k R - w R b_k) f_k + v,           v = sum_{right edges} c sum_i j b_dst f_src
// and for the commutator spec u, v enter through m += u Q - Q u - R u R^dag + u R R^dag,
// nn += Q^dag v - v Q^dag - R v R^dag + R R^dag v. Covector (m + nn^dag)/2, environment
// Herm(b_0 at the endpoint), value Re tr(f_{nch-1} at the endpoint), summed over the specs
// with coefficients (1, 1, g).
// Device organisation: one CTA per (node block, state x row block, spec) accumulates six
// sums on FP64 tensor cores (RowGemm): M1 = sum f_k W_k, P = sum w f_k b_k, N1 = sum W'_k f_k,
// P' = sum w b_k f_k, and for the commutator spec U, V. W_k = w R^dag b_k (+ the left-edge
// terms of a non-commutator spec) is formed per node as a full matrix in a per-CTA scratch,
// W'_k = w b_k R (+ right-edge terms) on the CTA's rows. The deferred products
// (m = M1 - P R^dag, nn = N1 - R P') and the commutator transforms run in the finalize kernel.
#include <cuda_runtime.h>
#include "common.cuh"
#include "gemm.cuh"
#include "pullback.h"

namespace rcmps {

__constant__ FullPullSpec c_pull_specs[kMaxPullSpecs];

template <int DP>
struct FGeo {
  static constexpr int MB = DP <= 64 ? DP : (DP == 96 ? 48 : 32);
  static constexpr int NW = DP == 16 ? 2 : DP == 48 ? 6 : DP == 96 ? 12 : 8;
  static constexpr int KC = DP <= 64 ? 16 : 8;
  static constexpr int NST = 4;
  static constexpr int LDA = DP + 4;
  static constexpr int NRB = DP / MB;
  using GM = RowGemm<DP, MB, NW, KC, NST>;
  static constexpr int NT = 32 * NW;
  static constexpr size_t BUF = (size_t)MB * LDA;
  static constexpr size_t SMEM = (2 * BUF + (size_t)NST * KC * (DP + kBPad)) * 16 + 128;
};

template <int DP>
__global__ void __launch_bounds__(FGeo<DP>::NT, 1)
pullback_full_kernel(FullPullbackArgs a) {
  using PG = FGeo<DP>;
  using GM = typename PG::GM;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double2* bufX = reinterpret_cast<double2*>(smem_raw);
  double2* bufY = bufX + PG::BUF;
  double2* ring = bufY + PG::BUF;
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + (size_t)PG::NST * PG::KC * (DP + kBPad));
  int* flag = reinterpret_cast<int*>(full + PG::NST);

  constexpr int MAT = DP * DP;
  const FullPullSpec& sp = c_pull_specs[blockIdx.z];
  const int blk = blockIdx.x;
  const int state = blockIdx.y / PG::NRB, rb = blockIdx.y % PG::NRB;
  const int n = a.nodes;
  const int i0 = blk * a.nodes_per_block, i1 = min(n, i0 + a.nodes_per_block);
  const long long vec = (long long)a.channels * MAT;
  const double2* samples = a.samples + (size_t)state * a.samples_stride;
  const double2* ops = a.ops + (size_t)state * a.ops_stride;
  const double2* R = ops + 2 * MAT;
  const double2* Rh = ops + 3 * MAT;
  const size_t cta = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blk;
  double2* wscr = a.scratch + cta * kMaxPullChannels * MAT;
  const int tid = threadIdx.x;

  GM gm;
  gm.ring = ring;
  gm.full = full;
  gm.wait_flag = flag;
  gm.gq = 0;
  if (tid == 0) *flag = 0;
  gm.init();
  __syncthreads();

  auto fwd = [&](int i, int k) { return samples + (size_t)i * vec + (size_t)(sp.fwd0 + k) * MAT; };
  auto adj = [&](int i, int k) { return samples + (size_t)(n - 1 - i) * vec + (size_t)(sp.adj0 + k) * MAT; };
  auto load_rows = [&](double2* dst, const double2* src, int row0, double scale) {
    for (int e = tid; e < PG::MB * DP; e += PG::NT) {
      const int r = e / DP, c = e % DP;
      dst[r * PG::LDA + c] = zscale(scale, src[(size_t)(row0 + r) * DP + c]);
    }
  };

  const int npass = sp.comm ? 6 : 4;
  ZFrag acc[GM::TPW], tmp[GM::TPW];
  for (int pass = 0; pass < npass; ++pass) {
#pragma unroll
    for (int j = 0; j < GM::TPW; ++j) acc[j].zero();
    if (pass == 0 && PG::NRB == 1) {
      load_rows(bufX, Rh, 0, 1.0);
      __syncthreads();
    }
    for (int i = i0; i < i1; ++i) {
      const double w = a.wj[2 * i], jv = a.wj[2 * i + 1];
      typename GM::Segs sb;
      sb.n = 1;
      sb.rows[0] = DP;
      if (pass == 0) {
        for (int k = 0; k < sp.nch; ++k) {
          // W_k = w R^dag b_k (+ sum of c j b_dst over the left edges from k) -> scratch slot k
          for (int rbw = 0; rbw < PG::NRB; ++rbw) {
            if (PG::NRB > 1) {
              load_rows(bufX, Rh, rbw * PG::MB, 1.0);
              __syncthreads();
            }
#pragma unroll
            for (int j = 0; j < GM::TPW; ++j) tmp[j].zero();
            sb.ptr[0] = adj(i, k);
            gm.run(tmp, bufX, PG::LDA, sb);
#pragma unroll
            for (int j = 0; j < GM::TPW; ++j)
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                int row, col;
                GM::coord(j, e, row, col);
                row += rbw * PG::MB;
                double2 v = zscale(w, tmp[j].value(e));
                if (!sp.comm)
                  for (int q = 0; q < sp.nedge; ++q)
                    if (sp.eleft[q] && sp.esrc[q] == k) v = zaxpy(jv * sp.ecoef[q], adj(i, sp.edst[q])[row * DP + col], v);
                wscr[k * MAT + row * DP + col] = v;
              }
          }
          fence_proxy_async_global();   // W_k is read next by bulk copies
          __syncthreads();
          load_rows(bufY, fwd(i, k), rb * PG::MB, 1.0);
          __syncthreads();
          sb.ptr[0] = wscr + k * MAT;
          gm.run(acc, bufY, PG::LDA, sb);
        }
      } else if (pass == 1) {
        for (int k = 0; k < sp.nch; ++k) {
          load_rows(bufY, fwd(i, k), rb * PG::MB, w);   // P += w f_k b_k
          __syncthreads();
          sb.ptr[0] = adj(i, k);
          gm.run(acc, bufY, PG::LDA, sb);
        }
      } else if (pass == 2) {
        for (int k = 0; k < sp.nch; ++k) {
          // W'_k rows = w b_k R (+ c j b_dst over the right edges from k); N1 += W'_k f_k
          load_rows(bufX, adj(i, k), rb * PG::MB, 1.0);
          __syncthreads();
#pragma unroll
          for (int j = 0; j < GM::TPW; ++j) tmp[j].zero();
          sb.ptr[0] = R;
          gm.run(tmp, bufX, PG::LDA, sb);
#pragma unroll
          for (int j = 0; j < GM::TPW; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              int row, col;
              GM::coord(j, e, row, col);
              const int grow = row + rb * PG::MB;
              double2 v = zscale(w, tmp[j].value(e));
              if (!sp.comm)
                for (int q = 0; q < sp.nedge; ++q)
                  if (!sp.eleft[q] && sp.esrc[q] == k) v = zaxpy(jv * sp.ecoef[q], adj(i, sp.edst[q])[grow * DP + col], v);
              bufY[row * PG::LDA + col] = v;
            }
          __syncthreads();
          sb.ptr[0] = fwd(i, k);
          gm.run(acc, bufY, PG::LDA, sb);
        }
      } else if (pass == 3) {
        for (int k = 0; k < sp.nch; ++k) {
          load_rows(bufX, adj(i, k), rb * PG::MB, w);   // P' += w b_k f_k
          __syncthreads();
          sb.ptr[0] = fwd(i, k);
          gm.run(acc, bufX, PG::LDA, sb);
        }
      } else {
        // commutator spec: U (pass 4) over the left edges, V (pass 5) over the right edges
        const bool left = pass == 4;
        for (int q = 0; q < sp.nedge; ++q) {
          if ((sp.eleft[q] != 0) != left) continue;
          const double cj = jv * sp.ecoef[q];
          if (left) load_rows(bufY, fwd(i, sp.esrc[q]), rb * PG::MB, cj);
          else load_rows(bufY, adj(i, sp.edst[q]), rb * PG::MB, cj);
          __syncthreads();
          sb.ptr[0] = left ? adj(i, sp.edst[q]) : fwd(i, sp.esrc[q]);
          gm.run(acc, bufY, PG::LDA, sb);
        }
      }
    }
    double2* out = a.partial + ((((size_t)state * gridDim.z + blockIdx.z) * gridDim.x + blk) * 6 + pass) * MAT;
#pragma unroll
    for (int j = 0; j < GM::TPW; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        int row, col;
        GM::coord(j, e, row, col);
        out[(row + rb * PG::MB) * DP + col] = acc[j].value(e);
      }
    __syncthreads();
  }
  gm.drain();
  if (tid == 0 && *flag) atomicExch(a.error_flag + state, 1);
}

// C = alpha op(A) op(B) (+ C), op = identity or conjugate transpose; dp x dp, one CTA.
__device__ void fmat_mul(double2* C, const double2* A, const double2* B, int dp, bool ah, bool bh, double alpha,
                         bool add) {
  for (int e = threadIdx.x; e < dp * dp; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    double2 s = make_double2(0.0, 0.0);
    for (int l = 0; l < dp; ++l) {
      const double2 x = ah ? zconj(A[l * dp + i]) : A[i * dp + l];
      const double2 y = bh ? zconj(B[j * dp + l]) : B[l * dp + j];
      s = zadd(s, zmul(x, y));
    }
    s = zscale(alpha, s);
    C[e] = add ? zadd(C[e], s) : s;
  }
  __syncthreads();
}

// One CTA per state: sum the partials of every spec, apply the deferred products and the
// commutator transforms, and write value, covector and environment (all specs summed).
__global__ void pullback_full_finalize(FullPullbackArgs a, int nblk, int nspec) {
  const int state = blockIdx.x;
  const int dp = a.dp, MAT = dp * dp, n = a.nodes;
  const long long vec = (long long)a.channels * MAT;
  const double2* samples = a.samples + (size_t)state * a.samples_stride;
  const double2* ops = a.ops + (size_t)state * a.ops_stride;
  const double2 *Q = ops, *R = ops + 2 * MAT;
  double2* t = a.fin + (size_t)state * 10 * MAT;
  double2 *M1 = t, *P = t + MAT, *N1 = t + 2 * MAT, *Pp = t + 3 * MAT, *U = t + 4 * MAT, *V = t + 5 * MAT,
          *T1 = t + 6 * MAT, *T2 = t + 7 * MAT, *cov = t + 8 * MAT, *env = t + 9 * MAT;
  double value = 0.0;
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    cov[e] = make_double2(0.0, 0.0);
    env[e] = make_double2(0.0, 0.0);
  }
  for (int s = 0; s < nspec; ++s) {
    const FullPullSpec& sp = c_pull_specs[s];
    const double coef = sp.coupling_scaled ? a.coupling[state] : 1.0;
    for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
      double2 acc[6] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}};
      for (int b = 0; b < nblk; ++b) {
        const double2* p = a.partial + ((((size_t)state * nspec + s) * nblk + b) * 6) * MAT;
        for (int q = 0; q < (sp.comm ? 6 : 4); ++q) acc[q] = zadd(acc[q], p[q * MAT + e]);
      }
      M1[e] = acc[0];
      P[e] = acc[1];
      N1[e] = acc[2];
      Pp[e] = acc[3];
      U[e] = acc[4];
      V[e] = acc[5];
    }
    __syncthreads();
    fmat_mul(M1, P, R, dp, false, true, -1.0, true);         // m = M1 - P R^dag
    fmat_mul(N1, R, Pp, dp, false, false, -1.0, true);       // nn = N1 - R P'
    if (sp.comm) {
      // m += U Q - Q U - R U R^dag + U R R^dag
      fmat_mul(M1, U, Q, dp, false, false, 1.0, true);
      fmat_mul(M1, Q, U, dp, false, false, -1.0, true);
      fmat_mul(T1, R, U, dp, false, false, 1.0, false);
      fmat_mul(M1, T1, R, dp, false, true, -1.0, true);
      fmat_mul(T2, U, R, dp, false, false, 1.0, false);
      fmat_mul(M1, T2, R, dp, false, true, 1.0, true);
      // nn += Q^dag V - V Q^dag - R V R^dag + R R^dag V
      fmat_mul(N1, Q, V, dp, true, false, 1.0, true);
      fmat_mul(N1, V, Q, dp, false, true, -1.0, true);
      fmat_mul(T1, R, V, dp, false, false, 1.0, false);
      fmat_mul(N1, T1, R, dp, false, true, -1.0, true);
      fmat_mul(T2, R, V, dp, true, false, 1.0, false);          // R^dag V
      fmat_mul(N1, R, T2, dp, false, false, 1.0, true);
    }
    const double2* last = samples + (size_t)(a.npoints - 1) * vec;
    const double2* b0 = last + (size_t)sp.adj0 * MAT;
    const double2* ftop = last + (size_t)(sp.fwd0 + sp.nch - 1) * MAT;
    for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
      const int i = e / dp, j = e % dp;
      cov[e] = zaxpy(0.5 * coef, zadd(M1[e], zconj(N1[j * dp + i])), cov[e]);
      env[e] = zaxpy(0.5 * coef, zadd(b0[e], zconj(b0[j * dp + i])), env[e]);
    }
    double tr = 0.0;
    for (int i = 0; i < dp; ++i) tr += ftop[i * dp + i].x;
    value += coef * tr;
    __syncthreads();
  }
  (void)n;
  double2* cov_out = a.cov_out + (size_t)state * MAT;
  double2* env_out = a.env_out + (size_t)state * MAT;
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    cov_out[e] = cov[e];
    env_out[e] = env[e];
  }
  if (threadIdx.x == 0) a.value_out[state] = value;
}

template <int DP>
static cudaError_t launch_pbf(const FullPullbackArgs& a, int nblk, int nspec, cudaStream_t s) {
  using PG = FGeo<DP>;
  auto k = pullback_full_kernel<DP>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PG::SMEM);
  if (e != cudaSuccess) return e;
  dim3 grid(nblk, a.nstates * PG::NRB, nspec);
  note_launch();
  k<<<grid, PG::NT, PG::SMEM, s>>>(a);
  return cudaGetLastError();
}

int pullback_full_row_blocks(int dp) {
  switch (dp) {
    case 16: return FGeo<16>::NRB;
    case 32: return FGeo<32>::NRB;
    case 48: return FGeo<48>::NRB;
    case 64: return FGeo<64>::NRB;
    case 96: return FGeo<96>::NRB;
    case 128: return FGeo<128>::NRB;
  }
  return 1;
}

cudaError_t pullback_full_set_specs(const FullPullSpec* specs, int nspec) {
  if (nspec < 1 || nspec > kMaxPullSpecs) return cudaErrorInvalidValue;
  return cudaMemcpyToSymbol(c_pull_specs, specs, nspec * sizeof(FullPullSpec));
}

cudaError_t pullback_full_launch(const FullPullbackArgs& a, int nblk, int nspec, cudaStream_t s) {
  cudaError_t e;
  switch (a.dp) {
    case 16: e = launch_pbf<16>(a, nblk, nspec, s); break;
    case 32: e = launch_pbf<32>(a, nblk, nspec, s); break;
    case 48: e = launch_pbf<48>(a, nblk, nspec, s); break;
    case 64: e = launch_pbf<64>(a, nblk, nspec, s); break;
    case 96: e = launch_pbf<96>(a, nblk, nspec, s); break;
    case 128: e = launch_pbf<128>(a, nblk, nspec, s); break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  note_launch();
  pullback_full_finalize<<<a.nstates, 256, 0, s>>>(a, nblk, nspec);
  return cudaGetLastError();
}

}  // namespace rcmps
