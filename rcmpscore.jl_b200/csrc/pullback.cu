// Quadrature pullback of the quartic term: covector, environment and value from the samples.
//
// Reference: rcmps_gpu ode_backend.py:589-637 (_pullback with the reduced interfaces of
// _reduced_quartic_pullback) and src/observables.jl:238-276. With forward samples
// f_0 = rho, f_1..f_3 at node i, adjoint samples b_0..b_3 at node n-1-i, b_4 = I, and
// w = weight 2|t|, j = weight source(t), c_k = (k+1) j:
//   m  = sum_i sum_k f_k (w R^dag b_k + c_k b_{k+1}) - (sum_i sum_k w f_k b_k) R^dag
//   nn = sum_i sum_k (w b_k R + c_k b_{k+1}) f_k - R (sum_i sum_k w b_k f_k)
// The k = 0 terms are linear in the adjoint samples (f_0 = rho is constant) and are formed
// once from B0 = sum w b_0 and B1 = sum j b_1 (pullback_bsum) in the finalize kernel, as are the deferred
// products with R^dag and R. The samples are Hermitian and the weights real, so in exact
// arithmetic nn = m^dag: the reference's covector (m + nn^dag)/2 equals m, and only m is formed
// (the two differ by rounding, about 1e-15 relative). Per node and k >= 1 this leaves three D^3
// products, run as two accumulation passes on FP64 tensor cores (RowGemm), each CTA owning one
// block of output rows and a range of nodes; partial sums are reduced in a fixed order.
#include <cuda_runtime.h>
#include <algorithm>
#include "common.cuh"
#include "gemm.cuh"
#include "pullback.h"

namespace rcmps {

template <int DP>
struct PGeo {
  static constexpr int MB = DP <= 64 ? DP : (DP == 96 ? 48 : 32);
  static constexpr int NW = DP == 16 ? 2 : DP == 48 ? 6 : DP == 96 ? 12 : 8;
  static constexpr int KC = DP <= 64 ? 16 : 8;
  static constexpr int NST = 4;
  static constexpr int LDA = DP + 4;
  static constexpr int NRB = DP / MB;
  using GM = RowGemm<DP, MB, NW, KC, NST>;
  static constexpr int NT = 32 * NW;
  static constexpr size_t BUF = (size_t)MB * LDA;      // double2 per A buffer
  static constexpr size_t RING = (size_t)NST * KC * (DP + kBPad);   // double2
  static constexpr size_t SMEM = (2 * BUF + RING) * 16 + 128;
  // W_k = w R^dag b_k + c b_{k+1} fits the ring area (DP rows of DP + kBPad) when the state has a
  // single row block: the second product then reads it from shared memory.
  static constexpr bool WSMEM = NRB == 1 && (size_t)DP * (DP + kBPad) <= RING;
};

template <int DP>
__global__ void __launch_bounds__(PGeo<DP>::NT, 1)
pullback_kernel(PullbackArgs a) {
  using PG = PGeo<DP>;
  using GM = typename PG::GM;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double2* bufX = reinterpret_cast<double2*>(smem_raw);
  double2* bufY = bufX + PG::BUF;
  double2* ring = bufY + PG::BUF;
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + PG::RING);
  uint64_t* ybar = full + PG::NST;   // rows of a sample block landed in bufY
  int* flag = reinterpret_cast<int*>(ybar + 1);

  constexpr int MAT = DP * DP, VEC = 7 * MAT;
  const int n = a.nodes;
  const int nblk = a.nblk;
  const int items = nblk * a.nstates * PG::NRB;   // (node block, state, row block) work items
  double2* wscr = a.scratch + (size_t)blockIdx.x * 3 * MAT;
  const int tid = threadIdx.x;

  GM gm;
  gm.ring = ring;
  gm.full = full;
  gm.wait_flag = flag;
  gm.gq = 0;
  if (tid == 0) {
    *flag = 0;
    mbar_init(ybar, 1);
  }
  gm.init();
  __syncthreads();
  uint32_t yphase = 0;
  // rows [row0, row0 + rows) of a D x D matrix into dst (bufX or bufY, leading dimension LDA) by
  // 1-D bulk copies, all in flight at once, completing on ybar (await_rows). Call with all
  // threads, after the block's last use of dst.
  auto load_rows_to = [&](double2* dst, const double2* src, int row0, int rows) {
    if (tid == 0) {
      fence_proxy_async_shared();
      mbar_expect_tx(ybar, (uint32_t)(rows * DP * 16));
      for (int r = 0; r < rows; ++r) bulk_g2s(dst + r * PG::LDA, src + (size_t)(row0 + r) * DP, DP * 16, ybar);
    }
  };
  auto load_rows_bulk = [&](const double2* src, int row0, int rows) { load_rows_to(bufY, src, row0, rows); };
  int ygave = -1;   // the phase of a bounded wait on ybar that gave up (its copies may still land)
  auto await_rows = [&]() {
    if (!mbar_wait(ybar, yphase, flag)) ygave = (int)yphase;
    yphase ^= 1u;
  };

  // a CTA takes items in turn (the grid may be smaller than the item count, so that the pullback
  // can leave SMs to concurrent work)
  for (int item = blockIdx.x; item < items; item += gridDim.x) {
    const int blk = item % nblk, ys = item / nblk;
    const int state = ys / PG::NRB, rb = ys % PG::NRB;
    const int i0 = blk * a.nodes_per_block, i1 = min(n, i0 + a.nodes_per_block);
    const double2* samples = a.samples + (size_t)state * a.samples_stride;
    const double2* ops = a.ops + (size_t)state * a.ops_stride;
    const double2* Rh = ops + 3 * MAT;
    // packed Z2 state: f_k and b_k (k = 1..3) have parity 1 for odd k, 0 for k = 2; R is odd
    const bool zs = a.packed && DP % 32 == 0 && a.dims[state] == DP &&
                    *reinterpret_cast<const int*>(a.packed + (size_t)state * a.packed_stride + a.packed_offset) != 0;
    auto zsk = [&](int row0, int pa, int pout) {
      typename GM::ZSkip z;
      z.on = zs ? 1 : 0;
      z.half = DP / 2;
      z.row0 = row0;
      z.pa = pa;
      z.pout = pout;
      return z;
    };

    auto fwd = [&](int i, int k) { return samples + (size_t)i * VEC + (size_t)(k - 1) * MAT; };       // f_k, k=1..3
    auto adj = [&](int i, int k) { return samples + (size_t)(n - 1 - i) * VEC + (size_t)(3 + k) * MAT; };  // b_k, k=0..3
    auto load_rows = [&](double2* dst, const double2* src, int row0, double scale) {
      for (int e = tid; e < PG::MB * DP; e += PG::NT) {
        const int r = e / DP, c = e % DP;
        dst[r * PG::LDA + c] = zscale(scale, src[(size_t)(row0 + r) * DP + c]);
      }
    };

    ZFrag acc[GM::TPW], tmp[GM::TPW];
    for (int pass = 0; pass < 2; ++pass) {   // m, P (nn = m^dag and P' = P^dag are not formed)
  #pragma unroll
      for (int j = 0; j < GM::TPW; ++j) acc[j].zero();
      if (pass == 0 && PG::NRB == 1) {
        load_rows(bufX, Rh, 0, 1.0);
        __syncthreads();
      }
      for (int i = i0; i < i1; ++i) {
        const double w = a.wj[2 * i], jv = a.wj[2 * i + 1];
        for (int k = 1; k <= 3; ++k) {
          const double c = jv * (k + 1);
          typename GM::Segs sb;
          sb.n = 1;
          sb.rows[0] = DP;
          if (pass == 0 && PG::WSMEM) {
            // W_k = w R^dag b_k + c b_{k+1} into the ring area, once the product's chunks are
            // consumed; b_{k+1} lands in bufY meanwhile, f_k after the epilogue
            double2* W = ring;
            constexpr int LDW = DP + kBPad;
            if (k < 3) load_rows_bulk(adj(i, k + 1), 0, DP);
  #pragma unroll
            for (int j = 0; j < GM::TPW; ++j) tmp[j].zero();
            sb.ptr[0] = adj(i, k);
            const int pk = k & 1;
            const auto z0 = zsk(0, 1, 1 ^ pk);   // R^dag b_k
            gm.run(tmp, bufX, PG::LDA, sb, z0);
            if (k < 3) await_rows();
            // a structurally zero block of W_k is never read by the live tiles of the next
            // product, so it is not written
            if (!GM::band_zero(z0)) {
  #pragma unroll
              for (int j = 0; j < GM::TPW; ++j)
  #pragma unroll
                for (int e = 0; e < 4; ++e) {
                  int row, col;
                  GM::coord(j, e, row, col);
                  double2 v = zscale(w, tmp[j].value(e));
                  if (k < 3) v = zaxpy(c, bufY[row * PG::LDA + col], v);
                  else if (row == col) v.x += c;
                  W[row * LDW + col] = v;
                }
            }
            __syncthreads();
            load_rows_bulk(fwd(i, k), 0, DP);
            await_rows();
            gm.run_smem(acc, bufY, PG::LDA, W, LDW, zsk(0, k & 1, 1));   // f_k W_k
          } else if (pass == 0) {
            // W_k = w R^dag b_k + c b_{k+1} (all rows) -> scratch
            for (int rbw = 0; rbw < PG::NRB; ++rbw) {
              // the row block of R^dag this product takes into bufX and, for the epilogue, the
              // same rows of b_{k+1} into bufY (free until f_k is loaded), on one barrier phase
              if (tid == 0) {
                fence_proxy_async_shared();
                mbar_expect_tx(ybar, (uint32_t)((k < 3 ? 2 : 1) * PG::MB * DP * 16));
                for (int r = 0; r < PG::MB; ++r) {
                  bulk_g2s(bufX + r * PG::LDA, Rh + (size_t)(rbw * PG::MB + r) * DP, DP * 16, ybar);
                  if (k < 3)
                    bulk_g2s(bufY + r * PG::LDA, adj(i, k + 1) + (size_t)(rbw * PG::MB + r) * DP, DP * 16, ybar);
                }
              }
              await_rows();
  #pragma unroll
              for (int j = 0; j < GM::TPW; ++j) tmp[j].zero();
              sb.ptr[0] = adj(i, k);
              const int pk = k & 1;
              const auto z0 = zsk(rbw * PG::MB, 1, 1 ^ pk);   // R^dag b_k
              gm.run(tmp, bufX, PG::LDA, sb, z0);
              // a structurally zero block of W_k is never read by the live tiles of the next
              // product, so it is not written
              if (!GM::band_zero(z0)) {
  #pragma unroll
                for (int j = 0; j < GM::TPW; ++j)
  #pragma unroll
                  for (int e = 0; e < 4; ++e) {
                    int row, col;
                    GM::coord(j, e, row, col);
                    double2 v = zscale(w, tmp[j].value(e));
                    if (k < 3) v = zaxpy(c, bufY[row * PG::LDA + col], v);
                    row += rbw * PG::MB;
                    if (k == 3 && row == col) v.x += c;
                    wscr[(k - 1) * MAT + row * DP + col] = v;
                  }
              }
              __syncthreads();   // bufX and bufY are refilled by the next row block
            }
            fence_proxy_async_global();   // W_k is read next by bulk copies
            __syncthreads();
            load_rows_bulk(fwd(i, k), rb * PG::MB, PG::MB);
            await_rows();
            sb.ptr[0] = wscr + (k - 1) * MAT;
            gm.run(acc, bufY, PG::LDA, sb, zsk(rb * PG::MB, k & 1, 1));   // f_k W_k
          } else {   // pass 1
            // P += w f_k b_k: the rows of f_k land in bufY and are scaled there
            load_rows_bulk(fwd(i, k), rb * PG::MB, PG::MB);
            await_rows();
            for (int e = tid; e < PG::MB * DP; e += PG::NT) {
              double2* y = bufY + (e / DP) * PG::LDA + e % DP;
              *y = zscale(w, *y);
            }
            __syncthreads();
            sb.ptr[0] = adj(i, k);
            gm.run(acc, bufY, PG::LDA, sb, zsk(rb * PG::MB, k & 1, 0));
          }
        }
      }
      // store this CTA's partial of matrix `pass` (m, P) on its rows
      double2* out = a.partial + (((size_t)state * nblk + blk) * 4 + pass) * MAT;
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
    if (tid == 0 && *flag) atomicExch(a.error_flag + state, 1);
  }
  // after a wait gave up, wait (bounded) for that phase's copies before the CTA leaves
  if (tid == 0 && ygave >= 0) mbar_wait(ybar, (uint32_t)ygave, nullptr);
  gm.drain();
}

// The environment alone, g Herm(b_0 at the endpoint), which the finalize kernel also writes: a
// caller that needs the environment before the pullback (the boundary solve) launches this right
// after the trajectory.
__global__ void quartic_env_kernel(PullbackArgs a) {
  const int state = blockIdx.x;
  const int dp = a.dp, MAT = dp * dp, VEC = 7 * MAT;
  const double2* env = a.samples + (size_t)state * a.samples_stride + (size_t)(a.npoints - 1) * VEC + 3 * MAT;
  double2* env_out = a.env_out + (size_t)state * MAT;
  const double g = a.coupling[state];
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    env_out[e] = zscale(0.5 * g, zadd(env[e], zconj(env[j * dp + i])));
  }
}

cudaError_t quartic_env_launch(const PullbackArgs& a, cudaStream_t s) {
  note_launch();
  quartic_env_kernel<<<a.nstates, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// B0 = sum_i w_i b_0 and B1 = sum_i j_i b_1 (adjoint samples at node n - 1 - i) into the
// finalize buffers, one element per thread in node order, many CTAs per state (the sums read every
// node's b_0 and b_1 from HBM: 2 n D^2 complex values per state).
constexpr int kBsumThreads = 128;
__global__ void __launch_bounds__(kBsumThreads) pullback_bsum(PullbackArgs a) {
  const int state = blockIdx.y;
  const int dp = a.dp, MAT = dp * dp, VEC = 7 * MAT, n = a.nodes;
  const int e = blockIdx.x * kBsumThreads + threadIdx.x;
  if (e >= MAT) return;
  const double2* samples = a.samples + (size_t)state * a.samples_stride;
  double2 b0 = make_double2(0, 0), b1 = make_double2(0, 0);
#pragma unroll 8
  for (int i = 0; i < n; ++i) {
    const double2* bs = samples + (size_t)(n - 1 - i) * VEC;
    b0 = zaxpy(a.wj[2 * i], __ldcs(bs + 3 * MAT + e), b0);
    b1 = zaxpy(a.wj[2 * i + 1], __ldcs(bs + 4 * MAT + e), b1);
  }
  double2* t = a.fin + (size_t)state * 8 * MAT;
  t[4 * MAT + e] = b0;
  t[5 * MAT + e] = b1;
}

// Naive dense helpers for the finalize step (a few D^3 products per state).
__device__ void dmat_mul(double2* C, const double2* A, const double2* B, int dp, bool ah, bool bh, double alpha,
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

// One CTA per state (after pullback_bsum): reduce partials, add the k = 0 terms and the deferred
// products, and write value, covector = g m (= g (m + nn^dag)/2) and environment = g Herm(b_0 at the endpoint).
__global__ void pullback_finalize(PullbackArgs a, int nblk) {
  const int state = blockIdx.x;
  const int dp = a.dp, MAT = dp * dp, VEC = 7 * MAT;
  const double2* samples = a.samples + (size_t)state * a.samples_stride;
  const double2* ops = a.ops + (size_t)state * a.ops_stride;
  const double2 *R = ops + 2 * MAT, *rho = ops + 7 * MAT;
  double2* t = a.fin + (size_t)state * 8 * MAT;
  double2 *m = t, *P = t + MAT, *B0 = t + 4 * MAT, *B1 = t + 5 * MAT, *T1 = t + 6 * MAT;
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    double2 s[2] = {{0, 0}, {0, 0}};
    for (int b = 0; b < nblk; ++b) {
      const double2* p = a.partial + (((size_t)state * nblk + b) * 4) * MAT;
      for (int q = 0; q < 2; ++q) s[q] = zadd(s[q], p[q * MAT + e]);
    }
    m[e] = s[0];
    P[e] = s[1];
  }
  __syncthreads();
  // m += rho R^dag B0 + rho B1 - (P + rho B0) R^dag
  dmat_mul(T1, R, B0, dp, true, false, 1.0, false);      // R^dag B0
  dmat_mul(m, rho, T1, dp, false, false, 1.0, true);
  dmat_mul(m, rho, B1, dp, false, false, 1.0, true);
  dmat_mul(P, rho, B0, dp, false, false, 1.0, true);      // P + rho B0
  dmat_mul(m, P, R, dp, false, true, -1.0, true);         // - (...) R^dag
  // nn = m^dag (B0, B1, rho Hermitian): the covector is g m
  const double g = a.coupling[state];
  const double2* env = samples + (size_t)(a.npoints - 1) * VEC + 3 * MAT;
  double2* cov_out = a.cov_out + (size_t)state * MAT;
  double2* env_out = a.env_out + (size_t)state * MAT;
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    cov_out[e] = zscale(g, m[e]);
    const double2 h = zadd(env[e], zconj(env[j * dp + i]));
    env_out[e] = zscale(0.5 * g, h);
  }
  if (threadIdx.x == 0) a.value_out[state] = g * a.traj_value[state];
}

template <int DP>
static cudaError_t launch_pb(const PullbackArgs& a, int nblk, cudaStream_t s) {
  using PG = PGeo<DP>;
  auto k = pullback_kernel<DP>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PG::SMEM);
  if (e != cudaSuccess) return e;
  const int items = nblk * a.nstates * PG::NRB;
  const int grid = a.ctas > 0 ? std::min(a.ctas, items) : items;
  note_launch();
  k<<<grid, PG::NT, PG::SMEM, s>>>(a);
  return cudaGetLastError();
}

size_t pullback_smem_bytes(int dp) {
  switch (dp) {
    case 16: return PGeo<16>::SMEM;
    case 32: return PGeo<32>::SMEM;
    case 48: return PGeo<48>::SMEM;
    case 64: return PGeo<64>::SMEM;
    case 96: return PGeo<96>::SMEM;
    case 128: return PGeo<128>::SMEM;
  }
  return 0;
}

int pullback_row_blocks(int dp) {
  switch (dp) {
    case 16: return PGeo<16>::NRB;
    case 32: return PGeo<32>::NRB;
    case 48: return PGeo<48>::NRB;
    case 64: return PGeo<64>::NRB;
    case 96: return PGeo<96>::NRB;
    case 128: return PGeo<128>::NRB;
  }
  return 1;
}

cudaError_t pullback_launch(const PullbackArgs& a, int nblk, cudaStream_t s) {
  cudaError_t e;
  switch (a.dp) {
    case 16: e = launch_pb<16>(a, nblk, s); break;
    case 32: e = launch_pb<32>(a, nblk, s); break;
    case 48: e = launch_pb<48>(a, nblk, s); break;
    case 64: e = launch_pb<64>(a, nblk, s); break;
    case 96: e = launch_pb<96>(a, nblk, s); break;
    case 128: e = launch_pb<128>(a, nblk, s); break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  note_launch();
  pullback_bsum<<<dim3((a.dp * a.dp + kBsumThreads - 1) / kBsumThreads, a.nstates), kBsumThreads, 0, s>>>(a);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  note_launch();
  pullback_finalize<<<a.nstates, 256, 0, s>>>(a, nblk);
  return cudaGetLastError();
}

}  // namespace rcmps
