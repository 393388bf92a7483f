// Kinetic infinite-line terms by shifted Arnoldi, all states and all four Krylov problems of a
// batch at once.
//
// Reference: rcmps_gpu kinetic_backend.py:236-592 (KineticContext, kinetic_raw),
// cooperative_arnoldi.py:51-126 (two-pass classical Gram-Schmidt on the device) and
// src/kinetic_krylov.jl:113-189. For op in (R, [Q,R]) the problems are
//   forward:  (I - c L)  X_c = rho op^dag      adjoint: (I - c L*) A_c = op^dag
// for the angular nodes c = cos(theta). Each problem has one Arnoldi basis shared by all
// shifts: CGS2 with the breakdown test |v| <= 10 eps max(|v before projection|, eps); the basis
// doubles (16, 32, ...) until the projected estimate max_c |c H[k,k-1] y_c[k-1]| / beta meets
// the tolerance, then every shifted solution is reconstructed and its true residual checked.
// Device organisation (this library): every phase is one launch over all active problems of a
// batch (the Lindblad actions and the reconstruction on FP64 tensor cores, the Gram-Schmidt
// passes as streaming reductions over the basis); the adjoint solutions are stored conjugate
// transposed (a_c = A_c^dag, using (L* A)^dag = L*(A^dag)) as the contraction needs them.
#include <cuda_runtime.h>
#include <cfloat>
#include "common.cuh"
#include "gemm.cuh"
#include "kinetic.h"

namespace rcmps {

// ======================================================================= Lindblad action
// out = L(X) = A1 X + X A1h + (A2 X) A2h            (mode 0)
// res = |X - c L(X) - rhs|^2 per row block          (mode 1)
template <int DP>
struct LGeo {
  static constexpr int T2 = DP / 8;
  static constexpr int NW = T2 > 8 ? 8 : T2;           // 2, 4, 6, 8, 12->8? (96: 12 tiles)
  static constexpr int KC = DP <= 64 ? 16 : 8;
  static constexpr int NST = DP <= 64 ? 2 : 4;         // two ring stages keep two CTAs per SM at DP <= 64
  static constexpr int LDP = DP + 4, LDA2 = 2 * DP + 4;
  static constexpr int NT = 32 * NW;
  static constexpr size_t SMEM = ((size_t)32 * LDP + 16 * LDA2 + (size_t)NST * KC * (DP + kBPad)) * 16 + 128;
  static constexpr int MINB = SMEM <= 110 * 1024 ? 2 : 1;   // resident CTAs per SM
};
template <>
struct LGeo<96> {
  static constexpr int NW = 12, KC = 8, NST = 4, LDP = 100, LDA2 = 196, NT = 384;
  static constexpr size_t SMEM = ((size_t)32 * LDP + 16 * LDA2 + (size_t)NST * KC * (96 + kBPad)) * 16 + 128;
  static constexpr int MINB = 1;
};

// The Arnoldi matvec task of step j of problem P: W = L(V_j), or L(Z_j) for a flexible GMRES
// problem whose preconditioned basis Z_j = M V_j was formed before; X = NULL skips the problem.
__device__ __forceinline__ LindbladTask arnoldi_task(const ArnoldiProblem& P, int j) {
  LindbladTask t;
  t.X = (P.active && !P.exhausted && j < P.target) ? (P.Z ? P.Z : P.V) + (size_t)j * P.ldv : nullptr;
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
  return t;
}

// tasks: one task per slot; or (tasks NULL) the Arnoldi step j of problems probs[0..ntasks).
template <int DP>
__global__ void __launch_bounds__(LGeo<DP>::NT, LGeo<DP>::MINB)
lindblad_kernel(const LindbladTask* __restrict__ tasks, const ArnoldiProblem* __restrict__ probs, int j, int ntasks,
                int mode) {
  using LG = LGeo<DP>;
  using GR = RowGemmRing<DP, LG::NW, LG::KC, LG::NST>;
  constexpr int MAT = DP * DP;   // used by the trace term
  constexpr int TPW1 = Tiling<DP, 32, LG::NW>::TPW, TPW2 = Tiling<DP, 16, LG::NW>::TPW;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double2* panel = reinterpret_cast<double2*>(smem_raw);       // [32][LDP]: A1 rows; A2 rows
  double2* aprime = panel + 32 * LG::LDP;                        // [16][LDA2]: X rows | T rows
  double2* ring = aprime + 16 * LG::LDA2;
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + (size_t)LG::NST * LG::KC * (DP + kBPad));
  int* flag = reinterpret_cast<int*>(full + LG::NST);
  const int tid = threadIdx.x;
  const int rb = blockIdx.x % (DP / 16);
  const int task = blockIdx.x / (DP / 16);
  if (task >= ntasks) return;
  const LindbladTask T = tasks ? tasks[task] : arnoldi_task(probs[task], j);
  if (!T.X) return;   // inactive slot
  const int row0 = rb * 16;
  // tr(trw X) for the GMRES operators, computed redundantly by every row block
  __shared__ double2 trace_sh;
  if (T.trw) {
    double tr_re = 0.0, tr_im = 0.0;
    for (int e = tid; e < MAT; e += LG::NT) {
      const int i = e / DP, j = e % DP;
      const double2 t = zmul(T.trw[e], T.X[j * DP + i]);
      tr_re += t.x;
      tr_im += t.y;
    }
    tr_re = warp_sum(tr_re);
    tr_im = warp_sum(tr_im);
    __shared__ double2 tred[16];
    if ((tid & 31) == 0) tred[tid >> 5] = make_double2(tr_re, tr_im);
    __syncthreads();
    if (tid == 0) {
      double2 t = make_double2(0, 0);
      for (int w = 0; w < LG::NW; ++w) t = zadd(t, tred[w]);
      trace_sh = t;
    }
    __syncthreads();
  }
  GR gr;
  gr.ring = ring;
  gr.full = full;
  gr.wait_flag = flag;
  if (tid == 0) *flag = 0;
  gr.init();
  for (int e = tid; e < 32 * DP; e += LG::NT) {
    const int r = e / DP, c = e % DP;
    const double2* src = r < 16 ? T.A1 : T.A2;
    panel[r * LG::LDP + c] = src[(row0 + (r & 15)) * DP + c];
  }
  for (int e = tid; e < 16 * DP; e += LG::NT) {
    const int r = e / DP, c = e % DP;
    aprime[r * LG::LDA2 + c] = T.X[(row0 + r) * DP + c];
  }
  __syncthreads();
  ZFrag acc1[TPW1];
#pragma unroll
  for (int j = 0; j < TPW1; ++j) acc1[j].zero();
  typename GR::Segs sb;
  sb.n = 1;
  sb.ptr[0] = T.X;
  sb.rows[0] = DP;
  gr.template run<32>(acc1, panel, LG::LDP, sb);
  // rows 0..15: A1 X (kept), rows 16..31: T = A2 X -> aprime[:, DP:]
  double2 keep[TPW1][4];
#pragma unroll
  for (int j = 0; j < TPW1; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int row, col;
      GR::template coord<32>(j, i, row, col);
      const double2 v = acc1[j].value(i);
      keep[j][i] = v;
      if (row >= 16) aprime[(row - 16) * LG::LDA2 + DP + col] = v;
    }
  __syncthreads();
  // X A1h + T A2h : [X rows | T rows] * [A1h; A2h]
  ZFrag acc2[TPW2];
#pragma unroll
  for (int j = 0; j < TPW2; ++j) acc2[j].zero();
  sb.n = 2;
  sb.ptr[0] = T.A1h;
  sb.rows[0] = DP;
  sb.ptr[1] = T.A2h;
  sb.rows[1] = DP;
  gr.template run<16>(acc2, aprime, LG::LDA2, sb);
  // combine: out = acc2 + A1 X (from acc1 rows < 16). Route acc1 rows < 16 through shared memory.
  double2* stage = panel;   // reuse: [16][LDP]
#pragma unroll
  for (int j = 0; j < TPW1; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int row, col;
      GR::template coord<32>(j, i, row, col);
      if (row < 16) stage[row * LG::LDP + col] = keep[j][i];
    }
  __syncthreads();
  double part = 0.0;
#pragma unroll
  for (int j = 0; j < TPW2; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int row, col;
      GR::template coord<16>(j, i, row, col);
      double2 lx = zadd(acc2[j].value(i), stage[row * LG::LDP + col]);
      const size_t off = (size_t)(row0 + row) * DP + col;
      if (mode == 0) {
        if (T.trw) {
          lx = make_double2(-lx.x, -lx.y);
          if (row0 + row == col && col < T.d) lx = zadd(lx, trace_sh);
        }
        T.out[off] = lx;
      } else {
        // r = X - c L(X) - rhs
        double2 r = zsub(zsub(T.X[off], zscale(T.shift, lx)), T.rhs[off]);
        part += zabs2(r);
      }
    }
  if (mode == 1) {
    part = warp_sum(part);
    __shared__ double red[16];
    if ((tid & 31) == 0) red[tid >> 5] = part;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int w = 0; w < LG::NW; ++w) s += red[w];
      T.res[rb] = s;
    }
  }
  gr.drain();
  if (tid == 0 && *flag && T.flag) atomicExch(T.flag, 1);
}

// ======================================================================= Gram-Schmidt passes
// One CTA per (chunk of CH rows, problem). Problem data: ArnoldiProblem.
constexpr int CH = 512;

// The second pass is run only when the first lost more than 1 - 1/sqrt(2) of the norm of w
// (the criterion of Daniel, Gragg, Kaufman and Stewart): |w after pass 0|^2 < |w before|^2 / 2.
// Otherwise w is orthogonal to the basis to working precision after one pass.
__device__ __forceinline__ bool cgs_needs_second_pass(const ArnoldiProblem& P, int nchunk) {
  double before = 0.0, after = 0.0;
  for (int c = 0; c < nchunk; ++c) {
    before += P.norms[c];
    after += P.norms[nchunk + c];
  }
  return !(after > 0.5 * before);
}

// partial[p][chunk][i] = sum_{r in chunk} conj(V_i[r]) w[r], i = 0..j;  norms: |w|^2 partial (pass 0)
__global__ void cgs_partial(ArnoldiProblem* __restrict__ probs, int nprob, int j, int nchunk, int pass) {
  const int p = blockIdx.y, ch = blockIdx.x;
  ArnoldiProblem& P = probs[p];
  if (!P.active || P.exhausted || j >= P.target) return;
  if (pass == 1) {
    // every CTA takes the same decision from the norms of pass 0; CTA 0 records it for the
    // subtraction, which overwrites those norms
    const bool again = cgs_needs_second_pass(P, nchunk);
    if (ch == 0 && threadIdx.x == 0) P.reorth = again ? 1 : 0;
    if (!again) return;
  }
  const int n = P.n;
  const int r0 = ch * CH, r1 = min(n, r0 + CH);
  __shared__ double2 w[CH];
  for (int r = r0 + threadIdx.x; r < r0 + CH; r += blockDim.x) w[r - r0] = r < r1 ? P.W[r] : make_double2(0, 0);
  // before the first projection w = L(V_j): keep it for the true residuals of the shifted solves
  if (pass == 0 && P.LV)
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) P.LV[(size_t)j * P.ldv + r] = w[r - r0];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // a warp takes two basis vectors at a time, four rows per lane per step: eight independent
  // 16-byte loads in flight per lane (the pass streams the basis from HBM)
  for (int i = warp; i <= j; i += 2 * nw) {
    const bool two = i + nw <= j;
    const double2* v0 = P.V + (size_t)i * P.ldv;
    const double2* v1 = P.V + (size_t)(two ? i + nw : i) * P.ldv;
    double re0 = 0.0, im0 = 0.0, re1 = 0.0, im1 = 0.0;
    int r = r0 + lane;
    for (; r + 96 < r1; r += 128) {
      double2 a[4], c[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = v0[r + 32 * u];
        c[u] = v1[r + 32 * u];
        b[u] = w[r - r0 + 32 * u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        re0 += a[u].x * b[u].x + a[u].y * b[u].y;
        im0 += a[u].x * b[u].y - a[u].y * b[u].x;
        re1 += c[u].x * b[u].x + c[u].y * b[u].y;
        im1 += c[u].x * b[u].y - c[u].y * b[u].x;
      }
    }
    for (; r < r1; r += 32) {
      const double2 a = v0[r], c = v1[r], b = w[r - r0];
      re0 += a.x * b.x + a.y * b.y;
      im0 += a.x * b.y - a.y * b.x;
      re1 += c.x * b.x + c.y * b.y;
      im1 += c.x * b.y - c.y * b.x;
    }
    re0 = warp_sum(re0);
    im0 = warp_sum(im0);
    re1 = warp_sum(re1);
    im1 = warp_sum(im1);
    if (lane == 0) {
      P.partial[(size_t)ch * P.kmax1 + i] = make_double2(re0, im0);
      if (two) P.partial[(size_t)ch * P.kmax1 + i + nw] = make_double2(re1, im1);
    }
  }
  if (pass == 0 && warp == 0) {
    double s = 0.0;
    for (int r = r0 + lane; r < r1; r += 32) s += zabs2(w[r - r0]);
    s = warp_sum(s);
    if (lane == 0) P.norms[ch] = s;   // |w|^2 before projection
  }
}

// h_i = sum_chunks partial; H[i][j] += h_i (chunk 0); w[r] -= sum_i V_i[r] h_i; |w|^2 partial
__global__ void cgs_subtract(ArnoldiProblem* __restrict__ probs, int nprob, int j, int nchunk, int pass) {
  const int p = blockIdx.y, ch = blockIdx.x;
  ArnoldiProblem& P = probs[p];
  if (!P.active || P.exhausted || j >= P.target) return;
  if (pass == 1 && !P.reorth) return;   // pass 0 left w orthogonal: its norms stand
  extern __shared__ double2 h[];
  for (int i = threadIdx.x; i <= j; i += blockDim.x) {
    double2 s = make_double2(0, 0);
    for (int c = 0; c < nchunk; ++c) s = zadd(s, P.partial[(size_t)c * P.kmax1 + i]);
    h[i] = s;
    if (ch == 0) P.H[(size_t)i * P.kmax + j] = zadd(P.H[(size_t)i * P.kmax + j], s);
  }
  __syncthreads();
  const int n = P.n;
  const int r0 = ch * CH, r1 = min(n, r0 + CH);
  double nrm = 0.0;
  for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    double2 acc = P.W[r];
    const double2* v = P.V + r;
    int i = 0;
    // four basis rows in flight per thread
    for (; i + 3 <= j; i += 4) {
      double2 x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) x[u] = v[(size_t)(i + u) * P.ldv];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double2 c = h[i + u];
        acc.x -= x[u].x * c.x - x[u].y * c.y;
        acc.y -= x[u].x * c.y + x[u].y * c.x;
      }
    }
    for (; i <= j; ++i) {
      const double2 x = v[(size_t)i * P.ldv], c = h[i];
      acc.x -= x.x * c.x - x.y * c.y;
      acc.y -= x.x * c.y + x.y * c.x;
    }
    P.W[r] = acc;
    nrm += zabs2(acc);
  }
  {
    __shared__ double red[32];
    nrm = warp_sum(nrm);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = nrm;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
      P.norms[nchunk + ch] = s;
    }
  }
}

// beta = |w|; H[j+1][j] = beta; breakdown test; V_{j+1} = w / beta (zero after a breakdown)
__global__ void cgs_finish(ArnoldiProblem* __restrict__ probs, int nprob, int j, int nchunk) {
  const int p = blockIdx.y, ch = blockIdx.x;
  ArnoldiProblem& P = probs[p];
  if (!P.active || P.exhausted || j >= P.target) return;
  double old = 0.0, now = 0.0;
  for (int c = 0; c < nchunk; ++c) {
    old += P.norms[c];
    now += P.norms[nchunk + c];
  }
  old = sqrt(old);
  const double beta = sqrt(now);
  const double eps = DBL_EPSILON;
  const bool exhausted = beta <= 10.0 * eps * fmax(old, eps) || j + 1 == P.n_phys;
  const bool finite = isfinite(beta);
  const int n = P.n;
  const int r0 = ch * CH, r1 = min(n, r0 + CH);
  double2* next = P.V + (size_t)(j + 1) * P.ldv;
  const double inv = 1.0 / fmax(beta, DBL_MIN);
  for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x)
    next[r] = exhausted ? make_double2(0, 0) : zscale(inv, P.W[r]);
  if (ch == 0 && threadIdx.x == 0) {
    P.H[(size_t)(j + 1) * P.kmax + j] = make_double2(beta, 0.0);
    P.k = j + 1;
    if (!finite) P.nonfinite = 1;
    if (exhausted) P.exhausted = 1;
  }
}

// One whole Gram-Schmidt step (both passes of cgs_partial/cgs_subtract and cgs_finish) in one
// launch: a cluster of G CTAs per problem, each holding its rows of w in shared memory; the
// projections h_i and the norms are summed across the cluster through distributed shared memory
// (in chunk order, as the three-launch form sums its partials). The basis is still streamed twice
// per pass; what goes is four launches and the global round trips between them.
constexpr int kCgsMaxCluster = 8;
constexpr int kCgsThreads = 256;

__host__ __device__ inline int cgs_cluster(int n) {
  const int g = (n + CH - 1) / CH;
  return g < kCgsMaxCluster ? g : kCgsMaxCluster;
}
__host__ __device__ inline int cgs_rows(int n) {   // rows per CTA, a multiple of 128
  const int g = cgs_cluster(n);
  return ((n + g - 1) / g + 127) / 128 * 128;
}

__global__ void __launch_bounds__(kCgsThreads) cgs_fused(ArnoldiProblem* __restrict__ probs, int nprob, int j) {
  const int p = blockIdx.y;
  ArnoldiProblem& P = probs[p];
  // uniform over the cluster (one problem per cluster)
  if (!P.active || P.exhausted || j >= P.target) return;
  extern __shared__ __align__(16) double2 dyn[];
  const int n = P.n, rows = cgs_rows(n), G = (int)cluster_size(), ch = (int)cluster_rank();
  double2* w = dyn;                        // [rows]
  double2* part = dyn + rows;              // [j + 1]: this CTA's projections
  double2* h = part + (j + 1);             // [j + 1]: the summed projections
  __shared__ double red[kCgsThreads / 32];
  __shared__ double xch[2];                // this CTA's |w|^2 before / after the current pass
  const int r0 = ch * rows, r1 = min(n, r0 + rows);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = kCgsThreads / 32;
  auto block_sum = [&](double v) {
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < nw; ++i) t += red[i];
    return t;
  };
  auto cluster_total = [&](int slot) {   // sum of xch[slot] over the cluster, in rank order
    double t = 0.0;
    for (int g = 0; g < G; ++g) t += dsmem_load(&xch[slot], (uint32_t)g);
    return t;
  };
  double s0 = 0.0;
  for (int r = threadIdx.x; r < rows; r += kCgsThreads) {
    const double2 v = r0 + r < r1 ? P.W[r0 + r] : make_double2(0, 0);
    w[r] = v;
    s0 += zabs2(v);
    // before the first projection w = L(V_j): kept for the true residuals of the shifted solves
    if (P.LV && r0 + r < r1) P.LV[(size_t)j * P.ldv + r0 + r] = v;
  }
  s0 = block_sum(s0);
  if (threadIdx.x == 0) xch[0] = s0;
  double before = 0.0, after = 0.0;
  for (int pass = 0; pass < 2; ++pass) {
    // projections of this CTA's rows: a warp takes two basis vectors at a time
    for (int i = warp; i <= j; i += 2 * nw) {
      const bool two = i + nw <= j;
      const double2* v0 = P.V + (size_t)i * P.ldv;
      const double2* v1 = P.V + (size_t)(two ? i + nw : i) * P.ldv;
      double re0 = 0.0, im0 = 0.0, re1 = 0.0, im1 = 0.0;
      int r = r0 + lane;
      for (; r + 96 < r1; r += 128) {
        double2 a[4], c[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          a[u] = v0[r + 32 * u];
          c[u] = v1[r + 32 * u];
          b[u] = w[r - r0 + 32 * u];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          re0 += a[u].x * b[u].x + a[u].y * b[u].y;
          im0 += a[u].x * b[u].y - a[u].y * b[u].x;
          re1 += c[u].x * b[u].x + c[u].y * b[u].y;
          im1 += c[u].x * b[u].y - c[u].y * b[u].x;
        }
      }
      for (; r < r1; r += 32) {
        const double2 a = v0[r], c = v1[r], b = w[r - r0];
        re0 += a.x * b.x + a.y * b.y;
        im0 += a.x * b.y - a.y * b.x;
        re1 += c.x * b.x + c.y * b.y;
        im1 += c.x * b.y - c.y * b.x;
      }
      re0 = warp_sum(re0);
      im0 = warp_sum(im0);
      re1 = warp_sum(re1);
      im1 = warp_sum(im1);
      if (lane == 0) {
        part[i] = make_double2(re0, im0);
        if (two) part[i + nw] = make_double2(re1, im1);
      }
    }
    cluster_sync();
    if (pass == 0) before = cluster_total(0);
    for (int i = threadIdx.x; i <= j; i += kCgsThreads) {
      double2 t = make_double2(0, 0);
      for (int g = 0; g < G; ++g) {
        t.x += dsmem_load(&part[i].x, (uint32_t)g);
        t.y += dsmem_load(&part[i].y, (uint32_t)g);
      }
      h[i] = t;
      if (ch == 0) P.H[(size_t)i * P.kmax + j] = zadd(P.H[(size_t)i * P.kmax + j], t);
    }
    cluster_sync();   // every CTA has read the others' projections (and xch[0]) before they change
    double nrm = 0.0;
    for (int r = threadIdx.x; r < r1 - r0; r += kCgsThreads) {
      double2 acc = w[r];
      const double2* v = P.V + r0 + r;
      int i = 0;
      for (; i + 3 <= j; i += 4) {
        double2 x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = v[(size_t)(i + u) * P.ldv];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const double2 c = h[i + u];
          acc.x -= x[u].x * c.x - x[u].y * c.y;
          acc.y -= x[u].x * c.y + x[u].y * c.x;
        }
      }
      for (; i <= j; ++i) {
        const double2 x = v[(size_t)i * P.ldv], c = h[i];
        acc.x -= x.x * c.x - x.y * c.y;
        acc.y -= x.x * c.y + x.y * c.x;
      }
      w[r] = acc;
      nrm += zabs2(acc);
    }
    nrm = block_sum(nrm);
    if (threadIdx.x == 0) xch[1] = nrm;
    cluster_sync();
    after = cluster_total(1);
    cluster_sync();   // xch[1] is rewritten by the second pass
    // the second pass only when the first lost more than 1 - 1/sqrt(2) of the norm (uniform)
    if (pass == 0 && after > 0.5 * before) break;
  }
  // beta = |w|; H[j+1][j] = beta; breakdown test; V_{j+1} = w / beta (zero after a breakdown)
  const double old = sqrt(before), beta = sqrt(after);
  const double eps = DBL_EPSILON;
  const bool exhausted = beta <= 10.0 * eps * fmax(old, eps) || j + 1 == P.n_phys;
  double2* next = P.V + (size_t)(j + 1) * P.ldv;
  const double inv = 1.0 / fmax(beta, DBL_MIN);
  for (int r = threadIdx.x; r < r1 - r0; r += kCgsThreads)
    next[r0 + r] = exhausted ? make_double2(0, 0) : zscale(inv, w[r]);
  if (ch == 0 && threadIdx.x == 0) {
    P.H[(size_t)(j + 1) * P.kmax + j] = make_double2(beta, 0.0);
    P.reorth = after > 0.5 * before ? 0 : 1;
    P.k = j + 1;
    if (!isfinite(beta)) P.nonfinite = 1;
    if (exhausted) P.exhausted = 1;
  }
}

// Arnoldi matvec tasks of step j: W = L(V_j) for every problem still extending (L(Z_j) for a
// flexible GMRES problem, whose preconditioned basis Z_j = M V_j was formed before).
__global__ void arnoldi_tasks(const ArnoldiProblem* __restrict__ probs, int nprob, int j, LindbladTask* tasks) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nprob) return;
  tasks[p] = arnoldi_task(probs[p], j);
}

// start: beta = |rhs|, V_0 = rhs / beta
__global__ void arnoldi_start(ArnoldiProblem* __restrict__ probs, int nprob) {
  const int p = blockIdx.x;
  ArnoldiProblem& P = probs[p];
  __shared__ double red[32];
  double s = 0.0;
  for (int r = threadIdx.x; r < P.n; r += blockDim.x) s += zabs2(P.rhs[r]);
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  const double beta = sqrt(t);
  const double inv = beta > 0.0 ? 1.0 / beta : 0.0;
  for (int r = threadIdx.x; r < P.n; r += blockDim.x) P.V[r] = zscale(inv, P.rhs[r]);
  if (threadIdx.x == 0) {
    P.beta = beta;
    P.k = 0;
    P.exhausted = beta == 0.0 ? 1 : 0;
    P.nonfinite = isfinite(beta) ? 0 : 1;
  }
}

// ======================================================================= projected solves
// One warp per (problem, shift): solve (I - c H_k) y = beta e1 by Gaussian elimination with the
// two-row partial pivoting an upper-Hessenberg matrix allows (kinetic_backend.py:94-184 solves
// the same system with one CTA per shift); the rows of U go to a per-warp scratch slot.
template <int MAXC>
__global__ void __launch_bounds__(256) hessenberg_solve(ArnoldiProblem* __restrict__ probs, int nprob,
                                 const double* __restrict__ shifts, int nshift, double2* __restrict__ scratch,
                                 long long slot_elems, int nslots) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  if (gw >= nslots) return;
  double2* U = scratch + (size_t)gw * slot_elems;   // k <= 32 MAXC
  for (long long task = gw; task < (long long)nprob * nshift; task += nwarps) {
    const int p = (int)(task / nshift), si = (int)(task % nshift);
    ArnoldiProblem& P = probs[p];
    if (!P.solve) continue;
    const int k = P.k;
    if (k > 32 * MAXC) {
      if (lane == 0) atomicMax(reinterpret_cast<unsigned long long*>(&P.estimate), __double_as_longlong(INFINITY));
      continue;
    }
    const double c = shifts[si];
    const double2* H = P.H;
    const int ldh = P.kmax;
    // working row u (columns i..k-1) distributed: column q held by lane q % 32, slot q / 32
    double2 u[MAXC];
#pragma unroll
    for (int m = 0; m < MAXC; ++m) {
      const int q = lane + 32 * m;
      u[m] = make_double2(0, 0);
      if (q < k) {
        const double2 hq = H[q];
        u[m] = make_double2((q == 0 ? 1.0 : 0.0) - c * hq.x, -c * hq.y);
      }
    }
    double2 bu = make_double2(P.beta, 0.0);
    int bad = 0;
    auto rowoff = [&](int i) -> long long { return (long long)i * k - (long long)i * (i - 1) / 2; };
    for (int i = 0; i < k - 1; ++i) {
      // row i+1 of A: -c H[i+1][q] + delta, nonzero from q = i
      double2 ui = make_double2(0, 0), ri = make_double2(0, 0);
      const double2 hsub = H[(size_t)(i + 1) * ldh + i];
      ri = make_double2(-c * hsub.x, -c * hsub.y);
      {
        const int m = i >> 5, owner = i & 31;
        double2 mine = make_double2(0, 0);
#pragma unroll
        for (int mm = 0; mm < MAXC; ++mm)
          if (mm == m) mine = u[mm];
        ui.x = __shfl_sync(0xffffffffu, mine.x, owner);
        ui.y = __shfl_sync(0xffffffffu, mine.y, owner);
      }
      const bool swap = hypot(ri.x, ri.y) > hypot(ui.x, ui.y);
      const double2 piv = swap ? ri : ui, oth = swap ? ui : ri;
      if ((piv.x == 0.0 && piv.y == 0.0) || !isfinite(piv.x) || !isfinite(piv.y)) {
        bad = 1;
        break;
      }
      // f = oth / piv (Smith division)
      double2 f;
      if (fabs(piv.x) >= fabs(piv.y)) {
        const double rr = piv.y / piv.x, den = piv.x + piv.y * rr;
        f = make_double2((oth.x + oth.y * rr) / den, (oth.y - oth.x * rr) / den);
      } else {
        const double rr = piv.x / piv.y, den = piv.y + piv.x * rr;
        f = make_double2((oth.x * rr + oth.y) / den, (oth.y * rr - oth.x) / den);
      }
      const double2 br = make_double2(0, 0);
      const double2 bpiv = swap ? br : bu, both = swap ? bu : br;
      const long long off = rowoff(i);
#pragma unroll
      for (int m = 0; m < MAXC; ++m) {
        const int q = lane + 32 * m;
        if (q >= i && q < k) {
          double2 rq;
          if (q == i) rq = ri;
          else {
            const double2 hq = H[(size_t)(i + 1) * ldh + q];
            rq = make_double2((q == i + 1 ? 1.0 : 0.0) - c * hq.x, -c * hq.y);
          }
          const double2 pq = swap ? rq : u[m], oq = swap ? u[m] : rq;
          U[off + (q - i)] = pq;                           // final row i of U
          u[m] = q == i ? make_double2(0, 0) : zsub(oq, zmul(f, pq));   // working row i+1
        }
      }
      if (lane == 0) U[slot_elems - k + i] = bpiv;        // b of row i
      bu = zsub(both, zmul(f, bpiv));
    }
    if (!bad) {
      const long long off = rowoff(k - 1);
      const int m = (k - 1) >> 5, owner = (k - 1) & 31;
      double2 mine = make_double2(0, 0);
#pragma unroll
      for (int mm = 0; mm < MAXC; ++mm)
        if (mm == m) mine = u[mm];
      if (lane == owner) U[off] = mine;
      if (lane == 0) U[slot_elems - k + (k - 1)] = bu;
    }
    __syncwarp();
    // back substitution; y stored in place of u's registers
    double2 y[MAXC];
#pragma unroll
    for (int m = 0; m < MAXC; ++m) y[m] = make_double2(0, 0);
    for (int i = k - 1; i >= 0 && !bad; --i) {
      const long long off = rowoff(i);
      double sr = 0.0, si_ = 0.0;
#pragma unroll
      for (int m = 0; m < MAXC; ++m) {
        const int q = lane + 32 * m;
        if (q > i && q < k) {
          const double2 t = zmul(U[off + (q - i)], y[m]);
          sr += t.x;
          si_ += t.y;
        }
      }
      sr = warp_sum(sr);
      si_ = warp_sum(si_);
      const double2 piv = U[off];
      const double2 b = U[slot_elems - k + i];
      const double2 num = make_double2(b.x - sr, b.y - si_);
      double2 yi;
      if ((piv.x == 0.0 && piv.y == 0.0) || !isfinite(piv.x) || !isfinite(piv.y)) {
        bad = 1;
        break;
      }
      if (fabs(piv.x) >= fabs(piv.y)) {
        const double rr = piv.y / piv.x, den = piv.x + piv.y * rr;
        yi = make_double2((num.x + num.y * rr) / den, (num.y - num.x * rr) / den);
      } else {
        const double rr = piv.x / piv.y, den = piv.y + piv.x * rr;
        yi = make_double2((num.x * rr + num.y) / den, (num.y * rr - num.x) / den);
      }
      if (!isfinite(yi.x) || !isfinite(yi.y)) {
        bad = 1;
        break;
      }
      const int m = i >> 5;
#pragma unroll
      for (int mm = 0; mm < MAXC; ++mm)
        if (mm == m && lane == (i & 31)) y[mm] = yi;
    }
    double2* yout = P.Yt + (size_t)si * P.kmax;
#pragma unroll
    for (int m = 0; m < MAXC; ++m) {
      const int q = lane + 32 * m;
      if (q < k) yout[q] = y[m];
    }
    // estimate |c H[k][k-1] y[k-1]| / beta
    if (lane == ((k - 1) & 31)) {
      const int m = (k - 1) >> 5;
      double2 yl = make_double2(0, 0);
#pragma unroll
      for (int mm = 0; mm < MAXC; ++mm)
        if (mm == m) yl = y[mm];
      const double2 hs = H[(size_t)k * ldh + (k - 1)];
      double est = fabs(c) * hypot(hs.x, hs.y) * hypot(yl.x, yl.y) / P.beta;
      if (bad || !isfinite(est)) est = INFINITY;
      // non-negative doubles order like their bit patterns
      atomicMax(reinterpret_cast<unsigned long long*>(&P.estimate), __double_as_longlong(est));
    }
    if (bad && lane == 0) atomicMax(reinterpret_cast<unsigned long long*>(&P.estimate),
                                    __double_as_longlong(INFINITY));
  }
}

// ======================================================================= reconstruction
// X[p][s][:] = sum_j Yt[p][s][j] V_p[j][:] on tensor cores (CTA tile 64 shifts x 64 columns) and,
// with the kept actions LV_j = L(V_j), the true residual r = X - c L(X) - rhs =
// sum_j Yt[p][s][j] (V_j - c LV_j) - rhs (L is linear): its squared norm per 64-column tile into
// res. Adjoint problems store the conjugate transpose of each solution matrix; their residual
// norm is that of the untransposed equation (the norm is invariant under the conjugate transpose).
__global__ void __launch_bounds__(256, 1) reconstruct_residual_kernel(ArnoldiProblem* __restrict__ probs, int nprob,
                                                                      const double* __restrict__ shifts, int nshift,
                                                                      double* __restrict__ res, int ntile) {
  constexpr int BM = 64, BN = 64, BK = 16, LDA = BK + 4, LDB = BN;
  extern __shared__ __align__(16) double2 rsm[];
  double2(*As)[BM * LDA] = reinterpret_cast<double2(*)[BM * LDA]>(rsm);
  double2(*Bs)[BK * LDB] = reinterpret_cast<double2(*)[BK * LDB]>(rsm + 2 * BM * LDA);
  double2(*Cs)[BK * LDB] = reinterpret_cast<double2(*)[BK * LDB]>(rsm + 2 * BM * LDA + 2 * BK * LDB);
  __shared__ double rowsum[8][16];
  const int p = blockIdx.z;
  ArnoldiProblem& P = probs[p];
  if (!P.reconstruct) return;
  const int n = P.n, k = P.k;
  const int s0 = blockIdx.y * BM, c0 = blockIdx.x * BN;
  if (s0 >= nshift || c0 >= n) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  ZFrag ax[4], aw[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    ax[j].zero();
    aw[j].zero();
  }
  const int mt = warp >> 1, nt0 = (warp & 1) * 4;   // warp: 16-row band mt, 4 tiles of 8 columns
  const int nk = (k + BK - 1) / BK;
  auto load = [&](int kc, int buf) {
    for (int e = tid; e < BM * BK; e += 256) {
      const int r = e / BK, q = e % BK, s = s0 + r, j = kc * BK + q;
      As[buf][r * LDA + q] = (s < nshift && j < k) ? P.Yt[(size_t)s * P.kmax + j] : make_double2(0, 0);
    }
    for (int e = tid; e < BK * BN; e += 256) {
      const int q = e / BN, cc = e % BN, j = kc * BK + q, col = c0 + cc;
      const bool in = j < k && col < n;
      Bs[buf][q * LDB + cc] = in ? P.V[(size_t)j * P.ldv + col] : make_double2(0, 0);
      Cs[buf][q * LDB + cc] = in ? P.LV[(size_t)j * P.ldv + col] : make_double2(0, 0);
    }
  };
  load(0, 0);
  __syncthreads();
  for (int kc = 0; kc < nk; ++kc) {
    const int buf = kc & 1;
    if (kc + 1 < nk) load(kc + 1, buf ^ 1);
#pragma unroll
    for (int ks = 0; ks < BK / 8; ++ks) {
      AFrag a;
      load_a(As[buf], LDA, mt * 16, ks * 8, lane, a);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        BFrag b, c;
        load_b(Bs[buf], LDB, ks * 8, (nt0 + j) * 8, lane, b);
        load_b(Cs[buf], LDB, ks * 8, (nt0 + j) * 8, lane, c);
        zmma(ax[j], a, b);
        zmma(aw[j], a, c);
      }
    }
    __syncthreads();
  }
  const int dp = P.dp;
  double part[2] = {0.0, 0.0};   // rows g and g + 8 of the warp's band
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int s = s0 + mt * 16 + frag_row(lane, i), col = c0 + (nt0 + j) * 8 + frag_col(lane, i);
      if (s < nshift && col < n) {
        const double2 v = ax[j].value(i);
        const double2 r = zsub(zsub(v, zscale(shifts[s], aw[j].value(i))), P.rhs[col]);
        part[i >> 1] += zabs2(r);
        double2* X = P.X + (size_t)s * n;
        if (P.adjoint) {
          const int rr = col / dp, cc = col % dp;
          X[(size_t)cc * dp + rr] = zconj(v);
        } else {
          X[col] = v;
        }
      }
    }
  // sum over the four lanes of a row, then over the two warps of a band
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    part[h] += __shfl_xor_sync(0xffffffffu, part[h], 1);
    part[h] += __shfl_xor_sync(0xffffffffu, part[h], 2);
  }
  if ((lane & 3) == 0) {
    rowsum[warp][lane >> 2] = part[0];
    rowsum[warp][8 + (lane >> 2)] = part[1];
  }
  __syncthreads();
  if (tid < BM) {
    const int band = tid >> 4, r = tid & 15, s = s0 + tid;
    if (s < nshift) res[((size_t)p * nshift + s) * ntile + blockIdx.x] = rowsum[2 * band][r] + rowsum[2 * band + 1][r];
  }
}

// ======================================================================= contraction
// Per (state, op, node block): the four sums of the gradient contraction with wc = w c:
//   S0 = sum wc (X R^dag) a,  S1 = sum wc X a,  S2 = sum wc (a R) X,  S3 = sum wc a X
// (kinetic_backend.py:565-569), as accumulation passes on tensor cores like the pullback's.
template <int DP>
struct CGeo {
  static constexpr int MB = DP <= 64 ? DP : (DP == 96 ? 48 : 32);
  static constexpr int NW = DP == 16 ? 2 : DP == 48 ? 6 : DP == 96 ? 12 : 8;
  static constexpr int KC = DP <= 64 ? 16 : 8;
  static constexpr int NST = 4;
  static constexpr int LDA = DP + 4;
  static constexpr int NRB = DP / MB;
  static constexpr int NT = 32 * NW;
  static constexpr size_t BUF = (size_t)MB * LDA;
  static constexpr size_t SMEM = (2 * BUF + (size_t)NST * KC * (DP + kBPad)) * 16 + 128;
};

template <int DP>
__global__ void __launch_bounds__(CGeo<DP>::NT, 1)
contract_kernel(ContractArgs a) {
  using CG = CGeo<DP>;
  using GM = RowGemm<DP, CG::MB, CG::NW, CG::KC, CG::NST>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double2* bufX = reinterpret_cast<double2*>(smem_raw);
  double2* bufY = bufX + CG::BUF;
  double2* ring = bufY + CG::BUF;
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + (size_t)CG::NST * CG::KC * (DP + kBPad));
  int* flag = reinterpret_cast<int*>(full + CG::NST);
  constexpr int MAT = DP * DP;
  const int blk = blockIdx.x;
  const int so = blockIdx.y / CG::NRB, rb = blockIdx.y % CG::NRB;   // so = state * 2 + op
  const int i0 = blk * a.nodes_per_block, i1 = min(a.nodes, i0 + a.nodes_per_block);
  const double2* X = a.X[so];       // [nodes][dp^2] forward solutions
  const double2* Aa = a.A[so];      // [nodes][dp^2] adjoint solutions, conjugate transposed
  const double2* R = a.R[so >> 1];
  const double2* Rh = a.Rh[so >> 1];
  const int tid = threadIdx.x;
  GM gm;
  gm.ring = ring;
  gm.full = full;
  gm.wait_flag = flag;
  if (tid == 0) *flag = 0;
  gm.init();
  __syncthreads();
  auto load_rows = [&](double2* dst, const double2* src, double scale) {
    for (int e = tid; e < CG::MB * DP; e += CG::NT) {
      const int r = e / DP, c = e % DP;
      dst[r * CG::LDA + c] = zscale(scale, src[(size_t)(rb * CG::MB + r) * DP + c]);
    }
  };
  ZFrag acc[GM::TPW], tmp[GM::TPW];
  for (int pass = 0; pass < 4; ++pass) {
#pragma unroll
    for (int j = 0; j < GM::TPW; ++j) acc[j].zero();
    for (int i = i0; i < i1; ++i) {
      const double wc = a.weights[i] * a.shifts[i];
      const double2* Xi = X + (size_t)i * MAT;
      const double2* Ai = Aa + (size_t)i * MAT;
      typename GM::Base::Segs sb;
      sb.n = 1;
      sb.rows[0] = DP;
      if (pass == 0 || pass == 2) {
        // T = (X_i or a_i)[rows] * (R^dag or R), scaled by wc -> bufY; acc += T * (a_i or X_i)
        load_rows(bufX, pass == 0 ? Xi : Ai, 1.0);
        __syncthreads();
#pragma unroll
        for (int j = 0; j < GM::TPW; ++j) tmp[j].zero();
        sb.ptr[0] = pass == 0 ? Rh : R;
        gm.run(tmp, bufX, CG::LDA, sb);
#pragma unroll
        for (int j = 0; j < GM::TPW; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            int row, col;
            GM::coord(j, e, row, col);
            bufY[row * CG::LDA + col] = zscale(wc, tmp[j].value(e));
          }
        __syncthreads();
        sb.ptr[0] = pass == 0 ? Ai : Xi;
        gm.run(acc, bufY, CG::LDA, sb);
      } else {
        load_rows(bufX, pass == 1 ? Xi : Ai, wc);
        __syncthreads();
        sb.ptr[0] = pass == 1 ? Ai : Xi;
        gm.run(acc, bufX, CG::LDA, sb);
      }
    }
    double2* out = a.partial + (((size_t)so * gridDim.x + blk) * 4 + pass) * MAT;
#pragma unroll
    for (int j = 0; j < GM::TPW; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        int row, col;
        GM::coord(j, e, row, col);
        out[(row + rb * CG::MB) * DP + col] = acc[j].value(e);
      }
    __syncthreads();
  }
  gm.drain();
  if (tid == 0 && *flag) atomicExch(a.error_flag + (so >> 1), 1);
}

__device__ void kmat_mul(double2* C, const double2* A, const double2* B, int dp, double alpha, bool add) {
  for (int e = threadIdx.x; e < dp * dp; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    double2 s = make_double2(0.0, 0.0);
    for (int l = 0; l < dp; ++l) s = zadd(s, zmul(A[i * dp + l], B[l * dp + j]));
    s = zscale(alpha, s);
    C[e] = add ? zadd(C[e], s) : s;
  }
  __syncthreads();
}

// One CTA per state: value, covector and environment of both kinetic terms
// (kinetic_backend.py:550-583).
__global__ void contract_finalize(ContractArgs a, int nblk) {
  const int s = blockIdx.x;
  const int dp = a.dp, MAT = dp * dp;
  const double2 *Q = a.Q[s], *Qh = a.Qh[s], *R = a.R[s], *Rh = a.Rh[s], *rho = a.rho[s];
  double2* t = a.fin + (size_t)s * 12 * MAT;
  double2 *m = t, *S1 = t + MAT, *nn = t + 2 * MAT, *S3 = t + 3 * MAT, *u = t + 4 * MAT, *sa = t + 5 * MAT,
          *v = t + 6 * MAT, *T1 = t + 7 * MAT, *T2 = t + 8 * MAT, *cov = t + 9 * MAT, *env = t + 10 * MAT,
          *opm = t + 11 * MAT;
  __shared__ double red[32];
  double value = 0.0;
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    cov[e] = make_double2(0, 0);
    env[e] = make_double2(0, 0);
  }
  __syncthreads();
  for (int op = 0; op < 2; ++op) {
    const int so = 2 * s + op;
    const double2 *X = a.X[so], *Aa = a.A[so];
    // op matrix: R or C = QR - RQ
    if (op == 0) {
      for (int e = threadIdx.x; e < MAT; e += blockDim.x) opm[e] = R[e];
      __syncthreads();
    } else {
      kmat_mul(opm, Q, R, dp, 1.0, false);
      kmat_mul(opm, R, Q, dp, -1.0, true);
    }
    double vpart = 0.0;
    for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
      double2 sm[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
      for (int b = 0; b < nblk; ++b) {
        const double2* pp = a.partial + (((size_t)so * nblk + b) * 4) * MAT;
        for (int q = 0; q < 4; ++q) sm[q] = zadd(sm[q], pp[q * MAT + e]);
      }
      m[e] = sm[0];
      S1[e] = sm[1];
      nn[e] = sm[2];
      S3[e] = sm[3];
      double2 uu = make_double2(0, 0), ss = make_double2(0, 0);
      const int i = e / dp, j = e % dp;
      const double2 opji = opm[j * dp + i];
      for (int c = 0; c < a.nodes; ++c) {
        const double w = a.weights[c];
        const double2 xv = X[(size_t)c * MAT + e];
        uu = zaxpy(w, xv, uu);
        ss = zaxpy(w, Aa[(size_t)c * MAT + e], ss);
        // Re tr(op X) = sum_ij Re(op_ji X_ij)
        vpart += w * (opji.x * xv.x - opji.y * xv.y);
      }
      u[e] = uu;
      sa[e] = ss;
    }
    __syncthreads();
    vpart = warp_sum(vpart);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vpart;
    __syncthreads();
    if (threadIdx.x == 0) {
      double tot = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
      value += tot;
    }
    __syncthreads();
    // m = S0 - S1 R^dag (+ u terms), nn = S2 - R S3 (+ v terms), v = sa rho
    kmat_mul(m, S1, Rh, dp, -1.0, true);
    kmat_mul(nn, R, S3, dp, -1.0, true);
    kmat_mul(v, sa, rho, dp, 1.0, false);
    if (op == 0) {
      for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
        m[e] = zadd(m[e], u[e]);
        nn[e] = zadd(nn[e], v[e]);
      }
      __syncthreads();
    } else {
      // m += u Q - Q u - R u R^dag + u R R^dag;  nn += Q^dag v - v Q^dag - R v R^dag + R R^dag v
      kmat_mul(m, u, Q, dp, 1.0, true);
      kmat_mul(m, Q, u, dp, -1.0, true);
      kmat_mul(T1, R, u, dp, 1.0, false);
      kmat_mul(m, T1, Rh, dp, -1.0, true);
      kmat_mul(T1, u, R, dp, 1.0, false);
      kmat_mul(m, T1, Rh, dp, 1.0, true);
      kmat_mul(nn, Qh, v, dp, 1.0, true);
      kmat_mul(nn, v, Qh, dp, -1.0, true);
      kmat_mul(T2, R, v, dp, 1.0, false);
      kmat_mul(nn, T2, Rh, dp, -1.0, true);
      kmat_mul(T2, R, Rh, dp, 1.0, false);
      kmat_mul(nn, T2, v, dp, 1.0, true);
    }
    // env_op = op^dag sa
    for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
      const int i = e / dp, j = e % dp;
      double2 acc = make_double2(0, 0);
      for (int l = 0; l < dp; ++l) acc = zadd(acc, zmul(zconj(opm[l * dp + i]), sa[l * dp + j]));
      T1[e] = acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
      const int i = e / dp, j = e % dp;
      cov[e] = zadd(cov[e], zscale(0.5, zadd(m[e], zconj(nn[j * dp + i]))));
      env[e] = zadd(env[e], zscale(0.5, zadd(T1[e], zconj(T1[j * dp + i]))));
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) a.value_out[s] = value;
}

// ======================================================================= problem set-up
// Per state: the commutator C = QR - RQ and the four right-hand sides
//   R fwd: rho R^dag, R adj: R^dag, C fwd: rho C^dag, C adj: C^dag (kinetic_backend.py:281-284).
__global__ void kinetic_rhs_kernel(KineticSetup a) {
  const int s = blockIdx.x, dp = a.dp, MAT = dp * dp;
  const double2 *Q = a.ops + (size_t)s * a.ops_stride, *R = Q + 2 * MAT, *rho = Q + 7 * MAT;
  double2* c = a.comm + (size_t)s * 2 * MAT;   // C, C^dag
  double2* rhs = a.rhs + (size_t)s * 4 * MAT;
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    double2 v = make_double2(0, 0);
    for (int l = 0; l < dp; ++l) v = zadd(v, zsub(zmul(Q[i * dp + l], R[l * dp + j]), zmul(R[i * dp + l], Q[l * dp + j])));
    c[e] = v;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    c[MAT + e] = zconj(c[j * dp + i]);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < MAT; e += blockDim.x) {
    const int i = e / dp, j = e % dp;
    double2 a0 = make_double2(0, 0), a2 = make_double2(0, 0);
    for (int l = 0; l < dp; ++l) {
      a0 = zadd(a0, zmul(rho[i * dp + l], zconj(R[j * dp + l])));
      a2 = zadd(a2, zmul(rho[i * dp + l], c[MAT + l * dp + j]));
    }
    rhs[e] = a0;
    rhs[MAT + e] = zconj(R[j * dp + i]);
    rhs[2 * MAT + e] = a2;
    rhs[3 * MAT + e] = c[MAT + e];
  }
}

// residual-check tasks -> per-problem worst relative residual
__global__ void residual_reduce(ArnoldiProblem* __restrict__ probs, int nprob, const double* __restrict__ res,
                                int nshift, int rbs) {
  const int p = blockIdx.x;
  ArnoldiProblem& P = probs[p];
  if (!P.reconstruct) return;
  double worst = 0.0;
  for (int s = threadIdx.x; s < nshift; s += blockDim.x) {
    double t = 0.0;
    for (int r = 0; r < rbs; ++r) t += res[((size_t)p * nshift + s) * rbs + r];
    const double rel = sqrt(t) / P.beta;
    worst = isfinite(rel) ? fmax(worst, rel) : INFINITY;
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) worst = fmax(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = worst;
  __syncthreads();
  if (threadIdx.x == 0) {
    double w = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) w = fmax(w, red[i]);
    P.residual = w;
  }
}

// ======================================================================= launchers
template <int DP>
static cudaError_t launch_l(const LindbladTask* tasks, const ArnoldiProblem* probs, int j, int ntasks, int mode,
                            cudaStream_t s) {
  using LG = LGeo<DP>;
  auto k = lindblad_kernel<DP>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LG::SMEM);
  if (e != cudaSuccess) return e;
  if (ntasks == 0) return cudaSuccess;
  note_launch();
  k<<<ntasks * (DP / 16), LG::NT, LG::SMEM, s>>>(tasks, probs, j, ntasks, mode);
  return cudaGetLastError();
}

static cudaError_t launch_l_dp(int dp, const LindbladTask* tasks, const ArnoldiProblem* probs, int j, int ntasks,
                               int mode, cudaStream_t s) {
  switch (dp) {
    case 16: return launch_l<16>(tasks, probs, j, ntasks, mode, s);
    case 32: return launch_l<32>(tasks, probs, j, ntasks, mode, s);
    case 48: return launch_l<48>(tasks, probs, j, ntasks, mode, s);
    case 64: return launch_l<64>(tasks, probs, j, ntasks, mode, s);
    case 96: return launch_l<96>(tasks, probs, j, ntasks, mode, s);
    case 128: return launch_l<128>(tasks, probs, j, ntasks, mode, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t lindblad_launch(int dp, const LindbladTask* d_tasks, int ntasks, int mode, cudaStream_t s) {
  return launch_l_dp(dp, d_tasks, nullptr, 0, ntasks, mode, s);
}

cudaError_t lindblad_arnoldi_launch(int dp, const ArnoldiProblem* d_probs, int nprob, int j, cudaStream_t s) {
  return launch_l_dp(dp, nullptr, d_probs, j, nprob, 0, s);
}

cudaError_t arnoldi_tasks_launch(const ArnoldiProblem* d_probs, int nprob, int j, LindbladTask* d_tasks,
                                cudaStream_t s) {
  note_launch();
  arnoldi_tasks<<<(nprob + 127) / 128, 128, 0, s>>>(d_probs, nprob, j, d_tasks);
  return cudaGetLastError();
}

cudaError_t arnoldi_start_launch(ArnoldiProblem* d_probs, int nprob, cudaStream_t s) {
  note_launch();
  arnoldi_start<<<nprob, 256, 0, s>>>(d_probs, nprob);
  return cudaGetLastError();
}

cudaError_t cgs_step_launch(ArnoldiProblem* d_probs, int nprob, int j, int n, cudaStream_t s) {
  const int nchunk = (n + CH - 1) / CH;
  dim3 grid(nchunk, nprob);
  const size_t hbytes = (size_t)(j + 1) * sizeof(double2);
  for (int pass = 0; pass < 2; ++pass) {
    note_launch();
    cgs_partial<<<grid, 256, 0, s>>>(d_probs, nprob, j, nchunk, pass);
    note_launch();
    cgs_subtract<<<grid, 256, hbytes, s>>>(d_probs, nprob, j, nchunk, pass);
  }
  note_launch();
  cgs_finish<<<grid, 256, 0, s>>>(d_probs, nprob, j, nchunk);
  return cudaGetLastError();
}

cudaError_t cgs_fused_launch(ArnoldiProblem* d_probs, int nprob, int j, int n, cudaStream_t s) {
  if (nprob == 0) return cudaSuccess;
  const int g = cgs_cluster(n), rows = cgs_rows(n);
  const size_t smem = ((size_t)rows + 2 * (size_t)(j + 1)) * sizeof(double2);
  cudaError_t e = cudaFuncSetAttribute(cgs_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(g, nprob, 1);
  cfg.blockDim = dim3(kCgsThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = g;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  note_launch();
  return cudaLaunchKernelEx(&cfg, cgs_fused, d_probs, nprob, j);
}

cudaError_t gram_schmidt_launch(ArnoldiProblem* d_probs, int nprob, int j, int n, int sms, cudaStream_t s) {
  // few problems: the step is latency-bound and one clustered launch wins; a large batch streams
  // the basis from HBM on whatever SMs the concurrent trajectory leaves, where the independent
  // CTAs of the three-kernel form keep those SMs busier than clusters waiting at their barriers
  if ((long long)nprob * cgs_cluster(n) <= 2ll * sms) return cgs_fused_launch(d_probs, nprob, j, n, s);
  return cgs_step_launch(d_probs, nprob, j, n, s);
}

cudaError_t hessenberg_launch(ArnoldiProblem* d_probs, int nprob, const double* d_shifts, int nshift,
                              double2* scratch, long long slot_elems, int nslots, int kmax, cudaStream_t s) {
  const int blocks = (nslots * 32 + 255) / 256;
  // MAXC = columns per lane: the smallest template that holds k columns (32 MAXC >= k)
  if (kmax <= 64) {
    note_launch();
    hessenberg_solve<2><<<blocks, 256, 0, s>>>(d_probs, nprob, d_shifts, nshift, scratch, slot_elems, nslots);
  }
  else if (kmax <= 128) {
    note_launch();
    hessenberg_solve<4><<<blocks, 256, 0, s>>>(d_probs, nprob, d_shifts, nshift, scratch, slot_elems, nslots);
  }
  else if (kmax <= 256) {
    note_launch();
    hessenberg_solve<8><<<blocks, 256, 0, s>>>(d_probs, nprob, d_shifts, nshift, scratch, slot_elems, nslots);
  }
  else if (kmax <= 512) {
    note_launch();
    hessenberg_solve<16><<<blocks, 256, 0, s>>>(d_probs, nprob, d_shifts, nshift, scratch, slot_elems, nslots);
  }
  else {
    note_launch();
    hessenberg_solve<32><<<blocks, 256, 0, s>>>(d_probs, nprob, d_shifts, nshift, scratch, slot_elems, nslots);
  }
  return cudaGetLastError();
}

cudaError_t reconstruct_residual_launch(ArnoldiProblem* d_probs, int nprob, const double* d_shifts, int nshift,
                                        int n, double* d_res, cudaStream_t s) {
  dim3 grid((n + 63) / 64, (nshift + 63) / 64, nprob);
  const int smem = (2 * 64 * 20 + 4 * 16 * 64) * 16;
  cudaError_t e = cudaFuncSetAttribute(reconstruct_residual_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  note_launch();
  reconstruct_residual_kernel<<<grid, 256, smem, s>>>(d_probs, nprob, d_shifts, nshift, d_res, (n + 63) / 64);
  return cudaGetLastError();
}

cudaError_t residual_reduce_launch(ArnoldiProblem* d_probs, int nprob, const double* d_res, int nshift, int rbs,
                                   cudaStream_t s) {
  note_launch();
  residual_reduce<<<nprob, 256, 0, s>>>(d_probs, nprob, d_res, nshift, rbs);
  return cudaGetLastError();
}

cudaError_t kinetic_rhs_launch(const KineticSetup& a, int nstates, cudaStream_t s) {
  note_launch();
  kinetic_rhs_kernel<<<nstates, 256, 0, s>>>(a);
  return cudaGetLastError();
}

template <int DP>
static cudaError_t launch_c(const ContractArgs& a, int nblk, cudaStream_t s) {
  using CG = CGeo<DP>;
  auto k = contract_kernel<DP>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CG::SMEM);
  if (e != cudaSuccess) return e;
  dim3 grid(nblk, 2 * a.nstates * CG::NRB);
  note_launch();
  k<<<grid, CG::NT, CG::SMEM, s>>>(a);
  return cudaGetLastError();
}

cudaError_t contract_launch(const ContractArgs& a, int nblk, cudaStream_t s) {
  cudaError_t e;
  switch (a.dp) {
    case 16: e = launch_c<16>(a, nblk, s); break;
    case 32: e = launch_c<32>(a, nblk, s); break;
    case 48: e = launch_c<48>(a, nblk, s); break;
    case 64: e = launch_c<64>(a, nblk, s); break;
    case 96: e = launch_c<96>(a, nblk, s); break;
    case 128: e = launch_c<128>(a, nblk, s); break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  note_launch();
  contract_finalize<<<a.nstates, 256, 0, s>>>(a, nblk);
  return cudaGetLastError();
}

}  // namespace rcmps
