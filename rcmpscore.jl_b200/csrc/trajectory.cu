// Persistent adaptive DOP853 trajectory of the reduced quartic system, many states per launch.
//
// Reference: rcmps_gpu persistent_trajectory_backend.py:207-283 (one cooperative grid per
// state, grid.sync between stages) and ode_backend.py:170-233, 500-586 (the equations and the
// integrator). This kernel is organised differently:
//   * one thread-block cluster per state (G = DP/16 CTAs, 16 rows of every channel per CTA);
//     clusters are independent, so a launch co-schedules many states and uneven trajectory
//     lengths need no grid-wide barrier;
//   * per stage one cluster barrier (after the stage vector is written), plus one per attempt
//     for the error-norm exchange through distributed shared memory;
//   * the right-hand side is 4 complex products per channel:
//       G1: [Qc; Rc](rows) * X_c             -> Qc X_c rows and P_c = Rc X_c rows
//       G2: [jac X_c | jac P_c + src coef_c X_s](rows) * [Qc^dag; Rc^dag]
//     out_c = jac Qc X_c + src coef_c P_s + G2 + src fixed_c, which is
//     jac L_c(X_c) + src (coef_c (Rc X_s + X_s Rc^dag) + fixed_c) with P_s = Rc X_s shared
//     between the jump of channel s and the insertion into channel c;
//   * products on FP64 tensor cores (mma.sync m16n8k8), B operands streamed by 1-D bulk copies
//     into a 4-stage shared-memory ring, A operands resident in shared memory;
//   * the scalar energy channel is integrated from per-CTA partial traces reduced once per
//     attempt (its value never feeds back into the matrix channels);
//   * the step controller runs identically in every CTA from the same reduced norms.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include "common.cuh"
#include "dop853_tables.h"
#include "source_table.h"
#include "trajectory.h"

namespace rcmps {

__constant__ double c_dop_a[256];
__constant__ double c_dop_b[16];
__constant__ double c_dop_c[16];
__constant__ double c_dop_e5[16];
__constant__ double c_dop_e3[16];
__constant__ double c_dop_d[64];
__constant__ double c_source[RCMPS_SOURCE_SEGMENTS * (RCMPS_SOURCE_DEGREE + 1)];

// 2|t| J(t^2) from the piecewise Chebyshev table (Clenshaw); |t| <= sqrt(40).
__device__ double source_value(double t) {
  const double a = fabs(t);
  const double width = RCMPS_SOURCE_AMAX / RCMPS_SOURCE_SEGMENTS;
  int seg = (int)(a / width);
  if (seg > RCMPS_SOURCE_SEGMENTS - 1) seg = RCMPS_SOURCE_SEGMENTS - 1;
  const double z = 2.0 * (a - seg * width) / width - 1.0;
  const double* c = c_source + seg * (RCMPS_SOURCE_DEGREE + 1);
  double b1 = 0.0, b2 = 0.0;
  for (int j = RCMPS_SOURCE_DEGREE; j > 0; --j) {
    const double b0 = 2.0 * z * b1 - b2 + c[j];
    b2 = b1;
    b1 = b0;
  }
  return z * b1 - b2 + c[0];
}

// The next double above t (nextafter(t, +inf)) for finite t.
__device__ __forceinline__ double next_up(double t) {
  if (t == 0.0) return 4.9406564584124654e-324;
  const long long b = __double_as_longlong(t);
  return __longlong_as_double(t > 0.0 ? b + 1 : b - 1);
}

// Insertion source channel and coefficient of each channel (ode_backend.py:193).
__device__ __forceinline__ int ins_src(int c) {
  return c == 1 ? 0 : c == 2 ? 1 : c == 3 ? 4 : c == 4 ? 5 : c == 5 ? 6 : -1;
}
__device__ __forceinline__ double ins_coef(int c) {
  return c == 1 ? 2.0 : c == 2 ? 3.0 : c == 3 ? 1.0 : c == 4 ? 2.0 : c == 5 ? 3.0 : 0.0;
}

// Tiling of one product pass: M rows (a multiple of 16) by DP columns over NW warps; a warp owns
// TPW consecutive 16x8 tiles of one band, or (when there are fewer tiles than warps) one tile and a
// 1/SK slice of the k-steps.
template <int DP, int M, int NW>
struct PassTiling {
  static constexpr int NTN = DP / 8;
  static constexpr int T = (M / 16) * NTN;
  static constexpr int SK = T >= NW ? 1 : NW / T;
  static constexpr int TPW = T >= NW ? T / NW : 1;
  static_assert(T % NW == 0 || NW % T == 0, "tiling");
  static_assert(SK > 1 || NTN % TPW == 0, "a warp's tiles share one band");
  static constexpr int SPLIT = SK > 1 ? T * (SK - 1) * 128 : 0;   // split-K scratch (double2)
};

template <int DP>
struct Geo {
  static constexpr int G = DP / 16;
  static constexpr int NW = (DP == 48 || DP == 96) ? 12 : (DP == 64 || DP == 128) ? 16 : 8;
  static constexpr int NT = 32 * NW;
  static constexpr int KC = DP <= 64 ? 16 : 8;       // rows of a streamed B chunk
  static constexpr int NST = 4;                       // ring stages
  static constexpr int LDB = DP + kBPad;              // padded row stride of a ring chunk
  static constexpr int LDP = DP + 4;                  // panel leading dimension (complex)
  static constexpr int LDA2 = 2 * DP + 4;             // A' leading dimension
  static constexpr int GS = DP <= 64 ? 2 : 1;         // channels per G2 pass
  static constexpr int NPASS = GS == 2 ? 4 : 7;       // G2 passes: {0,1},{2},{3,4},{5,6} or one per channel
  using T1 = PassTiling<DP, 32, NW>;
  using T2a = PassTiling<DP, 16 * GS, NW>;
  using T2b = PassTiling<DP, 16, NW>;
  static constexpr int CH1 = DP / KC, CH2 = 2 * DP / KC;   // chunks per G1 channel / G2 pass
  static constexpr int NCHUNK = 7 * CH1 + NPASS * CH2;
  static constexpr int MAT = DP * DP;                 // elements of one channel matrix
  static constexpr int VEC = 7 * MAT;                 // elements of one stage vector
  static constexpr int OWN = 7 * 16 * DP;             // elements owned by one CTA
  static constexpr int cmax(int a, int b) { return a > b ? a : b; }
  // shared memory (double2 units): one direction panel, the A' rows of a pass, the ring, split-K
  static constexpr int OFF_PANEL = 0;
  static constexpr int OFF_APRIME = OFF_PANEL + 32 * LDP;
  static constexpr int OFF_RING = OFF_APRIME + 16 * GS * LDA2;
  static constexpr int OFF_SPLIT = OFF_RING + NST * KC * LDB;
  static constexpr int END2 = OFF_SPLIT + cmax(T1::SPLIT, cmax(T2a::SPLIT, T2b::SPLIT));
  static constexpr size_t SMEM = (size_t)END2 * 16 + 2048;   // + barriers and scalars (see carve)
  // G2 pass p: first channel and channel count
  __device__ static int pass_first(int p) { return GS == 2 ? (p == 0 ? 0 : p == 1 ? 2 : p == 2 ? 3 : 5) : p; }
  __device__ static int pass_count(int p) { return GS == 2 ? (p == 1 ? 1 : 2) : 1; }
};

// Scalars of the controller, one copy per CTA (identical in all CTAs of a cluster).
struct Ctl {
  double t, h, h_next, t_new, err, min_h, max_h;
  double y_sc, prop_sc;                  // the scalar channel (total)
  double ksc[16];                        // total scalar k of the attempt, by stage
  double jac[16], src[16];               // per stage of the attempt
  long long attempts, accepted, rejected, dense_steps, next_point, first, last;
  int status, after_reject, accept, dense, done, wait_flag;
  int kslot[16];                         // k buffer of each stage (permuted on acceptance)
};

struct Xch {                             // exchanged through distributed shared memory
  double s5, s3;
  double kscp[13];
  int flag;
};

template <int DP>
struct Smem {
  double2* panel;     // [32][LDP]: the current direction's [Qc; Rc] rows
  double2* aprime;    // [16 GS][LDA2]
  double2* ring;      // [NST][KC*LDB]
  double2* split;     // split-K partial fragments
  uint64_t* full;     // [NST]
  Ctl* ctl;
  Xch* xch;
  double* red;        // [NW * 2] block reduction scratch
  double* kscp;       // [16] this CTA's partial scalar k by stage
};

template <int DP>
__device__ __forceinline__ Smem<DP> carve(unsigned char* base) {
  using GE = Geo<DP>;
  Smem<DP> s;
  double2* z = reinterpret_cast<double2*>(base);
  s.panel = z + GE::OFF_PANEL;
  s.aprime = z + GE::OFF_APRIME;
  s.ring = z + GE::OFF_RING;
  s.split = z + GE::OFF_SPLIT;
  constexpr size_t o_ctl = 64;
  constexpr size_t o_xch = o_ctl + ((sizeof(Ctl) + 15) / 16) * 16;
  constexpr size_t o_red = o_xch + ((sizeof(Xch) + 15) / 16) * 16;
  constexpr size_t o_ksc = o_red + 32 * sizeof(double) * 2;
  static_assert(o_ksc + 16 * sizeof(double) <= 2048, "shared tail");
  unsigned char* tail = base + (size_t)GE::END2 * 16;
  s.full = reinterpret_cast<uint64_t*>(tail);
  s.ctl = reinterpret_cast<Ctl*>(tail + o_ctl);
  s.xch = reinterpret_cast<Xch*>(tail + o_xch);
  s.red = reinterpret_cast<double*>(tail + o_red);
  s.kscp = reinterpret_cast<double*>(tail + o_ksc);
  return s;
}

// Block-wide sum of two doubles; the result is returned to every thread.
template <int DP>
__device__ void block_sum2(double& a, double& b, double* red) {
  using GE = Geo<DP>;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  __syncthreads();
  if (lane == 0) { red[2 * w] = a; red[2 * w + 1] = b; }
  __syncthreads();
  double x = 0.0, y = 0.0;
  for (int i = 0; i < GE::NW; ++i) { x += red[2 * i]; y += red[2 * i + 1]; }
  a = x;
  b = y;
}

template <int DP>
struct Rhs {
  using GE = Geo<DP>;
  const TrajState* st;
  Smem<DP> sm;
  int row0, tid, lane, warp;
  long long* gq;   // running chunk counter (uniform across the CTA)

  // Source pointer of chunk q (0 <= q < NCHUNK) of one right-hand side on stage vector zb.
  __device__ const double2* chunk_src(int q, const double2* zb) const {
    if (q < 7 * GE::CH1) {
      const int c = q / GE::CH1, k = q % GE::CH1;
      return zb + c * GE::MAT + k * GE::KC * DP;
    }
    q -= 7 * GE::CH1;
    const int p = q / GE::CH2, k = q % GE::CH2;
    const bool fwd = GE::pass_first(p) < 3;
    const double2* top = fwd ? st->Qh : st->Q;     // (Qc)^dag
    const double2* bot = fwd ? st->Rh : st->R;     // (Rc)^dag
    const int r = k * GE::KC;
    return r < DP ? top + r * DP : bot + (r - DP) * DP;
  }

  __device__ void issue(long long gidx, int q, const double2* zb) {
    const int slot = (int)(gidx % GE::NST);
    mbar_expect_tx(&sm.full[slot], GE::KC * DP * 16);
    const double2* src = chunk_src(q, zb);
    double2* dst = sm.ring + slot * GE::KC * GE::LDB;
#pragma unroll
    for (int r = 0; r < GE::KC; ++r) bulk_g2s(dst + r * GE::LDB, src + r * DP, DP * 16, &sm.full[slot]);
  }

  // Wait for chunk (global index gidx); bounded.
  __device__ const double2* await(long long gidx) {
    const int slot = (int)(gidx % GE::NST);
    const uint32_t parity = (uint32_t)((gidx / GE::NST) & 1);
    if (!mbar_wait(&sm.full[slot], parity, &sm.ctl->wait_flag)) {}
    return sm.ring + slot * GE::KC * GE::LDB;
  }

  __device__ void load_panel(int dir, double2* dst) const {
    const double2* qs = dir == 0 ? st->Q : st->Qh;
    const double2* rs = dir == 0 ? st->R : st->Rh;
    for (int e = tid; e < 32 * DP; e += GE::NT) {
      const int r = e / DP, col = e % DP;
      const double2* srcm = r < 16 ? qs : rs;
      dst[r * GE::LDP + col] = srcm[(row0 + (r & 15)) * DP + col];
    }
  }

  // Split-K reduction; warps with slice > 0 deposit, slice 0 adds.
  template <int TPW, int SK>
  __device__ void split_reduce(ZFrag* acc, int tile0, int slice) {
    if constexpr (SK > 1) {
      if (slice > 0) {
#pragma unroll
        for (int j = 0; j < TPW; ++j) {
          double2* p = sm.split + ((tile0 + j) * (SK - 1) + slice - 1) * 128;
#pragma unroll
          for (int i = 0; i < 4; ++i) p[i * 32 + lane] = make_double2(acc[j].re[i], acc[j].im[i]);
        }
      }
      __syncthreads();
      if (slice == 0) {
#pragma unroll
        for (int j = 0; j < TPW; ++j)
          for (int sl = 1; sl < SK; ++sl) {
            const double2* p = sm.split + ((tile0 + j) * (SK - 1) + sl - 1) * 128;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const double2 v = p[i * 32 + lane];
              acc[j].re[i] += v.x;
              acc[j].im[i] += v.y;
            }
          }
      }
      __syncthreads();
    }
  }

  // acc += A (M rows in shared memory, lda) * the next nch streamed chunks. Ends with the chunks'
  // slots released and the next chunks issued.
  template <class TL>
  __device__ void stream_product(ZFrag* acc, const double2* A, int lda, int nch, int& q, long long g0,
                                 const double2* zb) {
    constexpr int TPW = TL::TPW, SK = TL::SK;
    const int tile0 = SK > 1 ? warp / SK : warp * TPW;
    const int slice = SK > 1 ? warp % SK : 0;
    const int mt = tile0 / TL::NTN;
    for (int ch = 0; ch < nch; ++ch, ++q) {
      const double2* B = await(g0 + q);
#pragma unroll
      for (int ks = 0; ks < GE::KC / 8; ++ks) {
        const int kstep = ch * (GE::KC / 8) + ks;
        if (kstep % SK != slice) continue;
        double ar[4], ai[4], nai[4];
        load_a(A, lda, mt * 16, kstep * 8, lane, ar, ai, nai);
        double br[TPW][2], bi[TPW][2];
#pragma unroll
        for (int j = 0; j < TPW; ++j) load_b(B, GE::LDB, ks * 8, ((tile0 + j) % TL::NTN) * 8, lane, br[j], bi[j]);
        zmma_tiles<TPW>(acc, ar, ai, nai, br, bi);
      }
      __syncthreads();
      if (tid == 0 && q + GE::NST < GE::NCHUNK) issue(g0 + q + GE::NST, q + GE::NST, zb);
    }
    split_reduce<TPW, SK>(acc, tile0, slice);
  }

  // G2 pass over the channels first..first+NC-1 (same direction).
  template <int NC>
  __device__ void g2_pass(int first, const double2* zb, double2* kout, double jac, double src, int& q,
                          long long g0) {
    using TL = PassTiling<DP, 16 * NC, GE::NW>;
    constexpr int TPW = TL::TPW, SK = TL::SK;
    // A' = [jac X_c | jac P_c + src coef_c X_s] on this CTA's rows, channel i of the pass in rows 16 i..
    for (int e = tid; e < 16 * NC * DP; e += GE::NT) {
      const int r = e / DP, col = e % DP;
      const int c = first + r / 16;
      const int s = ins_src(c);
      const size_t off = (size_t)(row0 + (r & 15)) * DP + col;
      const double2 x = __ldcg(zb + (size_t)c * GE::MAT + off);
      double2 m = zscale(jac, __ldcg(st->P + (size_t)c * GE::MAT + off));
      if (s >= 0) m = zaxpy(src * ins_coef(c), __ldcg(zb + (size_t)s * GE::MAT + off), m);
      sm.aprime[r * GE::LDA2 + col] = zscale(jac, x);
      sm.aprime[r * GE::LDA2 + DP + col] = m;
    }
    __syncthreads();
    ZFrag acc[TPW];
#pragma unroll
    for (int j = 0; j < TPW; ++j) acc[j].zero();
    stream_product<TL>(acc, sm.aprime, GE::LDA2, GE::CH2, q, g0, zb);
    const int tile0 = SK > 1 ? warp / SK : warp * TPW;
    const int slice = SK > 1 ? warp % SK : 0;
    if (slice == 0) {
#pragma unroll
      for (int j = 0; j < TPW; ++j) {
        const int tile = tile0 + j, mt = tile / TL::NTN, nt = tile % TL::NTN;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r = mt * 16 + frag_row(lane, i), col = nt * 8 + frag_col(lane, i);
          const int c = first + r / 16;
          const int s = ins_src(c);
          const size_t loc = (size_t)(row0 + (r & 15)) * DP + col;
          const size_t off = (size_t)c * GE::MAT + loc;
          double2 v = zadd(make_double2(acc[j].re[i], acc[j].im[i]), kout[off]);
          if (s >= 0) v = zaxpy(src * ins_coef(c), __ldcg(st->P + (size_t)s * GE::MAT + loc), v);
          if (c == 0) v = zaxpy(src, st->fixed0[loc], v);
          if (c == 6) v = zaxpy(src, st->fixed6[loc], v);
          kout[off] = v;
        }
      }
    }
    __syncthreads();
  }

  // One right-hand side: k_out = f(t, z) on this CTA's rows. zb: the full stage vector
  // (written by every CTA of the cluster before the barrier that precedes this call).
  __device__ void operator()(const double2* zb, double2* kout, double jac, double src) {
    const long long g0 = *gq;
    if (tid == 0) {
      fence_proxy_async_global();
      for (int q = 0; q < GE::NST && q < GE::NCHUNK; ++q) issue(g0 + q, q, zb);
    }
    int q = 0;
    // ------------------------------------------------------------------ G1: [Qc; Rc] rows * X_c
    {
      using TL = typename GE::T1;
      constexpr int TPW = TL::TPW, SK = TL::SK;
      const int tile0 = SK > 1 ? warp / SK : warp * TPW;
      const int slice = SK > 1 ? warp % SK : 0;
      const int mt = tile0 / TL::NTN;     // 0: Qc rows, 1: Rc rows
      for (int c = 0; c < 7; ++c) {
        if (c == 0 || c == 3) {
          __syncthreads();
          load_panel(c == 0 ? 0 : 1, sm.panel);
          __syncthreads();
        }
        ZFrag acc[TPW];
#pragma unroll
        for (int j = 0; j < TPW; ++j) acc[j].zero();
        stream_product<TL>(acc, sm.panel, GE::LDP, GE::CH1, q, g0, zb);
        if (slice == 0) {
#pragma unroll
          for (int j = 0; j < TPW; ++j) {
            const int nt = (tile0 + j) % TL::NTN;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const int r = frag_row(lane, i), col = nt * 8 + frag_col(lane, i);
              const size_t off = (size_t)c * GE::MAT + (size_t)(row0 + r) * DP + col;
              const double2 v = make_double2(acc[j].re[i], acc[j].im[i]);
              if (mt == 0) kout[off] = zscale(jac, v);
              else st->P[off] = v;
            }
          }
        }
      }
    }
    __syncthreads();
    // ------------------------------------------------------------------ G2 passes
    for (int p = 0; p < GE::NPASS; ++p) {
      const int first = GE::pass_first(p);
      if constexpr (GE::GS == 2) {
        if (GE::pass_count(p) == 2) g2_pass<2>(first, zb, kout, jac, src, q, g0);
        else g2_pass<1>(first, zb, kout, jac, src, q, g0);
      } else {
        g2_pass<1>(first, zb, kout, jac, src, q, g0);
      }
    }
    *gq = g0 + GE::NCHUNK;
    __syncthreads();
  }
};

// Element e of this CTA's rows -> offset in a stage vector.
template <int DP>
__device__ __forceinline__ size_t own_offset(int e, int row0) {
  const int c = e / (16 * DP), rem = e % (16 * DP);
  return (size_t)c * DP * DP + (size_t)(row0 + rem / DP) * DP + (rem % DP);
}

template <int DP>
__global__ void __launch_bounds__(Geo<DP>::NT, 1)
trajectory_kernel(const TrajState* __restrict__ states, const double* __restrict__ points, int npoints,
                  TrajControls ctl_in) {
  using GE = Geo<DP>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem<DP> sm = carve<DP>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t rank = cluster_rank();
  const int sidx = (int)cluster_id_x();
  const TrajState* st = states + sidx;
  const int row0 = (int)rank * 16;
  Ctl& C = *sm.ctl;
  long long gq = 0;

  if (tid == 0) {
    for (int i = 0; i < GE::NST; ++i) mbar_init(&sm.full[i], 1);
    fence_mbar_init();
    C.t = -ctl_in.endpoint;
    C.h = fmin(ctl_in.initial_h, 2.0 * ctl_in.endpoint);
    C.min_h = INFINITY;
    C.max_h = 0.0;
    C.err = 0.0;
    C.y_sc = 0.0;
    C.attempts = C.accepted = C.rejected = C.dense_steps = C.next_point = 0;
    C.status = 0;
    C.after_reject = 0;
    C.done = 0;
    C.wait_flag = 0;
    C.jac[0] = 2.0 * ctl_in.endpoint;
    C.src[0] = source_value(-ctl_in.endpoint);
    for (int i = 0; i < 16; ++i) { C.ksc[i] = 0.0; sm.kscp[i] = 0.0; }
  }
  __syncthreads();
  Rhs<DP> rhs{st, sm, row0, tid, lane, warp, &gq};

  // slot permutation: C.kslot[s] is the k buffer of stage s; y and proposed swap on acceptance
  if (tid < 16) C.kslot[tid] = tid;
  __syncthreads();
  double2* ybuf = st->y;
  double2* pbuf = st->prop;
  auto kb = [&](int s) { return st->k + (size_t)C.kslot[s] * GE::VEC; };
  long long zcount = 0;
  auto zb = [&](long long n) { return st->z + (size_t)(n & 1) * GE::VEC; };

  // initial y = 0 on own rows, and f = RHS(-a, 0)
  for (int e = tid; e < GE::OWN; e += GE::NT) {
    const size_t off = own_offset<DP>(e, row0);
    ybuf[off] = make_double2(0.0, 0.0);
    zb(zcount)[off] = make_double2(0.0, 0.0);
  }
  fence_proxy_async_global();
  cluster_sync();
  rhs(zb(zcount), kb(0), C.jac[0], C.src[0]);
  ++zcount;

  const double N = 7.0 * st->d * st->d + 1.0;
  const double atol = st->atol, rtol = st->rtol;
  const long long max_steps = st->max_steps;
  const unsigned long long t_start = global_ns();

  while (true) {
    // ---------------------------------------------------------------- prepare the attempt
    if (tid == 0) {
      const double t = C.t, boundary = t < 0.0 ? 0.0 : ctl_in.endpoint;
      double h = fmin(C.h, boundary - t);
      if (C.attempts >= max_steps) C.status = kMaxSteps;
      else if (!isfinite(h) || h <= 10.0 * fabs(next_up(t) - t)) C.status = kStepUnderflow;
      if (!C.status) {
        ++C.attempts;
        C.min_h = fmin(C.min_h, h);
        C.max_h = fmax(C.max_h, h);
      }
      C.h = h;
      for (int s = 1; s < 16; ++s) {
        const double ts = s == 12 ? __dadd_rn(t, h) : __dadd_rn(t, __dmul_rn(c_dop_c[s], h));
        if (fabs(ts) > RCMPS_SOURCE_AMAX * (1.0 + 1e-14)) C.status = kSourceDomain;
        C.jac[s] = 2.0 * fabs(ts);
        C.src[s] = source_value(ts);
      }
    }
    __syncthreads();
    if (C.status) break;   // uniform across the cluster: every CTA computes the same
    const double h = C.h;

    // ---------------------------------------------------------------- stages 1..12
    for (int s = 1; s <= 12; ++s) {
      const double* w = s == 12 ? c_dop_b : c_dop_a + 16 * s;
      const int terms = s;   // a[s][0..s-1], b[0..11]
      double2* z = zb(zcount);
      double part = 0.0, dummy = 0.0;
      const double2* kp[12];
      double ha[12];
#pragma unroll
      for (int j = 0; j < 12; ++j) {
        kp[j] = kb(j);
        ha[j] = j < terms ? h * w[j] : 0.0;
      }
      for (int e = tid; e < GE::OWN; e += GE::NT) {
        const size_t off = own_offset<DP>(e, row0);
        double2 kv[12];
#pragma unroll
        for (int j = 0; j < 12; ++j) kv[j] = ha[j] != 0.0 ? __ldcg(kp[j] + off) : make_double2(0.0, 0.0);
        double2 v = ybuf[off];
#pragma unroll
        for (int j = 0; j < 12; ++j) v = zaxpy(ha[j], kv[j], v);
        z[off] = v;
        if (s == 12) pbuf[off] = v;
        if (e / (16 * DP) == 2) {
          const double2 sv = st->S[off - 2 * (size_t)GE::MAT];
          part += v.x * sv.x - v.y * sv.y;
        }
      }
      block_sum2<DP>(part, dummy, sm.red);
      if (tid == 0) sm.kscp[s] = 4.0 * C.src[s] * part;
      fence_proxy_async_global();
      cluster_sync();
      rhs(z, kb(s), C.jac[s], C.src[s]);
      ++zcount;
    }

    // ---------------------------------------------------------------- error norms
    {
      double s5 = 0.0, s3 = 0.0;
      for (int e = tid; e < GE::OWN; e += GE::NT) {
        const size_t off = own_offset<DP>(e, row0);
        double2 e5 = make_double2(0.0, 0.0), e3 = make_double2(0.0, 0.0);
#pragma unroll
        for (int s = 0; s <= 12; ++s) {
          const double2 kv = kb(s)[off];
          e5 = zaxpy(c_dop_e5[s], kv, e5);
          e3 = zaxpy(c_dop_e3[s], kv, e3);
        }
        const double2 yo = ybuf[off], yn = pbuf[off];
        const double scale = atol + rtol * fmax(hypot(yo.x, yo.y), hypot(yn.x, yn.y));
        s5 += zabs2(e5) / (scale * scale);
        s3 += zabs2(e3) / (scale * scale);
      }
      block_sum2<DP>(s5, s3, sm.red);
      if (tid == 0) {
        sm.xch->s5 = s5;
        sm.xch->s3 = s3;
        for (int s = 0; s < 13; ++s) sm.xch->kscp[s] = sm.kscp[s];
        // bit 0: a bounded wait gave up in this CTA; bit 1: this CTA's device clock passed the
        // watchdog. Both are OR-ed over the cluster, so every CTA takes the same decision.
        int f = C.wait_flag ? 1 : 0;
        if (ctl_in.max_ns && global_ns() - t_start >= ctl_in.max_ns) f |= 2;
        sm.xch->flag = f;
      }
      cluster_sync();
      if (tid == 0) {
        double t5 = 0.0, t3 = 0.0;
        double ks[13];
        for (int s = 1; s < 13; ++s) ks[s] = 0.0;
        int flag = 0;
        for (uint32_t g = 0; g < (uint32_t)GE::G; ++g) {
          t5 += dsmem_load(&sm.xch->s5, g);
          t3 += dsmem_load(&sm.xch->s3, g);
          for (int s = 1; s < 13; ++s) ks[s] += dsmem_load(&sm.xch->kscp[s], g);
          flag |= dsmem_load_int(&sm.xch->flag, g);
        }
        ks[0] = C.ksc[0];
        for (int s = 1; s < 13; ++s) C.ksc[s] = ks[s];
        // the scalar channel's own contribution
        double prop = C.y_sc, e5 = 0.0, e3 = 0.0;
        for (int s = 0; s < 12; ++s) prop += h * c_dop_b[s] * ks[s];
        for (int s = 0; s <= 12; ++s) { e5 += c_dop_e5[s] * ks[s]; e3 += c_dop_e3[s] * ks[s]; }
        const double scale = atol + rtol * fmax(fabs(C.y_sc), fabs(prop));
        t5 += (e5 / scale) * (e5 / scale);
        t3 += (e3 / scale) * (e3 / scale);
        C.prop_sc = prop;
        // controller (ode_backend.py:529-547; persistent_trajectory_backend.py:109-131)
        const double den = __dadd_rn(t5, __dmul_rn(0.01, t3));
        const double err = den > 0.0 ? __ddiv_rn(__dmul_rn(h, t5), __dsqrt_rn(__dmul_rn(den, N))) : 0.0;
        C.err = err;
        C.accept = 0;
        C.dense = 0;
        if (flag & 1) C.status = kWaitLimit;
        else if (flag & 2) C.status = kDeviceTimeout;
        else if (!isfinite(t5) || !isfinite(t3) || !isfinite(err)) C.status = kNonfiniteError;
        else {
          double factor = err > 0.0 ? fmin(10.0, __dmul_rn(0.9, pow(err, -1.0 / 8.0))) : 10.0;
          if (err > 1.0) {
            ++C.rejected;
            C.after_reject = 1;
            C.h_next = __dmul_rn(h, fmax(0.2, factor));
          } else {
            C.accept = 1;
            ++C.accepted;
            const double t = C.t, boundary = t < 0.0 ? 0.0 : ctl_in.endpoint;
            C.t_new = h == boundary - t ? boundary : __dadd_rn(t, h);
            if (C.after_reject) factor = fmin(1.0, factor);
            C.h_next = __dmul_rn(h, factor);
            C.after_reject = 0;
            long long first = C.next_point, last = first;
            while (last < npoints && points[last] <= C.t_new) ++last;
            C.first = first;
            C.last = last;
            if (last > first) {
              C.dense = 1;
              ++C.dense_steps;
            }
          }
        }
      }
      __syncthreads();
      if (C.status) break;
    }

    if (C.accept) {
      if (C.dense) {
        // dense stages 13..15
        for (int s = 13; s < 16; ++s) {
          double2* z = zb(zcount);
          for (int e = tid; e < GE::OWN; e += GE::NT) {
            const size_t off = own_offset<DP>(e, row0);
            double2 v = ybuf[off];
            for (int j = 0; j < s; ++j) {
              const double a = c_dop_a[16 * s + j];
              if (a != 0.0) v = zaxpy(h * a, kb(j)[off], v);
            }
            z[off] = v;
          }
          fence_proxy_async_global();
          cluster_sync();
          rhs(z, kb(s), C.jac[s], C.src[s]);
          ++zcount;
        }
        // order-7 interpolation at the nodes in (t, t_new]
        const double t = C.t, tn = C.t_new;
        const long long first = C.first, last = C.last;
        for (int e = tid; e < GE::OWN; e += GE::NT) {
          const size_t off = own_offset<DP>(e, row0);
          const double2 yo = ybuf[off], yn = pbuf[off], f0 = kb(0)[off], f12 = kb(12)[off];
          double2 cf[7];
          const double2 delta = zsub(yn, yo);
          cf[0] = delta;
          cf[1] = zsub(zscale(h, f0), delta);
          cf[2] = zsub(zscale(2.0, delta), zscale(h, zadd(f12, f0)));
#pragma unroll
          for (int row = 0; row < 4; ++row) {
            double2 v = make_double2(0.0, 0.0);
            for (int s = 0; s < 16; ++s) {
              const double dcoef = c_dop_d[16 * row + s];
              if (dcoef != 0.0) v = zaxpy(h * dcoef, kb(s)[off], v);
            }
            cf[3 + row] = v;
          }
          for (long long node = first; node < last; ++node) {
            double2* out = st->samples + (size_t)node * GE::VEC + off;
            if (points[node] == tn) {
              *out = yn;
            } else {
              const double x = (points[node] - t) / h;
              double2 acc = make_double2(0.0, 0.0);
#pragma unroll
              for (int i = 0; i < 7; ++i) acc = zscale(i % 2 == 0 ? x : 1.0 - x, zadd(acc, cf[6 - i]));
              *out = zadd(acc, yo);
            }
          }
        }
      }
      // commit: y <- proposed, f <- k12 (buffer swaps)
      double2* tmp = ybuf;
      ybuf = pbuf;
      pbuf = tmp;
      __syncthreads();
      if (tid == 0) {
        const int k0 = C.kslot[0];
        C.kslot[0] = C.kslot[12];
        C.kslot[12] = k0;
        C.y_sc = C.prop_sc;
        C.ksc[0] = C.ksc[12];
        C.t = C.t_new;
        C.next_point = C.last;
      }
    }
    __syncthreads();
    if (tid == 0) {
      C.h = C.h_next;
      if (C.t >= ctl_in.endpoint && C.next_point != npoints) C.status = kMissingSamples;
      if (C.t < ctl_in.endpoint && C.attempts >= max_steps) C.status = kMaxSteps;
      if (C.t >= ctl_in.endpoint) C.done = 1;
    }
    __syncthreads();
    if (C.status || C.done) break;
  }

  // wait (bounded) for any copies still in flight before the CTA's shared memory goes away
  __syncthreads();
  if (tid == 0 && C.wait_flag) {
    // a copy whose wait gave up may still be in flight: wait for each slot's last use, bounded
    for (long long g = gq - 1; g >= 0 && g >= gq - GE::NST; --g) {
      mbar_wait(&sm.full[g % GE::NST], (uint32_t)((g / GE::NST) & 1), nullptr);
    }
  }
  if (rank == 0 && tid == 0) {
    TrajStats* o = st->stats;
    o->status = C.status;
    o->attempts = C.attempts;
    o->accepted = C.accepted;
    o->rejected = C.rejected;
    o->dense_steps = C.dense_steps;
    o->next_point = C.next_point;
    o->t = C.t;
    o->h = C.h;
    o->min_h = C.min_h;
    o->max_h = C.max_h;
    o->last_error = C.err;
    o->value = C.y_sc;
  }
  // keep every CTA's shared memory alive until the others finished reading it
  cluster_sync();
}

template <int DP>
static cudaError_t launch_dp(const TrajState* d_states, int nstates, const double* d_points, int npoints,
                             const TrajControls& ctl, cudaStream_t stream) {
  using GE = Geo<DP>;
  auto kern = trajectory_kernel<DP>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GE::SMEM);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nstates * GE::G, 1, 1);
  cfg.blockDim = dim3(GE::NT, 1, 1);
  cfg.dynamicSmemBytes = GE::SMEM;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = GE::G;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  note_launch();
  return cudaLaunchKernelEx(&cfg, kern, d_states, d_points, npoints, ctl);
}

// Node weights of the pullback: wj[2i] = weight_i 2|t_i|, wj[2i+1] = weight_i source(t_i).
__global__ void node_weights_kernel(const double* points, const double* weights, int n, double* wj) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    wj[2 * i] = weights[i] * 2.0 * fabs(points[i]);
    wj[2 * i + 1] = weights[i] * source_value(points[i]);
  }
}

cudaError_t node_weights_launch(const double* d_points, const double* d_weights, int n, double* d_wj,
                                cudaStream_t stream) {
  note_launch();
  node_weights_kernel<<<(n + 255) / 256, 256, 0, stream>>>(d_points, d_weights, n, d_wj);
  return cudaGetLastError();
}

cudaError_t trajectory_set_tables() {
  cudaError_t e;
  if ((e = cudaMemcpyToSymbol(c_dop_a, rcmps_dop_a, sizeof(rcmps_dop_a))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_dop_b, rcmps_dop_b, sizeof(rcmps_dop_b))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_dop_c, rcmps_dop_c, sizeof(rcmps_dop_c))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_dop_e5, rcmps_dop_e5, sizeof(rcmps_dop_e5))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_dop_e3, rcmps_dop_e3, sizeof(rcmps_dop_e3))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_dop_d, rcmps_dop_d, sizeof(rcmps_dop_d))) != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_source, rcmps_source_table, sizeof(rcmps_source_table));
}

cudaError_t trajectory_launch(int dp, const TrajState* d_states, int nstates, const double* d_points,
                              int npoints, const TrajControls& ctl, cudaStream_t stream) {
  switch (dp) {
    case 16: return launch_dp<16>(d_states, nstates, d_points, npoints, ctl, stream);
    case 32: return launch_dp<32>(d_states, nstates, d_points, npoints, ctl, stream);
    case 48: return launch_dp<48>(d_states, nstates, d_points, npoints, ctl, stream);
    case 64: return launch_dp<64>(d_states, nstates, d_points, npoints, ctl, stream);
    case 96: return launch_dp<96>(d_states, nstates, d_points, npoints, ctl, stream);
    case 128: return launch_dp<128>(d_states, nstates, d_points, npoints, ctl, stream);
    default: return cudaErrorInvalidValue;
  }
}

size_t trajectory_smem_bytes(int dp) {
  switch (dp) {
    case 16: return Geo<16>::SMEM;
    case 32: return Geo<32>::SMEM;
    case 48: return Geo<48>::SMEM;
    case 64: return Geo<64>::SMEM;
    case 96: return Geo<96>::SMEM;
    case 128: return Geo<128>::SMEM;
    default: return 0;
  }
}

}  // namespace rcmps
