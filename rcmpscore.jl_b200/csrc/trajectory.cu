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
//     into a 4-stage shared-memory ring, A operands resident in shared memory; one producer warp
//     refills each ring slot once every MMA warp has released it (per-slot "full" and "empty"
//     mbarriers), so the MMA warps never meet at a block barrier inside a product;
//   * the scalar energy channel is integrated from per-CTA partial traces reduced once per
//     attempt (its value never feeds back into the matrix channels);
//   * the step controller runs identically in every CTA from the same reduced norms.
// The channel structure comes from a table (SysTab) so that one kernel serves two systems:
//   * the reduced quartic system above (7 channels + scalar; ode_backend.py:170-233);
//   * the all-ODE route of kinetic1 + kinetic2 + g phi^4 (26 channels, ode_backend.py:76-167):
//     per channel jac (ql X + X ql^dag + rl X rl^dag) + src (c_l ol_a X_a + c_r X_b ol_b^dag),
//     where ol = R folds into the P products and ol = [Q, R] (the commutator spec) adds a
//     G1 product C X and a third K block [.. | src c_r X_b] * C^dag to G2.
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>
#include <cstdio>
#include <cstring>
#include "common.cuh"
#include "dop853_tables.h"
#include "split.cuh"
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

// Channel tables of the two systems (filled by trajectory_set_tables).
//   g1: the G1 products in order: channel and panel kind (0 [Q;R] rows, 1 [Q^dag;R^dag] rows,
//       2 C rows, 3 C^dag rows; kinds 2, 3 give L_c = ol X_c for the commutator spec);
//   p_*[gs]: the G2 passes for the one-channel (gs 0) and two-channel (gs 1) tilings, k3 when
//       the pass has the third K block (commutator spec);
//   lsrc/lcoef/lkind: the left insertion c_l ol_a X_a (P_a for ol = R, L_a for the commutator);
//   rsrc/rcoef: the right insertion c_r X_b ol_b^dag; fixed: 1 fixed0, 2 fixed6;
//   init: initial value 0, rho (1) or the identity on the physical block (2);
//   grp_*[k]: the channel groups when a state's rows are also split by channel over 2^k CTAs
//       (contiguous channel ranges; a G2 pass never straddles two groups), grp_remote[k] when a
//       left insertion reads P_a of a channel in another group (the CTAs then meet at a cluster
//       barrier between the G1 products and the G2 epilogues).
constexpr int kSysQuartic = 0, kSysFull = 1, kSysPhi1 = 2;
constexpr int kMaxChannels = 26;
constexpr int kGroupLevels = 3;   // 1, 2 or 4 channel groups
struct SysTab {
  int nch, ng1;
  int g1_ch[32], g1_kind[32];
  int np[2];
  int p_first[2][32], p_count[2][32], p_k3[2][32];
  int dir[kMaxChannels], lsrc[kMaxChannels], lkind[kMaxChannels], rsrc[kMaxChannels];
  int fixed[kMaxChannels], init[kMaxChannels];
  double lcoef[kMaxChannels], rcoef[kMaxChannels];
  int grp_levels;                               // group levels available (1: whole-state CTAs only)
  int grp_first[kGroupLevels][4], grp_count[kGroupLevels][4], grp_remote[kGroupLevels];
};
__constant__ SysTab c_sys[3];

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

// Bytes after the engine's buffers: ring barriers, the controller's scalars, the exchange record,
// reduction scratch and the gathered exchange records of up to 16 CTAs.
constexpr size_t kTail = 4096;

template <int DP, int SYS>
struct Geo {
  static constexpr int NCH = SYS == kSysQuartic ? 7 : SYS == kSysFull ? 26 : 4;   // matrix channels
  static constexpr bool SCALAR = SYS == kSysQuartic;       // the quartic system's scalar channel
  static constexpr int KM = SYS == kSysFull ? 3 : 2;       // K blocks of the widest G2 pass
  static constexpr int G = DP / 16;
  static constexpr int NW = (DP == 48 || DP == 96) ? 12 : (DP == 64 || DP == 128) ? 16 : 8;
  static constexpr int NWT = NW + 1;                  // + one producer warp that only streams B chunks
  static constexpr int NT = 32 * NWT;
  static constexpr int KC = DP <= 64 ? 16 : 8;       // rows of a streamed B chunk
  static constexpr int NST = (SYS == kSysFull && DP == 128) ? 3 : 4;   // ring stages
  static constexpr int LDB = DP + kBPad;              // padded row stride of a ring chunk
  static constexpr int LDP = DP + 4;                  // panel leading dimension (complex)
  static constexpr int LDA2 = KM * DP + 4;            // A' leading dimension
  static constexpr int GS = DP <= 64 ? 2 : 1;         // channels per G2 pass
  using T1 = PassTiling<DP, 32, NW>;
  using T2a = PassTiling<DP, 16 * GS, NW>;
  using T2b = PassTiling<DP, 16, NW>;
  static constexpr int CH1 = DP / KC;                 // chunks per G1 product; a G2 pass has 2 or 3 CH1
  static constexpr int MAT = DP * DP;                 // elements of one channel matrix
  static constexpr int VEC = NCH * MAT;               // elements of one stage vector
  static constexpr int OWN = NCH * 16 * DP;           // elements owned by one CTA
  static constexpr int cmax(int a, int b) { return a > b ? a : b; }
  // shared memory (double2 units): the direction panels, the A' rows of a pass, the ring, split-K.
  // The quartic system keeps both directions' panels ([Q; R] and [Q^dag; R^dag] rows, constant
  // over the trajectory) resident when they fit; otherwise one panel is reloaded per direction.
  static constexpr int PANEL = 32 * LDP;
  static constexpr int SPLIT_MAX = cmax(T1::SPLIT, cmax(T2a::SPLIT, T2b::SPLIT));
  static constexpr size_t smem_with(int panels) {
    return ((size_t)panels * PANEL + 16 * GS * LDA2 + NST * KC * LDB + SPLIT_MAX) * 16 + kTail;
  }
  static constexpr int NPANEL = (SYS == kSysQuartic && smem_with(2) <= 232448) ? 2 : 1;
  static constexpr int OFF_PANEL = 0;
  static constexpr int OFF_APRIME = OFF_PANEL + NPANEL * PANEL;
  static constexpr int OFF_RING = OFF_APRIME + 16 * GS * LDA2;
  static constexpr int OFF_SPLIT = OFF_RING + NST * KC * LDB;
  static constexpr int END2 = OFF_SPLIT + SPLIT_MAX;
  static constexpr size_t SMEM = (size_t)END2 * 16 + kTail;   // + barriers and scalars (see carve)
  static_assert(SMEM <= 232448, "shared memory per CTA");
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

template <int DP, int SYS>
struct Smem {
  double2* panel;     // [NPANEL][32][LDP]: the direction panels ([Qc; Rc] rows)
  double2* aprime;    // [16 GS][LDA2]
  double2* ring;      // [NST][KC*LDB]
  double2* split;     // split-K partial fragments
  uint64_t* full;     // [NST] chunk landed in the slot
  uint64_t* empty;    // [NST] every MMA warp released the slot
  Ctl* ctl;
  Xch* xch;
  double* red;        // [NW * 2] block reduction scratch
  double* kscp;       // [16] this CTA's partial scalar k by stage
  double* gat;        // [16][16] the exchange records of the cluster's CTAs, gathered
};

template <int DP, int SYS>
__device__ __forceinline__ Smem<DP, SYS> carve(unsigned char* base) {
  using GE = Geo<DP, SYS>;
  Smem<DP, SYS> s;
  double2* z = reinterpret_cast<double2*>(base);
  s.panel = z + GE::OFF_PANEL;
  s.aprime = z + GE::OFF_APRIME;
  s.ring = z + GE::OFF_RING;
  s.split = z + GE::OFF_SPLIT;
  // tail: full[NST] at 0, empty[NST] at 64, then the controller scalars
  static_assert(GE::NST <= 8, "barrier slots");
  constexpr size_t o_ctl = 128;
  constexpr size_t o_xch = o_ctl + ((sizeof(Ctl) + 15) / 16) * 16;
  constexpr size_t o_red = o_xch + ((sizeof(Xch) + 15) / 16) * 16;
  constexpr size_t o_ksc = o_red + 32 * sizeof(double) * 2;
  constexpr size_t o_gat = o_ksc + 16 * sizeof(double);
  static_assert(o_gat + 256 * sizeof(double) <= kTail, "shared tail");
  unsigned char* tail = base + (size_t)GE::END2 * 16;
  s.full = reinterpret_cast<uint64_t*>(tail);
  s.empty = reinterpret_cast<uint64_t*>(tail + 64);
  s.ctl = reinterpret_cast<Ctl*>(tail + o_ctl);
  s.xch = reinterpret_cast<Xch*>(tail + o_xch);
  s.red = reinterpret_cast<double*>(tail + o_red);
  s.kscp = reinterpret_cast<double*>(tail + o_ksc);
  s.gat = reinterpret_cast<double*>(tail + o_gat);
  return s;
}

// Block-wide sum of two doubles; the result is returned to every thread.
template <int NW>
__device__ void block_sum2(double& a, double& b, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  __syncthreads();
  if (lane == 0) { red[2 * w] = a; red[2 * w + 1] = b; }
  __syncthreads();
  double x = 0.0, y = 0.0;
  for (int i = 0; i < NW; ++i) { x += red[2 * i]; y += red[2 * i + 1]; }
  a = x;
  b = y;
}

// NST: stages of the operand ring (a compile-time depth keeps the slot arithmetic of every wait
// and release a shift and a mask; the tile autotuner picks among the compiled depths).
template <int DP, int SYS, int NST>
struct Rhs {
  using GE = Geo<DP, SYS>;
  static_assert(NST >= 2 && NST <= GE::NST, "ring depth");
  const TrajState* st;
  Smem<DP, SYS> sm;
  int row0, tid, lane, warp;
  long long* gq;   // running chunk counter (uniform across the CTA)
  int nchunk;      // chunks of one right-hand side (uniform)
  int ce, cc;      // producer cursor (thread 0): entry (G1 products, then G2 passes), chunk in it
  static constexpr int nst = NST;   // ring stages in use
  // Packed Z2 state with d = DP and d/2 a multiple of 16 (zs): each CTA's 16 rows lie in one
  // parity half hh of the two halves of hz rows; the structurally zero output tiles and K
  // halves of every product are skipped.
  int zs, hz, hh;
  // The CTA's channels [c0, c1) (all of them unless the state's rows are split by channel too)
  // and whether a left insertion reads P of a channel another CTA computes (remote).
  int c0, c1, remote;

  __device__ static const SysTab& T() { return c_sys[SYS]; }
  __device__ static int gsi() { return GE::GS == 2 ? 1 : 0; }

  // Chunks of entry e: a G1 product (CH1) or a G2 pass (2 or 3 CH1).
  __device__ static int entry_chunks(int e) {
    const SysTab& t = T();
    if (e < t.ng1) return GE::CH1;
    return (t.p_k3[gsi()][e - t.ng1] ? 3 : 2) * GE::CH1;
  }
  __device__ static int entries() { return T().ng1 + T().np[gsi()]; }
  // Entry e (a G1 product or a G2 pass) belongs to this CTA's channels.
  __device__ bool mine(int e) const {
    const SysTab& t = T();
    const int c = e < t.ng1 ? t.g1_ch[e] : t.p_first[gsi()][e - t.ng1];
    return c >= c0 && c < c1;
  }
  __device__ int next_mine(int e) const {
    while (e < entries() && !mine(e)) ++e;
    return e;
  }
  __device__ int total_chunks() const {
    int n = 0;
    for (int e = 0; e < entries(); ++e)
      if (mine(e)) n += entry_chunks(e);
    return n;
  }

  // Source of the cursor's chunk on stage vector zb.
  __device__ const double2* cursor_src(const double2* zb) const {
    const SysTab& t = T();
    const int r = cc * GE::KC;
    if (ce < t.ng1) return zb + (size_t)t.g1_ch[ce] * GE::MAT + (size_t)r * DP;
    const int first = t.p_first[gsi()][ce - t.ng1];
    const bool fwd = t.dir[first] == 0;
    const int blk = r / DP, rr = r % DP;
    // G2 B operand [Qc^dag; Rc^dag; Oc^dag]: forward (Q^dag, R^dag, C^dag), adjoint (Q, R, C)
    const double2* m = blk == 0 ? (fwd ? st->Qh : st->Q) : blk == 1 ? (fwd ? st->Rh : st->R) : (fwd ? st->Ch : st->C);
    return m + (size_t)rr * DP;
  }

  __device__ void issue(long long gidx, const double2* zb) {
    const int slot = (int)(gidx % nst);
    mbar_expect_tx(&sm.full[slot], GE::KC * DP * 16);
    const double2* src = cursor_src(zb);
    double2* dst = sm.ring + slot * GE::KC * GE::LDB;
#pragma unroll
    for (int r = 0; r < GE::KC; ++r) bulk_g2s(dst + r * GE::LDB, src + r * DP, DP * 16, &sm.full[slot]);
    if (++cc == entry_chunks(ce)) {
      cc = 0;
      ce = next_mine(ce + 1);
    }
  }

  // Wait for chunk (global index gidx); bounded.
  __device__ const double2* await(long long gidx) {
    const int slot = (int)(gidx % nst);
    const uint32_t parity = (uint32_t)((gidx / nst) & 1);
    if (!mbar_wait(&sm.full[slot], parity, &sm.ctl->wait_flag)) {}
    return sm.ring + slot * GE::KC * GE::LDB;
  }

  // The CTA's rows of the G1 A operand: kind 0 [Q; R], 1 [Q^dag; R^dag] (32 rows), 2 C, 3 C^dag (16).
  __device__ void load_panel(int kind, double2* dst) const {
    const int rows = kind < 2 ? 32 : 16;
    for (int e = tid; e < rows * DP; e += GE::NT) {
      const int r = e / DP, col = e % DP;
      const double2* srcm = kind == 0 ? (r < 16 ? st->Q : st->R)
                            : kind == 1 ? (r < 16 ? st->Qh : st->Rh)
                            : kind == 2 ? st->C : st->Ch;
      dst[r * GE::LDP + col] = srcm[(row0 + (r & 15)) * DP + col];
    }
  }

  // Split-K reduction; warps with slice > 0 deposit, slice 0 adds.
  template <int TPW, int SK>
  __device__ void split_reduce(ZFrag* acc, int tile0, int slice) {
    if constexpr (SK > 1) {
      if (slice > 0 && warp < GE::NW) {
#pragma unroll
        for (int j = 0; j < TPW; ++j) {
          double2* p = sm.split + ((tile0 + j) * (SK - 1) + slice - 1) * 128;
#pragma unroll
          for (int i = 0; i < 4; ++i) p[i * 32 + lane] = acc[j].value(i);
        }
      }
      __syncthreads();
      if (slice == 0 && warp < GE::NW) {
#pragma unroll
        for (int j = 0; j < TPW; ++j)
          for (int sl = 1; sl < SK; ++sl) {
            const double2* p = sm.split + ((tile0 + j) * (SK - 1) + sl - 1) * 128;
#pragma unroll
            for (int i = 0; i < 4; ++i) acc[j].add(i, p[i * 32 + lane]);
          }
      }
      __syncthreads();
    }
  }

  // acc += A (M rows in shared memory, lda) * the next nch streamed chunks. Ends with the chunks'
  // slots released and the next chunks issued.
  // ztile: the warp's tiles are structurally zero (no math); kn0/kn1 >= 0: only K rows of that
  // half of the first / second K block contribute (packed Z2 states), -1: all.
  template <class TL>
  __device__ void stream_product(ZFrag* acc, const double2* A, int lda, int nch, int& q, long long g0,
                                 const double2* zb, bool ztile, int kn0, int kn1) {
    constexpr int TPW = TL::TPW, SK = TL::SK;
    const int tile0 = SK > 1 ? warp / SK : warp * TPW;
    const int slice = SK > 1 ? warp % SK : 0;
    const int mt = tile0 / TL::NTN;
    if (warp == GE::NW) {
      // producer warp: refill each slot once every MMA warp has released it
      if (lane == 0)
        for (int ch = 0; ch < nch; ++ch) {
          const long long g = g0 + q + ch;
          if (q + ch + nst < nchunk) {
            mbar_wait(&sm.empty[(int)(g % nst)], (uint32_t)((g / nst) & 1), &sm.ctl->wait_flag);
            issue(g + nst, zb);
          }
        }
      __syncwarp();
      q += nch;
      split_reduce<TPW, SK>(acc, tile0, slice);
      return;
    }
    for (int ch = 0; ch < nch; ++ch, ++q) {
      const double2* B = await(g0 + q);   // every warp waits, so a slot is refilled only once it landed
      bool live = !ztile;
      if (live && kn0 >= 0) {
        const int kr = ch * GE::KC;        // a chunk lies in one half: hz is a multiple of KC
        live = ((kr % DP) >= hz ? 1 : 0) == (kr < DP ? kn0 : kn1);
      }
      if (live) {
#pragma unroll
        for (int ks = 0; ks < GE::KC / 8; ++ks) {
          const int kstep = ch * (GE::KC / 8) + ks;
          if (kstep % SK != slice) continue;
          AFrag a;
          load_a(A, lda, mt * 16, kstep * 8, lane, a);
          BFrag b[TPW];
#pragma unroll
          for (int j = 0; j < TPW; ++j) load_b(B, GE::LDB, ks * 8, ((tile0 + j) % TL::NTN) * 8, lane, b[j]);
          zmma_tiles<TPW>(acc, a, b);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.empty[(int)((g0 + q) % nst)]);
    }
    split_reduce<TPW, SK>(acc, tile0, slice);
  }

  // G1 product of channel c with a panel of 32 rows ([Qc; Rc]: Qc X_c -> kout scaled by jac,
  // P_c = Rc X_c) or 16 rows (L_c = Oc X_c).
  template <int M>
  __device__ void g1_product(int c, const double2* panel, const double2* zb, double2* kout, double jac, int& q,
                             long long g0) {
    using TL = PassTiling<DP, M, GE::NW>;
    constexpr int TPW = TL::TPW, SK = TL::SK;
    const int tile0 = SK > 1 ? warp / SK : warp * TPW;
    const int slice = SK > 1 ? warp % SK : 0;
    const int mt = tile0 / TL::NTN;     // M = 32: 0 Qc rows, 1 Rc rows
    static_assert(DP % 32 != 0 || (DP / 16) % TPW == 0, "a warp's tiles lie in one column half");
    // packed Z2: Q X_c on rows of half hh lives in column half hh ^ p (p = 1 for odd channels)
    // and takes K rows of half hh; R X_c lives in (1 - hh) ^ p and takes K rows of 1 - hh
    bool zt = false;
    int kn0 = -1;
    if (zs && M == 32) {
      const int p = (c % 2 == 0) ? 1 : 0;
      const int colh = ((tile0 % TL::NTN) * 8) >= hz ? 1 : 0;
      zt = colh != (mt == 0 ? (hh ^ p) : ((1 - hh) ^ p));
      kn0 = mt == 0 ? hh : 1 - hh;
    }
    ZFrag acc[TPW];
#pragma unroll
    for (int j = 0; j < TPW; ++j) acc[j].zero();
    stream_product<TL>(acc, panel, GE::LDP, GE::CH1, q, g0, zb, zt, kn0, -1);
    if (slice == 0 && warp < GE::NW) {
#pragma unroll
      for (int j = 0; j < TPW; ++j) {
        const int nt = (tile0 + j) % TL::NTN;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r = frag_row(lane, i), col = nt * 8 + frag_col(lane, i);
          const size_t off = (size_t)c * GE::MAT + (size_t)(row0 + r) * DP + col;
          const double2 v = acc[j].value(i);
          if (M == 16) st->L[off] = v;
          else if (mt == 0) kout[off] = zscale(jac, v);
          else st->P[off] = v;
        }
      }
    }
  }

  // G2 pass over the channels first..first+NC-1 (same direction and spec). K3: the pass has the
  // third K block of the commutator spec.
  // wait: meet the other CTAs' G1 results here (the cluster barrier's wait half, after this
  // pass's products and before its epilogue reads P of another CTA's channel).
  template <int NC, bool K3>
  __device__ void g2_pass(int first, const double2* zb, double2* kout, double jac, double src, int& q,
                          long long g0, bool wait) {
    using TL = PassTiling<DP, 16 * NC, GE::NW>;
    constexpr int TPW = TL::TPW, SK = TL::SK;
    const SysTab& t = T();
    // A' = [jac X_c | jac P_c (+ src c_r X_b for ol = R) (| src c_r X_b for the commutator)]
    for (int e = tid; e < 16 * NC * DP; e += GE::NT) {
      const int r = e / DP, col = e % DP;
      const int c = first + r / 16;
      const int b = t.rsrc[c];
      const size_t off = (size_t)(row0 + (r & 15)) * DP + col;
      // packed Z2: X_c (row half hh) lives in column half hh ^ p, P_c and X_b in (1 - hh) ^ p;
      // the products read only those parts of A'
      bool need0 = true, need1 = true;
      if (!K3 && zs) {
        const int p = (c % 2 == 0) ? 1 : 0, colh = col >= hz ? 1 : 0;
        need0 = colh == (hh ^ p);
        need1 = !need0;
      }
      if (need0) sm.aprime[r * GE::LDA2 + col] = zscale(jac, __ldcg(zb + (size_t)c * GE::MAT + off));
      if (need1) {
        double2 m = zscale(jac, __ldcg(st->P + (size_t)c * GE::MAT + off));
        double2 ins = make_double2(0.0, 0.0);
        if (b >= 0) ins = zscale(src * t.rcoef[c], __ldcg(zb + (size_t)b * GE::MAT + off));
        if constexpr (K3) {
          sm.aprime[r * GE::LDA2 + DP + col] = m;
          sm.aprime[r * GE::LDA2 + 2 * DP + col] = ins;
        } else {
          sm.aprime[r * GE::LDA2 + DP + col] = zadd(m, ins);
        }
      }
    }
    __syncthreads();
    ZFrag acc[TPW];
#pragma unroll
    for (int j = 0; j < TPW; ++j) acc[j].zero();
    const int tile0 = SK > 1 ? warp / SK : warp * TPW;
    const int slice = SK > 1 ? warp % SK : 0;
    static_assert(DP % 32 != 0 || (DP / 16) % TPW == 0, "a warp's tiles lie in one column half");
    // packed Z2: channel c' of the warp's band (rows of half hh) lives in column half hh ^ p
    bool zt = false;
    int kn0 = -1, kn1 = -1;
    if (!K3 && zs) {
      const int cb = first + tile0 / TL::NTN;
      const int p = (cb % 2 == 0) ? 1 : 0;
      zt = (((tile0 % TL::NTN) * 8) >= hz ? 1 : 0) != (hh ^ p);
      kn0 = hh ^ p;
      kn1 = (1 - hh) ^ p;
    }
    stream_product<TL>(acc, sm.aprime, GE::LDA2, (K3 ? 3 : 2) * GE::CH1, q, g0, zb, zt, kn0, kn1);
    if (wait) cluster_wait_acquire();
    if (slice == 0 && warp < GE::NW) {
#pragma unroll
      for (int j = 0; j < TPW; ++j) {
        const int tile = tile0 + j, mt = tile / TL::NTN, nt = tile % TL::NTN;
        // a tile's rows lie in one channel: its insertion source and fixed term are uniform
        const int c = first + mt;
        const int a = t.lsrc[c], fx = t.fixed[c];
        if (zt) {   // structurally zero: every term of the sum is an exact zero
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int r = mt * 16 + frag_row(lane, i), col = nt * 8 + frag_col(lane, i);
            kout[(size_t)c * GE::MAT + (size_t)(row0 + (r & 15)) * DP + col] = make_double2(0.0, 0.0);
          }
          continue;
        }
        // every operand of the tile's four elements is loaded before the first store, so their
        // L2 round trips overlap (a store to kout between them would order each element's loads
        // after the previous element's store)
        const double2* ins = (t.lkind[c] ? st->L : st->P) + (size_t)(a >= 0 ? a : 0) * GE::MAT;
        const double2* fxp = fx == 2 ? st->fixed6 : st->fixed0;
        size_t loc[4];
        double2 kv[4], iv[4], fv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r = mt * 16 + frag_row(lane, i), col = nt * 8 + frag_col(lane, i);
          loc[i] = (size_t)(row0 + (r & 15)) * DP + col;
          kv[i] = __ldcg(kout + (size_t)c * GE::MAT + loc[i]);
          iv[i] = a >= 0 ? __ldcg(ins + loc[i]) : make_double2(0.0, 0.0);
          fv[i] = fx ? __ldg(fxp + loc[i]) : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          double2 v = zadd(acc[j].value(i), kv[i]);
          if (a >= 0) v = zaxpy(src * t.lcoef[c], iv[i], v);
          if (fx) v = zaxpy(src, fv[i], v);
          kout[(size_t)c * GE::MAT + loc[i]] = v;
        }
      }
    }
    __syncthreads();
  }

  // One right-hand side: k_out = f(t, z) on this CTA's rows. zb: the full stage vector
  // (written by every CTA of the cluster before the barrier that precedes this call).
  __device__ void operator()(const double2* zb, double2* kout, double jac, double src) {
    const SysTab& t = T();
    const long long g0 = *gq;
    if (tid == GE::NW * 32) {
      fence_proxy_async_global();
      ce = next_mine(0);
      cc = 0;
      for (int q = 0; q < nst && q < nchunk; ++q) issue(g0 + q, zb);
    }
    int q = 0;
    // ------------------------------------------------------------------ G1 products
    int kind_prev = -1;
    for (int e = 0; e < t.ng1; ++e) {
      const int c = t.g1_ch[e], kind = t.g1_kind[e];
      if (c < c0 || c >= c1) continue;
      const double2* panel = sm.panel;
      if constexpr (GE::NPANEL == 2) {
        panel += kind * GE::PANEL;   // both resident (loaded once per trajectory)
      } else if (kind != kind_prev) {
        __syncthreads();
        load_panel(kind, sm.panel);
        __syncthreads();
        kind_prev = kind;
      }
      if (kind < 2) g1_product<32>(c, panel, zb, kout, jac, q, g0);
      else if constexpr (GE::KM == 3) g1_product<16>(c, panel, zb, kout, jac, q, g0);
    }
    __syncthreads();
    // the G1 results (P) of every CTA are published here and awaited in the first G2 pass
    if (remote) cluster_arrive_release();
    bool wait = remote != 0;
    // ------------------------------------------------------------------ G2 passes
    const int gs = gsi();
    for (int p = 0; p < t.np[gs]; ++p) {
      const int first = t.p_first[gs][p];
      if (first < c0 || first >= c1) continue;
      const bool two = GE::GS == 2 && t.p_count[gs][p] == 2;
      if constexpr (GE::KM == 3) {
        if (t.p_k3[gs][p]) {
          if constexpr (GE::GS == 2) {
            if (two) g2_pass<2, true>(first, zb, kout, jac, src, q, g0, wait);
            else g2_pass<1, true>(first, zb, kout, jac, src, q, g0, wait);
          } else {
            g2_pass<1, true>(first, zb, kout, jac, src, q, g0, wait);
          }
          wait = false;
          continue;
        }
      }
      if constexpr (GE::GS == 2) {
        if (two) g2_pass<2, false>(first, zb, kout, jac, src, q, g0, wait);
        else g2_pass<1, false>(first, zb, kout, jac, src, q, g0, wait);
      } else {
        g2_pass<1, false>(first, zb, kout, jac, src, q, g0, wait);
      }
      wait = false;
    }
    if (wait) cluster_wait_acquire();   // (every group has a G2 pass; kept for a uniform barrier count)
    *gq = g0 + nchunk;
    __syncthreads();
  }
};

#include "trajectory_split.cuh"

// Element e of this CTA's rows -> offset in a stage vector.
template <int DP>
__device__ __forceinline__ size_t own_offset(int e, int row0) {
  const int c = e / (16 * DP), rem = e % (16 * DP);
  return (size_t)c * DP * DP + (size_t)(row0 + rem / DP) * DP + (rem % DP);
}

// Structurally zero element e of a packed Z2 state's own rows (row0: the CTA's first row; half:
// d/2): channel parity p (1 for c even), nonzero iff the row and column halves differ by p.
template <int DP>
__device__ __forceinline__ bool z2_zero_element(int e, int row0, int half) {
  const int c = e / (16 * DP), row = row0 + (e % (16 * DP)) / DP, col = e % DP;
  return (((row >= half) != (col >= half)) ? 1 : 0) != ((c % 2 == 0) ? 1 : 0);
}

// Shared memory of the kernel: the FP64 engine's panels and ring (Geo::SMEM), or the split
// engine's chunk buffers followed by the controller's tail (kTail bytes).
template <int DP, int SYS, int ENG>
constexpr size_t kernel_smem() {
  return ENG == 0 ? Geo<DP, SYS>::SMEM : ((split_engine::kEnd + 127) / 128) * 128 + kTail;
}

template <int DP, int SYS, int ENG>
__device__ __forceinline__ Smem<DP, SYS> carve_engine(unsigned char* base) {
  if constexpr (ENG == 0) {
    return carve<DP, SYS>(base);
  } else {
    // the controller's scalars after the split engine's region, at the offsets carve uses
    constexpr size_t tail = ((split_engine::kEnd + 127) / 128) * 128;
    Smem<DP, SYS> s = carve<DP, SYS>(base + tail - (size_t)Geo<DP, SYS>::END2 * 16);
    s.panel = s.aprime = s.ring = s.split = nullptr;
    return s;
  }
}

template <int DP, int SYS, int ENG, int NST = Geo<DP, SYS>::NST>
__global__ void __launch_bounds__(Geo<DP, SYS>::NT, 1)
trajectory_kernel(const TrajState* __restrict__ states, const double* __restrict__ points, int npoints,
                  TrajControls ctl_in) {
  using GE = Geo<DP, SYS>;
  static_assert(ENG == 0 || (SYS == kSysQuartic && DP == 64), "the split engine covers the quartic system at dp 64");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem<DP, SYS> sm = carve_engine<DP, SYS, ENG>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t rank = cluster_rank();
  const int sidx = (int)cluster_id_x();
  const TrajState* st = states + sidx;
  // cluster of G x CG CTAs: rows 16 (rank % G) .. + 15 of the channel group rank / G
  const uint32_t nrank = cluster_size();
  const int ngroups = (int)nrank / GE::G;
  const int glevel = ngroups == 4 ? 2 : ngroups == 2 ? 1 : 0;
  const int row0 = (int)(rank % GE::G) * 16;
  const int grp = (int)rank / GE::G;
  const int c0 = c_sys[SYS].grp_first[glevel][grp], c1 = c0 + c_sys[SYS].grp_count[glevel][grp];
  const int e0 = c0 * 16 * DP, e1 = c1 * 16 * DP;   // the CTA's elements (own_offset numbering)
  Ctl& C = *sm.ctl;
  long long gq = 0;
  if (SYS == kSysQuartic && st->z2 < 0) {
    // the packed Z2 route refused this state (no exact Z2 block structure): nothing is
    // integrated; every CTA of the cluster leaves here, before any cluster barrier
    if (rank == 0 && tid == 0) {
      TrajStats* o = st->stats;
      o->status = kInvalidInput;
      o->packed = 0;
      o->attempts = o->accepted = o->rejected = o->dense_steps = o->next_point = 0;
      o->t = o->h = o->min_h = o->max_h = o->last_error = o->value = 0.0;
    }
    return;
  }

  SplitSmem ssm{};
  if constexpr (ENG == 1) ssm = split_carve(smem_raw);
  if (tid == 0) {
    if constexpr (ENG == 0) {
      for (int i = 0; i < GE::NST; ++i) {
        mbar_init(&sm.full[i], 1);
        mbar_init(&sm.empty[i], GE::NW);
      }
    } else {
      split_barriers_init(ssm);
    }
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
  uint32_t tmem = 0;
  if constexpr (ENG == 1) {
    if (warp == 0) split::tmem_alloc(ssm.tslot, split_engine::kTmemCols);
    split::tc_fence_before();
    __syncthreads();
    split::tc_fence_after();
    tmem = *ssm.tslot;
  }
  __syncthreads();
  using RhsT = std::conditional_t<ENG == 0, Rhs<DP, SYS, NST>, RhsSplit<DP>>;
  RhsT rhs;
  if constexpr (ENG == 0) {
    rhs = Rhs<DP, SYS, NST>{st, sm, row0, tid, lane, warp, &gq, 0, 0, 0};
    rhs.c0 = c0;
    rhs.c1 = c1;
    rhs.remote = c_sys[SYS].grp_remote[glevel];
    rhs.nchunk = rhs.total_chunks();
  } else {
    rhs.st = st;
    rhs.ss = ssm;
    rhs.row0 = row0;
    rhs.rank = (int)rank;
    rhs.tid = tid;
    rhs.lane = lane;
    rhs.warp = warp;
    rhs.tmem = tmem;
    rhs.q = 0;
    rhs.u = 0;
    rhs.wait_flag = &C.wait_flag;
  }
  // The packed Z2 route counts, per channel, the upper off-diagonal block of an odd channel
  // (F1, F3, A2, A4: c even) and the two diagonal blocks of an even one, 10 (d/2)^2 entries plus
  // the scalar (persistent_trajectory_backend.py:68, 115); the structural zeros and the lower
  // blocks, the adjoints of the upper ones, stay out of the norm. When d = DP and d/2 is a
  // multiple of 16 the structural zeros are also skipped in the products and stage sums: they
  // stay exact zeros, written once below.
  const bool packed = SYS == kSysQuartic && st->z2 > 0;
  const int half = st->d / 2;
  const bool zskip = packed && st->d == DP && DP % 32 == 0;
  if constexpr (ENG == 0) {
    rhs.zs = zskip ? 1 : 0;
    rhs.hz = half;
    rhs.hh = zskip && row0 >= half ? 1 : 0;
  }
  if (zskip) {
    // every work vector's own rows start at zero: the skipped parts are never written again
    for (int e = e0 + tid; e < e1; e += GE::NT) {
      const size_t off = own_offset<DP>(e, row0);
      const double2 z0 = make_double2(0.0, 0.0);
      st->y[off] = z0;
      st->prop[off] = z0;
      st->P[off] = z0;
      for (int s = 0; s < 16; ++s) st->k[(size_t)s * GE::VEC + off] = z0;
      st->z[off] = z0;
      st->z[GE::VEC + off] = z0;
    }
  }

  // slot permutation: C.kslot[s] is the k buffer of stage s; y and proposed swap on acceptance
  if (tid < 16) C.kslot[tid] = tid;
  __syncthreads();
  double2* ybuf = st->y;
  double2* pbuf = st->prop;
  auto kb = [&](int s) { return st->k + (size_t)C.kslot[s] * GE::VEC; };
  long long zcount = 0;
  auto zb = [&](long long n) { return st->z + (size_t)(n & 1) * GE::VEC; };

  // initial y on own rows (zero, rho or the identity of the physical block), and f = RHS(-a, y)
  {
    const SysTab& tab = c_sys[SYS];
    for (int e = e0 + tid; e < e1; e += GE::NT) {
      const size_t off = own_offset<DP>(e, row0);
      const int c = e / (16 * DP), row = row0 + (e % (16 * DP)) / DP, col = e % DP;
      double2 v = make_double2(0.0, 0.0);
      if (tab.init[c] == 1) v = st->rho[row * DP + col];
      else if (tab.init[c] == 2 && row == col && row < st->d) v.x = 1.0;
      ybuf[off] = v;
      zb(zcount)[off] = v;
    }
  }
  if constexpr (ENG == 0 && GE::NPANEL == 2) {   // both direction panels, once per trajectory
    rhs.load_panel(0, sm.panel);
    rhs.load_panel(1, sm.panel + GE::PANEL);
  }
  fence_proxy_async_global();
  cluster_sync();
  rhs(zb(zcount), kb(0), C.jac[0], C.src[0]);
  ++zcount;

  const double N = packed ? 10.0 * half * half + 1.0
                          : (double)GE::NCH * st->d * st->d + (GE::SCALAR ? 1.0 : 0.0);
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
    }
    __syncthreads();
    // the stage times' Jacobian and source values, one stage per lane of warp 0
    if (tid >= 1 && tid < 16) {
      const int s = tid;
      const double t = C.t, h = C.h;
      const double ts = s == 12 ? __dadd_rn(t, h) : __dadd_rn(t, __dmul_rn(c_dop_c[s], h));
      if (fabs(ts) > RCMPS_SOURCE_AMAX * (1.0 + 1e-14)) C.status = kSourceDomain;
      C.jac[s] = 2.0 * fabs(ts);
      C.src[s] = source_value(ts);
    }
    __syncthreads();
    if (C.status) break;   // uniform across the cluster: every CTA computes the same
    const double h = C.h;

    // ---------------------------------------------------------------- stages 1..12
    for (int s = 1; s <= 12; ++s) {
      const double* w = s == 12 ? c_dop_b : c_dop_a + 16 * s;
      double2* z = zb(zcount);
      const int terms = s;   // a[s][0..s-1], b[0..11]
      double part = 0.0, dummy = 0.0;
      const double2* kp[12];
      double ha[12];
#pragma unroll
      for (int j = 0; j < 12; ++j) {
        kp[j] = kb(j);
        ha[j] = j < terms ? h * w[j] : 0.0;
      }
      for (int e = e0 + tid; e < e1; e += GE::NT) {
        if (zskip && z2_zero_element<DP>(e, row0, half)) continue;
        const size_t off = own_offset<DP>(e, row0);
        double2 kv[12];
#pragma unroll
        for (int j = 0; j < 12; ++j) kv[j] = ha[j] != 0.0 ? __ldcg(kp[j] + off) : make_double2(0.0, 0.0);
        double2 v = ybuf[off];
#pragma unroll
        for (int j = 0; j < 12; ++j) v = zaxpy(ha[j], kv[j], v);
        z[off] = v;
        if (s == 12) pbuf[off] = v;
        if constexpr (GE::SCALAR) {
          if (e / (16 * DP) == 2) {
            const double2 sv = st->S[off - 2 * (size_t)GE::MAT];
            part += v.x * sv.x - v.y * sv.y;
          }
        }
      }
      // the scalar channel's partial trace (channel 2's rows): only its CTAs reduce it
      if (GE::SCALAR && c0 <= 2 && 2 < c1) {
        block_sum2<GE::NWT>(part, dummy, sm.red);
        if (tid == 0) sm.kscp[s] = 4.0 * C.src[s] * part;
      }
      fence_proxy_async_global();
      cluster_sync();
      rhs(z, kb(s), C.jac[s], C.src[s]);
      ++zcount;
    }

    // ---------------------------------------------------------------- error norms
    {
      double s5 = 0.0, s3 = 0.0;
      const double2* ke_p[13];
#pragma unroll
      for (int j = 0; j < 13; ++j) ke_p[j] = kb(j);
      for (int e = e0 + tid; e < e1; e += GE::NT) {
        const size_t off = own_offset<DP>(e, row0);
        if (packed) {
          const int c = e / (16 * DP), row = row0 + (e % (16 * DP)) / DP, col = e % DP;
          const bool lo_r = row < half, lo_c = col < half;
          if ((c % 2 == 0) ? !(lo_r && !lo_c) : (lo_r != lo_c)) continue;
        }
        double2 kv[13];
#pragma unroll
        for (int j = 0; j <= 12; ++j) kv[j] = __ldcg(ke_p[j] + off);
        double2 e5 = make_double2(0.0, 0.0), e3 = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j <= 12; ++j) {
          e5 = zaxpy(c_dop_e5[j], kv[j], e5);
          e3 = zaxpy(c_dop_e3[j], kv[j], e3);
        }
        const double2 yo = ybuf[off], yn = pbuf[off];
        const double scale = atol + rtol * fmax(hypot(yo.x, yo.y), hypot(yn.x, yn.y));
        s5 += zabs2(e5) / (scale * scale);
        s3 += zabs2(e3) / (scale * scale);
      }
      block_sum2<GE::NWT>(s5, s3, sm.red);
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
      // every CTA's record, one distributed-shared-memory load per thread (a serial walk over 16
      // CTAs' records by one thread took tens of microseconds per attempt); summed below in rank
      // order as before
      for (int i = tid; i < (int)nrank * 16; i += GE::NT) {
        const uint32_t g = (uint32_t)(i >> 4);
        const int v = i & 15;
        double x = 0.0;
        if (v == 0) x = dsmem_load(&sm.xch->s5, g);
        else if (v == 1) x = dsmem_load(&sm.xch->s3, g);
        else if (v <= 13) x = dsmem_load(&sm.xch->kscp[v - 1], g);
        else if (v == 14) x = (double)dsmem_load_int(&sm.xch->flag, g);
        sm.gat[i] = x;
      }
      __syncthreads();
      if (tid == 0) {
        double t5 = 0.0, t3 = 0.0;
        double ks[13];
        for (int s = 1; s < 13; ++s) ks[s] = 0.0;
        int flag = 0;
        for (uint32_t g = 0; g < nrank; ++g) {
          const double* r = sm.gat + 16 * g;
          t5 += r[0];
          t3 += r[1];
          for (int s = 1; s < 13; ++s) ks[s] += r[s + 1];
          flag |= (int)r[14];
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
          const double2* kp[15];
          double ha[15];
#pragma unroll
          for (int j = 0; j < 15; ++j) {
            kp[j] = kb(j);
            ha[j] = j < s ? h * c_dop_a[16 * s + j] : 0.0;
          }
          for (int e = e0 + tid; e < e1; e += GE::NT) {
            const size_t off = own_offset<DP>(e, row0);
            double2 kv[15];
#pragma unroll
            for (int j = 0; j < 15; ++j) kv[j] = ha[j] != 0.0 ? __ldcg(kp[j] + off) : make_double2(0.0, 0.0);
            double2 v = ybuf[off];
#pragma unroll
            for (int j = 0; j < 15; ++j)
              if (ha[j] != 0.0) v = zaxpy(ha[j], kv[j], v);
            z[off] = v;
          }
          fence_proxy_async_global();
          cluster_sync();
          rhs(z, kb(s), C.jac[s], C.src[s]);
          ++zcount;
        }
        // order-7 interpolation at the nodes in (t, t_new]: every stage the dense matrix reads
        // (rcmps_dop_dense_mask, k0 and k12 among them) is loaded once per element, all at once
        const double t = C.t, tn = C.t_new;
        const long long first = C.first, last = C.last;
        const double2* kd_p[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) kd_p[j] = kb(j);
        for (int e = e0 + tid; e < e1; e += GE::NT) {
          const size_t off = own_offset<DP>(e, row0);
          double2 kd[16];
#pragma unroll
          for (int j = 0; j < 16; ++j)
            kd[j] = ((rcmps_dop_dense_mask >> j) & 1u) ? __ldcg(kd_p[j] + off) : make_double2(0.0, 0.0);
          const double2 yo = ybuf[off], yn = pbuf[off], f0 = kd[0], f12 = kd[12];
          double2 cf[7];
          const double2 delta = zsub(yn, yo);
          cf[0] = delta;
          cf[1] = zsub(zscale(h, f0), delta);
          cf[2] = zsub(zscale(2.0, delta), zscale(h, zadd(f12, f0)));
#pragma unroll
          for (int row = 0; row < 4; ++row) {
            double2 v = make_double2(0.0, 0.0);
#pragma unroll
            for (int j = 0; j < 16; ++j)
              if ((rcmps_dop_dense_mask >> j) & 1u) v = zaxpy(h * c_dop_d[16 * row + j], kd[j], v);
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
  if constexpr (ENG == 0) {
    if (tid == 0 && C.wait_flag) {
      // a copy whose wait gave up may still be in flight: wait for each slot's last use, bounded
      for (long long g = gq - 1; g >= 0 && g >= gq - rhs.nst; --g) {
        mbar_wait(&sm.full[g % rhs.nst], (uint32_t)((g / rhs.nst) & 1), nullptr);
      }
    }
  } else {
    // every unit's epilogue waited for its MMAs; after a wait that gave up, wait (bounded) once
    // more for the last unit's and the last copies' barriers, then release TMEM
    if (tid == 0 && C.wait_flag && rhs.u > 0) {
      using split_engine::kBufs;
      const long long uu = rhs.u - 1;
      mbar_wait(&ssm.acc[uu & 1], (uint32_t)((uu >> 1) & 1), nullptr);
      for (long long g = rhs.q - 1; g >= 0 && g >= rhs.q - kBufs; --g) {
        mbar_wait(&ssm.copy[g % kBufs], (uint32_t)((g / kBufs) & 1), nullptr);
        mbar_wait(&ssm.free[g % kBufs], (uint32_t)((g / kBufs) & 1), nullptr);
      }
    }
    split::tc_fence_before();
    __syncthreads();
    split::tc_fence_after();
    if (warp == 0) split::tmem_dealloc(tmem, split_engine::kTmemCols);
  }
  if (rank == 0 && tid == 0) {
    TrajStats* o = st->stats;
    o->status = C.status;
    o->packed = packed ? 1 : 0;
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

int trajectory_group_levels(int system);   // channel-group levels of a system's table (below)

// Launch configuration of `nstates` clusters of cluster_ctas CTAs each.
template <int DP, int SYS, int ENG>
static cudaLaunchConfig_t launch_config(int nstates, int cluster_ctas, cudaStream_t stream, cudaLaunchAttribute* attr) {
  using GE = Geo<DP, SYS>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nstates * cluster_ctas, 1, 1);
  cfg.blockDim = dim3(GE::NT, 1, 1);
  cfg.dynamicSmemBytes = kernel_smem<DP, SYS, ENG>();
  cfg.stream = stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster_ctas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

template <int DP, int SYS, int ENG, int NST = Geo<DP, SYS>::NST>
static cudaError_t prepare_kernel() {
  constexpr size_t smem = kernel_smem<DP, SYS, ENG>();
  static_assert(smem <= 232448, "shared memory per CTA");
  auto kern = trajectory_kernel<DP, SYS, ENG, NST>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

// Channel groups for nstates states (see trajectory_groups).
template <int DP, int SYS, int ENG>
static int choose_groups(int nstates, int requested) {
  using GE = Geo<DP, SYS>;
  static int levels = -1;
  if (levels < 0) levels = ENG == 0 ? trajectory_group_levels(SYS) : 1;
  auto allowed = [&](int cg) {
    const int level = cg == 4 ? 2 : cg == 2 ? 1 : 0;
    return (cg == 1 || cg == 2 || cg == 4) && level < levels && GE::G * cg <= 16;
  };
  // clusters of G x cg CTAs the device holds at once (0 when it cannot place one)
  auto resident = [&](int cg) {
    if (prepare_kernel<DP, SYS, ENG>() != cudaSuccess) return 0;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = launch_config<DP, SYS, ENG>(nstates, GE::G * cg, nullptr, attr);
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, trajectory_kernel<DP, SYS, ENG>, &cfg) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    return clusters;
  };
  if (requested > 0) {   // the largest supported count up to the request
    for (int cg = requested; cg > 1; cg /= 2)
      if (allowed(cg) && resident(cg) >= 1) return cg;
    return 1;
  }
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) return 1;
  for (int cg = 4; cg > 1; cg /= 2)
    if (allowed(cg) && (long long)nstates * GE::G * cg <= sms && resident(cg) >= nstates) return cg;
  return 1;
}

template <int DP, int SYS, int ENG, int NST>
static cudaError_t launch_kernel(const TrajState* d_states, int nstates, const double* d_points, int npoints,
                                 const TrajControls& ctl, cudaStream_t stream) {
  using GE = Geo<DP, SYS>;
  cudaError_t e = prepare_kernel<DP, SYS, ENG, NST>();
  if (e != cudaSuccess) return e;
  const int cg = choose_groups<DP, SYS, ENG>(nstates, ctl.groups);
  if (cg == 0) return cudaErrorInvalidValue;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = launch_config<DP, SYS, ENG>(nstates, GE::G * cg, stream, attr);
  note_launch();
  return cudaLaunchKernelEx(&cfg, trajectory_kernel<DP, SYS, ENG, NST>, d_states, d_points, npoints, ctl);
}

// The ring depth the launch asked for (ctl.ring 2 or 3; the quartic FP64 system compiles those),
// else the system's default depth.
template <int DP, int SYS, int ENG = 0>
static cudaError_t launch_dp(const TrajState* d_states, int nstates, const double* d_points, int npoints,
                             const TrajControls& ctl, cudaStream_t stream) {
  if constexpr (ENG == 0 && SYS == kSysQuartic) {
    if (ctl.ring == 2) return launch_kernel<DP, SYS, ENG, 2>(d_states, nstates, d_points, npoints, ctl, stream);
    if (ctl.ring == 3) return launch_kernel<DP, SYS, ENG, 3>(d_states, nstates, d_points, npoints, ctl, stream);
  }
  return launch_kernel<DP, SYS, ENG, Geo<DP, SYS>::NST>(d_states, nstates, d_points, npoints, ctl, stream);
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

// The channel tables of the systems (host side, copied to c_sys).
static void quartic_table(SysTab& t) {
  std::memset(&t, 0, sizeof(t));
  t.nch = 7;
  for (int c = 0; c < 7; ++c) {
    t.dir[c] = c < 3 ? 0 : 1;
    t.lsrc[c] = t.rsrc[c] = -1;
    t.g1_ch[c] = c;
    t.g1_kind[c] = t.dir[c];
  }
  t.ng1 = 7;
  // insertions c_s (R X_s + X_s R^dag) of ode_backend.py:193: 1<-0 (2), 2<-1 (3), 3<-4 (1), 4<-5 (2), 5<-6 (3)
  const int src[7] = {-1, 0, 1, 4, 5, 6, -1};
  const double coef[7] = {0, 2, 3, 1, 2, 3, 0};
  for (int c = 0; c < 7; ++c) {
    t.lsrc[c] = t.rsrc[c] = src[c];
    t.lcoef[c] = t.rcoef[c] = coef[c];
  }
  t.fixed[0] = 1;
  t.fixed[6] = 2;
  // G2 passes: one per channel, or the same-direction pairs {0,1}, {2}, {3,4}, {5,6}
  t.np[0] = 7;
  for (int c = 0; c < 7; ++c) { t.p_first[0][c] = c; t.p_count[0][c] = 1; }
  const int pf[4] = {0, 2, 3, 5}, pc[4] = {2, 1, 2, 2};
  t.np[1] = 4;
  for (int p = 0; p < 4; ++p) { t.p_first[1][p] = pf[p]; t.p_count[1][p] = pc[p]; }
}

struct SpecEdge { int a, b; bool left; double c; };
struct SpecDef { int nch; const SpecEdge* edges; int nedge; bool comm; };

// Table of forward and adjoint channels of a list of specs (ode_backend.py:76-167): forward
// channels from 0, adjoint channels from half = sum of the specs' channels.
static void spec_table(SysTab& t, const SpecDef* sp, int nsp) {
  std::memset(&t, 0, sizeof(t));
  int off[kMaxChannels], half = 0;
  for (int s = 0; s < nsp; ++s) {
    off[s] = half;
    half += sp[s].nch;
  }
  const int nch = 2 * half;
  t.nch = nch;
  for (int c = 0; c < nch; ++c) {
    t.dir[c] = c < half ? 0 : 1;
    t.lsrc[c] = t.rsrc[c] = -1;
  }
  bool is_comm[kMaxChannels] = {false}, lsource_comm[kMaxChannels] = {false};
  for (int s = 0; s < nsp; ++s) {
    for (int i = 0; i < sp[s].nch; ++i) is_comm[off[s] + i] = is_comm[half + off[s] + i] = sp[s].comm;
    t.init[off[s]] = 1;                              // rho in the first forward channel
    t.init[half + off[s] + sp[s].nch - 1] = 2;       // I in the last adjoint channel
    for (int q = 0; q < sp[s].nedge; ++q) {
      const SpecEdge& ed = sp[s].edges[q];
      const int fa = off[s] + ed.a, fb = off[s] + ed.b;
      const int aa = half + off[s] + ed.a, ab = half + off[s] + ed.b;
      if (ed.left) {
        t.lsrc[fb] = fa; t.lcoef[fb] = ed.c;       // forward b += c O X_a
        t.rsrc[aa] = ab; t.rcoef[aa] = ed.c;       // adjoint a += c X_b O
      } else {
        t.rsrc[fb] = fa; t.rcoef[fb] = ed.c;       // forward b += c X_a O^dag
        t.lsrc[aa] = ab; t.lcoef[aa] = ed.c;       // adjoint a += c O^dag X_b
      }
    }
  }
  for (int c = 0; c < nch; ++c)
    if (t.lsrc[c] >= 0 && is_comm[c]) {
      t.lkind[c] = 1;
      lsource_comm[t.lsrc[c]] = true;
    }
  // G1: forward [Q;R] products, forward C products, adjoint [Q^dag;R^dag], adjoint C^dag products
  int n = 0;
  for (int c = 0; c < half; ++c) { t.g1_ch[n] = c; t.g1_kind[n++] = 0; }
  for (int c = 0; c < half; ++c) if (lsource_comm[c]) { t.g1_ch[n] = c; t.g1_kind[n++] = 2; }
  for (int c = half; c < nch; ++c) { t.g1_ch[n] = c; t.g1_kind[n++] = 1; }
  for (int c = half; c < nch; ++c) if (lsource_comm[c]) { t.g1_ch[n] = c; t.g1_kind[n++] = 3; }
  t.ng1 = n;
  // G2 passes: one per channel, or pairs of consecutive channels of one spec
  t.np[0] = nch;
  for (int c = 0; c < nch; ++c) { t.p_first[0][c] = c; t.p_count[0][c] = 1; t.p_k3[0][c] = is_comm[c]; }
  int p = 0;
  for (int dir = 0; dir < 2; ++dir)
    for (int s = 0; s < nsp; ++s)
      for (int i = 0; i < sp[s].nch; i += 2) {
        const int c = dir * half + off[s] + i;
        t.p_first[1][p] = c;
        t.p_count[1][p] = i + 1 < sp[s].nch ? 2 : 1;
        t.p_k3[1][p] = sp[s].comm;
        ++p;
      }
  t.np[1] = p;
}

// Specs of the all-ODE route (ode_backend.py:60-73, 851-858): kinetic1 (4 channels, O = R),
// kinetic2 (4 channels, O = [Q, R]) and phi^4 (5 channels, O = R); forward channels 0..12,
// adjoint 13..25. A forward edge a -> b inserts forward a into forward b on its side; its trace
// dual inserts adjoint b into adjoint a on the other side (ode_backend.py:108-113).
static void full_table(SysTab& t) {
  const double r2 = 1.4142135623730951;
  const SpecEdge kin[4] = {{0, 1, true, r2}, {0, 2, false, r2}, {2, 3, true, r2}, {1, 3, false, r2}};
  SpecEdge quart[8];
  for (int k = 0; k < 4; ++k) {
    quart[2 * k] = {k, k + 1, true, (double)(k + 1)};
    quart[2 * k + 1] = {k, k + 1, false, (double)(k + 1)};
  }
  const SpecDef specs[3] = {{4, kin, 4, false}, {4, kin, 4, true}, {5, quart, 8, false}};
  spec_table(t, specs, 3);
}

// The first monomial phi_monomial(s, 1) of RcmpsCore (validate_sweep.py:23-32): F0 = rho and
// dF1 = 2|t| L(F1) dt + j(t) (R F0 + F0 R^dag) dt, with the two adjoint channels.
static void phi1_table(SysTab& t) {
  const SpecEdge phi[2] = {{0, 1, true, 1.0}, {0, 1, false, 1.0}};
  const SpecDef spec = {2, phi, 2, false};
  spec_table(t, &spec, 1);
}

// Channel groups of level k (2^k groups of contiguous channels: first[i], count[i]). The level is
// kept only when every G2 pass of both tilings lies inside one group; grp_remote[k] records a left
// insertion whose source channel lies in another group.
static bool set_groups(SysTab& t, int k, const int* first, const int* count) {
  const int ng = 1 << k;
  int owner[kMaxChannels];
  for (int c = 0; c < t.nch; ++c) owner[c] = -1;
  for (int g = 0, c = 0; g < ng; ++g) {
    if (first[g] != c || count[g] < 1) return false;
    for (int i = 0; i < count[g]; ++i) owner[c++] = g;
    if (g == ng - 1 && c != t.nch) return false;
  }
  for (int gs = 0; gs < 2; ++gs)
    for (int p = 0; p < t.np[gs]; ++p)
      if (owner[t.p_first[gs][p]] != owner[t.p_first[gs][p] + t.p_count[gs][p] - 1]) return false;
  int remote = 0;
  for (int c = 0; c < t.nch; ++c)
    if (t.lsrc[c] >= 0 && owner[t.lsrc[c]] != owner[c]) remote = 1;
  for (int g = 0; g < 4; ++g) {
    t.grp_first[k][g] = g < ng ? first[g] : 0;
    t.grp_count[k][g] = g < ng ? count[g] : 0;
  }
  t.grp_remote[k] = remote;
  return true;
}

static void whole_state_groups(SysTab& t) {
  const int first[1] = {0}, count[1] = {t.nch};
  set_groups(t, 0, first, count);
  t.grp_levels = 1;
}

// The quartic system by direction ({0,1,2} forward, {3..6} adjoint: no insertion crosses) and in
// four groups along the G2 pairs ({0,1}, {2}, {3,4}, {5,6}: the insertions 2 <- 1 and 4 <- 5 cross).
static void quartic_groups(SysTab& t) {
  whole_state_groups(t);
  const int f2[2] = {0, 3}, n2[2] = {3, 4};
  const int f4[4] = {0, 2, 3, 5}, n4[4] = {2, 1, 2, 2};
  if (set_groups(t, 1, f2, n2)) {
    t.grp_levels = 2;
    if (set_groups(t, 2, f4, n4)) t.grp_levels = 3;
  }
}

int trajectory_group_levels(int system) {
  SysTab t;
  if (system == kSysQuartic) {
    quartic_table(t);
    quartic_groups(t);
    return t.grp_levels;
  }
  return 1;
}

cudaError_t trajectory_set_tables() {
  cudaError_t e;
  if ((e = cudaMemcpyToSymbol(c_dop_a, rcmps_dop_a, sizeof(rcmps_dop_a))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_dop_b, rcmps_dop_b, sizeof(rcmps_dop_b))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_dop_c, rcmps_dop_c, sizeof(rcmps_dop_c))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_dop_e5, rcmps_dop_e5, sizeof(rcmps_dop_e5))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_dop_e3, rcmps_dop_e3, sizeof(rcmps_dop_e3))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_dop_d, rcmps_dop_d, sizeof(rcmps_dop_d))) != cudaSuccess) return e;
  SysTab tabs[3];
  quartic_table(tabs[0]);
  full_table(tabs[1]);
  phi1_table(tabs[2]);
  quartic_groups(tabs[0]);
  whole_state_groups(tabs[1]);
  whole_state_groups(tabs[2]);
  if ((e = cudaMemcpyToSymbol(c_sys, tabs, sizeof(tabs))) != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_source, rcmps_source_table, sizeof(rcmps_source_table));
}

template <int SYS>
static cudaError_t launch_sys(int dp, const TrajState* d_states, int nstates, const double* d_points,
                              int npoints, const TrajControls& ctl, cudaStream_t stream) {
  switch (dp) {
    case 16: return launch_dp<16, SYS>(d_states, nstates, d_points, npoints, ctl, stream);
    case 32: return launch_dp<32, SYS>(d_states, nstates, d_points, npoints, ctl, stream);
    case 48: return launch_dp<48, SYS>(d_states, nstates, d_points, npoints, ctl, stream);
    case 64: return launch_dp<64, SYS>(d_states, nstates, d_points, npoints, ctl, stream);
    case 96: return launch_dp<96, SYS>(d_states, nstates, d_points, npoints, ctl, stream);
    case 128: return launch_dp<128, SYS>(d_states, nstates, d_points, npoints, ctl, stream);
    default: return cudaErrorInvalidValue;
  }
}

size_t split_state_bytes() { return split_engine::kStateBytes; }

void split_state_pointers(unsigned char* block, TrajState& t) {
  using namespace split_engine;
  t.split_g1 = block;
  t.split_g2 = block + kG1Bytes;
  t.split_g1_scale = reinterpret_cast<const double*>(block + kG1Bytes + kG2Bytes);
  t.split_g2_scale = reinterpret_cast<const double*>(block + kG1Bytes + kG2Bytes + kG1ScaleBytes);
}

cudaError_t split_prep_launch(const TrajState* d_states, int nstates, cudaStream_t stream) {
  note_launch();
  split_prep_kernel<<<dim3(nstates, 10), 256, 0, stream>>>(d_states);
  return cudaGetLastError();
}

cudaError_t trajectory_launch(int system, int dp, const TrajState* d_states, int nstates, const double* d_points,
                              int npoints, const TrajControls& ctl, cudaStream_t stream, int engine) {
  if (engine == 1) {
    if (system != kSysQuartic || dp != 64) return cudaErrorInvalidValue;
    return launch_dp<64, kSysQuartic, 1>(d_states, nstates, d_points, npoints, ctl, stream);
  }
  if (system == kSysQuartic) return launch_sys<kSysQuartic>(dp, d_states, nstates, d_points, npoints, ctl, stream);
  if (system == kSysFull) return launch_sys<kSysFull>(dp, d_states, nstates, d_points, npoints, ctl, stream);
  if (system == kSysPhi1) return launch_sys<kSysPhi1>(dp, d_states, nstates, d_points, npoints, ctl, stream);
  return cudaErrorInvalidValue;
}

int trajectory_channels(int system) { return system == kSysFull ? 26 : system == kSysPhi1 ? 4 : 7; }

template <int SYS>
static int groups_sys(int dp, int nstates, int requested) {
  switch (dp) {
    case 16: return choose_groups<16, SYS, 0>(nstates, requested);
    case 32: return choose_groups<32, SYS, 0>(nstates, requested);
    case 48: return choose_groups<48, SYS, 0>(nstates, requested);
    case 64: return choose_groups<64, SYS, 0>(nstates, requested);
    case 96: return choose_groups<96, SYS, 0>(nstates, requested);
    case 128: return choose_groups<128, SYS, 0>(nstates, requested);
    default: return 0;
  }
}

int trajectory_groups(int system, int dp, int nstates, int requested, int engine) {
  if (engine == 1) return 1;
  if (system == kSysQuartic) return groups_sys<kSysQuartic>(dp, nstates, requested);
  if (system == kSysFull) return groups_sys<kSysFull>(dp, nstates, requested);
  if (system == kSysPhi1) return groups_sys<kSysPhi1>(dp, nstates, requested);
  return 0;
}

}  // namespace rcmps
