// Split-precision right-hand side of the reduced quartic system (padded dimension 64), the
// tensor-core engine of split.cuh in place of the FP64 mma.sync products of Rhs<DP, SYS>.
// Included by trajectory.cu after the definitions it uses (TrajState, SysTab, Geo, c_sys).
//
// Per right-hand side a CTA (16 own rows of every channel, row0 = 16 rank) runs 11 product units:
//   * G1 of channel c (7 units): [Qc; Rc](own rows) X_c, computed transposed as
//     (X_c^T)(64 x 64) ([Qc; Rc]^T)(64 x 32): A = X_c^T is sliced from the stage vector (per-column
//     scales of X_c), B = the panel^T is constant per state, rank and direction (sliced once by
//     split_prep_kernel); K_cat = 128 in four chunks of 32: rows 0-31 and 32-63 of Re X_c^T with
//     the matching rows of [Re B, Im B], then of Im X_c^T with [-Im B, Re B].
//     Output column n < 16: jac (Qc X_c) -> k_c; n >= 16: P_c = Rc X_c.
//   * G2 of the channel pairs {0,1}, {2}, {3,4}, {5,6} (4 units): out = X' F1 + Y' F2 with
//     X' = jac X_c, Y' = jac P_c + src coef_c X_s (own rows), F1 = Q^dag, F2 = R^dag forward and
//     Q, R adjoint; transposed: [F1^T | F2^T](64 x 128) [X'^T; Y'^T](128 x 16 nc). A is constant
//     (per-column scales of F1, F2 together), B is sliced from own rows (per-row scales of X', Y'
//     together); K_cat = 256 in eight chunks of 32: the two halves of each of the blocks Re F1^T,
//     Re F2^T, Im F1^T, Im F2^T with the matching rows of B_cat.
//     The epilogue adds k_c (jac Qc X_c from G1), the left insertion src coef P_a and the fixed
//     terms, as the FP64 kernel does.
// A unit is 4 (G1) or 8 (G2) chunks. The work is split between warps:
//   * builder warps 0-15 slice the per-stage operand of chunk q into shared-memory buffer q % 3
//     (A half and B half, 28 KB each: seven slices of 4 KB) once the MMAs of chunk q - 3 released
//     it, and arrive on the buffer's "full" barrier; they also run the epilogues;
//   * the issuer (lane 0 of warp 16) bulk-copies (cp.async.bulk) the constant half of chunk q + 1
//     ahead, waits for chunk q's full and copy barriers, issues its MMAs and commits them to the
//     buffer's "free" barrier (and, after a unit's last chunk, to the unit's accumulator barrier).
// Unit u accumulates in the lane half u % 2 of TMEM (6 accumulators of 64 columns). Its epilogue
// runs in the builders' program order during unit u + 1, two chunks in, when its MMAs have long
// completed, so the tensor pipe is not drained at unit boundaries; the builders' arrival on the
// full barrier of unit u + 2's first chunk comes after that epilogue, which orders its TMEM reads
// before the MMAs that overwrite the lane half. The epilogue's results (k_c and P_c rows) are
// ordered for the later builds and epilogues by a named barrier of the builder warps. Every wait
// on a barrier is bounded and sets the controller's wait flag.

namespace split_engine {

constexpr uint32_t kHalf = split::kSlices * split::block_bytes(64);   // one operand half
constexpr uint32_t kBuf = 2 * kHalf;                                   // A half + B half
constexpr int kBufs = 3;                                               // chunk buffers
constexpr int kG1Chunks = 128 / split::kChunkK, kG2Chunks = 256 / split::kChunkK;
constexpr int kKGroups = split::kChunkK / 8;                           // 8-element K groups per chunk
constexpr int kBuilders = 512;                                         // threads of warps 0-15
constexpr int kEpilogueChunk = 2;                                      // chunk of unit u + 1 after which unit u's epilogue runs
constexpr size_t kG1Bytes = (size_t)4 * 2 * kG1Chunks * kHalf;         // [rank][dir][chunk] panel^T slices
constexpr size_t kG2Bytes = (size_t)2 * kG2Chunks * kHalf;             // [dir][chunk] [F1^T | F2^T] slices
constexpr size_t kG1ScaleBytes = (size_t)4 * 2 * 32 * 8;               // [rank][dir][32] column scales
constexpr size_t kG2ScaleBytes = (size_t)2 * 64 * 8;                   // [dir][64] row scales
constexpr size_t kStateBytes = kG1Bytes + kG2Bytes + kG1ScaleBytes + kG2ScaleBytes;
// shared memory: chunk buffers, G1 scales [7][64], G2 scales [4][32], partial maxima [8][64],
// barriers (full, free, copy per buffer; accumulator per lane half), TMEM slot
constexpr size_t kOffG1 = kBufs * (size_t)kBuf;
constexpr size_t kOffG2 = kOffG1 + 7 * 64 * 8;
constexpr size_t kOffRed = kOffG2 + 4 * 32 * 8;
constexpr size_t kOffBar = kOffRed + 8 * 64 * 8;
constexpr size_t kOffSlot = kOffBar + (3 * kBufs + 2) * 8;
constexpr size_t kEnd = kOffSlot + 16;
constexpr uint32_t kTmemCols = 512;

}  // namespace split_engine

struct SplitSmem {
  unsigned char* buf;
  double* g1scale;     // [7][64] per column of X_c (the G1 products' M index)
  double* g2scale;     // [4][32] per own row of X', Y' of each G2 unit (its N index)
  double* red;         // [8][64] partial maxima
  uint64_t* full;      // [kBufs] sliced half written (one arrival per builder warp)
  uint64_t* free;      // [kBufs] MMAs of the buffer's chunk completed
  uint64_t* copy;      // [kBufs] constant half landed
  uint64_t* acc;       // [2] accumulator lane half complete
  uint32_t* tslot;     // TMEM base address written by tcgen05.alloc
};

__device__ __forceinline__ SplitSmem split_carve(unsigned char* base) {
  using namespace split_engine;
  SplitSmem s;
  s.buf = base;
  s.g1scale = reinterpret_cast<double*>(base + kOffG1);
  s.g2scale = reinterpret_cast<double*>(base + kOffG2);
  s.red = reinterpret_cast<double*>(base + kOffRed);
  s.full = reinterpret_cast<uint64_t*>(base + kOffBar);
  s.free = s.full + kBufs;
  s.copy = s.free + kBufs;
  s.acc = s.copy + kBufs;
  s.tslot = reinterpret_cast<uint32_t*>(base + kOffSlot);
  return s;
}

// Barrier initialization (thread 0): full counts one arrival per builder warp.
__device__ __forceinline__ void split_barriers_init(const SplitSmem& s) {
  using namespace split_engine;
  for (int b = 0; b < kBufs; ++b) {
    mbar_init(&s.full[b], kBuilders / 32);
    mbar_init(&s.free[b], 1);
    mbar_init(&s.copy[b], 1);
  }
  mbar_init(&s.acc[0], 1);
  mbar_init(&s.acc[1], 1);
}

// Named barrier of the builder warps only (the issuer warp keeps issuing).
__device__ __forceinline__ void builders_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(split_engine::kBuilders) : "memory");
}

// One product unit of a right-hand side.
struct SplitUnit {
  int g2;      // 0: G1 of channel c; 1: G2 of channels c .. c + nc - 1
  int c, nc, dir;
  int g2i;     // index of the G2 unit (0..3)
};

template <int DP>
struct RhsSplit {
  static_assert(DP == 64, "the split engine covers padded dimension 64");
  using GE = Geo<DP, kSysQuartic>;
  const TrajState* st;
  SplitSmem ss;
  int row0, rank, tid, lane, warp;
  uint32_t tmem;
  long long q, u;      // chunks and units issued so far (the barriers' phases)
  int* wait_flag;

  __device__ static const SysTab& T() { return c_sys[kSysQuartic]; }
  __device__ static int units() { return 7 + T().np[1]; }
  __device__ static SplitUnit unit(int k) {
    const SysTab& t = T();
    SplitUnit U;
    if (k < 7) {
      U.g2 = 0;
      U.c = k;
      U.nc = 1;
      U.g2i = 0;
    } else {
      U.g2 = 1;
      U.c = t.p_first[1][k - 7];
      U.nc = t.p_count[1][k - 7];
      U.g2i = k - 7;
    }
    U.dir = t.dir[U.c];
    return U;
  }
  __device__ static int chunks(const SplitUnit& U) { return U.g2 ? split_engine::kG2Chunks : split_engine::kG1Chunks; }

  // Y' = jac P_c + src coef_c X_b of own row r, column k (the same expression in the scale and
  // the slicing passes, so that every sliced value lies below its scale).
  __device__ double2 yprime(int cc, int r, int k, const double2* zb, double jac, double src) const {
    const size_t loc = (size_t)(row0 + r) * DP + k;
    double2 m = zscale(jac, __ldcg(st->P + (size_t)cc * GE::MAT + loc));
    const int b = T().rsrc[cc];
    if (b >= 0) m = zadd(m, zscale(src * T().rcoef[cc], __ldcg(zb + (size_t)b * GE::MAT + loc)));
    return m;
  }

  // Builders: scales of every column of the 7 channels of the stage vector (the G1 products'
  // A rows), one column per thread.
  __device__ void g1_scales(const double2* zb) {
    for (int col = tid; col < 7 * 64; col += split_engine::kBuilders) {
      const double2* X = zb + (size_t)(col / 64) * GE::MAT + (col % 64);
      double mx = 0.0;
#pragma unroll 8
      for (int k = 0; k < 64; ++k) {
        const double2 v = __ldcg(X + (size_t)k * DP);
        mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
      }
      ss.g1scale[col] = split::pow2_above(mx);
    }
    builders_sync();
  }

  // Builders: scales of the own rows of X' and Y' of G2 unit U (its B columns).
  __device__ void g2_scales(const SplitUnit& U, const double2* zb, double jac, double src) {
    const int rows = 16 * U.nc;
    if (tid < rows * 8) {
      const int n = tid >> 3, g = tid & 7, cc = U.c + n / 16, r = n % 16;
      const double2* X = zb + (size_t)cc * GE::MAT + (size_t)(row0 + r) * DP;
      double mx = 0.0;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int k = 8 * g + e;
        const double2 x = zscale(jac, __ldcg(X + k));
        const double2 y = yprime(cc, r, k, zb, jac, src);
        mx = fmax(mx, fmax(fmax(fabs(x.x), fabs(x.y)), fmax(fabs(y.x), fabs(y.y))));
      }
      ss.red[g * 64 + n] = mx;
    }
    builders_sync();
    if (tid < rows) {
      double mx = 0.0;
      for (int g = 0; g < 8; ++g) mx = fmax(mx, ss.red[g * 64 + tid]);
      ss.g2scale[U.g2i * 32 + tid] = split::pow2_above(mx);
    }
    builders_sync();
  }

  // Builders: the sliced half of chunk kc of unit U into dst.
  __device__ void build(const SplitUnit& U, int kc, const double2* zb, double jac, double src, unsigned char* dst) {
    using split_engine::kKGroups;
    const int koff = split::kChunkK * (kc % 2);   // complex K offset of the chunk within its block
    if (!U.g2) {
      // A = rows koff .. koff + 31 of Re (kc < 2) or Im X_c^T: item (column j of X_c, 8 rows)
      const double2* X = zb + (size_t)U.c * GE::MAT;
      if (tid < 64 * kKGroups) {
        const int j = tid & 63, k8 = tid >> 6;
        const double inv = 1.0 / ss.g1scale[U.c * 64 + j];
        double v[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const double2 x = __ldcg(X + (size_t)(koff + 8 * k8 + e) * DP + j);
          v[e] = (kc < 2 ? x.x : x.y) * inv;
        }
        split::slice8(v, dst + split::kmajor_offset(j, 8 * k8, 64), split::block_bytes(64));
      }
    } else {
      // B = block kc / 2 of the rows of B_cat ([Re, Im] of X'^T, of Y'^T, then [-Im, Re] of each),
      // rows koff .. koff + 31 of it: item (column n of B_cat, 8 rows)
      const int rows = 16 * U.nc, ncat = 2 * rows, block = kc / 2;
      if (tid < ncat * kKGroups) {
        const int n_cat = tid % ncat, k8 = tid / ncat;
        const int n = n_cat % rows, cc = U.c + n / 16, r = n % 16;
        const bool second = n_cat >= rows;
        const double inv = 1.0 / ss.g2scale[U.g2i * 32 + n];
        const double2* X = zb + (size_t)cc * GE::MAT + (size_t)(row0 + r) * DP;
        double v[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = koff + 8 * k8 + e;
          const double2 w = (block % 2 == 0) ? zscale(jac, __ldcg(X + k)) : yprime(cc, r, k, zb, jac, src);
          const double val = block < 2 ? (second ? w.y : w.x) : (second ? w.x : -w.y);
          v[e] = val * inv;
        }
        split::slice8(v, dst + split::kmajor_offset(n_cat, 8 * k8, ncat), split::block_bytes(ncat));
      }
    }
  }

  // Builders: results of unit U (issued as unit number uu) from its TMEM lane half into k and P;
  // ends with a named barrier of the builders.
  __device__ void epilogue(const SplitUnit& U, long long uu, double2* kout, double jac, double src) {
    const int ab = (int)(uu & 1);
    mbar_wait(&ss.acc[ab], (uint32_t)((uu >> 1) & 1), wait_flag);
    split::tc_fence_after();
    const bool narrow = U.g2 && U.nc == 1;   // N_cat = 32: real columns 0..15, imaginary 16..31
    const int ncat = narrow ? 32 : 64;
    if (warp < (narrow ? 4 : 8)) {
      const int quarter = warp & 3, h = warp >> 2;
      double sum[16];
      split::group_sums(split::acc_addr(tmem + ((uint32_t)(32 * quarter) << 16), ab, (uint32_t)(narrow ? 0 : 32 * h)),
                        (uint32_t)ncat, sum);
      const int j = 16 * quarter + (lane & 15);       // output column (the M index)
      const int part = narrow ? (lane >> 4) : h;       // 0 real, 1 imaginary
      const SysTab& t = T();
      const double sj = (U.g2 ? st->split_g2_scale[U.dir * 64 + j] : ss.g1scale[U.c * 64 + j]) * 0x1p-14;
      if (!U.g2) {
#pragma unroll 4
        for (int i = 0; i < 16; ++i) {
          const int n = narrow ? i : 16 * (lane >> 4) + i;   // the N index
          const double sn = st->split_g1_scale[(rank * 2 + U.dir) * 32 + n];
          const double val = sum[i] * sj * sn;
          const int r = n & 15;
          const size_t off = (size_t)U.c * GE::MAT + (size_t)(row0 + r) * DP + j;
          if (n < 16) reinterpret_cast<double*>(kout + off)[part] = jac * val;
          else reinterpret_cast<double*>(st->P + off)[part] = val;
        }
      } else {
        // four entries at a time: their operands (k, the insertion P_a, the fixed term) are all
        // loaded before the first of their stores, so the L2 round trips overlap
        for (int i0 = 0; i0 < 16; i0 += 4) {
          double kv[4], pv[4], fv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int n = narrow ? i0 + u : 16 * (lane >> 4) + i0 + u;
            const int cc = U.c + n / 16, r = n % 16;
            const size_t loc = (size_t)(row0 + r) * DP + j, off = (size_t)cc * GE::MAT + loc;
            const int a = t.lsrc[cc], fx = t.fixed[cc];
            kv[u] = reinterpret_cast<const double*>(kout + off)[part];
            pv[u] = a >= 0 ? reinterpret_cast<const double*>(st->P + (size_t)a * GE::MAT + loc)[part] : 0.0;
            fv[u] = fx ? reinterpret_cast<const double*>((fx == 2 ? st->fixed6 : st->fixed0) + loc)[part] : 0.0;
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int i = i0 + u;
            const int n = narrow ? i : 16 * (lane >> 4) + i;   // the N index
            const double sn = ss.g2scale[U.g2i * 32 + n];
            const double val = sum[i] * sj * sn;
            const int cc = U.c + n / 16, r = n % 16;
            const size_t off = (size_t)cc * GE::MAT + (size_t)(row0 + r) * DP + j;
            double v = val + kv[u];
            if (t.lsrc[cc] >= 0) v += src * t.lcoef[cc] * pv[u];
            if (t.fixed[cc]) v += src * fv[u];
            reinterpret_cast<double*>(kout + off)[part] = v;
          }
        }
      }
    }
    split::tc_fence_before();
    builders_sync();
  }

  // Issuer: the constant half of chunk (unit k, chunk kc), numbered qq, into its buffer.
  __device__ void issue_copy(const SplitUnit& U, int kc, long long qq) {
    using namespace split_engine;
    const int b = (int)(qq % kBufs);
    if (qq >= kBufs) mbar_wait(&ss.free[b], (uint32_t)((qq / kBufs - 1) & 1), wait_flag);
    const unsigned char* srcp = U.g2 ? st->split_g2 + (size_t)(U.dir * kG2Chunks + kc) * kHalf
                                     : st->split_g1 + (size_t)((rank * 2 + U.dir) * kG1Chunks + kc) * kHalf;
    unsigned char* dst = ss.buf + (size_t)b * kBuf + (U.g2 ? 0 : kHalf);
    mbar_expect_tx(&ss.copy[b], kHalf);
#pragma unroll
    for (int i = 0; i < split::kSlices; ++i)
      bulk_g2s(dst + i * split::block_bytes(64), srcp + i * split::block_bytes(64), split::block_bytes(64), &ss.copy[b]);
  }

  // One right-hand side: k_out = f(t, z) on this CTA's rows (the FP64 kernel's contract).
  __device__ void operator()(const double2* zb, double2* kout, double jac, double src) {
    using namespace split_engine;
    const int nu = units();
    if (warp == kBuilders / 32) {
      // ------------------------------------------------ issuer warp
      if (lane == 0) {
        long long qq = q, uu = u;
        int nk = 0, nkc = 0;          // the next chunk whose copy is to be issued
        auto advance = [&](int& k, int& kc) {
          if (++kc == chunks(unit(k))) {
            kc = 0;
            ++k;
          }
        };
        issue_copy(unit(0), 0, qq);
        advance(nk, nkc);
        for (int k = 0; k < nu; ++k, ++uu) {
          const SplitUnit U = unit(k);
          const int ab = (int)(uu & 1);
          for (int kc = 0; kc < chunks(U); ++kc, ++qq) {
            if (nk < nu) {             // the next chunk's constant half, one chunk ahead
              issue_copy(unit(nk), nkc, qq + 1);
              advance(nk, nkc);
            }
            const int b = (int)(qq % kBufs);
            const uint32_t ph = (uint32_t)((qq / kBufs) & 1);
            mbar_wait(&ss.full[b], ph, wait_flag);
            mbar_wait(&ss.copy[b], ph, wait_flag);
            split::tc_fence_after();
            const uint32_t bA = smem_u32(ss.buf + (size_t)b * kBuf), bB = bA + kHalf;
            const uint32_t acc = split::acc_addr(tmem, ab, 0);
            if (U.g2 && U.nc == 1) split::chunk_mmas<32>(acc, bA, bB, kc == 0);
            else split::chunk_mmas<64>(acc, bA, bB, kc == 0);
            split::mma_commit(&ss.free[b]);
            if (kc == chunks(U) - 1) split::mma_commit(&ss.acc[ab]);
          }
        }
      }
      __syncwarp();
    } else {
      // ------------------------------------------------ builder warps
      g1_scales(zb);
      long long qq = q, uu = u;
      SplitUnit prev{};
      for (int k = 0; k < nu; ++k, ++uu) {
        const SplitUnit U = unit(k);
        if (U.g2) g2_scales(U, zb, jac, src);
        for (int kc = 0; kc < chunks(U); ++kc, ++qq) {
          const int b = (int)(qq % kBufs);
          if (qq >= kBufs) mbar_wait(&ss.free[b], (uint32_t)((qq / kBufs - 1) & 1), wait_flag);
          unsigned char* bufp = ss.buf + (size_t)b * kBuf;
          build(U, kc, zb, jac, src, U.g2 ? bufp + kHalf : bufp);
          split::fence_proxy_async_smem();
          split::tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&ss.full[b]);
          if (kc == kEpilogueChunk && k > 0) epilogue(prev, uu - 1, kout, jac, src);
        }
        prev = U;
      }
      epilogue(prev, uu - 1, kout, jac, src);
    }
    // every thread leaves with the same counters
    for (int k = 0; k < nu; ++k) q += chunks(unit(k));
    u += nu;
    __syncthreads();
  }
};

// Slices of the constant operands of every state (split engine, padded dimension 64):
// blockIdx.y < 8: the G1 panel^T of rank y / 2 and direction y % 2; y = 8, 9: [F1^T | F2^T] of
// direction y - 8. One CTA of 256 threads per (state, y).
__global__ void __launch_bounds__(256) split_prep_kernel(const TrajState* __restrict__ states) {
  using namespace split_engine;
  constexpr int DP = 64;
  __shared__ double scale[64];
  __shared__ double part[4][64];
  const TrajState* st = states + blockIdx.x;
  const int y = blockIdx.y, tid = threadIdx.x;
  unsigned char* g1 = const_cast<unsigned char*>(st->split_g1);
  unsigned char* g2 = const_cast<unsigned char*>(st->split_g2);
  if (y < 8) {
    const int rank = y / 2, dir = y % 2;
    const double2* Qd = dir == 0 ? st->Q : st->Qh;
    const double2* Rd = dir == 0 ? st->R : st->Rh;
    auto panel = [&](int n, int k) {   // row n of [Q_dir; R_dir] restricted to the rank's rows
      return n < 16 ? Qd[(size_t)(16 * rank + n) * DP + k] : Rd[(size_t)(16 * rank + n - 16) * DP + k];
    };
    if (tid < 128) {
      const int n = tid & 31, g = tid >> 5;
      double mx = 0.0;
      for (int k = 16 * g; k < 16 * g + 16; ++k) {
        const double2 v = panel(n, k);
        mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
      }
      part[g][n] = mx;
    }
    __syncthreads();
    if (tid < 32) {
      const double s = split::pow2_above(fmax(fmax(part[0][tid], part[1][tid]), fmax(part[2][tid], part[3][tid])));
      scale[tid] = s;
      const_cast<double*>(st->split_g1_scale)[(rank * 2 + dir) * 32 + tid] = s;
    }
    __syncthreads();
    for (int kc = 0; kc < kG1Chunks; ++kc)
      for (int it = tid; it < 64 * kKGroups; it += 256) {
        const int n_cat = it & 63, k8 = it >> 6, n = n_cat & 31;
        const bool second = n_cat >= 32;
        const int koff = split::kChunkK * (kc % 2);
        const double inv = 1.0 / scale[n];
        double v[8];
        for (int e = 0; e < 8; ++e) {
          const double2 b = panel(n, koff + 8 * k8 + e);   // B[k][n] = panel[n][k]
          const double val = kc < 2 ? (second ? b.y : b.x) : (second ? b.x : -b.y);
          v[e] = val * inv;
        }
        split::slice8(v, g1 + (size_t)((rank * 2 + dir) * kG1Chunks + kc) * kHalf +
                             split::kmajor_offset(n_cat, 8 * k8, 64), split::block_bytes(64));
      }
  } else {
    const int dir = y - 8;
    const double2* F1 = dir == 0 ? st->Qh : st->Q;
    const double2* F2 = dir == 0 ? st->Rh : st->R;
    if (tid < 256) {
      const int j = tid & 63, g = tid >> 6;
      double mx = 0.0;
      for (int k = 16 * g; k < 16 * g + 16; ++k) {
        const double2 a = F1[(size_t)k * DP + j], b = F2[(size_t)k * DP + j];
        mx = fmax(mx, fmax(fmax(fabs(a.x), fabs(a.y)), fmax(fabs(b.x), fabs(b.y))));
      }
      part[g][j] = mx;
    }
    __syncthreads();
    if (tid < 64) {
      const double s = split::pow2_above(fmax(fmax(part[0][tid], part[1][tid]), fmax(part[2][tid], part[3][tid])));
      scale[tid] = s;
      const_cast<double*>(st->split_g2_scale)[dir * 64 + tid] = s;
    }
    __syncthreads();
    for (int kc = 0; kc < kG2Chunks; ++kc)
      for (int it = tid; it < 64 * kKGroups; it += 256) {
        const int j = it & 63, k8 = it >> 6, block = kc / 2, koff = split::kChunkK * (kc % 2);
        const double2* F = (block % 2 == 0) ? F1 : F2;   // A[j][k] = F[k][j]
        const double inv = 1.0 / scale[j];
        double v[8];
        for (int e = 0; e < 8; ++e) {
          const double2 a = F[(size_t)(koff + 8 * k8 + e) * DP + j];
          v[e] = (block < 2 ? a.x : a.y) * inv;
        }
        split::slice8(v, g2 + (size_t)(dir * kG2Chunks + kc) * kHalf + split::kmajor_offset(j, 8 * k8, 64),
                      split::block_bytes(64));
      }
  }
}
