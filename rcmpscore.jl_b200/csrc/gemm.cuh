// CTA-level complex FP64 GEMM on tensor cores: C(MB x DP) += A(MB x K) * B(K x DP).
// A lives in shared memory (row-major, leading dimension lda, lda % 8 == 4 for conflict-free
// fragment loads); B is a list of row-contiguous segments in global memory, streamed in
// KC-row chunks by 1-D bulk copies into an NST-stage ring. C stays in registers: warp w owns
// TPW consecutive 16x8 tiles of one 16-row band.
#pragma once
#include "common.cuh"

namespace rcmps {

template <int DP, int MB, int NW>
struct Tiling {
  static constexpr int TN = DP / 8, TM = MB / 16, T = TM * TN, TPW = T / NW;
  static_assert(T % NW == 0, "tiles per warp");
  static_assert(TN % TPW == 0, "a warp's tiles share one band");
};

// The ring and its counter are shared by products of different row counts (run<MB>).
template <int DP, int NW, int KC, int NST>
struct RowGemmRing {
  static constexpr int NT = 32 * NW;
  static constexpr int LDB = DP + kBPad;            // padded row stride of a chunk in the ring
  static constexpr uint32_t CHUNK_BYTES = KC * DP * 16;
  static constexpr int SLOT = KC * LDB;             // ring slot size (double2)

  double2* ring;        // [NST][KC*LDB]
  uint64_t* full;       // [NST]
  int* wait_flag;       // shared flag set when a bounded wait gives up
  long long gq;         // running chunk counter (uniform across the CTA)

  struct Segs {
    const double2* ptr[6];
    int rows[6];
    int n;
  };

  // Structural zeros of a product of two Z2 block-structured matrices (a packed Z2 state): with
  // `half` = D/2 rows per parity half, the A block starting at row `row0` and parities pa (of A)
  // and pout (of the product), output block (h, c) is zero unless c = h ^ pout, and a live
  // block takes only the K rows of half h ^ pa. on = 0: a dense product.
  struct ZSkip {
    int on = 0, half = 0, row0 = 0, pa = 0, pout = 0;
  };

  // Whether this warp's tiles (one 16-row band, TPW tiles in one column half) are structurally
  // zero; kh: the K half a live band takes (-1: every K row).
  template <int MB>
  __device__ static bool band_zero(const ZSkip& z, int& kh) {
    constexpr int TN = Tiling<DP, MB, NW>::TN, TPW = Tiling<DP, MB, NW>::TPW;
    kh = -1;
    if (!z.on || (z.half % 16) != 0 || ((z.half / 8) % TPW) != 0) return false;
    const int warp = threadIdx.x >> 5;
    const int tile0 = warp * TPW;
    const int h = (z.row0 + (tile0 / TN) * 16) >= z.half ? 1 : 0;
    const int c = ((tile0 % TN) * 8) >= z.half ? 1 : 0;
    kh = h ^ z.pa;
    return c != (h ^ z.pout);
  }

  __device__ static const double2* chunk_ptr(const Segs& s, int q) {
    int r = q * KC;
    for (int i = 0; i < s.n; ++i) {
      if (r < s.rows[i]) return s.ptr[i] + (size_t)r * DP;
      r -= s.rows[i];
    }
    return s.ptr[0];
  }

  __device__ void init() {
    if (threadIdx.x == 0) {
      for (int i = 0; i < NST; ++i) mbar_init(&full[i], 1);
      fence_mbar_init();
    }
    gq = 0;
  }

  __device__ void issue(const Segs& s, int q) {
    const long long g = gq + q;
    const int slot = (int)(g % NST);
    mbar_expect_tx(&full[slot], CHUNK_BYTES);
    const double2* src = chunk_ptr(s, q);
#pragma unroll
    for (int r = 0; r < KC; ++r) bulk_g2s(ring + slot * SLOT + r * LDB, src + r * DP, DP * 16, &full[slot]);
  }

  // acc[TPW] += A * B. Call with all threads; ends with a __syncthreads. z: the product's
  // structural zeros (packed Z2 states; a single K segment of DP rows), skipped.
  template <int MB>
  __device__ void run(ZFrag* acc, const double2* A, int lda, const Segs& s, const ZSkip& z = ZSkip()) {
    constexpr int TN = Tiling<DP, MB, NW>::TN, TPW = Tiling<DP, MB, NW>::TPW;
    int krows = 0;
    for (int i = 0; i < s.n; ++i) krows += s.rows[i];
    const int nch = krows / KC;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile0 = warp * TPW;
    const int mt = tile0 / TN;
    int kh = -1;
    const bool zt = (s.n == 1 && krows == DP) && band_zero<MB>(z, kh);
    if (!(s.n == 1 && krows == DP)) kh = -1;
    if (threadIdx.x == 0) {
      fence_proxy_async_global();
      fence_proxy_async_shared();   // the ring may have been read or written as plain shared memory
      for (int q = 0; q < NST && q < nch; ++q) issue(s, q);
    }
    for (int q = 0; q < nch; ++q) {
      const long long g = gq + q;
      const int slot = (int)(g % NST);
      mbar_wait(&full[slot], (uint32_t)((g / NST) & 1), wait_flag);
      const double2* B = ring + slot * SLOT;
      // every warp waits for every chunk (the slot is refilled after the barrier below); a
      // chunk lies in one K half since the half is a multiple of KC
      const bool live = !zt && (kh < 0 || ((q * KC >= z.half) ? 1 : 0) == kh);
      if (live) {
#pragma unroll
        for (int ks = 0; ks < KC / 8; ++ks) {
          AFrag a;
          load_a(A, lda, mt * 16, q * KC + ks * 8, lane, a);
          BFrag b[TPW];
#pragma unroll
          for (int j = 0; j < TPW; ++j) load_b(B, LDB, ks * 8, ((tile0 + j) % TN) * 8, lane, b[j]);
          zmma_tiles<TPW>(acc, a, b);
        }
      }
      __syncthreads();
      if (threadIdx.x == 0 && q + NST < nch) issue(s, q + NST);
    }
    gq += nch;
  }

  // acc[TPW] += A * B with B (DP x DP) resident in shared memory (leading dimension ldb), the
  // same k-steps in the same order as run(). Call with all threads; ends with a __syncthreads.
  template <int MB>
  __device__ void run_smem(ZFrag* acc, const double2* A, int lda, const double2* B, int ldb,
                           const ZSkip& z = ZSkip()) {
    constexpr int TN = Tiling<DP, MB, NW>::TN, TPW = Tiling<DP, MB, NW>::TPW;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile0 = warp * TPW;
    const int mt = tile0 / TN;
    int kh = -1;
    const bool zt = band_zero<MB>(z, kh);
    if (!zt) {
      for (int q = 0; q < DP / KC; ++q) {
        if (kh >= 0 && ((q * KC >= z.half) ? 1 : 0) != kh) continue;
#pragma unroll
        for (int ks = 0; ks < KC / 8; ++ks) {
          AFrag a;
          load_a(A, lda, mt * 16, q * KC + ks * 8, lane, a);
          BFrag b[TPW];
#pragma unroll
          for (int j = 0; j < TPW; ++j) load_b(B + (size_t)q * KC * ldb, ldb, ks * 8, ((tile0 + j) % TN) * 8, lane, b[j]);
          zmma_tiles<TPW>(acc, a, b);
        }
      }
    }
    __syncthreads();
  }

  // Coordinates of fragment entry i of tile j for this thread: row in [0, MB), col in [0, DP).
  template <int MB>
  __device__ static void coord(int j, int i, int& row, int& col) {
    constexpr int TN = Tiling<DP, MB, NW>::TN, TPW = Tiling<DP, MB, NW>::TPW;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile = warp * TPW + j;
    row = (tile / TN) * 16 + frag_row(lane, i);
    col = (tile % TN) * 8 + frag_col(lane, i);
  }

  // After a wait gave up, wait (bounded) for the copies that may still be in flight.
  __device__ void drain() {
    if (threadIdx.x == 0 && *wait_flag) {
      for (long long g = gq - 1; g >= 0 && g >= gq - NST; --g)
        mbar_wait(&full[g % NST], (uint32_t)((g / NST) & 1), nullptr);
    }
    __syncthreads();
  }
};

// Single-row-count convenience form (the pullback's passes).
template <int DP, int MB, int NW, int KC, int NST>
struct RowGemm : RowGemmRing<DP, NW, KC, NST> {
  using Base = RowGemmRing<DP, NW, KC, NST>;
  static constexpr int TPW = Tiling<DP, MB, NW>::TPW;
  __device__ void run(ZFrag* acc, const double2* A, int lda, const typename Base::Segs& s,
                      const typename Base::ZSkip& z = typename Base::ZSkip()) {
    Base::template run<MB>(acc, A, lda, s, z);
  }
  __device__ void run_smem(ZFrag* acc, const double2* A, int lda, const double2* B, int ldb,
                           const typename Base::ZSkip& z = typename Base::ZSkip()) {
    Base::template run_smem<MB>(acc, A, lda, B, ldb, z);
  }
  __device__ static bool band_zero(const typename Base::ZSkip& z) {
    int kh;
    return Base::template band_zero<MB>(z, kh);
  }
  __device__ static void coord(int j, int i, int& row, int& col) { Base::template coord<MB>(j, i, row, col); }
};

}  // namespace rcmps
