// Split-precision complex products on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// A double-precision complex product C = A B is emulated by exact products of 7-bit integer
// slices held in BF16 (the Ozaki scheme): every row m of A is scaled by a power of two s_m so
// that |A[m][k]| < s_m, and every column n of B by t_n; the scaled values v (|v| < 1) are cut
// into kSlices slices v = 2^-7 sum_i u_i 2^-7i + r, each u_i an integer (u_0 in [-128, 128], the
// others in [-64, 64]: the remainder is rounded to the nearest integer, exactly in FP64, so the
// cut is unbiased and |r| <= 2^-7kSlices / 2). The slices are stored pre-weighted,
// w_i = u_i 2^-7i, which BF16 holds exactly. Then
//     C[m][n] = s_m t_n 2^-14 sum_{i,l} (sum_k wA_i[m][k] wB_l[k][n]),
// and the pairs with i + l <= kSlices - 1 are kept: with seven slices the error is about 2^-50
// of s_m t_n per term. (Six slices, 2^-43, meet a 1e-10 energy bar but not the DOP853 step
// control at rtol 1e-12, whose error estimate cancels to about 1e-12 of the stage values: the
// product rounding then dominates it and the controller takes about ten times the steps.)
// The pair products accumulate in FP32 in TMEM, one accumulator per group s = i + l for
// s = 0 .. 4 (exact: every group sum is an integer times 2^-7s, of magnitude at most
// 128^2 K + 2 128 64 K + (s - 1) 64^2 K < 2^24 for K <= 256) and one shared accumulator for
// s >= 5, whose terms are at most 2^-35 of the leading group, so that its FP32 rounding stays
// below 2^-57 of the result. The accumulators are summed in FP64 and rescaled.
//
// Complex arithmetic is folded into K: with A_cat = [Ar | Ai] (M x 2K) and
// B_cat = [[Br, Bi], [-Bi, Br]] (2K x 2N), A_cat B_cat = [Re C | Im C].
//
// Shared-memory operand layout (K-major, no swizzle): an operand block of MN rows and kChunkK K
// elements (BF16) is a grid of core matrices of 128 bytes (8 rows of 16 bytes); core matrix
// (mn / 8, k / 8) sits at ((k / 8) (MN / 8) + mn / 8) 128 bytes, so the descriptor's stride byte
// offset (between core matrices adjacent in MN) is 128 and its leading byte offset (adjacent in
// K) is MN / 8 * 128. One MMA instruction covers K = 16, i.e. two core matrices.
//
// Accumulators (M = 64, cta_group::1): row m of a 64-row accumulator based at lane b (0 or 16)
// lives in TMEM lane b + (m % 16) + 32 (m / 16), so two accumulators share the same columns in
// the two lane halves of every 32-lane quarter; warp w reads the lanes of its quarter w % 4, 16
// at a time (tcgen05.ld 16x32bx2).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"

namespace rcmps {
namespace split {

constexpr int kSlices = 7;      // slices per operand: 49 bits
constexpr int kBits = 7;        // bits per slice
constexpr int kGroups = 6;      // accumulators: s = 0 .. 4 and s >= 5
constexpr int kM = 64;          // rows of every product (the MMA's M)
constexpr int kChunkK = 32;     // K elements (BF16) of one staged chunk
constexpr int kPairs = kSlices * (kSlices + 1) / 2;

// Byte offset of element (mn, k) in a K-major operand block of MN rows x kChunkK K.
RCMPS_DEVICE_INLINE uint32_t kmajor_offset(int mn, int k, int MN) {
  return (uint32_t)((((k >> 3) * (MN >> 3)) + (mn >> 3)) * 128 + (mn & 7) * 16 + (k & 7) * 2);
}
// Bytes of one slice of an operand block of MN rows x kChunkK K.
__host__ __device__ constexpr uint32_t block_bytes(int MN) { return (uint32_t)MN * kChunkK * 2; }

// Shared-memory matrix descriptor (sm_100 format, version 1, no swizzle).
RCMPS_DEVICE_INLINE uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// Instruction descriptor of kind::f16: BF16 x BF16 -> FP32, A and B K-major, M = 64, N.
__host__ __device__ constexpr uint32_t idesc_bf16_m64(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
}

// ------------------------------------------------------------------ tcgen05 primitives
RCMPS_DEVICE_INLINE void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
RCMPS_DEVICE_INLINE void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
RCMPS_DEVICE_INLINE void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
RCMPS_DEVICE_INLINE void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
RCMPS_DEVICE_INLINE void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D (TMEM) = A B (+ D when accumulate), issued by one thread.
RCMPS_DEVICE_INLINE void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                  uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}
// Arrive on `bar` once every MMA this thread issued so far has completed.
RCMPS_DEVICE_INLINE void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// 16 lanes of a 32-lane quarter from lane `taddr`'s lane on (16 or 0 within the quarter):
// threads 0-15 read columns [c, c + 16) of lanes +0..15 and threads 16-31 columns
// [c + 16, c + 32) of the same lanes (warp-wide), waited for.
RCMPS_DEVICE_INLINE void tmem_load16x2(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.16x32bx2.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16], 16;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Sums over the kGroups accumulators (at taddr + g * ncat) of the 16 values tmem_load16x2
// gives this thread, in FP64, smallest group first.
RCMPS_DEVICE_INLINE void group_sums(uint32_t taddr, uint32_t ncat, double* out) {
  float v[16];
#pragma unroll
  for (int n = 0; n < 16; ++n) out[n] = 0.0;
#pragma unroll
  for (int g = kGroups - 1; g >= 0; --g) {
    tmem_load16x2(taddr + (uint32_t)g * ncat, v);
#pragma unroll
    for (int n = 0; n < 16; ++n) out[n] += (double)v[n];
  }
}
// TMEM address of accumulator buffer `ab` (lane half ab of every quarter), column `col`.
RCMPS_DEVICE_INLINE uint32_t acc_addr(uint32_t tmem, int ab, uint32_t col) {
  return tmem + ((uint32_t)(16 * ab) << 16) + col;
}

// ------------------------------------------------------------------ slicing
// Power-of-two scale 2^e with |x| < 2^e for every x of magnitude <= maxabs (1 for 0).
RCMPS_DEVICE_INLINE double pow2_above(double maxabs) {
  if (!(maxabs > 0.0)) return 1.0;
  int e;
  frexp(maxabs, &e);
  return ldexp(1.0, e);
}

// Cut 8 values (already divided by their scale, |v| < 1) into kSlices pre-weighted BF16
// slices (nearest-integer remainders); slice i of the 8 values is written as one 16-byte row to
// dst + i * stride.
RCMPS_DEVICE_INLINE void slice8(const double* v, unsigned char* dst, uint32_t stride) {
  double r[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) r[e] = v[e];
  constexpr double kWeight[8] = {1.0, 0x1p-7, 0x1p-14, 0x1p-21, 0x1p-28, 0x1p-35, 0x1p-42, 0x1p-49};
  static_assert(kSlices <= 8 && kBits == 7, "slice weights");
#pragma unroll
  for (int i = 0; i < kSlices; ++i) {
    const double w = kWeight[i];
    uint32_t packed[4];
#pragma unroll
    for (int e = 0; e < 8; e += 2) {
      r[e] *= 128.0;
      r[e + 1] *= 128.0;
      const double t0 = rint(r[e]), t1 = rint(r[e + 1]);
      r[e] -= t0;
      r[e + 1] -= t1;
      // t w has at most 8 significant bits: one exact conversion
      const __nv_bfloat16 b0 = __double2bfloat16(t0 * w), b1 = __double2bfloat16(t1 * w);
      packed[e / 2] = (uint32_t)__bfloat16_as_ushort(b0) | ((uint32_t)__bfloat16_as_ushort(b1) << 16);
    }
    *reinterpret_cast<uint4*>(dst + (size_t)i * stride) = make_uint4(packed[0], packed[1], packed[2], packed[3]);
  }
}

// ------------------------------------------------------------------ MMAs of one staged chunk
// Every kept pair (i, l) of the chunk's slices, K = kChunkK in MMAs of K = 16, into the
// kGroups group accumulators at tmem_acc + g * NCAT columns. first_chunk: the unit's first chunk (each
// group's first MMA overwrites its accumulator). a_base / b_base: shared addresses of slice 0.
template <int NCAT>
RCMPS_DEVICE_INLINE void chunk_mmas(uint32_t tmem_acc, uint32_t a_base, uint32_t b_base, bool first_chunk) {
  constexpr uint32_t a_lbo = (kM / 8) * 128, b_lbo = (NCAT / 8) * 128;
  constexpr uint32_t idesc = idesc_bf16_m64(NCAT);
  bool written[kGroups] = {};
#pragma unroll
  for (int s = 0; s < kSlices; ++s) {
#pragma unroll
    for (int i = 0; i <= s; ++i) {
      const int l = s - i;
      const int g = s < kGroups - 1 ? s : kGroups - 1;
#pragma unroll
      for (int kk = 0; kk < kChunkK / 16; ++kk) {
        const uint64_t ad = smem_desc(a_base + i * block_bytes(kM) + kk * 2 * a_lbo, a_lbo, 128);
        const uint64_t bd = smem_desc(b_base + l * block_bytes(NCAT) + kk * 2 * b_lbo, b_lbo, 128);
        const uint32_t acc = (first_chunk && !written[g]) ? 0u : 1u;
        mma_bf16(tmem_acc + (uint32_t)(g * NCAT), ad, bd, idesc, acc);
        written[g] = true;
      }
    }
  }
}

}  // namespace split
}  // namespace rcmps
