// Batched d x d complex products (d <= 64) by the split-precision tensor-core engine
// (split.cuh): C_b = A_b B_b for every b, each product on one CTA.
//
// Each product is two units (the column halves of C, 32 complex columns each), accumulated in the
// two lane halves of TMEM (kGroups accumulators of 64 FP32 columns each); each unit is four
// staged chunks (K_cat = 128 in chunks of 32: the real, then the imaginary part of A with the
// matching row blocks of B_cat), so a
// CTA runs the same pipeline as the trajectory's split right-hand side: chunk q is sliced into
// shared-memory buffer q % 2 while the MMAs of chunk q - 1 run, and the epilogue of unit u - 1
// (TMEM -> FP64 recombination) runs while the MMAs of unit u do.
#include <cuda_runtime.h>
#include <cstdint>
#include "../../include/rcmps_b200.h"
#include "context.h"
#include "split.cuh"

namespace rcmps {

namespace {

constexpr int kProdThreads = 512;
constexpr uint32_t kBufBytes = split::kSlices * (split::block_bytes(64) + split::block_bytes(64));
constexpr size_t kProdSmem = 2 * (size_t)kBufBytes + (64 + 2 * 32) * 8 + 4 * 8 + 16;

__global__ void __launch_bounds__(kProdThreads, 1)
split_product_kernel(const double2* __restrict__ A, const double2* __restrict__ B, double2* __restrict__ C, int d,
                     int* __restrict__ status) {
  using namespace split;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* bufs = smem;
  double* sA = reinterpret_cast<double*>(smem + 2 * kBufBytes);   // [64] row scales of A
  double* sB = sA + 64;                                           // [2][32] column scales of B, per unit
  uint64_t* mma_done = reinterpret_cast<uint64_t*>(sB + 64);      // [2] chunk buffers
  uint64_t* acc_full = mma_done + 2;                              // [2] accumulator buffers
  uint32_t* tslot = reinterpret_cast<uint32_t*>(acc_full + 2);
  __shared__ int wait_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t mat = (size_t)d * d;
  const double2* a = A + blockIdx.x * mat;
  const double2* b = B + blockIdx.x * mat;
  double2* c = C + blockIdx.x * mat;
  auto load = [&](const double2* m, int r, int col) {
    return (r < d && col < d) ? m[(size_t)r * d + col] : make_double2(0.0, 0.0);
  };

  if (tid == 0) {
    mbar_init(&mma_done[0], 1);
    mbar_init(&mma_done[1], 1);
    mbar_init(&acc_full[0], 1);
    mbar_init(&acc_full[1], 1);
    fence_mbar_init();
    wait_flag = 0;
  }
  if (warp == 0) tmem_alloc(tslot, 512);
  // row scales of A
  if (tid < 64) {
    double mx = 0.0;
    for (int k = 0; k < 64; ++k) {
      const double2 v = load(a, tid, k);
      mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
    }
    sA[tid] = pow2_above(mx);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  auto epilogue = [&](int u) {
    const int ab = u & 1;
    mbar_wait(&acc_full[ab], (uint32_t)((u >> 1) & 1), &wait_flag);
    tc_fence_after();
    if (warp < 8) {
      // warp w: lane quarter w % 4 (rows 16 (w % 4) + lane % 16), N_cat columns [32 h, 32 h + 32)
      // with h = w / 4 (h 0: real parts, 1: imaginary parts); lanes 16-31 take the upper 16
      const int quarter = warp & 3, h = warp >> 2;
      double sum[16];
      group_sums(acc_addr(tmem + ((uint32_t)(32 * quarter) << 16), ab, (uint32_t)(32 * h)), 64, sum);
      const int m = 16 * quarter + (lane & 15);
      if (m < d) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = 16 * (lane >> 4) + j, col = 32 * u + n;
          if (col < d) {
            const double val = sum[j] * sA[m] * sB[ab * 32 + n] * 0x1p-14;
            reinterpret_cast<double*>(c + (size_t)m * d + col)[h] = val;
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();
  };

  int q = 0;
  for (int u = 0; u < 2; ++u) {
    const int ab = u & 1;
    // column scales of this unit's 32 columns of B
    if (tid < 32) {
      double mx = 0.0;
      for (int k = 0; k < 64; ++k) {
        const double2 v = load(b, k, 32 * u + tid);
        mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
      }
      sB[ab * 32 + tid] = pow2_above(mx);
    }
    __syncthreads();
    // K_cat = [Re A | Im A] = 128 columns, in chunks of kChunkK: chunk kc holds part kc / 2 (0 the
    // real part of A with the rows [Br, Bi] of B_cat, 1 the imaginary part with [-Bi, Br]) at
    // complex columns koff = 32 (kc % 2) ..
    constexpr int kChunks = 128 / kChunkK, kGroupsK = kChunkK / 8;
    for (int kc = 0; kc < kChunks; ++kc, ++q) {
      const int buf = q & 1, part = kc / 2, koff = kChunkK * (kc % 2);
      if (q >= 2) mbar_wait(&mma_done[buf], (uint32_t)(((q >> 1) - 1) & 1), &wait_flag);
      unsigned char* bA = bufs + (size_t)buf * kBufBytes;
      unsigned char* bB = bA + kSlices * block_bytes(64);
      // A items (row m, 8 consecutive k), then B items (column n of B_cat, 8 consecutive k)
      for (int it = tid; it < 2 * 64 * kGroupsK; it += kProdThreads) {
        double v[8];
        if (it < 64 * kGroupsK) {
          const int m = it / kGroupsK, k0 = (it % kGroupsK) * 8;
          const double inv = 1.0 / sA[m];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const double2 x = load(a, m, koff + k0 + e);
            v[e] = (part == 0 ? x.x : x.y) * inv;
          }
          slice8(v, bA + kmajor_offset(m, k0, 64), block_bytes(64));
        } else {
          const int j = it - 64 * kGroupsK, n = j / kGroupsK, k0 = (j % kGroupsK) * 8;
          const int col = 32 * u + (n & 31);
          const double inv = 1.0 / sB[ab * 32 + (n & 31)];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const double2 x = load(b, koff + k0 + e, col);
            const double val = part == 0 ? (n < 32 ? x.x : x.y) : (n < 32 ? -x.y : x.x);
            v[e] = val * inv;
          }
          slice8(v, bB + kmajor_offset(n, k0, 64), block_bytes(64));
        }
      }
      fence_proxy_async_smem();
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        chunk_mmas<64>(acc_addr(tmem, ab, 0), smem_u32(bA), smem_u32(bB), kc == 0);
        mma_commit(&mma_done[buf]);
        if (kc == kChunks - 1) mma_commit(&acc_full[ab]);
      }
    }
    if (u >= 1) epilogue(u - 1);
  }
  epilogue(1);
  // every MMA has completed (the last epilogue waited for it); release TMEM
  if (warp == 0) tmem_dealloc(tmem, 512);
  if (tid == 0 && wait_flag) atomicExch(status, 1);
}

}  // namespace

cudaError_t split_product_launch(const double* A, const double* B, double* C, int d, int n, int* d_status,
                                 cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(split_product_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kProdSmem);
  if (e != cudaSuccess) return e;
  note_launch();
  split_product_kernel<<<n, kProdThreads, kProdSmem, stream>>>(reinterpret_cast<const double2*>(A),
                                                               reinterpret_cast<const double2*>(B),
                                                               reinterpret_cast<double2*>(C), d, d_status);
  return cudaGetLastError();
}

}  // namespace rcmps

using namespace rcmps;

extern "C" int rcmps_split_product_batch(rcmps_context* ctx, int n, int d, const double* A, const double* B,
                                         double* C, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  if (n < 0 || d < 1 || d > 64) return fail(ctx, RCMPS_INVALID_ARGUMENT, "rcmps_split_product_batch: 1 <= d <= 64");
  if (n == 0) return RCMPS_OK;
  if (!A || !B || !C) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->slot[2].stream;
  if (aux_reserve(ctx, 256) != cudaSuccess) return fail(ctx, RCMPS_OUT_OF_MEMORY, "status word");
  int* d_status = static_cast<int*>(ctx->aux);
  cudaError_t e = cudaMemsetAsync(d_status, 0, sizeof(int), s);
  if (!e) e = split_product_launch(A, B, C, d, n, d_status, s);
  int h_status = 0;
  if (!e) e = cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (!e) e = cudaStreamSynchronize(s);
  if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("split product: ") + cudaGetErrorString(e));
  if (h_status) return fail(ctx, RCMPS_WAIT_LIMIT, "split product: a bounded wait gave up");
  return RCMPS_OK;
}
