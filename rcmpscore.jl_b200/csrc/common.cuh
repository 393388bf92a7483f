// Device primitives shared by the fg_phi4 kernels (sm_100a only).
//
// Complex matrices are row-major arrays of double2 (re, im), the layout of a C-ordered NumPy
// complex128 array. Products run on the FP64 tensor-core instruction mma.sync m16n8k8 (A 16x8
// row, B 8x8 col, C 16x8; fragment layout checked on B200 against a CPU product), three real
// products per complex product (ZFrag).
// Every wait on an mbarrier is bounded: on timeout it raises the kernel's error flag and
// returns, so control flow (and every cluster barrier) stays uniform.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#ifndef RCMPS_DEVICE_INLINE
#define RCMPS_DEVICE_INLINE __device__ __forceinline__
#endif

namespace rcmps {

// Kernel launches issued by the library in this process (every launch site calls note_launch).
void note_launch();
void note_launches(long long count);   // kernels replayed by one graph launch
long long thread_launch_count();   // launches noted by the calling host thread

// ------------------------------------------------------------------ status codes
// The numbers of the reference's device controller (device_control_backend.py:23-27 of
// rcmps_gpu) plus the wait limit and the solver and input failures of this library.
enum Status : int {
  kOk = 0,
  kMaxSteps = 1,
  kStepUnderflow = 2,
  kNonfiniteError = 3,
  kSourceDomain = 4,
  kMissingSamples = 5,
  kDeviceTimeout = 6,       // device-clock watchdog (max_device_seconds)
  kWaitLimit = 7,           // a bounded mbarrier wait gave up
  kKrylovFailure = 8,       // shifted Arnoldi did not reach its true residual
  kSolveFailure = 9,        // GMRES / dense solve did not reach its residual
  kNonfiniteResult = 10,
  kInvalidInput = 20,       // a state the requested route does not accept (RCMPS_INVALID_ARGUMENT)
};

// ------------------------------------------------------------------ complex helpers
RCMPS_DEVICE_INLINE double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
RCMPS_DEVICE_INLINE double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
RCMPS_DEVICE_INLINE double2 zscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
RCMPS_DEVICE_INLINE double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
RCMPS_DEVICE_INLINE double2 zconj(double2 a) { return make_double2(a.x, -a.y); }
RCMPS_DEVICE_INLINE double zabs2(double2 a) { return a.x * a.x + a.y * a.y; }
RCMPS_DEVICE_INLINE double2 zaxpy(double s, double2 x, double2 y) {
  return make_double2(fma(s, x.x, y.x), fma(s, x.y, y.y));
}

// ------------------------------------------------------------------ FP64 tensor-core tile
// D(16x8) += A(16x8, row) * B(8x8, col); lane = 4 g + t:
//   a = {A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4]}, b = {B[t][g], B[t+4][g]},
//   c = {C[g][2t], C[g][2t+1], C[g+8][2t], C[g+8][2t+1]}.
RCMPS_DEVICE_INLINE void dmma16x8x8(double* c, const double* a, const double* b) {
  asm(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// A complex 16x8 accumulator in the C-fragment layout, kept as the three real sums of the
// 3-multiplication complex product (Gauss): p = sum Ar Br, q = sum Ai Bi,
// s = sum (Ar + Ai)(Br + Bi), so that re = p - q and im = s - p - q. Three real MMAs per complex
// k-step instead of four, on three independent accumulators.
struct ZFrag {
  double p[4];
  double q[4];
  double s[4];
  RCMPS_DEVICE_INLINE void zero() {
#pragma unroll
    for (int i = 0; i < 4; ++i) p[i] = q[i] = s[i] = 0.0;
  }
  RCMPS_DEVICE_INLINE double re(int i) const { return p[i] - q[i]; }
  RCMPS_DEVICE_INLINE double im(int i) const { return s[i] - p[i] - q[i]; }
  RCMPS_DEVICE_INLINE double2 value(int i) const { return make_double2(re(i), im(i)); }
  // acc += v for entry i
  RCMPS_DEVICE_INLINE void add(int i, double2 v) {
    p[i] += v.x;
    s[i] += v.x + v.y;
  }
};

// A fragments of a complex 16x8 A tile: real part, imaginary part and their sum.
struct AFrag {
  double r[4], i[4], s[4];
};
// B fragments of a complex 8x8 B tile: real part, imaginary part and their sum.
struct BFrag {
  double r[2], i[2], s[2];
};

// acc[j] += A * B_j for TPW tiles sharing the A fragment; the MMAs are issued so that
// consecutive ones update different accumulators.
template <int TPW>
RCMPS_DEVICE_INLINE void zmma_tiles(ZFrag* acc, const AFrag& a, const BFrag* b) {
#pragma unroll
  for (int j = 0; j < TPW; ++j) {
    dmma16x8x8(acc[j].p, a.r, b[j].r);
    dmma16x8x8(acc[j].q, a.i, b[j].i);
    dmma16x8x8(acc[j].s, a.s, b[j].s);
  }
}
RCMPS_DEVICE_INLINE void zmma(ZFrag& acc, const AFrag& a, const BFrag& b) { zmma_tiles<1>(&acc, a, &b); }

// Load the A fragment of rows [m0, m0+16) and columns [k0, k0+8) of a row-major complex
// matrix with leading dimension lda (in complex elements) from shared memory.
RCMPS_DEVICE_INLINE void load_a(const double2* A, int lda, int m0, int k0, int lane, AFrag& a) {
  const int g = lane >> 2, t = lane & 3;
  const double2* p = A + (m0 + g) * lda + k0 + t;
  double2 v0 = p[0], v1 = p[8 * lda], v2 = p[4], v3 = p[8 * lda + 4];
  a.r[0] = v0.x; a.r[1] = v1.x; a.r[2] = v2.x; a.r[3] = v3.x;
  a.i[0] = v0.y; a.i[1] = v1.y; a.i[2] = v2.y; a.i[3] = v3.y;
#pragma unroll
  for (int i = 0; i < 4; ++i) a.s[i] = a.r[i] + a.i[i];
}

// Load the B fragment of rows [k0, k0+8) and columns [n0, n0+8) of a row-major complex matrix.
RCMPS_DEVICE_INLINE void load_b(const double2* B, int ldb, int k0, int n0, int lane, BFrag& b) {
  const int g = lane >> 2, t = lane & 3;
  double2 v0 = B[(k0 + t) * ldb + n0 + g], v1 = B[(k0 + t + 4) * ldb + n0 + g];
  b.r[0] = v0.x; b.r[1] = v1.x;
  b.i[0] = v0.y; b.i[1] = v1.y;
  b.s[0] = v0.x + v0.y; b.s[1] = v1.x + v1.y;
}

// Element coordinates (row, col) of C-fragment entry i for a lane.
RCMPS_DEVICE_INLINE int frag_row(int lane, int i) { return (lane >> 2) + ((i & 2) ? 8 : 0); }
RCMPS_DEVICE_INLINE int frag_col(int lane, int i) { return 2 * (lane & 3) + (i & 1); }

// ------------------------------------------------------------------ shared-memory addresses
RCMPS_DEVICE_INLINE uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ------------------------------------------------------------------ mbarrier + bulk copy
RCMPS_DEVICE_INLINE void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
RCMPS_DEVICE_INLINE void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
RCMPS_DEVICE_INLINE void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
RCMPS_DEVICE_INLINE void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
RCMPS_DEVICE_INLINE bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of `parity` to complete. Returns false (and sets *flag) on timeout.
constexpr long long kWaitIterations = 1ll << 24;
RCMPS_DEVICE_INLINE bool mbar_wait(uint64_t* bar, uint32_t parity, int* flag) {
  for (long long i = 0; i < kWaitIterations; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (flag) atomicExch(flag, 1);
  return false;
}
// Row padding of streamed B chunks in shared memory: a row stride of (cols + 2) complex values
// (= 32 mod 128 bytes) puts the four k-rows a B fragment reads in different banks.
constexpr int kBPad = 2;

// 1-D bulk copy global -> shared of this CTA, completing on `bar`. 16-byte aligned, size % 16 == 0.
RCMPS_DEVICE_INLINE void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
RCMPS_DEVICE_INLINE void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}
// Orders this thread's (and, after a barrier, the block's) generic accesses of shared memory
// before later bulk copies into the same bytes.
RCMPS_DEVICE_INLINE void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ------------------------------------------------------------------ clusters
RCMPS_DEVICE_INLINE uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
RCMPS_DEVICE_INLINE uint32_t cluster_id_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
RCMPS_DEVICE_INLINE uint32_t cluster_size() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
// Full cluster barrier with release/acquire semantics at cluster scope (orders global and
// shared::cluster accesses of every thread of the cluster).
RCMPS_DEVICE_INLINE void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// The two halves of cluster_sync, for work placed between them: every thread of every CTA of the
// cluster executes one arrive and then one wait.
RCMPS_DEVICE_INLINE void cluster_arrive_release() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
RCMPS_DEVICE_INLINE void cluster_wait_acquire() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Read a double from the shared memory of CTA `rank` of this cluster at the address that `p`
// has in this CTA.
RCMPS_DEVICE_INLINE double dsmem_load(const double* p, uint32_t rank) {
  uint32_t local = smem_u32(p), remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(rank));
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(remote) : "memory");
  return v;
}
RCMPS_DEVICE_INLINE int dsmem_load_int(const int* p, uint32_t rank) {
  uint32_t local = smem_u32(p), remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(rank));
  int v;
  asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(remote) : "memory");
  return v;
}

// ------------------------------------------------------------------ timer
RCMPS_DEVICE_INLINE unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ------------------------------------------------------------------ reductions
RCMPS_DEVICE_INLINE double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace rcmps
