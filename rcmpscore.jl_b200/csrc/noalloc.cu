// Finish step (boundary Poisson correction + metric solve) for one state without any allocation.
//
// Why: some callers cannot allocate device memory at the moment they need the gradient. Examples
// are a host whose memory planner reserves every byte up front (an inference-style server, or a
// framework whose caching allocator owns the device), a plugin whose enqueue callback may not
// allocate, and a process running near its memory limit, where a cudaMalloc in the middle of an
// optimizer step would fail or stall. rcmps_finish_gradient_batch draws its workspace from the
// context's arena, which grows with cudaMalloc; this variant instead works entirely inside one
// fixed array that lives in the library's device image.
//
// The scratch array below is reserved on every GPU that loads the library, for as long as the
// process runs: kNoAllocBytes = 2 MiB. That bounds the supported size to one state with d <= 32.
// Every call uses the same array, so calls that overlap on the GPU (two streams, two host
// threads) race on it; the caller must order them. Whatever must start at zero (the GMRES
// solution, the status words) is cleared by each call; nothing else carries over.
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include "../../include/rcmps_b200.h"
#include "context.h"
#include "kinetic.h"
#include "prep.h"
#include "quartic.h"
#include "solvers.h"

namespace rcmps {

constexpr size_t kNoAllocBytes = size_t(2) << 20;   // 2 MiB of device scratch
constexpr int kNoAllocMaxD = 32;
constexpr int kNoAllocM = 64;                        // GMRES restart length, as the batched solve
constexpr int kNoAllocRestarts = 200;

// The scratch itself. Host code must not pass this name to a kernel: on the host it is only a
// stand-in, and its device address comes from cudaGetSymbolAddress (one lookup per device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {nullptr};

struct Bump {
  char* base;
  size_t used = 0;
  size_t cap;
  void* take(size_t bytes) {
    const size_t off = align256(used);
    if (off + bytes > cap) return nullptr;
    used = off + bytes;
    return base + off;
  }
};
}  // namespace

// Device address of the scratch array on the current device; looked up on the first call per
// device and kept for the life of the process (a cudaDeviceReset of that device would leave the
// kept address stale, which the header rules out). Every call synchronizes its stream, so no call
// may run inside a stream capture.
static cudaError_t noalloc_scratch(int device, char** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[device] = p;
  }
  *out = static_cast<char*>(g_noalloc_ptr[device]);
  return cudaSuccess;
}

}  // namespace rcmps

using namespace rcmps;

extern "C" int rcmps_finish_gradient_noalloc(rcmps_context* ctx, int d, const double* R, const double* K,
                                             const double* rho, const double* covector,
                                             const double* environment, const rcmps_settings* settings,
                                             double* gradient, rcmps_state_stats* stats, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  if (!settings || !R || !K || !rho || !covector || !environment || !gradient || !stats)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  if (d < 1 || d > kNoAllocMaxD)
    return fail(ctx, RCMPS_INVALID_ARGUMENT,
                "rcmps_finish_gradient_noalloc supports 1 <= d <= " + std::to_string(kNoAllocMaxD) +
                    " (its fixed scratch is " + std::to_string(kNoAllocBytes >> 20) + " MiB); d = " + std::to_string(d));
  const double tol = settings->boundary_tolerance;
  if (!(tol > 0.0) || !(settings->metric_reg >= 0.0))
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "invalid boundary controls");
  cudaError_t e = cudaSetDevice(ctx->device);
  char* base = nullptr;
  if (!e) e = noalloc_scratch(ctx->device, &base);
  if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("no-alloc scratch address: ") + cudaGetErrorString(e));
  std::memset(stats, 0, sizeof(*stats));
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->slot[2].stream;
  const int dp = padded_dim(d), m = kNoAllocM;   // 16 or 32, as the batched entry pads
  const size_t mat = (size_t)dp * dp;
  const int nchunk = (dp * dp + 511) / 512;
  Bump B{base, 0, kNoAllocBytes};
  int* d_dims = (int*)B.take(sizeof(int));
  long long* d_off = (long long*)B.take(sizeof(long long));
  double2* d_in = (double2*)B.take(5 * mat * 16);      // R, K, rho, covector, environment (padded)
  double2* d_ops = (double2*)B.take(8 * mat * 16);
  double2* d_b = (double2*)B.take(mat * 16);
  double2* d_tmp = (double2*)B.take(4 * mat * 16);
  int* d_status = (int*)B.take(sizeof(int));
  ArnoldiProblem* d_prob = (ArnoldiProblem*)B.take(sizeof(ArnoldiProblem));
  double2* V = (double2*)B.take((m + 1) * mat * 16);
  double2* Hm = (double2*)B.take((size_t)(m + 1) * m * 16);
  double2* W = (double2*)B.take(mat * 16);
  double2* part = (double2*)B.take((size_t)nchunk * (m + 1) * 16);
  double* norms = (double*)B.take(2 * nchunk * 8);
  double2* x = (double2*)B.take(mat * 16);
  double2* g = (double2*)B.take((m + 1) * 16);
  double2* cs = (double2*)B.take(m * 16);
  double2* sn = (double2*)B.take(m * 16);
  int* flag = (int*)B.take(sizeof(int));
  LindbladTask* task = (LindbladTask*)B.take(sizeof(LindbladTask));
  if (!task) return fail(ctx, RCMPS_OUT_OF_MEMORY, "no-alloc scratch layout exceeds its fixed size");

  // host staging from stack memory (no pinned allocation)
  int h_dims = d;
  long long h_off = 0;
  e = cudaMemcpyAsync(d_dims, &h_dims, sizeof(int), cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(d_off, &h_off, sizeof(long long), cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemsetAsync(d_status, 0, sizeof(int), s);
  if (!e) e = cudaMemsetAsync(flag, 0, sizeof(int), s);
  if (!e) e = cudaMemsetAsync(x, 0, mat * 16, s);
  double* dR = (double*)d_in;
  double* dK = (double*)(d_in + mat);
  double* dP = (double*)(d_in + 2 * mat);
  double* dC = (double*)(d_in + 3 * mat);
  double* dE = (double*)(d_in + 4 * mat);
  if (!e) e = launch_pad(R, d_off, d_dims, dR, dp, mat, 1, s);
  if (!e) e = launch_pad(K, d_off, d_dims, dK, dp, mat, 1, s);
  if (!e) e = launch_pad(rho, d_off, d_dims, dP, dp, mat, 1, s);
  if (!e) e = launch_pad(covector, d_off, d_dims, dC, dp, mat, 1, s);
  if (!e) e = launch_pad(environment, d_off, d_dims, dE, dp, mat, 1, s);
  if (!e) e = launch_prepare(dR, dK, dP, (double*)d_ops, dp, mat, 8 * mat, 1, s);
  FinishArgs fa;
  fa.dp = dp;
  fa.dims = d_dims;
  fa.ops = d_ops;
  fa.ops_stride = (long long)(8 * mat);
  fa.env = (double2*)dE;
  fa.cov = (double2*)dC;
  fa.b = d_b;
  fa.x = x;
  fa.tmp = d_tmp;
  fa.metric_reg = settings->metric_reg;
  fa.status = d_status;
  if (!e) e = boundary_rhs_launch(fa, 1, s);
  // the GMRES problem: -L*(X) + tr(rho X) I_d = b
  ArnoldiProblem A;
  std::memset(&A, 0, sizeof(A));
  A.V = V;
  A.ldv = (long long)mat;
  A.H = Hm;
  A.W = W;
  A.partial = part;
  A.norms = norms;
  A.x = x;
  A.g = g;
  A.cs = cs;
  A.sn = sn;
  A.flag = flag;
  A.n = dp * dp;
  A.n_phys = d * d;
  A.d = d;
  A.dp = dp;
  A.kmax = m;
  A.kmax1 = m + 1;
  A.target = m < d * d ? m : d * d;
  A.gtol = tol;
  A.bnorm = -1.0;
  A.A1 = d_ops + mat;
  A.A1h = d_ops;
  A.A2 = d_ops + 3 * mat;
  A.A2h = d_ops + 2 * mat;
  A.trw = d_ops + 7 * mat;
  A.b = d_b;
  if (!e) e = cudaMemcpyAsync(d_prob, &A, sizeof(A), cudaMemcpyHostToDevice, s);
  for (int it = 0; it <= kNoAllocRestarts && !e; ++it) {
    e = gmres_x_tasks_launch(d_prob, 1, task, s);
    if (!e) e = lindblad_launch(dp, task, 1, 0, s);
    if (!e) e = gmres_residual_launch(d_prob, 1, dp * dp, s);
    if (!e) e = cudaMemcpyAsync(&A, d_prob, sizeof(A), cudaMemcpyDeviceToHost, s);
    if (!e) e = cudaStreamSynchronize(s);
    if (e || A.converged || it == kNoAllocRestarts) break;
    for (int j = 0; j < m && !e; ++j) {
      e = arnoldi_tasks_launch(d_prob, 1, j, task, s);
      if (!e) e = lindblad_launch(dp, task, 1, 0, s);
      if (!e) e = cgs_step_launch(d_prob, 1, j, dp * dp, s);
      if (!e) e = gmres_givens_launch(d_prob, 1, j, s);
    }
    if (!e) e = gmres_update_launch(d_prob, 1, dp * dp, m, s);
  }
  if (!e) e = finish_launch(fa, 1, s);
  if (!e) e = launch_unpad_acc((double*)(d_tmp + 3 * mat), (long long)(4 * mat), dp, d_off, d_dims, gradient, 1,
                               false, s);
  int h_status = 0;
  if (!e) e = cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (!e) e = cudaStreamSynchronize(s);
  if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("no-alloc finish: ") + cudaGetErrorString(e));
  stats->gmres_iterations = A.iters;
  stats->gmres_matvecs = A.iters + A.restarts;
  stats->boundary_residual = A.residual;
  const bool ok = A.converged || A.residual <= 20.0 * tol * (A.bnorm > 1.0 ? A.bnorm : 1.0);
  if (A.nonfinite || !std::isfinite(A.residual) || !ok) {
    stats->status = RCMPS_SOLVE_FAILURE;
    stats->failed_component = 4;
  } else if (h_status) {
    stats->status = h_status;
    stats->failed_component = 4;
  }
  return stats->status;
}
