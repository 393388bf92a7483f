// C ABI of the library: context, settings, workspace planning and the entry points of
// include/rcmps_b200.h. Host code only orchestrates device work; no arithmetic of the
// evaluation runs on the host.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <future>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "../../include/rcmps_b200.h"
#include "common.cuh"
#include "context.h"
#include "prep.h"
#include "kinetic_host.h"
#include "quartic.h"
#include "solvers_host.h"
#include "trajectory.h"

namespace rcmps {

static std::atomic<long long> g_launches{0};
// launches of this host thread (a graph capture counts the kernels it records)
static thread_local long long t_launches = 0;
void note_launch() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  ++t_launches;
}
void note_launches(long long count) { g_launches.fetch_add(count, std::memory_order_relaxed); }
long long thread_launch_count() { return t_launches; }

cudaError_t arena_reserve(rcmps_slot& sl, size_t bytes) {
  if (bytes <= sl.arena_bytes) return cudaSuccess;
  if (sl.arena) {
    cudaError_t e = cudaStreamSynchronize(sl.stream);
    if (e != cudaSuccess) return e;
    cudaFree(sl.arena);
    sl.arena = nullptr;
    sl.arena_bytes = 0;
  }
  const size_t want = align256(bytes + bytes / 8);
  cudaError_t e = cudaMalloc(&sl.arena, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    e = cudaMalloc(&sl.arena, align256(bytes));
    if (e != cudaSuccess) {
      cudaGetLastError();
      sl.arena = nullptr;
      return e;
    }
    sl.arena_bytes = align256(bytes);
    return cudaSuccess;
  }
  sl.arena_bytes = want;
  return cudaSuccess;
}

cudaError_t pinned_reserve(rcmps_slot& sl, size_t bytes) {
  if (bytes <= sl.pinned_bytes) return cudaSuccess;
  if (sl.pinned) {
    cudaStreamSynchronize(sl.stream);
    cudaFreeHost(sl.pinned);
  }
  sl.pinned = nullptr;
  sl.pinned_bytes = 0;
  cudaError_t e = cudaMallocHost(&sl.pinned, bytes);
  if (e == cudaSuccess) sl.pinned_bytes = bytes;
  return e;
}

cudaError_t aux_reserve(rcmps_context* ctx, size_t bytes) {
  if (bytes <= ctx->aux_bytes) return cudaSuccess;
  for (auto& sl : ctx->slot) cudaStreamSynchronize(sl.stream);
  if (ctx->aux) cudaFree(ctx->aux);
  ctx->aux = nullptr;
  ctx->aux_bytes = 0;
  cudaError_t e = cudaMalloc(&ctx->aux, align256(bytes));
  if (e == cudaSuccess) ctx->aux_bytes = align256(bytes);
  else cudaGetLastError();
  return e;
}

cudaError_t host_io_reserve(rcmps_context* ctx, size_t bytes) {
  if (bytes <= ctx->host_io_bytes) return cudaSuccess;
  for (auto& sl : ctx->slot) cudaStreamSynchronize(sl.stream);
  if (ctx->host_io) cudaFree(ctx->host_io);
  ctx->host_io = nullptr;
  ctx->host_io_bytes = 0;
  cudaError_t e = cudaMalloc(&ctx->host_io, align256(bytes));
  if (e == cudaSuccess) ctx->host_io_bytes = align256(bytes);
  else cudaGetLastError();
  return e;
}

int fail(rcmps_context* ctx, int code, const std::string& message) {
  if (ctx) {
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->error = message;
  }
  return code;
}

int padded_dim(int d) {
  if (d < 1) return 0;
  if (d <= 16) return 16;
  if (d <= 32) return 32;
  if (d <= 48) return 48;
  if (d <= 64) return 64;
  if (d <= 96) return 96;
  if (d <= 128) return 128;
  return 0;
}

// Gauss-Legendre nodes and weights on [-1, 1] by Newton's method on the Legendre recurrence.
static void gauss_legendre_compute(int n, std::vector<double>& x, std::vector<double>& w);

// Gauss-Legendre nodes and weights on [-1, 1], computed once per n and kept (the Newton iteration
// costs tens of milliseconds at n = 512, and every call of the library needs the same rules).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  static std::mutex mu;
  static std::map<int, std::pair<std::vector<double>, std::vector<double>>> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(n);
  if (it == cache.end()) {
    std::vector<double> cx, cw;
    gauss_legendre_compute(n, cx, cw);
    it = cache.emplace(n, std::make_pair(std::move(cx), std::move(cw))).first;
  }
  x = it->second.first;
  w = it->second.second;
}

static void gauss_legendre_compute(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(pi * (i + 0.75) / (n + 0.5));
    double dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = 0.0;
      for (int j = 1; j <= n; ++j) {
        const double p2 = p1;
        p1 = p0;
        p0 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p2) / j;
      }
      dp = n * (z * p0 - p1) / (z * z - 1.0);
      const double dz = p0 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-17) {
        // one more evaluation at the converged node for the weight
        p0 = 1.0;
        p1 = 0.0;
        for (int j = 1; j <= n; ++j) {
          const double p2 = p1;
          p1 = p0;
          p0 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p2) / j;
        }
        dp = n * (z * p0 - p1) / (z * z - 1.0);
        break;
      }
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

// Points of the quartic trajectory: the 2 n_quad Gauss nodes in t (ascending) and the endpoint
// sqrt(W) (ode_backend.py:37-44 and persistent_trajectory_backend.py:450-451); weights of the nodes.
void trajectory_points(double half_window, int n_quad, std::vector<double>& points, std::vector<double>& weights) {
  std::vector<double> x, w;
  gauss_legendre(n_quad, x, w);
  const double half = std::sqrt(half_window) / 2.0;
  points.resize(2 * n_quad + 1);
  weights.resize(2 * n_quad);
  for (int i = 0; i < n_quad; ++i) {
    const double p = (x[i] + 1.0) * half, q = w[i] * half;
    points[n_quad - 1 - i] = -p;
    weights[n_quad - 1 - i] = q;
    points[n_quad + i] = p;
    weights[n_quad + i] = q;
  }
  points[2 * n_quad] = std::sqrt(half_window);
}

int check_settings(rcmps_context* ctx, const rcmps_settings* s) {
  if (!s) return fail(ctx, RCMPS_INVALID_ARGUMENT, "settings is NULL");
  if (!(s->half_window > 0.0 && s->half_window <= 40.0))
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "half_window must be in (0, 40] (the source table covers |t| <= sqrt(40))");
  if (s->n_quad < 8) return fail(ctx, RCMPS_INVALID_ARGUMENT, "n_quad must be >= 8");
  if (!(s->atol > 0.0) || !(s->rtol >= 100 * 2.220446049250313e-16) || s->max_steps < 1)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "invalid ODE controls (atol > 0, rtol >= 100 eps, max_steps >= 1)");
  if (!(s->initial_step > 0.0) || !std::isfinite(s->initial_step))
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "initial_step must be positive");
  if (!(s->max_device_seconds >= 0.0)) return fail(ctx, RCMPS_INVALID_ARGUMENT, "max_device_seconds must be >= 0");
  if (s->symmetry < 0 || s->symmetry > 2)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "symmetry must be 0 (unpacked), 1 (packed Z2) or 2 (packed where Z2)");
  if (s->precision < 0 || s->precision > 1)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "precision must be 0 (FP64 tensor cores) or 1 (split BF16 slices)");
  if (s->trajectory_groups != 0 && s->trajectory_groups != 1 && s->trajectory_groups != 2 && s->trajectory_groups != 4)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "trajectory_groups must be 0 (automatic), 1, 2 or 4");
  if (s->boundary_preconditioner != 0 && s->boundary_preconditioner != 1)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "boundary_preconditioner must be 0 (none) or 1 (no-jump inverse)");
  return RCMPS_OK;
}

int check_dims(rcmps_context* ctx, int n, const int* dims) {
  if (n < 0) return fail(ctx, RCMPS_INVALID_ARGUMENT, "n_states must be >= 0");
  if (n > 0 && !dims) return fail(ctx, RCMPS_INVALID_ARGUMENT, "dims is NULL");
  for (int i = 0; i < n; ++i)
    if (padded_dim(dims[i]) == 0)
      return fail(ctx, RCMPS_INVALID_ARGUMENT,
                  "bond dimension " + std::to_string(dims[i]) + " of state " + std::to_string(i) +
                      " is outside 1..128");
  return RCMPS_OK;
}

// energy = vq + vk; covector = cq + ck; environment = eq + ek (packed arrays of `total` complex values);
// a NULL output is skipped
__global__ void sum_parts_kernel(int n, long long total, const double* vq, const double* vk, const double2* cq,
                                 const double2* ck, const double2* eq, const double2* ek, double* energy,
                                 double2* cov, double2* env) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n && energy) energy[i] = vq[i] + vk[i];
  for (long long e = i; e < total; e += (long long)gridDim.x * blockDim.x) {
    if (cov) cov[e] = zadd(cq[e], ck[e]);
    if (env) env[e] = zadd(eq[e], ek[e]);
  }
}

// FP64 tensor-core throughput: an in-register chain of independent mma.sync m16n8k8 per warp.
__global__ void fp64_peak_kernel(double* out, int iters) {
  double a[4], b[2], c[8][4];
  for (int j = 0; j < 4; ++j) a[j] = 1e-3 * (threadIdx.x + j);
  b[0] = 1.0;
  b[1] = 0.5;
  for (int t = 0; t < 8; ++t)
    for (int j = 0; j < 4; ++j) c[t][j] = 0.0;
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int t = 0; t < 8; ++t) dmma16x8x8(c[t], a, b);
  double s = 0.0;
  for (int t = 0; t < 8; ++t)
    for (int j = 0; j < 4; ++j) s += c[t][j];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace rcmps

using namespace rcmps;

// The solves run on the context's solve stream (slot 2), ordered after the caller's earlier work
// on `stream` and before its later work, so that their GMRES restart cycles can be captured as
// CUDA graphs whatever stream the caller passes (the legacy default stream cannot be captured).
// stream == NULL: the context's stream itself, no ordering.
static cudaStream_t solve_stream_enter(rcmps_context* ctx, void* stream) {
  cudaStream_t s2 = ctx->slot[2].stream;
  if (stream) {
    cudaEventRecord(ctx->slot[2].ev[3], static_cast<cudaStream_t>(stream));
    cudaStreamWaitEvent(s2, ctx->slot[2].ev[3], 0);
  }
  return s2;
}
static int solve_stream_leave(rcmps_context* ctx, void* stream, int rc) {
  if (stream) {
    cudaEventRecord(ctx->slot[2].ev[3], ctx->slot[2].stream);
    cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), ctx->slot[2].ev[3], 0);
  }
  return rc;
}

extern "C" {

void rcmps_default_settings(rcmps_settings* s) {
  if (!s) return;
  s->half_window = 30.0;
  s->n_quad = 512;
  s->atol = 1e-13;
  s->rtol = 1e-12;
  s->initial_step = 0.01;
  s->max_steps = 1000000;
  s->max_device_seconds = 30.0;
  s->kinetic_nodes = 512;
  s->krylov_tolerance = 1e-12;
  s->krylov_initialdim = 16;
  s->krylov_maxdim = 1024;
  s->metric_reg = 1e-3;
  s->boundary_tolerance = 1e-13;
  s->symmetry = 0;
  s->precision = 0;
  s->trajectory_groups = 0;
  s->boundary_preconditioner = 1;
}

int rcmps_context_create(int device, rcmps_context** out) {
  if (!out) return RCMPS_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return RCMPS_CUDA_ERROR;
  }
  rcmps_context* ctx = new rcmps_context();
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
  for (auto& sl : ctx->slot) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
    for (auto& ev : sl.ev)
      if (e == cudaSuccess) e = cudaEventCreate(&ev);
  }
  ctx->stream = ctx->slot[0].stream;
  if (e == cudaSuccess) e = trajectory_set_tables();
  if (e == cudaSuccess) e = quartic_init();
  if (e != cudaSuccess) {
    rcmps_context_destroy(ctx);
    return RCMPS_CUDA_ERROR;
  }
  ctx->tables = true;
  *out = ctx;
  return RCMPS_OK;
}

int rcmps_context_destroy(rcmps_context* ctx) {
  if (!ctx) return RCMPS_OK;
  cudaSetDevice(ctx->device);
  for (auto& sl : ctx->slot) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.arena) cudaFree(sl.arena);
    if (sl.pinned) cudaFreeHost(sl.pinned);
    for (auto& ev : sl.ev)
      if (ev) cudaEventDestroy(ev);
    if (sl.stream) cudaStreamDestroy(sl.stream);
  }
  if (ctx->aux) cudaFree(ctx->aux);
  if (ctx->host_io) cudaFree(ctx->host_io);
  for (auto& g : ctx->gmres_graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  delete ctx;
  return RCMPS_OK;
}

const char* rcmps_context_error(const rcmps_context* ctx) { return ctx ? ctx->error.c_str() : "no context"; }

const char* rcmps_status_name(int s) {
  switch (s) {
    case RCMPS_OK: return "success";
    case RCMPS_MAX_STEPS: return "max_steps";
    case RCMPS_STEP_UNDERFLOW: return "step_underflow";
    case RCMPS_NONFINITE_ERROR: return "nonfinite_error";
    case RCMPS_SOURCE_DOMAIN: return "source_domain";
    case RCMPS_MISSING_SAMPLES: return "missing_samples";
    case RCMPS_DEVICE_TIMEOUT: return "device_clock_timeout";
    case RCMPS_WAIT_LIMIT: return "wait_limit";
    case RCMPS_KRYLOV_FAILURE: return "krylov_failure";
    case RCMPS_SOLVE_FAILURE: return "solve_failure";
    case RCMPS_NONFINITE_RESULT: return "nonfinite_result";
    case RCMPS_INVALID_ARGUMENT: return "invalid_argument";
    case RCMPS_CUDA_ERROR: return "cuda_error";
    case RCMPS_OUT_OF_MEMORY: return "out_of_memory";
    default: return "unknown";
  }
}

int rcmps_last_timings(const rcmps_context* ctx, float* ms, int n) {
  if (!ctx || !ms) return RCMPS_INVALID_ARGUMENT;
  for (int i = 0; i < n && i < 8; ++i) ms[i] = ctx->last_ms[i];
  return RCMPS_OK;
}

int rcmps_quartic_samples(rcmps_context* ctx, int d, const double* R, const double* K, const double* rho,
                          const rcmps_settings* settings, double* samples, rcmps_state_stats* stats,
                          void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_settings(ctx, settings);
  if (rc) return rc;
  rc = check_dims(ctx, 1, &d);
  if (rc) return rc;
  if (!R || !K || !rho || !samples) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL matrix pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->slot[0].stream;
  QuarticJob job;
  job.n = 1;
  job.dims = &d;
  job.R = R;
  job.K = K;
  job.rho = rho;
  job.settings = *settings;
  job.samples_out = samples;
  rcmps_state_stats st;
  std::memset(&st, 0, sizeof(st));
  if (stats) std::memset(stats, 0, sizeof(*stats));
  job.stats = stats ? stats : &st;
  return quartic_run(ctx, job, s);
}

int rcmps_quartic_batch(rcmps_context* ctx, int n, const int* dims, const double* couplings, const double* R,
                        const double* K, const double* rho, const rcmps_settings* settings, double* value,
                        double* covector, double* environment, rcmps_state_stats* stats, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_settings(ctx, settings);
  if (rc) return rc;
  rc = check_dims(ctx, n, dims);
  if (rc) return rc;
  if (n == 0) return RCMPS_OK;
  if (!R || !K || !rho || !stats) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  for (int i = 0; i < n; ++i) std::memset(&stats[i], 0, sizeof(rcmps_state_stats));
  QuarticJob job;
  job.n = n;
  job.dims = dims;
  job.couplings = couplings;
  job.R = R;
  job.K = K;
  job.rho = rho;
  job.settings = *settings;
  job.value = value;
  job.covector = covector;
  job.environment = environment;
  job.stats = stats;
  return quartic_run(ctx, job, s);
}

int rcmps_phi4_ode_batch(rcmps_context* ctx, int n, const int* dims, const double* couplings, const double* R,
                         const double* K, const double* rho, const rcmps_settings* settings, double* value,
                         double* covector, double* environment, rcmps_state_stats* stats, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_settings(ctx, settings);
  if (rc) return rc;
  rc = check_dims(ctx, n, dims);
  if (rc) return rc;
  if (n == 0) return RCMPS_OK;
  if (!R || !K || !rho || !stats) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  for (int i = 0; i < n; ++i) std::memset(&stats[i], 0, sizeof(rcmps_state_stats));
  QuarticJob job;
  job.system = 1;
  job.n = n;
  job.dims = dims;
  job.couplings = couplings;
  job.R = R;
  job.K = K;
  job.rho = rho;
  job.settings = *settings;
  job.value = value;
  job.covector = covector;
  job.environment = environment;
  job.stats = stats;
  return quartic_run(ctx, job, s);
}

int rcmps_phi_ode_batch(rcmps_context* ctx, int n, const int* dims, const double* R, const double* K,
                        const double* rho, const rcmps_settings* settings, double* phi, rcmps_state_stats* stats,
                        void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_settings(ctx, settings);
  if (rc) return rc;
  rc = check_dims(ctx, n, dims);
  if (rc) return rc;
  if (n == 0) return RCMPS_OK;
  if (!R || !K || !rho || !phi || !stats) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  for (int i = 0; i < n; ++i) std::memset(&stats[i], 0, sizeof(rcmps_state_stats));
  QuarticJob job;
  job.system = 2;
  job.n = n;
  job.dims = dims;
  job.R = R;
  job.K = K;
  job.rho = rho;
  job.settings = *settings;
  job.settings.symmetry = 0;   // the packed route is the quartic term's only
  job.value = phi;
  job.stats = stats;
  return quartic_run(ctx, job, s);
}

int rcmps_kinetic_batch(rcmps_context* ctx, int n, const int* dims, const double* R, const double* K,
                        const double* rho, const rcmps_settings* settings, double* value, double* covector,
                        double* environment, rcmps_state_stats* stats, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_settings(ctx, settings);
  if (rc) return rc;
  rc = check_dims(ctx, n, dims);
  if (rc) return rc;
  if (n == 0) return RCMPS_OK;
  if (!R || !K || !rho || !stats) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  for (int i = 0; i < n; ++i) std::memset(&stats[i], 0, sizeof(rcmps_state_stats));
  KineticJob job;
  job.n = n;
  job.dims = dims;
  job.R = R;
  job.K = K;
  job.rho = rho;
  job.settings = *settings;
  job.value = value;
  job.covector = covector;
  job.environment = environment;
  job.stats = stats;
  rc = kinetic_run(ctx, job, s);
  return rc;
}

int rcmps_finish_gradient_batch(rcmps_context* ctx, int n, const int* dims, const double* R, const double* K,
                                const double* rho, const double* covector, const double* environment,
                                const rcmps_settings* settings, double* gradient, rcmps_state_stats* stats,
                                void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_settings(ctx, settings);
  if (rc) return rc;
  rc = check_dims(ctx, n, dims);
  if (rc) return rc;
  if (n == 0) return RCMPS_OK;
  if (!R || !K || !rho || !covector || !environment || !gradient || !stats)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = solve_stream_enter(ctx, stream);
  for (int i = 0; i < n; ++i) std::memset(&stats[i], 0, sizeof(rcmps_state_stats));
  FinishJob job;
  job.n = n;
  job.dims = dims;
  job.R = R;
  job.K = K;
  job.rho = rho;
  job.covector = covector;
  job.environment = environment;
  job.settings = *settings;
  job.gradient = gradient;
  job.stats = stats;
  return solve_stream_leave(ctx, stream, finish_run(ctx, job, s));
}

// restart cycles of the learned-preconditioner pass of the boundary solve before the fallback
constexpr int kLearnedRestarts = 8;

int rcmps_boundary_environment_batch(rcmps_context* ctx, int n, const int* dims, const double* R, const double* K,
                                     const double* rho, const double* environment, const double* x0,
                                     const rcmps_gmres_network* network, const rcmps_settings* settings, double* H,
                                     rcmps_state_stats* stats, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_settings(ctx, settings);
  if (rc) return rc;
  rc = check_dims(ctx, n, dims);
  if (rc) return rc;
  if (n == 0) return RCMPS_OK;
  if (!R || !K || !rho || !environment || !H || !stats) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  if (network) {
    if (!network->W1 || !network->W2 || network->rank < 1 || network->rank > 32768 || !std::isfinite(network->identity))
      return fail(ctx, RCMPS_INVALID_ARGUMENT, "network: weights, 1 <= rank <= 32768, finite identity");
    for (int i = 0; i < n; ++i)
      if (2 * dims[i] * dims[i] != network->n)
        return fail(ctx, RCMPS_INVALID_ARGUMENT, "network: every state needs 2 d^2 = n (state " + std::to_string(i) + ")");
  }
  cudaSetDevice(ctx->device);
  for (int i = 0; i < n; ++i) std::memset(&stats[i], 0, sizeof(rcmps_state_stats));
  FinishJob job;
  job.n = n;
  job.dims = dims;
  job.R = R;
  job.K = K;
  job.rho = rho;
  job.environment = environment;
  job.x0 = x0;
  job.net = network;
  job.settings = *settings;
  job.stats = stats;
  job.slot = 2;
  cudaStream_t s2 = solve_stream_enter(ctx, stream);
  if (!network) return solve_stream_leave(ctx, stream, boundary_run(ctx, job, H, s2));
  // the learned preconditioner first, for a few restart cycles; unpreconditioned GMRES is the
  // fallback: every state that did not converge is solved again from where the first pass left it
  job.max_restarts = kLearnedRestarts;
  rc = boundary_run(ctx, job, H, s2);
  if (rc == RCMPS_SOLVE_FAILURE) {
    std::vector<rcmps_state_stats> first(stats, stats + n);
    for (int i = 0; i < n; ++i) std::memset(&stats[i], 0, sizeof(rcmps_state_stats));
    job.net = nullptr;
    job.x0 = H;
    job.max_restarts = 200;
    rc = boundary_run(ctx, job, H, s2);
    for (int i = 0; i < n; ++i) stats[i].gmres_iterations += first[i].gmres_iterations;
  }
  return solve_stream_leave(ctx, stream, rc);
}

int rcmps_stationary_state_batch(rcmps_context* ctx, int n, const int* dims, const double* R, const double* K,
                                 double tolerance, double* rho, rcmps_state_stats* stats, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_dims(ctx, n, dims);
  if (rc) return rc;
  if (n == 0) return RCMPS_OK;
  if (!R || !K || !rho || !stats) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = solve_stream_enter(ctx, stream);
  for (int i = 0; i < n; ++i) std::memset(&stats[i], 0, sizeof(rcmps_state_stats));
  StationaryJob job;
  job.n = n;
  job.dims = dims;
  job.R = R;
  job.K = K;
  job.tolerance = tolerance;
  job.rho = rho;
  job.stats = stats;
  return solve_stream_leave(ctx, stream, stationary_run(ctx, job, s));
}

int rcmps_stationary_correction_batch(rcmps_context* ctx, int n, const int* dims, const double* R,
                                      const double* K, const double* rho_previous, double tolerance, double* rho,
                                      rcmps_state_stats* stats, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_dims(ctx, n, dims);
  if (rc) return rc;
  if (n == 0) return RCMPS_OK;
  if (!R || !K || !rho_previous || !rho || !stats) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t s = solve_stream_enter(ctx, stream);
  for (int i = 0; i < n; ++i) std::memset(&stats[i], 0, sizeof(rcmps_state_stats));
  StationaryJob job;
  job.n = n;
  job.dims = dims;
  job.R = R;
  job.K = K;
  job.tolerance = tolerance;
  job.rho = rho;
  job.rho_previous = rho_previous;
  job.stats = stats;
  return solve_stream_leave(ctx, stream, stationary_run(ctx, job, s));
}

// SMs the quartic pullback leaves free for the boundary solve that overlaps it
constexpr int kBoundarySMs = 32;

int rcmps_fg_phi4_batch(rcmps_context* ctx, int n, const int* dims, const double* couplings, const double* R,
                        const double* K, const double* rho, const rcmps_settings* settings, double* energy,
                        double* gradient, double* covector, double* environment, rcmps_state_stats* stats,
                        void* stream) {
  return rcmps_fg_phi4_batch_controls(ctx, n, dims, couplings, R, K, rho, settings, nullptr, energy, gradient,
                                      covector, environment, stats, stream);
}

int rcmps_fg_phi4_batch_controls(rcmps_context* ctx, int n, const int* dims, const double* couplings,
                                 const double* R, const double* K, const double* rho,
                                 const rcmps_settings* settings, const rcmps_state_controls* controls,
                                 double* energy, double* gradient, double* covector, double* environment,
                                 rcmps_state_stats* stats, void* stream) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_settings(ctx, settings);
  if (rc) return rc;
  rc = check_dims(ctx, n, dims);
  if (rc) return rc;
  for (int i = 0; controls && i < n; ++i) {
    const double at = controls[i].atol > 0.0 ? controls[i].atol : settings->atol;
    const double rt = controls[i].rtol > 0.0 ? controls[i].rtol : settings->rtol;
    if (!std::isfinite(at) || !std::isfinite(rt) || !(rt >= 100 * 2.220446049250313e-16))
      return fail(ctx, RCMPS_INVALID_ARGUMENT,
                  "controls[" + std::to_string(i) + "]: atol > 0 and rtol >= 100 eps, both finite");
  }
  if (n == 0) return RCMPS_OK;
  if (!R || !K || !rho || !energy || !gradient || !stats || !couplings)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  long long total = 0;
  for (int i = 0; i < n; ++i) total += (long long)dims[i] * dims[i];
  // aux: vq, vk [n]; cq, ck, eq, ek, cov, env [total complex]
  const size_t vbytes = align256((size_t)n * 8), cbytes = align256((size_t)total * 16);
  if (aux_reserve(ctx, 2 * vbytes + 6 * cbytes) != cudaSuccess)
    return fail(ctx, RCMPS_OUT_OF_MEMORY, "fg_phi4 intermediate buffers");
  char* a = static_cast<char*>(ctx->aux);
  double* vq = (double*)a;
  double* vk = (double*)(a + vbytes);
  double* cq = (double*)(a + 2 * vbytes);
  double* ck = (double*)(a + 2 * vbytes + cbytes);
  double* eq = (double*)(a + 2 * vbytes + 2 * cbytes);
  double* ek = (double*)(a + 2 * vbytes + 3 * cbytes);
  double* csum = covector ? covector : (double*)(a + 2 * vbytes + 4 * cbytes);
  double* esum = environment ? environment : (double*)(a + 2 * vbytes + 5 * cbytes);
  // the inputs are ordered on the caller's stream
  cudaStream_t cs = stream ? static_cast<cudaStream_t>(stream) : nullptr;
  cudaEvent_t ready = ctx->slot[2].ev[3];
  cudaEventRecord(ready, cs);
  for (auto& sl : ctx->slot) cudaStreamWaitEvent(sl.stream, ready, 0);
  cudaEventRecord(ctx->slot[2].ev[0], ctx->slot[0].stream);
  for (int i = 0; i < n; ++i) std::memset(&stats[i], 0, sizeof(rcmps_state_stats));
  std::vector<rcmps_state_stats> kst(n);
  std::memset(kst.data(), 0, n * sizeof(rcmps_state_stats));
  QuarticJob qj;
  qj.n = n;
  qj.dims = dims;
  qj.couplings = couplings;
  qj.R = R;
  qj.K = K;
  qj.rho = rho;
  qj.settings = *settings;
  qj.controls = controls;
  qj.value = vq;
  qj.covector = cq;
  qj.environment = eq;
  qj.stats = stats;
  qj.slot = 0;
  qj.memory_share = 0.4;
  KineticJob kj;
  kj.n = n;
  kj.dims = dims;
  kj.R = R;
  kj.K = K;
  kj.rho = rho;
  kj.settings = *settings;
  kj.value = vk;
  kj.covector = ck;
  kj.environment = ek;
  kj.stats = kst.data();
  kj.slot = 1;
  kj.memory_share = 0.3;
  // The kinetic term runs on its own thread and stream, the quartic term on another. The boundary
  // solve needs only the environment, which the quartic term writes right after its trajectory:
  // the solve starts then and runs while the quartic pullback produces the covector.
  int krc = RCMPS_OK, qrc = RCMPS_OK;
  std::promise<bool> env_promise;
  std::future<bool> env_future = env_promise.get_future();
  bool env_signalled = false;
  qj.env_ready = ctx->slot[0].ev[3];
  // the pullback leaves SMs to the boundary solve that runs beside it
  qj.pullback_ctas = std::max(1, ctx->sms - kBoundarySMs);
  qj.on_env = [&] {
    env_signalled = true;
    env_promise.set_value(true);
  };
  std::thread kworker([&] {
    cudaSetDevice(ctx->device);
    krc = kinetic_run(ctx, kj, ctx->slot[1].stream);
  });
  std::thread qworker([&] {
    cudaSetDevice(ctx->device);
    qrc = quartic_run(ctx, qj, ctx->slot[0].stream);
    if (!env_signalled) env_promise.set_value(false);
  });
  cudaStream_t s2 = ctx->slot[2].stream;
  const int nsum = (int)std::min<long long>(4096, (total + 255) / 256 + 1);
  std::vector<rcmps_state_stats> fst(n);
  std::memset(fst.data(), 0, n * sizeof(rcmps_state_stats));
  FinishJob fj;
  fj.n = n;
  fj.dims = dims;
  fj.R = R;
  fj.K = K;
  fj.rho = rho;
  fj.covector = csum;
  fj.environment = esum;
  fj.settings = *settings;
  fj.gradient = gradient;
  fj.stats = fst.data();
  fj.slot = 2;
  FinishPlan plan;
  // the solve's operators and the no-jump preconditioner's eigenbasis need only R, K and rho:
  // they are prepared on the solve stream while the two terms run
  cudaEventRecord(ctx->slot[2].ev[4], s2);
  int frc = finish_prepare(ctx, fj, s2, plan);
  cudaEventRecord(ctx->slot[2].ev[5], s2);
  kworker.join();
  const bool env_ok = env_future.get();
  const bool solve = env_ok && krc == RCMPS_OK && frc == RCMPS_OK;
  if (solve) {
    cudaStreamWaitEvent(s2, qj.env_ready, 0);
    cudaEventRecord(ctx->slot[2].ev[1], s2);
    note_launch();
    sum_parts_kernel<<<nsum, 256, 0, s2>>>(n, total, vq, vk, (double2*)cq, (double2*)ck, (double2*)eq, (double2*)ek,
                                           nullptr, nullptr, (double2*)esum);
    frc = finish_solve(ctx, fj, s2, plan);
    cudaEventRecord(ctx->slot[2].ev[6], s2);
  }
  qworker.join();
  for (int i = 0; i < n; ++i) {
    stats[i].kinetic_value = kst[i].kinetic_value;
    for (int q = 0; q < 4; ++q) stats[i].krylov_basis[q] = kst[i].krylov_basis[q];
    stats[i].krylov_residual = kst[i].krylov_residual;
    if (!stats[i].status && kst[i].status) {
      stats[i].status = kst[i].status;
      stats[i].failed_component = kst[i].failed_component;
    }
  }
  if (qrc || krc) return qrc ? qrc : krc;
  if (frc) return frc;
  if (!solve) return fail(ctx, RCMPS_CUDA_ERROR, "fg_phi4: the quartic environment was not produced");
  if (frc == RCMPS_OK) {
    note_launch();
    sum_parts_kernel<<<nsum, 256, 0, s2>>>(n, total, vq, vk, (double2*)cq, (double2*)ck, (double2*)eq,
                                           (double2*)ek, energy, (double2*)csum, nullptr);
    cudaStreamWaitEvent(s2, ctx->slot[0].ev[2], 0);   // the covector is complete with the pullback
    frc = finish_complete(ctx, fj, s2, plan);
  }
  cudaEventRecord(ctx->slot[2].ev[2], s2);
  cudaEventSynchronize(ctx->slot[2].ev[2]);
  cudaEventElapsedTime(&ctx->last_ms[3], ctx->slot[2].ev[1], ctx->slot[2].ev[2]);
  cudaEventElapsedTime(&ctx->last_ms[4], ctx->slot[2].ev[0], ctx->slot[2].ev[2]);
  cudaEventElapsedTime(&ctx->last_ms[5], ctx->slot[2].ev[4], ctx->slot[2].ev[5]);
  cudaEventElapsedTime(&ctx->last_ms[6], ctx->slot[2].ev[1], ctx->slot[2].ev[6]);
  for (int i = 0; i < n; ++i) {
    stats[i].gmres_iterations = fst[i].gmres_iterations;
    stats[i].gmres_matvecs = fst[i].gmres_matvecs;
    stats[i].boundary_residual = fst[i].boundary_residual;
    if (!stats[i].status && fst[i].status) {
      stats[i].status = fst[i].status;
      stats[i].failed_component = fst[i].failed_component;
    }
  }
  // the results are complete on the caller's stream too
  cudaEventRecord(ready, s2);
  cudaStreamWaitEvent(cs, ready, 0);
  return frc;
}

int rcmps_fg_phi4_batch_host(rcmps_context* ctx, int n, const int* dims, const double* couplings, const double* R,
                             const double* K, const double* rho, const rcmps_settings* settings, double* energy,
                             double* gradient, double* covector, double* environment, rcmps_state_stats* stats) {
  if (!ctx) return RCMPS_INVALID_ARGUMENT;
  int rc = check_dims(ctx, n, dims);
  if (rc) return rc;
  if (n == 0) return RCMPS_OK;
  if (!R || !K || !rho || !energy || !gradient) return fail(ctx, RCMPS_INVALID_ARGUMENT, "NULL pointer");
  cudaSetDevice(ctx->device);
  long long total = 0;
  for (int i = 0; i < n; ++i) total += (long long)dims[i] * dims[i];
  const size_t cb = (size_t)total * 16;
  // device copies of inputs and outputs in a grow-only buffer of the context (reused by later
  // calls of the same or smaller size)
  cudaError_t e = host_io_reserve(ctx, 6 * cb + (size_t)n * 8 + 256);
  if (e) return fail(ctx, RCMPS_OUT_OF_MEMORY, "host entry buffers");
  char* d = static_cast<char*>(ctx->host_io);
  double *dR = (double*)d, *dK = (double*)(d + cb), *dP = (double*)(d + 2 * cb), *dG = (double*)(d + 3 * cb),
         *dC = (double*)(d + 4 * cb), *dE = (double*)(d + 5 * cb), *dEn = (double*)(d + 6 * cb);
  cudaStream_t s = ctx->slot[0].stream;
  e = cudaMemcpyAsync(dR, R, cb, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(dK, K, cb, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(dP, rho, cb, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaStreamSynchronize(s);
  if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("host entry copies: ") + cudaGetErrorString(e));
  rc = rcmps_fg_phi4_batch(ctx, n, dims, couplings, dR, dK, dP, settings, dEn, dG, dC, dE, stats, s);
  if (!e) e = cudaMemcpyAsync(energy, dEn, (size_t)n * 8, cudaMemcpyDeviceToHost, s);
  if (!e) e = cudaMemcpyAsync(gradient, dG, cb, cudaMemcpyDeviceToHost, s);
  if (!e && covector) e = cudaMemcpyAsync(covector, dC, cb, cudaMemcpyDeviceToHost, s);
  if (!e && environment) e = cudaMemcpyAsync(environment, dE, cb, cudaMemcpyDeviceToHost, s);
  if (!e) e = cudaStreamSynchronize(s);
  if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("host entry copies: ") + cudaGetErrorString(e));
  return rc;
}

long long rcmps_workspace_bytes(const rcmps_context* ctx, int n, const int* dims, const rcmps_settings* settings) {
  if (!ctx || !dims || !settings || n < 0) return -1;
  long long total = 0;
  for (int i = 0; i < n; ++i) {
    const int dp = padded_dim(dims[i]);
    if (!dp) return -1;
    const long long mat = (long long)dp * dp * 16;
    const long long npoints = 2LL * settings->n_quad + 1;
    const int kmax = std::min(settings->krylov_maxdim, dims[i] * dims[i]);
    total += (npoints + 200) * 7 * mat;                                       // quartic
    total += 4 * ((kmax + 1) * mat + (long long)settings->kinetic_nodes * mat) + 64 * mat;   // kinetic
  }
  return total;
}

long long rcmps_launch_count(void) { return g_launches.load(); }

int rcmps_trajectory_tuning(const rcmps_context* ctx, int system, int dp, int* ring, float* ms) {
  if (!ctx || !ring || system < 0 || system > 2) return RCMPS_INVALID_ARGUMENT;
  int i = -1;
  const int dps[6] = {16, 32, 48, 64, 96, 128};
  for (int k = 0; k < 6; ++k)
    if (dps[k] == dp) i = k;
  if (i < 0) return RCMPS_INVALID_ARGUMENT;
  const int g = ctx->traj_groups[system][i], level = g == 4 ? 2 : g == 2 ? 1 : 0;
  *ring = ctx->traj_ring[system][i][level];
  for (int r = 0; ms && r < 3; ++r) ms[r] = ctx->traj_ring_ms[system][i][level][r];
  return RCMPS_OK;
}

int rcmps_trajectory_groups(const rcmps_context* ctx, int system, int dp, int* groups) {
  if (!ctx || !groups || system < 0 || system > 2) return RCMPS_INVALID_ARGUMENT;
  const int dps[6] = {16, 32, 48, 64, 96, 128};
  for (int k = 0; k < 6; ++k)
    if (dps[k] == dp) {
      *groups = ctx->traj_groups[system][k];
      return RCMPS_OK;
    }
  return RCMPS_INVALID_ARGUMENT;
}

double rcmps_fp64_peak_tflops(rcmps_context* ctx) {
  if (!ctx) return 0.0;
  cudaSetDevice(ctx->device);
  const int blocks = 2 * ctx->sms, threads = 256, iters = 4096;
  double* out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * threads * 8)) return 0.0;
  cudaStream_t s = ctx->slot[0].stream;
  note_launch();
  fp64_peak_kernel<<<blocks, threads, 0, s>>>(out, iters);   // warm-up
  cudaEventRecord(ctx->slot[0].ev[0], s);
  note_launch();
  fp64_peak_kernel<<<blocks, threads, 0, s>>>(out, iters);
  cudaEventRecord(ctx->slot[0].ev[1], s);
  cudaEventSynchronize(ctx->slot[0].ev[1]);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->slot[0].ev[0], ctx->slot[0].ev[1]);
  cudaFree(out);
  const double flops = 2.0 * 16 * 8 * 8 * 8.0 * iters * (double)blocks * (threads / 32);
  return ms > 0.f ? flops / (ms * 1e-3) / 1e12 : 0.0;
}

}  // extern "C"
