// C ABI of the library: context, settings, workspace planning and the entry points of
// include/rcmps_b200.h. Host code only orchestrates device work; no arithmetic of the
// evaluation runs on the host.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include "../../include/rcmps_b200.h"
#include "context.h"
#include "prep.h"
#include "kinetic_host.h"
#include "quartic.h"
#include "trajectory.h"

namespace rcmps {

cudaError_t arena_reserve(rcmps_context* ctx, size_t bytes) {
  if (bytes <= ctx->arena_bytes) return cudaSuccess;
  if (ctx->arena) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(ctx->side);
    if (e != cudaSuccess) return e;
    cudaFree(ctx->arena);
    ctx->arena = nullptr;
    ctx->arena_bytes = 0;
  }
  const size_t want = align256(bytes + bytes / 8);
  cudaError_t e = cudaMalloc(&ctx->arena, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    e = cudaMalloc(&ctx->arena, align256(bytes));
    if (e != cudaSuccess) {
      ctx->arena = nullptr;
      return e;
    }
    ctx->arena_bytes = align256(bytes);
    return cudaSuccess;
  }
  ctx->arena_bytes = want;
  return cudaSuccess;
}

cudaError_t pinned_reserve(rcmps_context* ctx, size_t bytes) {
  if (bytes <= ctx->pinned_bytes) return cudaSuccess;
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  ctx->pinned = nullptr;
  ctx->pinned_bytes = 0;
  cudaError_t e = cudaMallocHost(&ctx->pinned, bytes);
  if (e == cudaSuccess) ctx->pinned_bytes = bytes;
  return e;
}

int fail(rcmps_context* ctx, int code, const std::string& message) {
  if (ctx) ctx->error = message;
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
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
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

}  // namespace rcmps

using namespace rcmps;

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
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_a);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_b);
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
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->side) cudaStreamSynchronize(ctx->side);
  if (ctx->arena) cudaFree(ctx->arena);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->ev_a) cudaEventDestroy(ctx->ev_a);
  if (ctx->ev_b) cudaEventDestroy(ctx->ev_b);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->side) cudaStreamDestroy(ctx->side);
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
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
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
  cudaEventRecord(ctx->ev_a, s);
  rc = kinetic_run(ctx, job, s);
  cudaEventRecord(ctx->ev_b, s);
  cudaEventSynchronize(ctx->ev_b);
  cudaEventElapsedTime(&ctx->last_ms[2], ctx->ev_a, ctx->ev_b);
  return rc;
}

}  // extern "C"
