// Library context: device, streams and a grow-only device workspace (internal).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>

struct rcmps_context {
  int device = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;          // default work stream of the context
  cudaStream_t side = nullptr;            // second stream (kinetic work overlaps the quartic)
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  void* arena = nullptr;                  // workspace
  size_t arena_bytes = 0;
  void* pinned = nullptr;                 // small pinned host buffer for statuses
  size_t pinned_bytes = 0;
  std::string error;
  bool tables = false;
  float last_ms[8] = {0};                 // device times of the last call's phases
};

namespace rcmps {
// Ensure the arena holds at least `bytes`; returns a cudaError_t.
cudaError_t arena_reserve(rcmps_context* ctx, size_t bytes);
// Ensure the pinned host buffer holds at least `bytes`.
cudaError_t pinned_reserve(rcmps_context* ctx, size_t bytes);
int fail(rcmps_context* ctx, int code, const std::string& message);
inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
int padded_dim(int d);   // 16, 32, 48, 64, 96, 128, or 0 if d is unsupported
}  // namespace rcmps
