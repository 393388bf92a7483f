// Library context: device, streams and a grow-only device workspace (internal).
#pragma once
#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include <vector>

// One independent lane of work: its stream, device workspace, pinned staging buffer and events.
// Slot 0 runs the quartic term, slot 1 the kinetic terms (concurrently), slot 2 the solves.
struct rcmps_slot {
  cudaStream_t stream = nullptr;
  void* arena = nullptr;
  size_t arena_bytes = 0;
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  cudaEvent_t ev[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

// One restart cycle of the batched GMRES captured as a CUDA graph, for the problems and tasks at
// these device addresses and these sizes.
struct rcmps_gmres_graph {
  const void* probs = nullptr;
  const void* tasks = nullptr;
  int np = 0, dp = 0, m = 0;
  const void* net = nullptr;            // the learned preconditioner in the graph, if any: its weights,
  const void* net2 = nullptr;           // rank and identity weight (all baked into the kernels)
  int net_rank = 0;
  float net_identity = 0.f;
  const void* pre = nullptr;            // the no-jump preconditioner's sets, if any
  long long kernels = 0;                // kernels the graph replays
  cudaGraphExec_t exec = nullptr;
};

struct rcmps_context {
  int device = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;          // the caller-facing stream of the context (= slot 0)
  rcmps_slot slot[3];
  void* aux = nullptr;                    // per-call intermediate results of the composite entry
  size_t aux_bytes = 0;
  void* host_io = nullptr;                // device copies of the host-buffer entry's inputs and outputs
  size_t host_io_bytes = 0;
  rcmps_gmres_graph gmres_graphs[4];      // cached GMRES restart cycles (replaced in turn)
  int gmres_graph_next = 0;
  std::string error;
  std::mutex mu;                          // guards `error` (the composite entry runs two host threads)
  bool tables = false;
  float last_ms[8] = {0};                 // device times of the last call's phases
  // trajectory tile autotuning: the operand-ring depth chosen per (system, padded dimension,
  // channel-group level 1/2/4) after its first three launches, and the device ms per 1000
  // right-hand sides (of each launch's longest trajectory) those launches took at the depths 2,
  // 3, 4; the channel groups of the last launch per (system, padded dimension)
  int traj_ring[3][6][3] = {};
  float traj_ring_ms[3][6][3][3] = {};
  int traj_groups[3][6] = {};
};

namespace rcmps {
// Ensure slot `k` holds at least `bytes` of device workspace; returns a cudaError_t.
cudaError_t arena_reserve(rcmps_slot& slot, size_t bytes);
// Ensure slot `k` has at least `bytes` of pinned host staging.
cudaError_t pinned_reserve(rcmps_slot& slot, size_t bytes);
cudaError_t aux_reserve(rcmps_context* ctx, size_t bytes);
cudaError_t host_io_reserve(rcmps_context* ctx, size_t bytes);
int fail(rcmps_context* ctx, int code, const std::string& message);
void note_launches(long long count);   // kernels replayed by one graph launch
long long thread_launch_count();   // launches noted by the calling host thread
inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
int padded_dim(int d);   // 16, 32, 48, 64, 96, 128, or 0 if d is unsupported
}  // namespace rcmps
