// Host orchestration of the quartic term: states grouped by padded dimension, each group in
// sub-batches that fit the device workspace; per sub-batch: pad, prepare, one trajectory launch
// (all states co-scheduled), pullback, finalize, unpad.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include "../../include/rcmps_b200.h"
#include "context.h"
#include "prep.h"
#include "pullback.h"
#include "quartic.h"
#include "trajectory.h"

namespace rcmps {

cudaError_t quartic_init() { return cudaSuccess; }

namespace {

struct Layout {
  size_t total = 0;
  size_t add(size_t bytes) {
    const size_t off = total;
    total += align256(bytes);
    return off;
  }
};

constexpr int kNodesPerBlock = 32;

// Per-system sizes: channels of a stage vector, operator matrices, stage vectors of the
// trajectory workspace (y, prop, k[16], z[2], P, and L for the all-ODE route), pullback
// scratch, partial and finalize matrices per state.
struct SysSizes {
  int nch, nops, nwork;
  size_t wscr, part, fin;   // in dp x dp matrices per state
};
SysSizes sys_sizes(int system, int dp, int nblk) {
  SysSizes z;
  z.nch = trajectory_channels(system);
  if (system == 0) {
    z.nops = kOps;
    z.nwork = 21;
    z.wscr = (size_t)nblk * pullback_row_blocks(dp) * 3;
    z.part = (size_t)nblk * 4;
    z.fin = 8;
  } else if (system == 2) {   // <phi>: the trajectory and its endpoint only
    z.nops = kOps;
    z.nwork = 21;
    z.wscr = z.part = z.fin = 0;
  } else {
    z.nops = kOpsFull;
    z.nwork = 22;
    z.wscr = (size_t)nblk * pullback_full_row_blocks(dp) * kMaxPullSpecs * kMaxPullChannels;
    z.part = (size_t)kMaxPullSpecs * nblk * 6;
    z.fin = 10;
  }
  return z;
}

// The split-precision engine runs the quartic trajectory of the states of padded dimension 64
// when the settings ask for it.
bool split_engine_for(const rcmps_settings& S, int system, int dp) { return S.precision == 1 && system == 0 && dp == 64; }

size_t state_bytes(int system, int dp, int npoints, int nodes, bool split = false) {
  const size_t mat = (size_t)dp * dp * 16;
  const int nblk = (nodes + kNodesPerBlock - 1) / kNodesPerBlock;
  const SysSizes z = sys_sizes(system, dp, nblk);
  size_t b = 0;
  b += 3 * mat;                                 // padded R, K, rho
  b += z.nops * mat;                            // operators
  b += (size_t)z.nwork * z.nch * mat;           // trajectory workspace
  b += (size_t)npoints * z.nch * mat;           // samples
  b += (z.wscr + z.part + z.fin + 2) * mat;     // pullback scratch, partials, finalize, cov/env
  b += 1024;                                    // small per-state records
  if (split) b += split_state_bytes();          // BF16 slices of the constant operands
  return b;
}

// Channel specs of the all-ODE route for the pullback (ode_backend.py:60-73): kinetic1 (R),
// kinetic2 (commutator), g phi^4; forward channels from 0, adjoint from 13.
void full_pull_specs(FullPullSpec* sp) {
  std::memset(sp, 0, 3 * sizeof(FullPullSpec));
  const double r2 = 1.4142135623730951;
  const int kin_src[4] = {0, 0, 2, 1}, kin_dst[4] = {1, 2, 3, 3}, kin_left[4] = {1, 0, 1, 0};
  for (int s = 0; s < 2; ++s) {
    sp[s].nch = 4;
    sp[s].fwd0 = 4 * s;
    sp[s].adj0 = 13 + 4 * s;
    sp[s].comm = s;
    sp[s].nedge = 4;
    for (int q = 0; q < 4; ++q) {
      sp[s].esrc[q] = kin_src[q];
      sp[s].edst[q] = kin_dst[q];
      sp[s].eleft[q] = kin_left[q];
      sp[s].ecoef[q] = r2;
    }
  }
  sp[2].nch = 5;
  sp[2].fwd0 = 8;
  sp[2].adj0 = 21;
  sp[2].nedge = 8;
  sp[2].coupling_scaled = 1;
  for (int k = 0; k < 4; ++k)
    for (int side = 0; side < 2; ++side) {
      const int q = 2 * k + side;
      sp[2].esrc[q] = k;
      sp[2].edst[q] = k + 1;
      sp[2].eleft[q] = side == 0;
      sp[2].ecoef[q] = k + 1;
    }
}

}  // namespace

int dp_index(int dp) {
  switch (dp) {
    case 16: return 0;
    case 32: return 1;
    case 48: return 2;
    case 64: return 3;
    case 96: return 4;
    default: return 5;
  }
}

// Tile autotuning of the FP64 trajectory kernel: the depth of its operand ring (2, 3 or 4 staged
// B chunks, compiled variants of the quartic system). It tunes on the caller's own launches: while
// a (system, padded dimension, channel-group level) is undecided in a context, its launches take
// the depths 4, 2 and 3 in turn and each records its device time per 1000 right-hand sides of the
// launch's longest trajectory (the launch lasts as long as that one); after the third the fastest
// is kept, the default 4 unless another is faster by more than 2%. The timing thus includes
// whatever runs beside the trajectory (the kinetic term). The depth changes the schedule, not the
// arithmetic: results are identical for every depth.
static int group_level(int groups) { return groups == 4 ? 2 : groups == 2 ? 1 : 0; }

static int ring_for_launch(const rcmps_context* ctx, int system, int dp, int level) {
  if (system != 0) return 4;
  const int chosen = ctx->traj_ring[system][dp_index(dp)][level];
  if (chosen) return chosen;
  const float* t = ctx->traj_ring_ms[system][dp_index(dp)][level];
  for (int depth : {4, 2, 3})
    if (t[depth - 2] <= 0.f) return depth;
  return 4;
}

static void ring_record(rcmps_context* ctx, int system, int dp, int level, int depth, float ms, long long rhs) {
  if (system != 0 || ctx->traj_ring[system][dp_index(dp)][level] || rhs <= 0 || !(ms > 0.f)) return;
  float* t = ctx->traj_ring_ms[system][dp_index(dp)][level];
  t[depth - 2] = 1000.f * ms / (float)rhs;
  if (t[0] <= 0.f || t[1] <= 0.f || t[2] <= 0.f) return;
  int choice = 4;
  float best = t[2];
  for (int r = 2; r <= 3; ++r)
    if (t[r - 2] < 0.98f * best) {
      best = t[r - 2];
      choice = r;
    }
  ctx->traj_ring[system][dp_index(dp)][level] = choice;
}

int quartic_run(rcmps_context* ctx, QuarticJob& job, cudaStream_t stream) {
  const rcmps_settings& S = job.settings;
  std::vector<double> points, weights;
  trajectory_points(S.half_window, S.n_quad, points, weights);
  const int npoints = (int)points.size(), nodes = 2 * S.n_quad;
  const int nblk = (nodes + kNodesPerBlock - 1) / kNodesPerBlock;

  // offsets of the packed inputs/outputs
  std::vector<long long> off(job.n + 1, 0);
  for (int i = 0; i < job.n; ++i) off[i + 1] = off[i] + (long long)job.dims[i] * job.dims[i];

  std::map<int, std::vector<int>> groups;
  for (int i = 0; i < job.n; ++i) groups[padded_dim(job.dims[i])].push_back(i);

  rcmps_slot& SL = ctx->slot[job.slot];
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t budget = std::max<size_t>((size_t)1 << 30, (free_b + SL.arena_bytes) * job.memory_share);

  cudaEvent_t e0 = SL.ev[0], e1 = SL.ev[1], e2 = SL.ev[2];
  float traj_ms = 0.f, pull_ms = 0.f;

  const int system = job.system;
  if (system == 1) {
    FullPullSpec specs[3];
    full_pull_specs(specs);
    if (pullback_full_set_specs(specs, 3) != cudaSuccess) return fail(ctx, RCMPS_CUDA_ERROR, "pullback specs");
  }
  for (auto& kv : groups) {
    const int dp = kv.first;
    const std::vector<int>& all = kv.second;
    const bool split = split_engine_for(S, system, dp);
    const size_t per = state_bytes(system, dp, npoints, nodes, split);
    const SysSizes zs = sys_sizes(system, dp, nblk);
    const int NCH = zs.nch;
    const size_t fixed = (size_t)(npoints + 3 * nodes) * 8 + 4096;
    int cap = (int)std::max<size_t>(1, (budget - std::min(budget, fixed)) / per);
    for (size_t start = 0; start < all.size(); start += cap) {
      const int n = (int)std::min<size_t>(cap, all.size() - start);
      const bool early_env = system == 0 && job.on_env && job.environment && job.env_ready;
      const bool last_batch = kv.first == groups.rbegin()->first && start + n >= all.size();
      const std::vector<int> idx(all.begin() + start, all.begin() + start + n);
      const size_t mat = (size_t)dp * dp;   // complex elements
      Layout L;
      const size_t o_dims = L.add(n * sizeof(int));
      const size_t o_off = L.add(n * sizeof(long long));
      const size_t o_idx = L.add(n * sizeof(int));
      const size_t o_points = L.add(npoints * 8);
      const size_t o_weights = L.add(nodes * 8);
      const size_t o_wj = L.add(2 * nodes * 8);
      const size_t o_coup = L.add(n * 8);
      const size_t o_tval = L.add(n * 8);
      const size_t o_vout = L.add(n * 8);
      const size_t o_flag = L.add(n * sizeof(int));
      const size_t o_states = L.add(n * sizeof(TrajState));
      const size_t o_tstats = L.add(n * sizeof(TrajStats));
      const size_t o_in = L.add(3 * n * mat * 16);
      const size_t o_ops = L.add((size_t)n * zs.nops * mat * 16);
      const size_t o_work = L.add((size_t)n * zs.nwork * NCH * mat * 16);
      const size_t o_samp = L.add((size_t)n * npoints * NCH * mat * 16);
      const size_t o_wscr = L.add((size_t)n * zs.wscr * mat * 16);
      const size_t o_part = L.add((size_t)n * zs.part * mat * 16);
      const size_t o_fin = L.add((size_t)n * zs.fin * mat * 16);
      const size_t o_cov = L.add((size_t)n * mat * 16);
      const size_t o_env = L.add((size_t)n * mat * 16);
      const size_t o_split = L.add(split ? (size_t)n * split_state_bytes() : 0);
      cudaError_t e = arena_reserve(SL, L.total);
      if (e != cudaSuccess)
        return fail(ctx, RCMPS_OUT_OF_MEMORY, "quartic workspace: " + std::to_string(L.total) + " bytes");
      char* base = static_cast<char*>(SL.arena);
      auto P = [&](size_t o) { return static_cast<void*>(base + o); };

      // host-side tables through a pinned staging buffer
      Layout H;
      const size_t h_o_dims = H.add(n * sizeof(int));
      const size_t h_o_off = H.add(n * 8);
      const size_t h_o_idx = H.add(n * sizeof(int));
      const size_t h_o_points = H.add(npoints * 8);
      const size_t h_o_weights = H.add(nodes * 8);
      const size_t h_o_coup = H.add(n * 8);
      const size_t h_o_states = H.add(n * sizeof(TrajState));
      const size_t h_o_tstats = H.add(n * sizeof(TrajStats));
      const size_t h_o_flag = H.add(n * sizeof(int));
      const size_t h_o_vals = H.add(n * 8);
      const size_t h_o_z2 = H.add(n * sizeof(int));
      if (pinned_reserve(SL, H.total) != cudaSuccess) return fail(ctx, RCMPS_CUDA_ERROR, "pinned host buffer");
      char* h = static_cast<char*>(SL.pinned);
      int* h_dims = reinterpret_cast<int*>(h + h_o_dims);
      long long* h_off = reinterpret_cast<long long*>(h + h_o_off);
      int* h_idx = reinterpret_cast<int*>(h + h_o_idx);
      double* h_points = reinterpret_cast<double*>(h + h_o_points);
      double* h_weights = reinterpret_cast<double*>(h + h_o_weights);
      double* h_coup = reinterpret_cast<double*>(h + h_o_coup);
      TrajState* h_states = reinterpret_cast<TrajState*>(h + h_o_states);
      TrajStats* h_tstats = reinterpret_cast<TrajStats*>(h + h_o_tstats);
      int* h_flag = reinterpret_cast<int*>(h + h_o_flag);
      double* h_vals = reinterpret_cast<double*>(h + h_o_vals);
      for (int i = 0; i < n; ++i) {
        h_dims[i] = job.dims[idx[i]];
        h_off[i] = off[idx[i]];
        h_idx[i] = idx[i];
        h_coup[i] = job.couplings ? job.couplings[idx[i]] : 1.0;
      }
      std::memcpy(h_points, points.data(), npoints * 8);
      std::memcpy(h_weights, weights.data(), nodes * 8);
      double2* d_in = static_cast<double2*>(P(o_in));
      double2* d_ops = static_cast<double2*>(P(o_ops));
      double2* d_work = static_cast<double2*>(P(o_work));
      double2* d_samp = static_cast<double2*>(P(o_samp));
      const size_t vec = (size_t)NCH * mat;   // one stage vector
      for (int i = 0; i < n; ++i) {
        TrajState& t = h_states[i];
        std::memset(&t, 0, sizeof(t));
        const double2* ops = d_ops + (size_t)i * zs.nops * mat;
        t.Q = ops + kQ * mat;
        t.Qh = ops + kQh * mat;
        t.R = ops + kR * mat;
        t.Rh = ops + kRh * mat;
        t.fixed0 = ops + kFixed0 * mat;
        t.fixed6 = ops + kFixed6 * mat;
        t.S = ops + kS * mat;
        t.rho = ops + kRho * mat;
        if (system == 1) {
          t.C = ops + kC * mat;
          t.Ch = ops + kCh * mat;
        }
        double2* w = d_work + (size_t)i * zs.nwork * vec;
        t.y = w;
        t.prop = w + vec;
        t.k = w + 2 * vec;
        t.z = w + 18 * vec;
        t.P = w + 20 * vec;
        t.L = system == 1 ? w + 21 * vec : nullptr;
        t.samples = d_samp + (size_t)i * npoints * vec;
        t.stats = reinterpret_cast<TrajStats*>(base + o_tstats) + i;
        if (split) split_state_pointers(reinterpret_cast<unsigned char*>(base + o_split) + (size_t)i * split_state_bytes(), t);
        t.atol = S.atol;
        t.rtol = S.rtol;
        if (job.controls) {   // per-state tolerances (checked by the entry point)
          const rcmps_state_controls& c = job.controls[idx[i]];
          if (c.atol > 0.0) t.atol = c.atol;
          if (c.rtol > 0.0) t.rtol = c.rtol;
        }
        t.max_steps = S.max_steps;
        t.d = h_dims[i];
      }
      e = cudaMemcpyAsync(P(o_dims), h_dims, n * sizeof(int), cudaMemcpyHostToDevice, stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(P(o_off), h_off, n * 8, cudaMemcpyHostToDevice, stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(P(o_idx), h_idx, n * sizeof(int), cudaMemcpyHostToDevice, stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(P(o_points), h_points, npoints * 8, cudaMemcpyHostToDevice, stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(P(o_weights), h_weights, nodes * 8, cudaMemcpyHostToDevice, stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(P(o_coup), h_coup, n * 8, cudaMemcpyHostToDevice, stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(P(o_states), h_states, n * sizeof(TrajState), cudaMemcpyHostToDevice, stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(P(o_flag), 0, n * sizeof(int), stream);
      const long long in_stride = (long long)mat;
      double* dR = reinterpret_cast<double*>(d_in);
      double* dK = reinterpret_cast<double*>(d_in + n * mat);
      double* dP = reinterpret_cast<double*>(d_in + 2 * n * mat);
      if (e == cudaSuccess) e = launch_pad(job.R, (long long*)P(o_off), (int*)P(o_dims), dR, dp, in_stride, n, stream);
      if (e == cudaSuccess) e = launch_pad(job.K, (long long*)P(o_off), (int*)P(o_dims), dK, dp, in_stride, n, stream);
      if (e == cudaSuccess) e = launch_pad(job.rho, (long long*)P(o_off), (int*)P(o_dims), dP, dp, in_stride, n, stream);
      if (e == cudaSuccess)
        e = launch_prepare(dR, dK, dP, reinterpret_cast<double*>(d_ops), dp, in_stride, (long long)zs.nops * mat, n,
                           stream);
      if (e == cudaSuccess && system == 1)
        e = launch_commutator(reinterpret_cast<double*>(d_ops), dp, (long long)zs.nops * mat, n, stream);
      if (e == cudaSuccess && split) e = split_prep_launch((TrajState*)P(o_states), n, stream);
      // the packed Z2 route: each state's flag in its TrajState (the dense route keeps 0)
      if (e == cudaSuccess && system == 0 && S.symmetry != 0)
        e = launch_z2_check(dR, dK, dP, (int*)P(o_dims), dp, in_stride, n, S.symmetry,
                            reinterpret_cast<int*>(base + o_states + offsetof(TrajState, z2)),
                            (long long)(sizeof(TrajState) / sizeof(int)), stream);
      if (e == cudaSuccess && system == 0 && S.symmetry == 1) {
        // the strict route fails before any integration, as the reference raises in the
        // constructor of its packed system
        int* h_z2 = reinterpret_cast<int*>(h + h_o_z2);
        e = cudaMemcpy2DAsync(h_z2, sizeof(int), base + o_states + offsetof(TrajState, z2), sizeof(TrajState),
                              sizeof(int), n, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e == cudaSuccess)
          for (int i = 0; i < n; ++i)
            if (h_z2[i] < 0) {
              job.stats[idx[i]].status = RCMPS_INVALID_ARGUMENT;
              job.stats[idx[i]].failed_component = 1;
              return fail(ctx, RCMPS_INVALID_ARGUMENT,
                          "state " + std::to_string(idx[i]) +
                              ": the packed Z2 route requires an even D and the exact block structure "
                              "(R odd, K and rho even, rho Hermitian to 1e-13); no projection is performed");
            }
      }
      if (e == cudaSuccess)
        e = node_weights_launch((double*)P(o_points), (double*)P(o_weights), nodes, (double*)P(o_wj), stream);
      TrajControls tc;
      tc.endpoint = points.back();
      tc.initial_h = S.initial_step;
      tc.max_ns = (unsigned long long)(S.max_device_seconds * 1e9);
      tc.groups = trajectory_groups(system, dp, n, S.trajectory_groups, split ? 1 : 0);
      ctx->traj_groups[system][dp_index(dp)] = tc.groups;
      if (!split) tc.ring = ring_for_launch(ctx, system, dp, group_level(tc.groups));
      if (e == cudaSuccess) e = cudaEventRecord(e0, stream);
      if (e == cudaSuccess)
        e = trajectory_launch(system, dp, (TrajState*)P(o_states), n, (double*)P(o_points), npoints, tc, stream,
                              split ? 1 : 0);
      if (e == cudaSuccess) e = cudaEventRecord(e1, stream);
      if (e != cudaSuccess) return fail(ctx, RCMPS_CUDA_ERROR, std::string("trajectory launch: ") + cudaGetErrorString(e));
      // copy the trajectory values into a plain array for the finalize step
      // (TrajStats::value of each state)
      e = cudaMemcpy2DAsync(P(o_tval), 8, reinterpret_cast<char*>(P(o_tstats)) + offsetof(TrajStats, value),
                            sizeof(TrajStats), 8, n, cudaMemcpyDeviceToDevice, stream);
      if (system == 0) {
        PullbackArgs pa;
        pa.dp = dp;
        pa.nstates = n;
        pa.nodes = nodes;
        pa.npoints = npoints;
        pa.nodes_per_block = kNodesPerBlock;
        pa.nblk = nblk;
        pa.ctas = job.pullback_ctas;
        pa.samples = d_samp;
        pa.samples_stride = (long long)npoints * vec;
        pa.ops = d_ops;
        pa.ops_stride = (long long)zs.nops * mat;
        pa.wj = (double*)P(o_wj);
        pa.coupling = (double*)P(o_coup);
        pa.traj_value = (double*)P(o_tval);
        pa.scratch = (double2*)P(o_wscr);
        pa.partial = (double2*)P(o_part);
        pa.fin = (double2*)P(o_fin);
        pa.cov_out = (double2*)P(o_cov);
        pa.env_out = (double2*)P(o_env);
        pa.value_out = (double*)P(o_vout);
        pa.error_flag = (int*)P(o_flag);
        pa.packed = reinterpret_cast<const char*>(P(o_tstats));   // the route the trajectory took
        pa.packed_stride = (int)sizeof(TrajStats);
        pa.packed_offset = (int)offsetof(TrajStats, packed);
        pa.dims = (int*)P(o_dims);
        if (early_env) {
          if (e == cudaSuccess) e = quartic_env_launch(pa, stream);
          if (e == cudaSuccess)
            e = launch_unpad_acc(reinterpret_cast<double*>(P(o_env)), (long long)mat, dp, (long long*)P(o_off),
                                 (int*)P(o_dims), job.environment, n, job.accumulate, stream);
          if (e == cudaSuccess && last_batch) {
            e = cudaEventRecord(job.env_ready, stream);
            if (e == cudaSuccess) job.on_env();
          }
        }
        if (e == cudaSuccess) e = pullback_launch(pa, nblk, stream);
      } else if (system == 2) {
        // <phi> = Re tr F1 at the endpoint (the last sample point, channel 1)
        if (e == cudaSuccess)
          e = launch_endpoint_trace(d_samp, (long long)npoints * vec, (long long)(npoints - 1) * vec + mat, dp,
                                    (int*)P(o_dims), (double*)P(o_vout), n, stream);
      } else {
        FullPullbackArgs pa;
        pa.dp = dp;
        pa.nstates = n;
        pa.nodes = nodes;
        pa.npoints = npoints;
        pa.nodes_per_block = kNodesPerBlock;
        pa.channels = NCH;
        pa.samples = d_samp;
        pa.samples_stride = (long long)npoints * vec;
        pa.ops = d_ops;
        pa.ops_stride = (long long)zs.nops * mat;
        pa.wj = (double*)P(o_wj);
        pa.coupling = (double*)P(o_coup);
        pa.scratch = (double2*)P(o_wscr);
        pa.partial = (double2*)P(o_part);
        pa.fin = (double2*)P(o_fin);
        pa.cov_out = (double2*)P(o_cov);
        pa.env_out = (double2*)P(o_env);
        pa.value_out = (double*)P(o_vout);
        pa.error_flag = (int*)P(o_flag);
        if (e == cudaSuccess) e = pullback_full_launch(pa, nblk, kMaxPullSpecs, stream);
      }
      if (e == cudaSuccess) e = cudaEventRecord(e2, stream);
      if (e != cudaSuccess) return fail(ctx, RCMPS_CUDA_ERROR, std::string("pullback launch: ") + cudaGetErrorString(e));
      // outputs
      if (job.covector)
        e = launch_unpad_acc(reinterpret_cast<double*>(P(o_cov)), (long long)mat, dp, (long long*)P(o_off),
                             (int*)P(o_dims), job.covector, n, job.accumulate, stream);
      if (e == cudaSuccess && job.environment && !early_env)
        e = launch_unpad_acc(reinterpret_cast<double*>(P(o_env)), (long long)mat, dp, (long long*)P(o_off),
                             (int*)P(o_dims), job.environment, n, job.accumulate, stream);
      if (e == cudaSuccess && job.value)
        e = launch_scatter_values((double*)P(o_vout), n, (int*)P(o_idx), job.value, job.accumulate, stream);
      if (e == cudaSuccess && job.samples_out && system == 0)
        e = launch_export_samples(d_samp, dp, h_dims[0], npoints, (double*)P(o_tval), job.samples_out, stream);
      if (e == cudaSuccess && system != 0)   // the value comes from the pullback or the endpoint
        e = cudaMemcpyAsync(h_vals, P(o_vout), n * 8, cudaMemcpyDeviceToHost, stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(h_tstats, P(o_tstats), n * sizeof(TrajStats), cudaMemcpyDeviceToHost, stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(h_flag, P(o_flag), n * sizeof(int), cudaMemcpyDeviceToHost, stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) return fail(ctx, RCMPS_CUDA_ERROR, std::string("quartic: ") + cudaGetErrorString(e));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      traj_ms += ms;
      if (!split) {
        long long longest = 0;
        for (int i = 0; i < n; ++i)
          longest = std::max(longest, 1 + 12 * h_tstats[i].attempts + 3 * h_tstats[i].dense_steps);
        ring_record(ctx, system, dp, group_level(tc.groups), tc.ring, ms, longest);
      }
      cudaEventElapsedTime(&ms, e1, e2);
      pull_ms += ms;
      for (int i = 0; i < n; ++i) {
        const TrajStats& t = h_tstats[i];
        rcmps_state_stats& o = job.stats[idx[i]];
        o.attempts = t.attempts;
        o.accepted = t.accepted;
        o.rejected = t.rejected;
        o.dense_steps = t.dense_steps;
        o.rhs_calls = 1 + 12 * t.attempts + 3 * t.dense_steps;
        o.t_end = t.t;
        o.last_step = t.h;
        o.min_step = t.min_h;
        o.max_step = t.max_h;
        o.packed_z2 = t.packed;
        o.quartic_value = system == 0 ? (job.couplings ? job.couplings[idx[i]] : 1.0) * t.value : h_vals[i];
        if (t.status && !o.status) {
          o.status = t.status;
          o.failed_component = 1;
        } else if (h_flag[i] && !o.status) {
          o.status = RCMPS_WAIT_LIMIT;
          o.failed_component = 2;
        }
      }
    }
  }
  ctx->last_ms[0] = traj_ms;
  ctx->last_ms[1] = pull_ms;
  for (int i = 0; i < job.n; ++i)
    if (job.stats[i].status) return job.stats[i].status;
  return RCMPS_OK;
}

}  // namespace rcmps
