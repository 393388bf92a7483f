// Host orchestration of the batched GMRES solves: the boundary Poisson correction with the
// metric solve (finish_gradient, numerics.py:103-126) and the stationary density
// (stationary_state, numerics.py:74-100).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include "../../include/rcmps_b200.h"
#include "context.h"
#include "kinetic.h"
#include "nojump.h"
#include "prep.h"
#include "quartic.h"
#include "solvers.h"
#include "solvers_host.h"
#include "warmstart.h"

namespace rcmps {

namespace {
struct Layout {
  size_t total = 0;
  size_t add(size_t bytes) {
    const size_t off = total;
    total += align256(bytes);
    return off;
  }
};
constexpr int GCHROWS = 512;
}  // namespace

// The learned preconditioner of a flexible GMRES: the network's weights and its FP32 buffers.
struct GmresNet {
  const float* W1 = nullptr;   // rank x n
  const float* W2 = nullptr;   // n x rank
  int n = 0, rank = 0, d = 0;
  float identity = 0.f;
  float *X32 = nullptr, *H32 = nullptr, *Y32 = nullptr;   // n x NP, rank x NP, n x NP
};

// The no-jump preconditioner of a GMRES: every problem's set and the apply kernel's scratch.
struct GmresNoJump {
  const NoJumpSet* sets = nullptr;   // device [NP]
  double2* W = nullptr;              // device [NP][dp^2]
};

// The m Arnoldi steps of one restart cycle: launches that depend on nothing the host learns
// between them (converged problems are skipped inside the kernels). With a learned
// preconditioner every step first forms Z_j = M V_j (pack, two GEMMs, unpack); with the no-jump
// preconditioner Z_j = P(V_j) (one clustered launch).
static cudaError_t gmres_cycle_launches(ArnoldiProblem* d_probs, int NP, int dp, int m, int sms, cudaStream_t stream,
                                        const GmresNet* net = nullptr, const GmresNoJump* nj = nullptr) {
  const int nvec = dp * dp;
  cudaError_t e = cudaSuccess;
  for (int j = 0; j < m && !e; ++j) {
    if (nj) e = nojump_apply_launch(d_probs, NP, j, nj->sets, nj->W, dp, stream);
    if (!e && net) {
      e = net_pack_launch(d_probs, NP, j, net->d, dp, net->X32, stream);
      if (!e) e = warmstart_gemm(false, false, net->rank, NP, net->n, 1.f, net->W1, net->n, net->X32, NP, 0.f, net->H32,
                                 NP, stream);
      if (!e) e = warmstart_gemm(false, false, net->n, NP, net->rank, 1.f, net->W2, net->rank, net->H32, NP, 0.f,
                                 net->Y32, NP, stream);
      if (!e) e = net_unpack_launch(d_probs, NP, j, net->d, dp, net->Y32, net->identity, stream);
      if (e) break;
    }
    e = lindblad_arnoldi_launch(dp, d_probs, NP, j, stream);
    if (!e) e = gram_schmidt_launch(d_probs, NP, j, nvec, sms, stream);
    if (!e) e = gmres_givens_launch(d_probs, NP, j, stream);
  }
  return e;
}

// One restart cycle, replayed from a CUDA graph that is captured on first use for these device
// addresses and sizes and kept by the context (the cycle's several hundred launches then cost
// one). If capture is not possible the cycle is launched directly.
static cudaError_t gmres_cycle(rcmps_context* ctx, ArnoldiProblem* d_probs, int NP, int dp, int m,
                               LindbladTask* d_tasks, cudaStream_t stream, const GmresNet* net = nullptr,
                               const GmresNoJump* nj = nullptr) {
  const void* key = net ? static_cast<const void*>(net->W1) : nullptr;
  const void* kpre = nj ? static_cast<const void*>(nj->sets) : nullptr;
  const void* key2 = net ? static_cast<const void*>(net->W2) : nullptr;
  const int krank = net ? net->rank : 0;
  const float kid = net ? net->identity : 0.f;
  for (auto& g : ctx->gmres_graphs)
    if (g.exec && g.probs == d_probs && g.tasks == d_tasks && g.np == NP && g.dp == dp && g.m == m &&
        g.net == key && g.net2 == key2 && g.net_rank == krank && g.net_identity == kid && g.pre == kpre) {
      note_launches(g.kernels);
      return cudaGraphLaunch(g.exec, stream);
    }
  const long long before = thread_launch_count();
  cudaGraph_t graph = nullptr;
  if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return gmres_cycle_launches(d_probs, NP, dp, m, ctx->sms, stream, net, nj);
  }
  cudaError_t e = gmres_cycle_launches(d_probs, NP, dp, m, ctx->sms, stream, net, nj);
  const cudaError_t ec = cudaStreamEndCapture(stream, &graph);
  cudaGraphExec_t exec = nullptr;
  if (!e && !ec && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    rcmps_gmres_graph& g = ctx->gmres_graphs[ctx->gmres_graph_next];
    ctx->gmres_graph_next = (ctx->gmres_graph_next + 1) % 4;
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.probs = d_probs;
    g.tasks = d_tasks;
    g.np = NP;
    g.dp = dp;
    g.m = m;
    g.net = key;
    g.net2 = key2;
    g.net_rank = krank;
    g.net_identity = kid;
    g.pre = kpre;
    g.kernels = thread_launch_count() - before;
    g.exec = exec;
    return cudaGraphLaunch(exec, stream);
  }
  // capture or instantiation failed: nothing was launched by the capture; launch directly
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();
  return gmres_cycle_launches(d_probs, NP, dp, m, ctx->sms, stream, net, nj);
}

// Restarted GMRES(m) over NP problems that share dp; hp/d_probs hold set-up problems with x = 0.
// Returns 0, or a CUDA error code. Convergence per problem is in hp[p].converged / residual.
static cudaError_t gmres_run(rcmps_context* ctx, ArnoldiProblem* hp, ArnoldiProblem* d_probs, int NP, int dp,
                             int m, int maxrestart, LindbladTask* d_tasks, cudaStream_t stream,
                             bool bnorm_from_b = false, const GmresNet* net = nullptr,
                             const GmresNoJump* nj = nullptr) {
  const int nvec = dp * dp;
  cudaError_t e = cudaMemcpyAsync(d_probs, hp, NP * sizeof(ArnoldiProblem), cudaMemcpyHostToDevice, stream);
  // a warm start: the first residual is not |b|, so |b| is measured for the stopping target
  if (!e && bnorm_from_b) e = gmres_bnorm_launch(d_probs, NP, stream);
  for (int it = 0; it <= maxrestart && !e; ++it) {
    e = gmres_x_tasks_launch(d_probs, NP, d_tasks, stream);
    if (!e) e = lindblad_launch(dp, d_tasks, NP, 0, stream);
    if (!e) e = gmres_residual_launch(d_probs, NP, nvec, stream);
    if (!e) e = cudaMemcpyAsync(hp, d_probs, NP * sizeof(ArnoldiProblem), cudaMemcpyDeviceToHost, stream);
    if (!e) e = cudaStreamSynchronize(stream);
    if (e) break;
    bool all = true;
    for (int p = 0; p < NP; ++p) all &= hp[p].converged != 0;
    if (all || it == maxrestart) break;
    e = gmres_cycle(ctx, d_probs, NP, dp, m, d_tasks, stream, net, nj);
    if (!e) e = gmres_update_launch(d_probs, NP, nvec, m, stream);
  }
  return e;
}

// Fill the GMRES fields of NP problems (dp, m) in the layout of slot `base`.
struct GmresBuffers {
  size_t o_probs, o_V, o_H, o_W, o_part, o_norms, o_x, o_g, o_cs, o_sn, o_flags, o_tasks;
};
static GmresBuffers gmres_layout(Layout& L, int NP, int dp, int m) {
  const size_t mat = (size_t)dp * dp;
  const int nchunk = (dp * dp + GCHROWS - 1) / GCHROWS;
  GmresBuffers b;
  b.o_probs = L.add(NP * sizeof(ArnoldiProblem));
  b.o_V = L.add((size_t)NP * (m + 1) * mat * 16);
  b.o_H = L.add((size_t)NP * (m + 1) * m * 16);
  b.o_W = L.add((size_t)NP * mat * 16);
  b.o_part = L.add((size_t)NP * nchunk * (m + 1) * 16);
  b.o_norms = L.add((size_t)NP * 2 * nchunk * 8);
  b.o_x = L.add((size_t)NP * mat * 16);
  b.o_g = L.add((size_t)NP * (m + 1) * 16);
  b.o_cs = L.add((size_t)NP * m * 16);
  b.o_sn = L.add((size_t)NP * m * 16);
  b.o_flags = L.add(NP * 4);
  b.o_tasks = L.add(NP * sizeof(LindbladTask));
  return b;
}
static void gmres_problem(ArnoldiProblem& A, char* base, const GmresBuffers& b, int p, int dp, int d, int m,
                          double tol) {
  const size_t mat = (size_t)dp * dp;
  const int nchunk = (dp * dp + GCHROWS - 1) / GCHROWS;
  std::memset(&A, 0, sizeof(A));
  A.V = (double2*)(base + b.o_V) + (size_t)p * (m + 1) * mat;
  A.ldv = (long long)mat;
  A.H = (double2*)(base + b.o_H) + (size_t)p * (m + 1) * m;
  A.W = (double2*)(base + b.o_W) + (size_t)p * mat;
  A.partial = (double2*)(base + b.o_part) + (size_t)p * nchunk * (m + 1);
  A.norms = (double*)(base + b.o_norms) + (size_t)p * 2 * nchunk;
  A.x = (double2*)(base + b.o_x) + (size_t)p * mat;
  A.g = (double2*)(base + b.o_g) + (size_t)p * (m + 1);
  A.cs = (double2*)(base + b.o_cs) + (size_t)p * m;
  A.sn = (double2*)(base + b.o_sn) + (size_t)p * m;
  A.flag = (int*)(base + b.o_flags) + p;
  A.n = dp * dp;
  A.n_phys = d * d;
  A.d = d;
  A.dp = dp;
  A.kmax = m;
  A.kmax1 = m + 1;
  A.target = std::min(m, d * d);
  A.gtol = tol;
  A.bnorm = -1.0;
}

static FinishArgs finish_args(const FinishPlan& plan, const FinishPlan::Group& g, char* base, double metric_reg);

// The boundary solve needs only the environment; the covector enters after it. finish_solve runs
// the Poisson GMRES of every state and finish_complete applies the covector and the metric solve,
// so that a caller may produce the covector while the solve runs.
struct FinishPlan::Group {
  int dp = 0, n = 0;
  std::vector<int> idx;
  size_t o_dims = 0, o_off = 0, o_in = 0, o_ops = 0, o_b = 0, o_tmp = 0, o_status = 0;
  size_t o_z = 0, o_x32 = 0, o_h32 = 0, o_y32 = 0;   // learned preconditioner (flexible GMRES)
  size_t o_nj = 0, o_njv = 0, o_njs = 0, o_njw = 0, h_njs = 0;   // no-jump preconditioner
  const NoJumpSet* nj_sets = nullptr;
  double2* nj_W = nullptr;
  GmresBuffers gb{};
  size_t h_dims = 0, h_off = 0, h_probs = 0, h_status = 0;
};

static FinishArgs finish_args(const FinishPlan& plan, const FinishPlan::Group& g, char* base, double metric_reg) {
  (void)plan;
  const size_t mat = (size_t)g.dp * g.dp;
  double2* d_in = (double2*)(base + g.o_in);
  FinishArgs fa;
  fa.dp = g.dp;
  fa.dims = (int*)(base + g.o_dims);
  fa.ops = (double2*)(base + g.o_ops);
  fa.ops_stride = (long long)(8 * mat);
  fa.env = d_in + 4 * g.n * mat;
  fa.cov = d_in + 3 * g.n * mat;
  fa.b = (double2*)(base + g.o_b);
  fa.x = (double2*)(base + g.gb.o_x);
  fa.tmp = (double2*)(base + g.o_tmp);
  fa.metric_reg = metric_reg;
  fa.status = (int*)(base + g.o_status);
  return fa;
}

FinishPlan::FinishPlan() = default;
FinishPlan::~FinishPlan() = default;

int finish_prepare(rcmps_context* ctx, FinishJob& job, cudaStream_t stream, FinishPlan& plan) {
  const rcmps_settings& S = job.settings;
  // the no-jump preconditioner takes the reference's restart length min(40, d^2)
  // (numerics.py:55-71); the unpreconditioned and learned solves GMRES(64)
  const bool nojump = !job.net && S.boundary_preconditioner == 1;
  const int m = nojump ? 40 : 64;
  plan.nojump = nojump;
  plan.m = m;
  const double tol = S.boundary_tolerance;
  if (!(tol > 0.0) || !(S.metric_reg >= 0.0)) return fail(ctx, RCMPS_INVALID_ARGUMENT, "invalid boundary controls");
  plan.off.assign(job.n + 1, 0);
  for (int i = 0; i < job.n; ++i) plan.off[i + 1] = plan.off[i] + (long long)job.dims[i] * job.dims[i];
  std::map<int, std::vector<int>> groups;
  for (int i = 0; i < job.n; ++i) groups[padded_dim(job.dims[i])].push_back(i);
  // one workspace region and one staging region per padded dimension, all held at once
  plan.groups.clear();
  Layout L, H;
  for (auto& kv : groups) {
    FinishPlan::Group g;
    g.dp = kv.first;
    g.idx = kv.second;
    g.n = (int)g.idx.size();
    const size_t mat = (size_t)g.dp * g.dp;
    const int n = g.n;
    g.o_dims = L.add(n * 4);
    g.o_off = L.add(n * 8);
    g.o_in = L.add(5 * n * mat * 16);
    g.o_ops = L.add(n * 8 * mat * 16);
    g.o_b = L.add(n * mat * 16);
    g.o_tmp = L.add(n * 4 * mat * 16);
    g.o_status = L.add(n * 4);
    g.gb = gmres_layout(L, n, g.dp, m);
    if (nojump) {   // flexible GMRES through the no-jump sets
      g.o_z = L.add((size_t)n * m * mat * 16);
      g.o_nj = L.add((size_t)n * kNoJumpMats * mat * 16);
      g.o_njv = L.add((size_t)n * (g.dp + 2) * 16 + (size_t)n * 8 + (size_t)n * 4);
      g.o_njs = L.add((size_t)n * sizeof(NoJumpSet));
      g.o_njw = L.add((size_t)n * mat * 16);
      g.h_njs = H.add((size_t)n * sizeof(NoJumpSet));
    }
    if (job.net) {   // flexible GMRES: the preconditioned basis and the network's buffers
      g.o_z = L.add((size_t)n * m * mat * 16);
      g.o_x32 = L.add((size_t)job.net->n * n * 4);
      g.o_h32 = L.add((size_t)job.net->rank * n * 4);
      g.o_y32 = L.add((size_t)job.net->n * n * 4);
    }
    g.h_dims = H.add(n * 4);
    g.h_off = H.add(n * 8);
    g.h_probs = H.add(n * sizeof(ArnoldiProblem));
    g.h_status = H.add(n * 4);
    plan.groups.push_back(std::move(g));
  }
  rcmps_slot& SL = ctx->slot[job.slot];
  cudaError_t e = arena_reserve(SL, L.total);
  if (e) return fail(ctx, RCMPS_OUT_OF_MEMORY, "boundary workspace");
  if (pinned_reserve(SL, H.total)) return fail(ctx, RCMPS_CUDA_ERROR, "pinned host buffer");
  char* base = static_cast<char*>(SL.arena);
  char* h = static_cast<char*>(SL.pinned);
  auto P = [&](size_t o) { return static_cast<void*>(base + o); };
  for (auto& g : plan.groups) {
    const int dp = g.dp, n = g.n;
    const size_t mat = (size_t)dp * dp;
    int* hd = (int*)(h + g.h_dims);
    long long* ho = (long long*)(h + g.h_off);
    for (int i = 0; i < n; ++i) {
      hd[i] = job.dims[g.idx[i]];
      ho[i] = plan.off[g.idx[i]];
    }
    double2* d_in = (double2*)P(g.o_in);
    double* dR = (double*)d_in;
    double* dK = (double*)(d_in + n * mat);
    double* dP = (double*)(d_in + 2 * n * mat);
    e = cudaMemcpyAsync(P(g.o_dims), hd, n * 4, cudaMemcpyHostToDevice, stream);
    if (!e) e = cudaMemcpyAsync(P(g.o_off), ho, n * 8, cudaMemcpyHostToDevice, stream);
    if (!e) e = cudaMemsetAsync(P(g.o_status), 0, n * 4, stream);
    if (!e) e = launch_pad(job.R, (long long*)P(g.o_off), (int*)P(g.o_dims), dR, dp, mat, n, stream);
    if (!e) e = launch_pad(job.K, (long long*)P(g.o_off), (int*)P(g.o_dims), dK, dp, mat, n, stream);
    if (!e) e = launch_pad(job.rho, (long long*)P(g.o_off), (int*)P(g.o_dims), dP, dp, mat, n, stream);
    if (!e) e = launch_prepare(dR, dK, dP, (double*)P(g.o_ops), dp, mat, 8 * mat, n, stream);
    if (!e && nojump) {
      NoJumpSet* hs = (NoJumpSet*)(h + g.h_njs);
      double2* mats = (double2*)P(g.o_nj);
      double2* vecs = (double2*)P(g.o_njv);
      double* shifts = (double*)(vecs + (size_t)n * (dp + 2));
      int* status = (int*)(shifts + n);
      for (int i = 0; i < n; ++i) {
        NoJumpSet& t = hs[i];
        const double2* ops = (double2*)P(g.o_ops) + (size_t)i * 8 * mat;
        double2* b = mats + (size_t)i * kNoJumpMats * mat;
        t.Q = ops + kQ * mat;
        t.R = ops + kR * mat;
        t.rho = ops + kRho * mat;
        double2** outs[kNoJumpMats] = {&t.V, &t.Vh, &t.Vinv, &t.Vinvh, &t.nS, &t.z, &t.H, &t.U, &t.W, &t.M, &t.T};
        for (int q = 0; q < kNoJumpMats; ++q) *outs[q] = b + (size_t)q * mat;
        t.lambda = vecs + (size_t)i * (dp + 2);
        t.den = t.lambda + dp;
        t.shift = shifts + i;
        t.status = status + i;
        t.d = hd[i];
        t.dp = dp;
      }
      e = cudaMemcpyAsync(P(g.o_njs), hs, (size_t)n * sizeof(NoJumpSet), cudaMemcpyHostToDevice, stream);
      if (!e) e = nojump_setup_launch((const NoJumpSet*)P(g.o_njs), n, dp, stream);
      g.nj_sets = (const NoJumpSet*)P(g.o_njs);
      g.nj_W = (double2*)P(g.o_njw);
    }
    if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("boundary set-up: ") + cudaGetErrorString(e));
  }
  plan.prepared = true;
  return RCMPS_OK;
}

// The Poisson GMRES of every state (after finish_prepare, which it runs first if the caller has
// not): the environment and the right-hand side, then the batched solve per padded dimension.
int finish_solve(rcmps_context* ctx, FinishJob& job, cudaStream_t stream, FinishPlan& plan) {
  if (!plan.prepared) {
    const int rc = finish_prepare(ctx, job, stream, plan);
    if (rc) return rc;
  }
  const rcmps_settings& S = job.settings;
  const double tol = S.boundary_tolerance;
  const int m = plan.m, maxrestart = job.max_restarts;
  const bool nojump = plan.nojump;
  rcmps_slot& SL = ctx->slot[job.slot];
  char* base = static_cast<char*>(SL.arena);
  char* h = static_cast<char*>(SL.pinned);
  auto P = [&](size_t o) { return static_cast<void*>(base + o); };
  cudaError_t e = cudaSuccess;
  for (auto& g : plan.groups) {
    const int dp = g.dp, n = g.n;
    const size_t mat = (size_t)dp * dp;
    int* hd = (int*)(h + g.h_dims);
    ArnoldiProblem* hp = (ArnoldiProblem*)(h + g.h_probs);
    double* dE = (double*)((double2*)P(g.o_in) + 4 * n * mat);
    e = cudaMemsetAsync(P(g.gb.o_x), 0, (size_t)n * mat * 16, stream);
    if (!e && job.x0)
      e = launch_pad(job.x0, (long long*)P(g.o_off), (int*)P(g.o_dims), (double*)P(g.gb.o_x), dp, mat, n, stream);
    if (!e) e = launch_pad(job.environment, (long long*)P(g.o_off), (int*)P(g.o_dims), dE, dp, mat, n, stream);
    GmresNoJump nj;
    nj.sets = g.nj_sets;
    nj.W = g.nj_W;
    FinishArgs fa = finish_args(plan, g, base, S.metric_reg);
    if (!e) e = boundary_rhs_launch(fa, n, stream);
    if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("boundary set-up: ") + cudaGetErrorString(e));
    for (int i = 0; i < n; ++i) {
      ArnoldiProblem& A = hp[i];
      gmres_problem(A, base, g.gb, i, dp, hd[i], m, tol);
      const double2* ops = (double2*)P(g.o_ops) + (size_t)i * 8 * mat;
      A.A1 = ops + 1 * mat;   // L*: Q^dag X + X Q + R^dag X R
      A.A1h = ops;
      A.A2 = ops + 3 * mat;
      A.A2h = ops + 2 * mat;
      A.trw = ops + 7 * mat;  // + tr(rho X) I
      A.b = fa.b + (size_t)i * mat;
      if (job.net || nojump) A.Z = (double2*)P(g.o_z) + (size_t)i * m * mat;
    }
    GmresNet net;
    if (job.net) {
      net.W1 = job.net->W1;
      net.W2 = job.net->W2;
      net.n = job.net->n;
      net.rank = job.net->rank;
      net.identity = job.net->identity;
      net.d = hd[0];
      net.X32 = (float*)P(g.o_x32);
      net.H32 = (float*)P(g.o_h32);
      net.Y32 = (float*)P(g.o_y32);
    }
    e = gmres_run(ctx, hp, (ArnoldiProblem*)P(g.gb.o_probs), n, dp, m, maxrestart, (LindbladTask*)P(g.gb.o_tasks),
                  stream, job.x0 != nullptr, job.net ? &net : nullptr, nojump ? &nj : nullptr);
    if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("boundary GMRES: ") + cudaGetErrorString(e));
  }
  return RCMPS_OK;
}

int boundary_run(rcmps_context* ctx, FinishJob& job, double* H, cudaStream_t stream) {
  FinishPlan plan;
  int rc = finish_solve(ctx, job, stream, plan);
  if (rc) return rc;
  const double tol = job.settings.boundary_tolerance;
  rcmps_slot& SL = ctx->slot[job.slot];
  char* base = static_cast<char*>(SL.arena);
  char* h = static_cast<char*>(SL.pinned);
  cudaError_t e = cudaSuccess;
  for (auto& g : plan.groups) {
    const size_t mat = (size_t)g.dp * g.dp;
    e = launch_unpad_acc(reinterpret_cast<double*>(base + g.gb.o_x), (long long)mat, g.dp,
                         reinterpret_cast<long long*>(base + g.o_off), reinterpret_cast<int*>(base + g.o_dims), H, g.n,
                         false, stream);
    if (e) break;
  }
  if (!e) e = cudaStreamSynchronize(stream);
  if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("boundary solution: ") + cudaGetErrorString(e));
  for (auto& g : plan.groups) {
    const ArnoldiProblem* hp = reinterpret_cast<const ArnoldiProblem*>(h + g.h_probs);
    for (int i = 0; i < g.n; ++i) {
      rcmps_state_stats& st = job.stats[g.idx[i]];
      const ArnoldiProblem& A = hp[i];
      st.gmres_iterations = A.iters;
      st.gmres_matvecs = A.iters + A.restarts;
      st.boundary_residual = A.residual;
      const bool ok = A.converged || A.residual <= 20.0 * tol * std::max(1.0, A.bnorm);
      if (!st.status && (A.nonfinite || !std::isfinite(A.residual) || !ok)) {
        st.status = RCMPS_SOLVE_FAILURE;
        st.failed_component = 4;
      }
    }
  }
  for (int i = 0; i < job.n; ++i)
    if (job.stats[i].status) return job.stats[i].status;
  return RCMPS_OK;
}

int finish_complete(rcmps_context* ctx, FinishJob& job, cudaStream_t stream, FinishPlan& plan) {
  const rcmps_settings& S = job.settings;
  const double tol = S.boundary_tolerance;
  rcmps_slot& SL = ctx->slot[job.slot];
  char* base = static_cast<char*>(SL.arena);
  char* h = static_cast<char*>(SL.pinned);
  auto P = [&](size_t o) { return static_cast<void*>(base + o); };
  cudaError_t e = cudaSuccess;
  for (auto& g : plan.groups) {
    const int dp = g.dp, n = g.n;
    const size_t mat = (size_t)dp * dp;
    const ArnoldiProblem* hp = (const ArnoldiProblem*)(h + g.h_probs);
    int* hs = (int*)(h + g.h_status);
    double* dC = (double*)((double2*)P(g.o_in) + 3 * n * mat);
    FinishArgs fa = finish_args(plan, g, base, S.metric_reg);
    e = launch_pad(job.covector, (long long*)P(g.o_off), (int*)P(g.o_dims), dC, dp, mat, n, stream);
    if (!e) e = finish_launch(fa, n, stream);
    if (!e) e = launch_unpad_acc((double*)(fa.tmp + 3 * mat), (long long)(4 * mat), dp, (long long*)P(g.o_off),
                                 (int*)P(g.o_dims), job.gradient, n, false, stream);
    if (!e) e = cudaMemcpyAsync(hs, P(g.o_status), n * 4, cudaMemcpyDeviceToHost, stream);
    if (!e) e = cudaStreamSynchronize(stream);
    if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("finish: ") + cudaGetErrorString(e));
    for (int i = 0; i < n; ++i) {
      rcmps_state_stats& st = job.stats[g.idx[i]];
      const ArnoldiProblem& A = hp[i];
      st.gmres_iterations = A.iters;
      st.gmres_matvecs = A.iters + A.restarts;
      st.boundary_residual = A.residual;
      const bool ok = A.converged || A.residual <= 20.0 * tol * std::max(1.0, A.bnorm);
      if (st.status) continue;
      if (A.nonfinite || !std::isfinite(A.residual) || !ok) {
        st.status = RCMPS_SOLVE_FAILURE;
        st.failed_component = 4;
      } else if (hs[i]) {
        st.status = hs[i];
        st.failed_component = 4;
      }
    }
  }
  for (int i = 0; i < job.n; ++i)
    if (job.stats[i].status) return job.stats[i].status;
  return RCMPS_OK;
}

int finish_run(rcmps_context* ctx, FinishJob& job, cudaStream_t stream) {
  FinishPlan plan;
  const int rc = finish_solve(ctx, job, stream, plan);
  if (rc) return rc;
  return finish_complete(ctx, job, stream, plan);
}

int stationary_run(rcmps_context* ctx, StationaryJob& job, cudaStream_t stream) {
  const int m = 64, maxrestart = 200;
  const double tol = job.tolerance;
  if (!(tol > 0.0)) return fail(ctx, RCMPS_INVALID_ARGUMENT, "stationary tolerance must be positive");
  std::vector<long long> off(job.n + 1, 0);
  for (int i = 0; i < job.n; ++i) off[i + 1] = off[i] + (long long)job.dims[i] * job.dims[i];
  std::map<int, std::vector<int>> groups;
  for (int i = 0; i < job.n; ++i) groups[padded_dim(job.dims[i])].push_back(i);
  rcmps_slot& SL = ctx->slot[job.slot];
  for (auto& kv : groups) {
    const int dp = kv.first;
    const std::vector<int>& idx = kv.second;
    const int n = (int)idx.size();
    const size_t mat = (size_t)dp * dp;
    Layout L;
    const size_t o_dims = L.add(n * 4), o_off = L.add(n * 8);
    const size_t o_in = L.add(3 * n * mat * 16), o_ops = L.add(n * 8 * mat * 16);
    const size_t o_b = L.add(n * mat * 16), o_trw = L.add(n * mat * 16), o_rho = L.add(n * mat * 16),
                 o_tmp = L.add(n * mat * 16), o_lres = L.add((size_t)n * (dp / 16) * 8), o_herm = L.add(n * 16),
                 o_status = L.add(n * 4), o_rt = L.add(n * sizeof(LindbladTask));
    GmresBuffers gb = gmres_layout(L, n, dp, m);
    cudaError_t e = arena_reserve(SL, L.total);
    if (e) return fail(ctx, RCMPS_OUT_OF_MEMORY, "stationary workspace");
    char* base = static_cast<char*>(SL.arena);
    auto P = [&](size_t o) { return static_cast<void*>(base + o); };
    Layout H;
    const size_t h_dims = H.add(n * 4), h_off = H.add(n * 8), h_probs = H.add(n * sizeof(ArnoldiProblem)),
                 h_status = H.add(n * 4), h_lres = H.add((size_t)n * (dp / 16) * 8), h_herm = H.add(n * 16),
                 h_rt = H.add(n * sizeof(LindbladTask)), h_b = H.add(n * mat * 16);
    if (pinned_reserve(SL, H.total)) return fail(ctx, RCMPS_CUDA_ERROR, "pinned host buffer");
    char* h = static_cast<char*>(SL.pinned);
    int* hd = (int*)(h + h_dims);
    long long* ho = (long long*)(h + h_off);
    ArnoldiProblem* hp = (ArnoldiProblem*)(h + h_probs);
    int* hs = (int*)(h + h_status);
    double* hl = (double*)(h + h_lres);
    double* hh = (double*)(h + h_herm);
    LindbladTask* hrt = (LindbladTask*)(h + h_rt);
    double2* hb = (double2*)(h + h_b);
    // b = I_d / d and the trace weights trw = I_d / d
    std::memset(hb, 0, n * mat * 16);
    for (int i = 0; i < n; ++i) {
      hd[i] = job.dims[idx[i]];
      ho[i] = off[idx[i]];
      for (int q = 0; q < hd[i]; ++q) hb[(size_t)i * mat + (size_t)q * dp + q] = make_double2(1.0 / hd[i], 0.0);
    }
    double2* d_in = (double2*)P(o_in);
    double* dR = (double*)d_in;
    double* dK = (double*)(d_in + n * mat);
    e = cudaMemcpyAsync(P(o_dims), hd, n * 4, cudaMemcpyHostToDevice, stream);
    if (!e) e = cudaMemcpyAsync(P(o_off), ho, n * 8, cudaMemcpyHostToDevice, stream);
    if (!e) e = cudaMemcpyAsync(P(o_b), hb, n * mat * 16, cudaMemcpyHostToDevice, stream);
    if (!e) e = cudaMemcpyAsync(P(o_trw), hb, n * mat * 16, cudaMemcpyHostToDevice, stream);
    if (!e) e = cudaMemsetAsync(P(o_status), 0, n * 4, stream);
    if (!e && job.rho_previous)   // warm start: x0 = rho_previous, GMRES corrects it
      e = launch_pad(job.rho_previous, (long long*)P(o_off), (int*)P(o_dims), (double*)P(gb.o_x), dp, mat, n,
                     stream);
    else if (!e)
      e = cudaMemsetAsync(P(gb.o_x), 0, (size_t)n * mat * 16, stream);
    if (!e) e = cudaMemsetAsync(d_in + 2 * n * mat, 0, n * mat * 16, stream);   // rho placeholder
    if (!e) e = launch_pad(job.R, (long long*)P(o_off), (int*)P(o_dims), dR, dp, mat, n, stream);
    if (!e) e = launch_pad(job.K, (long long*)P(o_off), (int*)P(o_dims), dK, dp, mat, n, stream);
    if (!e) e = launch_prepare(dR, dK, (double*)(d_in + 2 * n * mat), (double*)P(o_ops), dp, mat, 8 * mat, n, stream);
    if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("stationary set-up: ") + cudaGetErrorString(e));
    for (int i = 0; i < n; ++i) {
      ArnoldiProblem& A = hp[i];
      gmres_problem(A, base, gb, i, dp, hd[i], m, tol);
      const double2* ops = (double2*)P(o_ops) + (size_t)i * 8 * mat;
      A.A1 = ops;             // L: Q X + X Q^dag + R X R^dag
      A.A1h = ops + 1 * mat;
      A.A2 = ops + 2 * mat;
      A.A2h = ops + 3 * mat;
      A.trw = (double2*)P(o_trw) + (size_t)i * mat;   // + tr(X)/d I
      A.b = (double2*)P(o_b) + (size_t)i * mat;
      // warm start: the target |b - A x| <= tolerance is absolute, as the reference's correction
      // solve with rtol = atol = tolerance / max(1, |rhs|) (stationary_correction.py:60-66)
      if (job.rho_previous) A.bnorm = 1.0;
    }
    e = gmres_run(ctx, hp, (ArnoldiProblem*)P(gb.o_probs), n, dp, m, maxrestart, (LindbladTask*)P(gb.o_tasks),
                  stream);
    if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("stationary GMRES: ") + cudaGetErrorString(e));
    StationaryArgs sa;
    sa.dp = dp;
    sa.dims = (int*)P(o_dims);
    sa.x = (double2*)P(gb.o_x);
    sa.rho = (double2*)P(o_rho);
    sa.tmp = (double2*)P(o_tmp);
    sa.herm = (double*)P(o_herm);
    sa.scale = (double*)P(o_herm) + n;
    sa.ops = (double2*)P(o_ops);
    sa.ops_stride = (long long)(8 * mat);
    sa.tolerance = tol;
    sa.status = (int*)P(o_status);
    e = stationary_finish_launch(sa, n, stream);
    // |L(rho)|: the residual mode computes |X - shift L(X) - rhs|^2; with rhs = X and shift = 1 it
    // is |L(rho)|^2.
    for (int i = 0; i < n; ++i) {
      const double2* ops = (double2*)P(o_ops) + (size_t)i * 8 * mat;
      LindbladTask& t = hrt[i];
      std::memset(&t, 0, sizeof(t));
      t.X = sa.rho + (size_t)i * mat;
      t.A1 = ops;
      t.A1h = ops + mat;
      t.A2 = ops + 2 * mat;
      t.A2h = ops + 3 * mat;
      t.rhs = t.X;
      t.res = (double*)P(o_lres) + (size_t)i * (dp / 16);
      t.shift = 1.0;
      t.flag = (int*)P(gb.o_flags) + i;
    }
    if (!e) e = cudaMemcpyAsync(P(o_rt), hrt, n * sizeof(LindbladTask), cudaMemcpyHostToDevice, stream);
    if (!e) e = lindblad_launch(dp, (LindbladTask*)P(o_rt), n, 1, stream);
    if (!e) e = launch_unpad_acc((double*)P(o_rho), (long long)mat, dp, (long long*)P(o_off), (int*)P(o_dims),
                                 job.rho, n, false, stream);
    if (!e) e = cudaMemcpyAsync(hs, P(o_status), n * 4, cudaMemcpyDeviceToHost, stream);
    if (!e) e = cudaMemcpyAsync(hl, P(o_lres), (size_t)n * (dp / 16) * 8, cudaMemcpyDeviceToHost, stream);
    if (!e) e = cudaMemcpyAsync(hh, P(o_herm), n * 16, cudaMemcpyDeviceToHost, stream);
    if (!e) e = cudaStreamSynchronize(stream);
    if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("stationary finish: ") + cudaGetErrorString(e));
    for (int i = 0; i < n; ++i) {
      rcmps_state_stats& st = job.stats[idx[i]];
      const ArnoldiProblem& A = hp[i];
      double l2 = 0.0;
      for (int r = 0; r < dp / 16; ++r) l2 += hl[(size_t)i * (dp / 16) + r];
      st.gmres_iterations = A.iters;
      st.boundary_residual = std::sqrt(l2);   // |L(rho)|
      const double scale = hh[n + i];
      if (st.status) continue;
      const bool ok = A.converged || A.residual <= 20.0 * tol * std::max(1.0, A.bnorm);
      if (!ok || A.nonfinite) {
        st.status = RCMPS_SOLVE_FAILURE;
        st.failed_component = 5;
      } else if (hs[i]) {
        st.status = hs[i];
        st.failed_component = 5;
      } else if (!(std::sqrt(l2) <= tol * scale)) {
        st.status = RCMPS_SOLVE_FAILURE;
        st.failed_component = 5;
      }
    }
  }
  for (int i = 0; i < job.n; ++i)
    if (job.stats[i].status) return job.stats[i].status;
  return RCMPS_OK;
}

}  // namespace rcmps
