// Host orchestration of the kinetic terms: Arnoldi rounds with basis doubling, projected solves,
// reconstruction and true residuals, then the contraction (kinetic_backend.py:438-592 of
// rcmps_gpu: KineticContext.solutions and kinetic_raw). The host only decides between device
// phases from per-problem flags it reads back (three small reads per round).
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
#include "kinetic_host.h"
#include "prep.h"
#include "quartic.h"

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
constexpr int kContractNodesPerBlock = 16;
constexpr int CHROWS = 512;   // rows of a Gram-Schmidt chunk (kinetic.cu CH)

size_t kinetic_state_bytes(int dp, int kmax, int nshift) {
  const size_t mat = (size_t)dp * dp * 16;
  const int nchunk = (dp * dp + CHROWS - 1) / CHROWS;
  const int nblk = (nshift + kContractNodesPerBlock - 1) / kContractNodesPerBlock;
  size_t b = 3 * mat + 8 * mat + 2 * mat + 4 * mat;                 // inputs, ops, C, rhs
  b += 4 * ((size_t)(2 * kmax + 1) * mat + (size_t)(kmax + 1) * kmax * 16 + mat + (size_t)nchunk * (kmax + 1) * 16 +
            (size_t)nshift * kmax * 16 + (size_t)nshift * mat);      // per problem (V, L(V), H, ...)
  b += 4 * (size_t)nshift * ((dp * dp + 63) / 64) * 8;
  b += 2 * (size_t)nblk * 4 * mat + 12 * mat;                        // contraction
  return b + 4096;
}
}  // namespace

void angular_grid(int nodes, std::vector<double>& shifts, std::vector<double>& weights) {
  std::vector<double> x, w;
  gauss_legendre(nodes, x, w);
  shifts.resize(nodes);
  weights.resize(nodes);
  const double quarter_pi = 0.78539816339744830962;
  for (int i = 0; i < nodes; ++i) {
    shifts[i] = std::cos(quarter_pi * (x[i] + 1.0));
    weights[i] = 0.5 * w[i];
  }
}

int kinetic_run(rcmps_context* ctx, KineticJob& job, cudaStream_t stream) {
  const rcmps_settings& S = job.settings;
  const int nshift = S.kinetic_nodes;
  if (nshift < 2) return fail(ctx, RCMPS_INVALID_ARGUMENT, "kinetic_nodes must be >= 2");
  if (!(S.krylov_tolerance > 0.0) || S.krylov_initialdim < 1 || S.krylov_maxdim < S.krylov_initialdim)
    return fail(ctx, RCMPS_INVALID_ARGUMENT, "invalid Krylov controls");
  std::vector<double> shifts, weights;
  angular_grid(nshift, shifts, weights);
  std::vector<long long> off(job.n + 1, 0);
  for (int i = 0; i < job.n; ++i) off[i + 1] = off[i] + (long long)job.dims[i] * job.dims[i];
  std::map<int, std::vector<int>> groups;
  for (int i = 0; i < job.n; ++i) groups[padded_dim(job.dims[i])].push_back(i);
  rcmps_slot& SL = ctx->slot[job.slot];
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t budget = std::max<size_t>((size_t)1 << 30, (free_b + SL.arena_bytes) * job.memory_share);
  cudaEventRecord(SL.ev[0], stream);
  const size_t scratch_budget = (size_t)1 << 30;

  for (auto& kv : groups) {
    const int dp = kv.first;
    const std::vector<int>& all = kv.second;
    int dmax = 0;
    for (int i : all) dmax = std::max(dmax, job.dims[i]);
    const int kmax = std::min(S.krylov_maxdim, dmax * dmax);
    const size_t per = kinetic_state_bytes(dp, kmax, nshift);
    const int cap = (int)std::max<size_t>(1, (budget - std::min(budget, scratch_budget)) / per);
    for (size_t start = 0; start < all.size(); start += cap) {
      const int n = (int)std::min<size_t>(cap, all.size() - start);
      const std::vector<int> idx(all.begin() + start, all.begin() + start + n);
      const int NP = 4 * n;
      const size_t mat = (size_t)dp * dp;
      const int nvec = dp * dp;
      const int nchunk = (nvec + CHROWS - 1) / CHROWS;
      const int ntile = (nvec + 63) / 64;   // column tiles of the residual partial sums
      const int nblk = (nshift + kContractNodesPerBlock - 1) / kContractNodesPerBlock;
      Layout L;
      const size_t o_dims = L.add(n * 4), o_off = L.add(n * 8), o_idx = L.add(n * 4);
      const size_t o_shift = L.add(nshift * 8), o_weight = L.add(nshift * 8);
      const size_t o_in = L.add(3 * n * mat * 16), o_ops = L.add(n * 8 * mat * 16);
      const size_t o_comm = L.add(n * 2 * mat * 16), o_rhs = L.add(n * 4 * mat * 16);
      const size_t o_probs = L.add(NP * sizeof(ArnoldiProblem));
      const size_t o_V = L.add((size_t)NP * (kmax + 1) * mat * 16);
      const size_t o_LV = L.add((size_t)NP * kmax * mat * 16);
      const size_t o_H = L.add((size_t)NP * (kmax + 1) * kmax * 16);
      const size_t o_W = L.add((size_t)NP * mat * 16);
      const size_t o_part = L.add((size_t)NP * nchunk * (kmax + 1) * 16);
      const size_t o_norms = L.add((size_t)NP * 2 * nchunk * 8);
      const size_t o_Yt = L.add((size_t)NP * nshift * kmax * 16);
      const size_t o_X = L.add((size_t)NP * nshift * mat * 16);
      const size_t o_flags = L.add(NP * 4 + n * 4);
      const size_t o_mtasks = L.add(NP * sizeof(LindbladTask));
      const size_t o_res = L.add((size_t)NP * nshift * ntile * 8);
      const size_t o_cpart = L.add((size_t)2 * n * nblk * 4 * mat * 16);
      const size_t o_fin = L.add((size_t)n * 12 * mat * 16);
      const size_t o_val = L.add(n * 8);
      const size_t o_ptrs = L.add((size_t)(4 * n + 5 * n) * sizeof(void*));
      const size_t o_scr = L.add(scratch_budget);
      cudaError_t e = arena_reserve(SL, L.total);
      if (e != cudaSuccess)
        return fail(ctx, RCMPS_OUT_OF_MEMORY, "kinetic workspace: " + std::to_string(L.total) + " bytes");
      char* base = static_cast<char*>(SL.arena);
      auto P = [&](size_t o) { return static_cast<void*>(base + o); };
      double2* d_in = (double2*)P(o_in);
      double2* d_ops = (double2*)P(o_ops);
      double2* d_comm = (double2*)P(o_comm);
      double2* d_rhs = (double2*)P(o_rhs);
      ArnoldiProblem* d_probs = (ArnoldiProblem*)P(o_probs);
      int* d_flags = (int*)P(o_flags);

      // host staging
      Layout H;
      const size_t h_dims = H.add(n * 4), h_off = H.add(n * 8), h_shift = H.add(nshift * 8),
                   h_weight = H.add(nshift * 8), h_probs = H.add(NP * sizeof(ArnoldiProblem)),
                   h_ptrs = H.add((size_t)9 * n * sizeof(void*)),
                   h_flag = H.add(n * 4), h_idx = H.add(n * 4);
      if (pinned_reserve(SL, H.total) != cudaSuccess) return fail(ctx, RCMPS_CUDA_ERROR, "pinned host buffer");
      char* h = static_cast<char*>(SL.pinned);
      int* hd = (int*)(h + h_dims);
      long long* ho = (long long*)(h + h_off);
      double* hs = (double*)(h + h_shift);
      double* hw = (double*)(h + h_weight);
      ArnoldiProblem* hp = (ArnoldiProblem*)(h + h_probs);
      const void** hptr = (const void**)(h + h_ptrs);
      int* hflag = (int*)(h + h_flag);
      int* hidx = (int*)(h + h_idx);
      for (int i = 0; i < n; ++i) {
        hd[i] = job.dims[idx[i]];
        ho[i] = off[idx[i]];
        hidx[i] = idx[i];
      }
      std::memcpy(hs, shifts.data(), nshift * 8);
      std::memcpy(hw, weights.data(), nshift * 8);
      e = cudaMemcpyAsync(P(o_dims), hd, n * 4, cudaMemcpyHostToDevice, stream);
      if (!e) e = cudaMemcpyAsync(P(o_off), ho, n * 8, cudaMemcpyHostToDevice, stream);
      if (!e) e = cudaMemcpyAsync(P(o_idx), hidx, n * 4, cudaMemcpyHostToDevice, stream);
      if (!e) e = cudaMemcpyAsync(P(o_shift), hs, nshift * 8, cudaMemcpyHostToDevice, stream);
      if (!e) e = cudaMemcpyAsync(P(o_weight), hw, nshift * 8, cudaMemcpyHostToDevice, stream);
      if (!e) e = cudaMemsetAsync(P(o_flags), 0, NP * 4 + n * 4, stream);
      if (!e) e = cudaMemsetAsync(P(o_H), 0, (size_t)NP * (kmax + 1) * kmax * 16, stream);
      double* dR = reinterpret_cast<double*>(d_in);
      double* dK = reinterpret_cast<double*>(d_in + n * mat);
      double* dP = reinterpret_cast<double*>(d_in + 2 * n * mat);
      if (!e) e = launch_pad(job.R, (long long*)P(o_off), (int*)P(o_dims), dR, dp, mat, n, stream);
      if (!e) e = launch_pad(job.K, (long long*)P(o_off), (int*)P(o_dims), dK, dp, mat, n, stream);
      if (!e) e = launch_pad(job.rho, (long long*)P(o_off), (int*)P(o_dims), dP, dp, mat, n, stream);
      if (!e) e = launch_prepare(dR, dK, dP, reinterpret_cast<double*>(d_ops), dp, mat, 8 * mat, n, stream);
      KineticSetup ks{dp, d_ops, (long long)(8 * mat), d_comm, d_rhs};
      if (!e) e = kinetic_rhs_launch(ks, n, stream);
      if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("kinetic set-up: ") + cudaGetErrorString(e));

      // problems: p = 4 i + q, q: 0 R fwd, 1 R adj, 2 C fwd, 3 C adj
      for (int i = 0; i < n; ++i) {
        const double2* ops = d_ops + (size_t)i * 8 * mat;
        for (int q = 0; q < 4; ++q) {
          const int p = 4 * i + q;
          ArnoldiProblem& A = hp[p];
          std::memset(&A, 0, sizeof(A));
          A.V = (double2*)P(o_V) + (size_t)p * (kmax + 1) * mat;
          A.LV = (double2*)P(o_LV) + (size_t)p * kmax * mat;
          A.ldv = (long long)mat;
          A.H = (double2*)P(o_H) + (size_t)p * (kmax + 1) * kmax;
          A.W = (double2*)P(o_W) + (size_t)p * mat;
          A.rhs = d_rhs + (size_t)i * 4 * mat + (size_t)q * mat;
          A.partial = (double2*)P(o_part) + (size_t)p * nchunk * (kmax + 1);
          A.norms = (double*)P(o_norms) + (size_t)p * 2 * nchunk;
          A.Yt = (double2*)P(o_Yt) + (size_t)p * nshift * kmax;
          A.X = (double2*)P(o_X) + (size_t)p * nshift * mat;
          const bool adj = q & 1;
          A.A1 = ops + (adj ? 1 : 0) * mat;    // Q or Q^dag
          A.A1h = ops + (adj ? 0 : 1) * mat;
          A.A2 = ops + (adj ? 3 : 2) * mat;    // R or R^dag
          A.A2h = ops + (adj ? 2 : 3) * mat;
          A.flag = d_flags + p;
          A.n = nvec;
          A.n_phys = hd[i] * hd[i];
          A.dp = dp;
          A.kmax = kmax;
          A.kmax1 = kmax + 1;
          A.adjoint = adj ? 1 : 0;
        }
      }
      e = cudaMemcpyAsync(d_probs, hp, NP * sizeof(ArnoldiProblem), cudaMemcpyHostToDevice, stream);
      if (!e) e = arnoldi_start_launch(d_probs, NP, stream);
      if (!e) e = cudaMemcpyAsync(hp, d_probs, NP * sizeof(ArnoldiProblem), cudaMemcpyDeviceToHost, stream);
      if (!e) e = cudaStreamSynchronize(stream);
      if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("kinetic start: ") + cudaGetErrorString(e));

      std::vector<int> done(NP, 0), failed(NP, 0);
      for (int p = 0; p < NP; ++p) {
        const int nphys = hp[p].n_phys;
        hp[p].target = std::min(S.krylov_initialdim, nphys);
        if (hp[p].beta == 0.0) done[p] = 1;   // zero right-hand side: zero solutions
        if (hp[p].nonfinite) failed[p] = 1;
      }
      int rounds = 0;
      while (true) {
        bool any = false;
        for (int p = 0; p < NP; ++p) any |= !done[p] && !failed[p];
        if (!any) break;
        if (++rounds > 64) return fail(ctx, RCMPS_KRYLOV_FAILURE, "kinetic: too many Arnoldi rounds");
        // ---- extend every open problem from k to target
        int jlo = 1 << 30, jhi = 0;
        for (int p = 0; p < NP; ++p) {
          ArnoldiProblem& A = hp[p];
          A.active = !done[p] && !failed[p] && !A.exhausted && A.k < A.target;
          A.solve = !done[p] && !failed[p];
          A.reconstruct = 0;
          A.estimate = 0.0;
          if (A.active) {
            jlo = std::min(jlo, A.k);
            jhi = std::max(jhi, A.target);
          }
        }
        e = cudaMemcpyAsync(d_probs, hp, NP * sizeof(ArnoldiProblem), cudaMemcpyHostToDevice, stream);
        for (int j = jlo; j < jhi && !e; ++j) {
          e = lindblad_arnoldi_launch(dp, d_probs, NP, j, stream);
          if (!e) e = gram_schmidt_launch(d_probs, NP, j, nvec, ctx->sms, stream);
        }
        // ---- projected solves of every open problem
        int kcur = 1;
        if (!e) e = cudaMemcpyAsync(hp, d_probs, NP * sizeof(ArnoldiProblem), cudaMemcpyDeviceToHost, stream);
        if (!e) e = cudaStreamSynchronize(stream);
        if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("kinetic Arnoldi: ") + cudaGetErrorString(e));
        for (int p = 0; p < NP; ++p) {
          ArnoldiProblem& A = hp[p];
          if (A.nonfinite && !done[p]) failed[p] = RCMPS_NONFINITE_RESULT;
          A.active = 0;
          A.solve = !done[p] && !failed[p] && A.k > 0;
          A.estimate = 0.0;
          if (A.solve) kcur = std::max(kcur, A.k);
        }
        const long long slot = (long long)kcur * (kcur + 1) / 2 + kcur;
        const int ntask = NP * nshift;
        const int nslots = (int)std::max<long long>(32, std::min<long long>(ntask, scratch_budget / (slot * 16)));
        e = cudaMemcpyAsync(d_probs, hp, NP * sizeof(ArnoldiProblem), cudaMemcpyHostToDevice, stream);
        if (!e) e = hessenberg_launch(d_probs, NP, (double*)P(o_shift), nshift, (double2*)P(o_scr), slot, nslots,
                                      kcur, stream);
        if (!e) e = cudaMemcpyAsync(hp, d_probs, NP * sizeof(ArnoldiProblem), cudaMemcpyDeviceToHost, stream);
        if (!e) e = cudaStreamSynchronize(stream);
        if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("kinetic projected solves: ") + cudaGetErrorString(e));
        // ---- reconstruct and check the candidates
        bool anyrec = false;
        for (int p = 0; p < NP; ++p) {
          ArnoldiProblem& A = hp[p];
          A.solve = 0;
          if (done[p] || failed[p]) continue;
          const int maxdim = std::min(S.krylov_maxdim, A.n_phys);
          const bool terminal = A.exhausted || A.k >= maxdim;
          A.reconstruct = std::isfinite(A.estimate) && (A.estimate <= S.krylov_tolerance || terminal);
          anyrec |= A.reconstruct;
        }
        if (anyrec) {
          // reconstruction and true residuals in one pass over the basis and its kept actions
          e = cudaMemcpyAsync(d_probs, hp, NP * sizeof(ArnoldiProblem), cudaMemcpyHostToDevice, stream);
          if (!e) e = reconstruct_residual_launch(d_probs, NP, (double*)P(o_shift), nshift, nvec, (double*)P(o_res), stream);
          if (!e) e = residual_reduce_launch(d_probs, NP, (double*)P(o_res), nshift, ntile, stream);
          if (!e) e = cudaMemcpyAsync(hp, d_probs, NP * sizeof(ArnoldiProblem), cudaMemcpyDeviceToHost, stream);
          if (!e) e = cudaStreamSynchronize(stream);
          if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("kinetic residuals: ") + cudaGetErrorString(e));
        }
        for (int p = 0; p < NP; ++p) {
          ArnoldiProblem& A = hp[p];
          if (done[p] || failed[p]) continue;
          const int maxdim = std::min(S.krylov_maxdim, A.n_phys);
          const bool terminal = A.exhausted || A.k >= maxdim;
          if (A.reconstruct) {
            if (std::isfinite(A.residual) && A.residual <= S.krylov_tolerance) {
              done[p] = 1;
              continue;
            }
            if (A.exhausted) {
              failed[p] = RCMPS_KRYLOV_FAILURE;
              continue;
            }
          }
          if (terminal) {
            failed[p] = RCMPS_KRYLOV_FAILURE;
            continue;
          }
          A.target = std::min(2 * A.k, maxdim);
        }
      }
      for (int i = 0; i < n; ++i) {
        rcmps_state_stats& st = job.stats[idx[i]];
        double worst = 0.0;
        for (int q = 0; q < 4; ++q) {
          const ArnoldiProblem& A = hp[4 * i + q];
          st.krylov_basis[q] = A.k;
          if (A.reconstruct || A.residual > 0) worst = std::max(worst, A.residual);
          if (failed[4 * i + q] && !st.status) {
            st.status = failed[4 * i + q];
            st.failed_component = 3;
          }
        }
        st.krylov_residual = worst;
      }
      bool any_failed = false;
      for (int p = 0; p < NP; ++p) any_failed |= failed[p] != 0;
      if (any_failed) {
        ctx->error = "kinetic: a shifted Arnoldi problem did not reach its true residual";
        cudaStreamSynchronize(stream);
        return RCMPS_KRYLOV_FAILURE;
      }
      // zero solutions for zero right-hand sides
      for (int p = 0; p < NP; ++p)
        if (hp[p].beta == 0.0 && !e) e = cudaMemsetAsync(hp[p].X, 0, (size_t)nshift * mat * 16, stream);
      // ---- contraction
      const void** pX = hptr;             // [2n]
      const void** pA = hptr + 2 * n;     // [2n]
      const void** pQ = hptr + 4 * n;
      const void** pQh = hptr + 5 * n;
      const void** pR = hptr + 6 * n;
      const void** pRh = hptr + 7 * n;
      const void** prho = hptr + 8 * n;
      for (int i = 0; i < n; ++i) {
        const double2* ops = d_ops + (size_t)i * 8 * mat;
        pX[2 * i] = hp[4 * i + 0].X;
        pA[2 * i] = hp[4 * i + 1].X;
        pX[2 * i + 1] = hp[4 * i + 2].X;
        pA[2 * i + 1] = hp[4 * i + 3].X;
        pQ[i] = ops;
        pQh[i] = ops + mat;
        pR[i] = ops + 2 * mat;
        pRh[i] = ops + 3 * mat;
        prho[i] = ops + 7 * mat;
      }
      const void** dptr = (const void**)P(o_ptrs);
      if (!e) e = cudaMemcpyAsync(dptr, hptr, (size_t)9 * n * sizeof(void*), cudaMemcpyHostToDevice, stream);
      ContractArgs ca;
      ca.dp = dp;
      ca.nstates = n;
      ca.nodes = nshift;
      ca.nodes_per_block = kContractNodesPerBlock;
      ca.X = (const double2* const*)dptr;
      ca.A = (const double2* const*)(dptr + 2 * n);
      ca.Q = (const double2* const*)(dptr + 4 * n);
      ca.Qh = (const double2* const*)(dptr + 5 * n);
      ca.R = (const double2* const*)(dptr + 6 * n);
      ca.Rh = (const double2* const*)(dptr + 7 * n);
      ca.rho = (const double2* const*)(dptr + 8 * n);
      ca.weights = (double*)P(o_weight);
      ca.shifts = (double*)P(o_shift);
      ca.partial = (double2*)P(o_cpart);
      ca.fin = (double2*)P(o_fin);
      ca.value_out = (double*)P(o_val);
      ca.error_flag = d_flags + NP;
      if (!e) e = contract_launch(ca, nblk, stream);
      // outputs: covector (fin slot 9) and environment (slot 10) of each state, unpadded
      if (!e && job.covector)
        e = launch_unpad_acc(reinterpret_cast<double*>((double2*)P(o_fin) + 9 * mat), (long long)(12 * mat), dp,
                             (long long*)P(o_off), (int*)P(o_dims), job.covector, n, job.accumulate, stream);
      if (!e && job.environment)
        e = launch_unpad_acc(reinterpret_cast<double*>((double2*)P(o_fin) + 10 * mat), (long long)(12 * mat), dp,
                             (long long*)P(o_off), (int*)P(o_dims), job.environment, n, job.accumulate, stream);
      if (!e && job.value)
        e = launch_scatter_values((double*)P(o_val), n, (int*)P(o_idx), job.value, job.accumulate, stream);
      std::vector<double> vals(n);
      if (!e) e = cudaMemcpyAsync(hflag, d_flags + NP, n * 4, cudaMemcpyDeviceToHost, stream);
      if (!e) e = cudaMemcpyAsync(vals.data(), P(o_val), n * 8, cudaMemcpyDeviceToHost, stream);
      if (!e) e = cudaStreamSynchronize(stream);
      if (e) return fail(ctx, RCMPS_CUDA_ERROR, std::string("kinetic contraction: ") + cudaGetErrorString(e));
      for (int i = 0; i < n; ++i) {
        rcmps_state_stats& st = job.stats[idx[i]];
        st.kinetic_value = vals[i];
        if (!std::isfinite(vals[i]) && !st.status) {
          st.status = RCMPS_NONFINITE_RESULT;
          st.failed_component = 3;
        }
        if (hflag[i] && !st.status) {
          st.status = RCMPS_WAIT_LIMIT;
          st.failed_component = 3;
        }
      }
    }
  }
  cudaEventRecord(SL.ev[1], stream);
  cudaEventSynchronize(SL.ev[1]);
  cudaEventElapsedTime(&ctx->last_ms[2], SL.ev[0], SL.ev[1]);
  for (int i = 0; i < job.n; ++i)
    if (job.stats[i].status) return job.stats[i].status;
  return RCMPS_OK;
}

}  // namespace rcmps
