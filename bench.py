"""Benchmark: fg_phi4 evaluations per second (energy + finished gradient) on B200.

Workload (default): 32 states at D = 64 — 16 random + 16 Z2-symmetric (i.i.d. standard complex
Gaussian entries times 0.2, NumPy PCG64 seeds), g = 2 — at the reference optimizer's settings
(W = 30, n_quad = 512, atol/rtol 1e-13/1e-12, 512 kinetic nodes, Krylov 1e-12, metric_reg 1e-3).
A step is one batched fg_phi4 call over all states; rho is computed once (untimed) by the
library's stationary solve. Inputs and workspaces (about 30 GB) exceed the 126 MB L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With N > 1 (torchrun, one rank per GPU) every rank evaluates its own shard of states: no data-path
collective (weak scaling); the elapsed time is the maximum over ranks. --impl reference times the
CPU oracle (the NumPy restatement of the reference's path) on all host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT), str(ROOT / "rcmpscore.jl_b200")]

import numpy as np  # noqa: E402

METRIC = "fg_phi4 evals/s at D=64 (energy + finished gradient), FP64"
METRIC_SPLIT = ("fg_phi4 evals/s at D=64 (energy + finished gradient), split-precision trajectory products "
                "(BF16 slices on tcgen05) vs FP64, |dE/E|<=1e-10")
FLOPS_PER_RHS_D3 = 224      # 28 complex D^3 products (8 flops per complex multiply-add) per right-hand side
# BF16 tensor flops the split engine executes per right-hand side of one D = 64 state (4 CTAs):
# per CTA and chunk 28 slice pairs x 2 MMAs of M = 64, K = 16 and N = N_cat; chunks: 7 G1 units x 4
# (N_cat 64), 3 paired G2 units x 8 (N_cat 64), 1 single G2 unit x 8 (N_cat 32)
SPLIT_FLOPS_PER_RHS = 4 * 28 * 2 * 2 * 64 * 16 * (7 * 4 * 64 + 3 * 8 * 64 + 1 * 8 * 32)


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------- CPU oracle sample
def _cpu_eval(args):
    """One full fg_phi4 evaluation (quartic trajectory + pullback, kinetic, boundary/metric
    solve) of one workload state with the oracle on one core; returns its seconds. rho is
    computed first, untimed, as the B200 arm computes it before its timed region."""
    d, seed, z2, g = args
    sys.path[:0] = [str(ROOT), str(ROOT / "rcmpscore.jl_b200")]
    from threadpoolctl import threadpool_limits
    from oracle import fg_phi4_oracle as O
    from rcmps_b200.batch import random_state, z2_state
    with threadpool_limits(limits=1):   # one core per evaluation: BLAS single-threaded
        R, K = (z2_state if z2 else random_state)(d, seed)
        Q = O.left_canonical_q(R, K)
        rho = O.stationary_state(Q, R, tolerance=1e-13, method="krylov")
        t0 = time.perf_counter()
        # Z2 states on the packed route, as the reference's persistent trajectory takes them, and
        # the boundary solve preconditioned as the reference solves it
        O.fg_phi4(R, K, rho, g, method="preconditioned", packed_z2=z2)
        return time.perf_counter() - t0


def cpu_eval_plan(workload):
    """(d, seed, z2, g) of every state of d64_mixed or d64_single (the seeds of rcmps_b200.batch)."""
    if workload == "d64_single":
        return [(64, 0, False, 2.0)]
    if workload != "d64_mixed":
        return None
    return [(64, i, False, 2.0) for i in range(16)] + [(64, 100 + i, True, 2.0) for i in range(16)]


def single_state_latency(steps):
    """Latency of one evaluation of the first random D = 64 state of the workload through the
    public single-state call (rcmps_b200.objective.objective, host arrays in and out), the call an
    L-BFGS trial makes: wall time per call after one untimed call, the device phases of the last
    call, and the trajectory's layout (CTAs per state)."""
    import ctypes as C
    from rcmps_b200 import objective
    from rcmps_b200.batch import random_state
    R, K = random_state(64, 0)
    Q = -1j * K - R.conj().T @ R / 2
    rho, _ = objective.stationary_state(Q, R, tolerance=1e-13)
    args = objective.default_args()
    e, _, st = objective.objective(R, K, rho, 2.0, args)
    walls = []
    for _ in range(steps):
        t0 = time.perf_counter()
        e, _, st = objective.objective(R, K, rho, 2.0, args)
        walls.append(time.perf_counter() - t0)
    ctx = objective.context()
    t = ctx.timings()
    groups = C.c_int(0)
    ctx.lib.rcmps_trajectory_groups(ctx.handle, 0, 64, C.byref(groups))
    return {"workload": "1 random state D=64 (seed 0, scaling 0.2), g=2, the benchmark's settings",
            "api": "rcmps_b200.objective.objective (host arrays in and out)", "steps": steps,
            "ms_per_eval": 1000 * statistics.mean(walls), "ms_min": 1000 * min(walls),
            "phases_ms_last_call": {"trajectory": t[0], "pullback": t[1], "kinetic": t[2], "boundary_finish": t[3],
                                    "whole_call": t[4], "boundary_prepare_beside_trajectory": t[5],
                                    "boundary_gmres": t[6]},
            "trajectory_ctas_per_state": 4 * groups.value, "channel_groups": groups.value,
            "rhs_calls": st["rhs_calls"], "accepted": st["accepted"], "rejected": st["rejected"], "energy": e}


# ----------------------------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    """The oracle (the NumPy restatement of the reference's path) on the host cores: one state per
    worker process and step, every evaluation complete; rank 0 only."""
    if rank != 0:
        return
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    from rcmps_b200.batch import config_states
    desc = config_states(args.workload)[3]
    plan = cpu_eval_plan(args.workload)
    workers = min(cores, len(plan))
    for var in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"      # inherited by the spawned workers: one core each
    ctx = mp.get_context("spawn")
    walls = []
    with ctx.Pool(workers) as pool:
        for step in range(args.warmup + args.steps):
            chunk = [plan[(step * workers + i) % len(plan)] for i in range(workers)]
            t0 = time.perf_counter()
            pool.map(_cpu_eval, chunk)
            wall = time.perf_counter() - t0
            if step >= args.warmup:
                walls.append(wall)
    value = workers * len(walls) / sum(walls)
    sample = (f"each step: {workers} workload states, one complete fg_phi4 evaluation per worker process "
              f"(oracle, single-threaded BLAS), states taken in turn from the {len(plan)}-state workload")
    line = {"metric": METRIC, "value": value, "unit": "evals/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * statistics.mean(walls),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "half_window": 30.0, "n_quad": 512, "kinetic_nodes": 512},
            "cpu_baseline": {"value": value, "unit": "evals/s", "cores": workers, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- B200 arm
def run_b200(args, rank, world, local_rank):
    import torch
    from rcmps_b200 import _lib
    from rcmps_b200.batch import config_states, shard
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    ctx = _lib.Context(local_rank)
    lib = ctx.lib
    R, K, g, desc = config_states(args.workload)
    tolerances = None
    if args.workload == "uneven200":      # per-state (atol, rtol) pairs in the same launch
        from rcmps_b200.batch import uneven_states
        tolerances = uneven_states(len(R))[3]
    dims_all = [len(r) for r in R]
    mine = shard(dims_all, rank, world)
    R = [R[i] for i in mine]
    K = [K[i] for i in mine]
    g = [g[i] for i in mine]
    controls = None
    if tolerances is not None:
        controls = (_lib.StateControls * len(mine))(*(_lib.StateControls(*tolerances[i]) for i in mine))
    dims = [len(r) for r in R]
    n = len(dims)
    total = sum(d * d for d in dims)
    # the quartic route of each state as the reference takes it: packed Z2 for the Z2 states,
    # the unpacked channels for the others
    split = args.precision == "split"
    s = _lib.default_settings(symmetry=2 if args.quartic_route == "auto" else 0, precision=1 if split else 0,
                              half_window=args.half_window, n_quad=args.n_quad,
                              trajectory_groups=args.trajectory_groups)
    cdims = (C.c_int * n)(*dims)
    cg = (C.c_double * n)(*g)
    pack = lambda L: torch.from_numpy(np.concatenate([np.ascontiguousarray(x).ravel() for x in L])).cuda()
    dR, dK = pack(R), pack(K)
    drho = torch.zeros_like(dR)
    stats = (_lib.StateStats * n)()
    torch.cuda.synchronize()
    rc = lib.rcmps_stationary_state_batch(ctx.handle, n, cdims, dR.data_ptr(), dK.data_ptr(), C.c_double(1e-13),
                                          drho.data_ptr(), stats, None)
    if rc:
        raise RuntimeError(f"stationary states failed: {ctx.error()}")
    energy = torch.zeros(n, dtype=torch.float64, device="cuda")
    grad = torch.zeros(total, dtype=torch.complex128, device="cuda")
    stream = torch.cuda.current_stream()
    sptr = C.c_void_p(stream.cuda_stream)

    quartic_only = args.component == "quartic"
    cov = torch.zeros(total, dtype=torch.complex128, device="cuda") if quartic_only else None

    def step(settings=s):
        if quartic_only:   # the quartic term alone (trajectory + pullback): the small profiling case
            rc = lib.rcmps_quartic_batch(ctx.handle, n, cdims, cg, dR.data_ptr(), dK.data_ptr(), drho.data_ptr(),
                                         C.byref(settings), energy.data_ptr(), cov.data_ptr(), grad.data_ptr(), stats,
                                         sptr)
        else:
            rc = lib.rcmps_fg_phi4_batch_controls(ctx.handle, n, cdims, cg, dR.data_ptr(), dK.data_ptr(),
                                                  drho.data_ptr(), C.byref(settings), controls, energy.data_ptr(),
                                                  grad.data_ptr(), None, None, stats, sptr)
        if rc:
            raise RuntimeError(f"{args.component} failed: {_lib.STATUS_NAMES.get(rc)} {ctx.error()}")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    traj_ms, pull_ms, kin_ms, fin_ms, call_ms, prep_ms, gmres_ms = [], [], [], [], [], [], []
    barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = lib.rcmps_launch_count()   # library launches before the timed region
    with ClockSampler(local_rank) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
            t = ctx.timings()
            traj_ms.append(t[0])
            pull_ms.append(t[1])
            kin_ms.append(t[2])
            fin_ms.append(t[3])
            prep_ms.append(t[5])
            gmres_ms.append(t[6])
            call_ms.append(t[4])
        end.record(stream)
        barrier()
    launches = (lib.rcmps_launch_count() - launches0) // args.steps
    elapsed = start.elapsed_time(end)
    if dist is not None:
        t = torch.tensor([elapsed], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    total_states = len(dims_all)
    value = total_states * args.steps / (elapsed / 1000.0)
    rhs_calls = [stats[i].rhs_calls for i in range(n)]
    # roofline of the dominant kernel: the trajectory (FP64 tensor cores, mma.sync m16n8k8)
    # a packed Z2 state needs a quarter of the products: each output block and each K half of a
    # product is one of two parity blocks, the other is a structural zero
    packed = [bool(stats[i].packed_z2) for i in range(n)]
    flops = sum(FLOPS_PER_RHS_D3 * rhs_calls[i] * dims[i] ** 3 * (0.25 if packed[i] else 1.0) for i in range(n))
    traj = statistics.mean(traj_ms)
    achieved = flops / (traj / 1000.0) / 1e12
    peak = lib.rcmps_fp64_peak_tflops(ctx.handle)
    def split_roofline_of(traj_ms_split, rhs):
        # the split engine runs on the BF16 tensor pipe: executed BF16 flops against the measured
        # sustained cuBLAS BF16 throughput (the kernel runs inside a long step)
        bf16 = sum(SPLIT_FLOPS_PER_RHS * rhs[i] for i in range(n) if dims[i] == 64)
        fp64eq = sum(FLOPS_PER_RHS_D3 * rhs[i] * dims[i] ** 3 * (0.25 if packed[i] else 1.0) for i in range(n))
        peaks = {}
        pf = ROOT / "MEASURED_PEAKS.json"
        if pf.exists():
            try:
                peaks = json.loads(pf.read_text())
            except (OSError, ValueError):
                peaks = {}
        bpeak = peaks.get("bf16_tflops_sustained") or 1400.0
        rate = bf16 / (traj_ms_split / 1000.0) / 1e12
        return {"bound": "tensor", "achieved": rate, "peak": bpeak, "unit": "TFLOP/s", "frac": rate / bpeak,
                "traffic": None,
                "kernel": "trajectory_kernel<64, quartic, split> (tcgen05.mma kind::f16, BF16 slices)",
                "peak_source": ("MEASURED_PEAKS.json bf16_tflops_sustained (of measured)"
                                if peaks.get("bf16_tflops_sustained") else "fallback 1.4 PFLOP/s"),
                "flops_per_launch": bf16, "launch_ms": traj_ms_split,
                "fp64_equivalent_tflops": fp64eq / (traj_ms_split / 1000.0) / 1e12}

    split_roofline = split_roofline_of(traj, rhs_calls) if split else None
    # DRAM traffic of one launch: bytes per right-hand side of one state times this launch's
    # right-hand sides. The rate comes from an ncu capture of this very launch where one was taken
    # (the default 32-state workload and layout: its stage vectors exceed L2 and are re-read from
    # DRAM), otherwise from a two-state capture at the same D, a lower bound for larger batches.
    traffic = None
    tf = ROOT / "profiles" / "trajectory_traffic.json"
    if tf.exists():
        try:
            rec = json.loads(tf.read_text())
            full = rec.get("measured_launches", {}).get(args.workload)
            default_layout = (not split and args.trajectory_groups == 0 and args.quartic_route == "auto"
                              and args.half_window == 30.0 and args.n_quad == 512 and not quartic_only)
            if full and default_layout:
                traffic = full["dram_bytes_per_state_rhs"] * sum(rhs_calls[i] for i in range(n))
            else:
                per = rec.get("dram_bytes_per_state_rhs", {})
                if all(str(d) in per for d in dims):
                    traffic = sum(per[str(dims[i])] * rhs_calls[i] for i in range(n))
        except (OSError, ValueError, KeyError):
            traffic = None

    # end to end through the host-buffer C entry: copies of inputs and results inside the timed region
    e2e = None
    if not quartic_only:
        hR = torch.from_numpy(np.concatenate([x.ravel() for x in R])).pin_memory()
        hK = torch.from_numpy(np.concatenate([x.ravel() for x in K])).pin_memory()
        hP = drho.cpu().pin_memory()
        hE = torch.zeros(n, dtype=torch.float64).pin_memory()
        hG = torch.zeros(total, dtype=torch.complex128).pin_memory()
        e2e_steps = args.steps

        rho_host = None
        if tolerances is not None:
            from rcmps_b200 import objective
            rho_np = hP.numpy()
            offs = np.cumsum([0] + [d * d for d in dims])
            rho_host = [rho_np[offs[i]:offs[i + 1]].reshape(dims[i], dims[i]) for i in range(n)]

        def host_step():
            if tolerances is not None:   # per-state tolerances: the Python entry on host arrays
                objective.fg_phi4_batch(R, K, rho_host, g, s, tolerances=[tolerances[i] for i in mine])
                return
            rc = lib.rcmps_fg_phi4_batch_host(ctx.handle, n, cdims, cg, hR.data_ptr(), hK.data_ptr(), hP.data_ptr(),
                                              C.byref(s), hE.data_ptr(), hG.data_ptr(), None, None, stats)
            if rc:
                raise RuntimeError(f"fg_phi4 (host buffers) failed: {ctx.error()}")

        host_step()   # untimed: the host entry's first call
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            host_step()
        barrier()
        wall = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([wall], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            wall = float(t.item())
        e2e = {"value": total_states * e2e_steps / wall, "unit": "evals/s",
               "h2d_bytes_per_step": 3 * total * 16 * world, "d2h_bytes_per_step": (n * 8 + total * 16) * world}

    def split_error_of():
        """Per-state error of the split form against the FP64 form on the same states (untimed)."""
        s_split = _lib.default_settings(symmetry=s.symmetry, precision=1, half_window=s.half_window, n_quad=s.n_quad)
        s64 = _lib.default_settings(symmetry=s.symmetry, precision=0, half_window=s.half_window, n_quad=s.n_quad)
        step(s_split)
        E_s, G_s = energy.cpu().numpy().copy(), grad.cpu().numpy().copy()
        acc_s = [stats[i].accepted for i in range(n)]
        step(s64)
        E_f, G_f = energy.cpu().numpy(), grad.cpu().numpy()
        acc_f = [stats[i].accepted for i in range(n)]
        rho_h = drho.cpu().numpy()
        rows, o = [], 0
        for i in range(n):
            d = dims[i]
            rho_i = rho_h[o:o + d * d].reshape(d, d)
            m = rho_i + 1e-3 * np.eye(d)
            dg = (G_s[o:o + d * d] - G_f[o:o + d * d]).reshape(d, d)
            gf = G_f[o:o + d * d].reshape(d, d)
            metric = lambda x: float(np.sqrt(max(0.0, 2.0 * np.real(np.vdot(x, x @ m)))))
            rows.append({"state": mine[i], "rel_energy": abs(E_s[i] - E_f[i]) / abs(E_f[i]),
                         "rel_gradient": metric(dg) / max(1.0, metric(gf)),
                         "accepted_split": acc_s[i], "accepted_fp64": acc_f[i]})
            o += d * d
        return {"against": "the FP64 tensor-core form of this library on the same states",
                "max_rel_energy": max(r["rel_energy"] for r in rows),
                "max_rel_gradient": max(r["rel_gradient"] for r in rows), "per_state": rows}

    split_error = split_error_of() if split and not quartic_only else None

    # the split-precision arm beside the FP64 one in the default run: the same workload and timing
    split_arm = None
    if (not split and not quartic_only and args.split_arm_steps > 0 and args.workload == "d64_mixed"
            and any(d == 64 for d in dims)):
        s_split = _lib.default_settings(symmetry=s.symmetry, precision=1, half_window=s.half_window, n_quad=s.n_quad)
        step(s_split)                          # warm-up
        barrier()
        t_ms = []
        st0, st1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st0.record(stream)
        for _ in range(args.split_arm_steps):
            step(s_split)
            t_ms.append(ctx.timings()[0])
        st1.record(stream)
        barrier()
        el = st0.elapsed_time(st1)
        if dist is not None:
            t = torch.tensor([el], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        rhs_s = [stats[i].rhs_calls for i in range(n)]
        v_split = total_states * args.split_arm_steps / (el / 1000.0)
        split_arm = {"metric": METRIC_SPLIT, "value": v_split, "unit": "evals/s",
                     "steps": args.split_arm_steps, "warmup": 1, "ms_per_step": el / args.split_arm_steps,
                     "ratio_to_fp64": v_split / value, "trajectory_ms": statistics.mean(t_ms),
                     "roofline": split_roofline_of(statistics.mean(t_ms), rhs_s), "split_error": split_error_of()}

    # the latency of one lone state through the single-state call (the L-BFGS caller's view)
    single = None
    if not quartic_only and world == 1 and args.workload == "d64_mixed" and args.single_steps > 0:
        single = single_state_latency(args.single_steps)

    # the learned GMRES preconditioner of the boundary solve: trained on the plain solver's triples
    # along a seeded optimizer-like path, measured on a held-out state of it against the fallback
    learned = None
    if not quartic_only and args.learned_d > 0 and world == 1 and args.workload == "d64_mixed":
        from rcmps_b200.warmstart import path_experiment
        learned = path_experiment(args.learned_d, train_states=args.learned_states, rhs_per_state=512, test_rhs=64,
                                  epochs=args.learned_epochs)
        learned["config"] = (f"D={args.learned_d}: {args.learned_states} states of a seeded path (relative steps "
                             "1e-2), 512 traceless Gaussian right-hand sides each, 64 held-out right-hand sides of the "
                             "next state; target |r| <= 1e-13 max(1, |b|)")

    cpu = None
    plan = cpu_eval_plan(args.workload)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and plan:
        t_eval = _cpu_eval(plan[0])
        cpu = {"value": 1.0 / t_eval, "unit": "evals/s", "cores": 1, "kind": "port",
               "sample": (f"one complete fg_phi4 evaluation of workload state 0 (D={plan[0][0]}, random, seed "
                          f"{plan[0][1]}) with the oracle on one core: {t_eval:.1f} s")}
    if rank == 0:
        metric = METRIC_SPLIT if split else METRIC
        if args.workload == "uneven200":
            metric = ("fg_phi4 evals/s, 200 states D in {16..128} with per-state atol/rtol in one batched call, "
                      + ("split" if split else "FP64"))
        if quartic_only:
            metric = "quartic term (trajectory + pullback) evals/s at D=64, " + ("split" if split else "FP64")
        line = {"metric": metric, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": elapsed / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": desc, "states_per_gpu": n, "half_window": args.half_window,
                           "n_quad": args.n_quad,
                           "kinetic_nodes": 512, "atol": 1e-13, "rtol": 1e-12, "krylov_tolerance": 1e-12,
                           "l2": "inputs and workspaces exceed L2 (126 MB); no flush needed", "parallelism":
                           f"state shards over {world} GPU(s)",
                           "quartic_route": ("packed Z2 for the Z2 states (error norm over 10 (D/2)^2 + 1 entries, "
                                             "structural zeros skipped), unpacked channels for the random states"
                                             if args.quartic_route == "auto" else
                                             "unpacked channels for every state")},
                "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                             "frac": achieved / peak if peak else None, "traffic": traffic,
                             "kernel": "trajectory_kernel<64> (FP64 mma.sync m16n8k8)",
                             "peak_source": "FP64 mma.sync throughput measured in this run (rcmps_fp64_peak_tflops)",
                             "flops_per_launch": flops, "launch_ms": traj},
                "phases_ms": {"trajectory": traj, "pullback": statistics.mean(pull_ms),
                              "kinetic": statistics.mean(kin_ms), "boundary_finish": statistics.mean(fin_ms),
                              "whole_call": statistics.mean(call_ms),
                              "boundary_prepare_beside_trajectory": statistics.mean(prep_ms),
                              "boundary_gmres": statistics.mean(gmres_ms)},
                "steps_per_state": {"rhs_calls_mean": statistics.mean(rhs_calls), "accepted_mean":
                                    statistics.mean(stats[i].accepted for i in range(n)),
                                    "gmres_iterations_mean": statistics.mean(stats[i].gmres_iterations for i in range(n)),
                                    "krylov_basis_max": max(max(stats[i].krylov_basis) for i in range(n)),
                                    "packed_z2_states": sum(packed),
                                    "rhs_calls_max_unpacked": max([rhs_calls[i] for i in range(n) if not packed[i]],
                                                                  default=0),
                                    "rhs_calls_max_packed": max([rhs_calls[i] for i in range(n) if packed[i]],
                                                                default=0)},
                "gpu_launches": None, "gpu_launches_note": "library kernel launches per step (rcmps_launch_count)", "clocks": clocks.summary(), "e2e": e2e, "cpu_baseline": cpu}
        line["gpu_launches"] = launches
        line["launches_before_timed"] = launches0
        tuning = {}
        for dp in sorted(set(((d + 15) // 16) * 16 if d <= 64 else (96 if d <= 96 else 128) for d in dims)):
            ring, ms = C.c_int(0), (C.c_float * 3)()
            if lib.rcmps_trajectory_tuning(ctx.handle, 0, dp, C.byref(ring), ms) == 0 and ring.value:
                tuning[str(dp)] = {"ring_stages": ring.value,
                                   "ms_per_1000_rhs_at_depth_2_3_4": [round(x, 3) for x in ms]}
        line["config"]["autotuned_tiles"] = tuning
        line["config"]["precision"] = ("split: trajectory products of the D=64 states on tcgen05 BF16 slices "
                                       "(7 x 7 bits), FP64 step control, sums and solves" if split else
                                       "FP64 tensor cores (DMMA)")
        if split_arm is not None:
            line["split_precision_arm"] = split_arm
        if learned is not None:
            line["learned_gmres"] = learned
        if single is not None:
            line["single_state"] = single
        if split:
            line["dtype"] = "f64 (split bf16 trajectory products)"
            line["roofline_fp64_form"] = line["roofline"]
            line["roofline"] = split_roofline
            line["split_error"] = split_error
        print(json.dumps(line), flush=True)


def main():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("b200", "reference"), default="b200")
    p.add_argument("--workload", default="d64_mixed")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--quartic-route", choices=("auto", "unpacked"), default="auto",
                   help="auto: the packed Z2 route for the Z2 states (the reference's default for them); "
                        "unpacked: the seven unpacked channels for every state")
    p.add_argument("--half-window", type=float, default=30.0,
                   help="window W of the integration (profiling cases only; the benchmark uses 30)")
    p.add_argument("--n-quad", type=int, default=512,
                   help="Gauss nodes per half window (profiling cases only; the benchmark uses 512)")
    p.add_argument("--precision", choices=("fp64", "split"), default="fp64",
                   help="trajectory products: FP64 tensor cores, or split BF16 slices on tcgen05 (D = 64)")
    p.add_argument("--learned-d", type=int, default=32,
                   help="bond dimension of the learned-preconditioner measurement (0: none)")
    p.add_argument("--learned-states", type=int, default=8, help="training states of that measurement")
    p.add_argument("--learned-epochs", type=int, default=100, help="training epochs of that measurement")
    p.add_argument("--split-arm-steps", type=int, default=3,
                   help="steps of the split-precision arm timed after the FP64 one (0: none)")
    p.add_argument("--trajectory-groups", type=int, choices=(0, 1, 2, 4), default=0,
                   help="CTAs per 16-row block of a state's trajectory cluster (0: chosen per launch)")
    p.add_argument("--single-steps", type=int, default=3,
                   help="timed calls of the single-state latency measurement (0: none)")
    p.add_argument("--component", choices=("fg", "quartic"), default="fg",
                   help="time the whole evaluation (default) or the quartic term alone")
    args = p.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        run_b200(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
