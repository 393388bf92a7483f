"""Accuracy refinement of an optimized state on the B200 library: the reference's final validation.

Mirrors gpu/src/rcmps_gpu/optimizer/validate_sweep.py of rcmps_gpu:
  * five objective evaluations of the state: three at the run's own controls (one cold, two
    warm) and two refined ones at W = 40, n_quad = 1024, atol 1e-14, rtol 1e-13 with 512 and
    1024 kinetic nodes (validate_sweep.py:91-97);
  * per row the energy, the finished gradient's metric norm and its differences from the first
    row and from the cached gradient of the checkpoint, <phi> in closed form at the row's window,
    and the pass test of the reference (validate_sweep.py:120-124);
  * <phi> again by the ODE of the first monomial at the refined controls (phi_by_ode).
Every evaluation runs on the GPU through the library; <phi> in closed form is a trace of two
D x D host matrices times a one-dimensional source integral (ode_backend.py:782-797).
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import math
import time
from pathlib import Path
from types import SimpleNamespace

import numpy as np

from . import _lib, objective

__all__ = ["source_integral", "phi_expectation", "phi_by_ode", "ROWS", "REFINED", "validate_state", "main"]

# Rows of the validation (validate_sweep.py:91-97): name, kinetic nodes (None: the run's own).
ROWS = (("standard_cold", None), ("standard_warm_1", None), ("standard_warm_2", None),
        ("refined_512", 512), ("refined_1024", 1024))
# The refined integration controls.
REFINED = dict(window=40.0, quadrature=1024, atol=1e-14, rtol=1e-13)


def source_integral(half_window):
    """Integral of the source over x in [-W, W]: 2^-1/2 (its integral over the line) minus twice
    the tail integral of K_{1/4}(x) x^{-1/4} beyond W, normalised by 2^{9/4} sqrt(pi) Gamma(5/4)
    (ode_backend.py:782-790)."""
    from scipy.integrate import quad
    from scipy.special import gamma, kv
    if not half_window > 0:
        raise ValueError("positive half_window required")
    tail = quad(lambda x: kv(0.25, x) / x ** 0.25, half_window, np.inf, epsabs=0, epsrel=1e-12, limit=200)[0]
    return 2 ** -0.5 - 2.0 * tail / (2 ** 2.25 * math.sqrt(math.pi) * gamma(1.25))


def phi_expectation(R, rho, half_window):
    """<phi> on the window W: tr F1(a) of the first monomial = source_integral(W) tr(R rho + rho
    R^dag) exactly, since the Lindbladian preserves the trace (ode_backend.py:793-797)."""
    R, rho = np.asarray(R), np.asarray(rho)
    return 2.0 * source_integral(half_window) * float(np.real(np.trace(rho @ R)))


def phi_by_ode(r, k, rho, controls):
    """<phi> as RcmpsCore's phi_monomial(s, 1) computes it, on the GPU: F0 = rho and
    dF1 = 2|t| L(F1) dt + j(t) (R F0 + F0 R^dag) dt with their adjoint channels, by the DOP853
    trajectory kernel; the value is Re tr F1 at the endpoint (validate_sweep.py:23-32).
    controls: window, quadrature, atol, rtol, max_steps. Returns (value, stats)."""
    import torch
    d = objective._check_matrices(r, k, rho)
    ctx = objective.context()
    s = _lib.default_settings(half_window=float(controls.window), n_quad=int(controls.quadrature),
                              atol=float(controls.atol), rtol=float(controls.rtol),
                              max_steps=int(getattr(controls, "max_steps", 1_000_000)))
    dR, dK, dP = objective._device([r]), objective._device([k]), objective._device([rho])
    phi = torch.zeros(1, dtype=torch.float64, device="cuda")
    stats = (_lib.StateStats * 1)()
    t0 = time.perf_counter()
    rc = ctx.lib.rcmps_phi_ode_batch(ctx.handle, 1, (C.c_int * 1)(d), dR.data_ptr(), dK.data_ptr(), dP.data_ptr(),
                                     C.byref(s), phi.data_ptr(), stats, objective._stream())
    objective._raise_for(rc, ctx, stats[0], "phi by ODE")
    value = float(phi.cpu().item())
    st = stats[0].as_dict()
    st.update(accepted_steps=st["accepted"], rejected_steps=st["rejected"], total_seconds=time.perf_counter() - t0)
    return value, st


def _norm(rho, x, reg):
    return float(np.sqrt(max(0.0, objective.metric(rho, x, x, reg))))


def validate_state(r, k, rho, coupling, args, *, cached_energy=None, cached_gradient=None, saved_energy=None,
                   gradient_target=None):
    """The five validation rows and <phi> of one state (validate_sweep.py:84-145). args: the
    run's controls (window, quadrature, atol, rtol, max_steps, nodes, krylov_tolerance, maxdim,
    metric_reg, packed_z2 or reduced). Without a cached energy/gradient the first row stands in
    for them. Returns the report dict; report["passed"] tells whether every row passed."""
    reg = float(getattr(args, "metric_reg", 1e-3))
    target = gradient_target if gradient_target is not None else getattr(args, "gradient_tolerance", None)
    report = dict(gradient_target=target, cached_energy=cached_energy, saved_cpu_energy=saved_energy,
                  evaluations=[], cpu_objective_rerun=False)
    gradients = {}
    standard_energy = standard_gradient = None
    for name, nodes in ROWS:
        controls = SimpleNamespace(**vars(args))
        if nodes is not None:
            controls.nodes = nodes
            for key, value in REFINED.items():
                setattr(controls, key, value)
        begin = time.perf_counter()
        energy, gradient, stats = objective.objective(r, k, rho, coupling, controls)
        seconds = time.perf_counter() - begin
        if standard_gradient is None:
            standard_energy, standard_gradient = energy, gradient
        ref_energy = cached_energy if cached_energy is not None else standard_energy
        ref_gradient = cached_gradient if cached_gradient is not None else standard_gradient
        row = dict(name=name, controls={key: getattr(controls, key) for key in
                                        ("nodes", "window", "quadrature", "atol", "rtol")},
                   seconds=seconds, energy=energy, gradient_norm=_norm(rho, gradient, reg),
                   phi=phi_expectation(r, rho, controls.window),
                   energy_difference_standard=abs(energy - standard_energy),
                   energy_difference_cached=abs(energy - ref_energy),
                   energy_difference_saved_cpu=abs(energy - saved_energy) if saved_energy is not None else None,
                   gradient_metric_difference_standard=_norm(rho, gradient - standard_gradient, reg),
                   gradient_metric_difference_cached=_norm(rho, gradient - ref_gradient, reg),
                   stats=stats)
        row["gradient_target_reached"] = bool(target is not None and row["gradient_norm"] <= target)
        # the reference's pass test; the library has no fallback solves, and every shifted solve
        # meets the Krylov tolerance or the evaluation raises
        row["passed"] = bool(np.isfinite(energy) and np.isfinite(gradient).all() and
                             row["gradient_metric_difference_cached"] <= 3e-7 and
                             row["energy_difference_cached"] <= 1e-8 and
                             stats["krylov_residual"] <= controls.krylov_tolerance)
        gradients[name] = gradient
        report["evaluations"].append(row)
    report["passed"] = all(x["passed"] for x in report["evaluations"])
    report["standard_warm_median_seconds"] = float(np.median(
        [x["seconds"] for x in report["evaluations"] if x["name"].startswith("standard_warm")]))
    final = report["evaluations"][-1]
    controls = SimpleNamespace(**{**vars(args), **final["controls"]})
    phi, phi_stats = phi_by_ode(r, k, rho, controls)
    report.update(symmetry="Z2" if getattr(args, "packed_z2", False) else "none", phi=final["phi"], phi_ode=phi,
                  phi_ode_difference=abs(phi - final["phi"]),
                  phi_ode_stats={key: phi_stats[key] for key in ("accepted_steps", "rejected_steps", "total_seconds")})
    report["gradients"] = gradients
    return report


def main(argv=None):
    """validate_sweep's command line on the library: checkpoint (JSON report + NPZ of a stopped
    run of the reference's optimizer), the run's initial portable state, --output."""
    from .io import Integration, Manifold, StateRecord, read_portable, write_portable
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("checkpoint")
    parser.add_argument("initial_reference")
    parser.add_argument("--comparison-reference")
    parser.add_argument("--output", required=True)
    cli = parser.parse_args(argv)
    checkpoint = Path(cli.checkpoint)
    run = json.loads(checkpoint.read_text())
    if not run.get("stop_reason"):
        raise ValueError("Optimization is still running")
    state = np.load(checkpoint.with_suffix(".npz"))
    if int(state["iteration"]) != len(run["history"]):
        raise ValueError("JSON/NPZ checkpoint generations differ")
    args = objective.default_args(**run["controls"])
    initial = read_portable(cli.initial_reference, arrays=False)
    comparison = read_portable(cli.comparison_reference, arrays=False) if cli.comparison_reference else None
    if comparison and comparison.D != initial.D:
        raise ValueError("Comparison reference dimension differs")
    r, k, rho, cached_gradient = (state[name] for name in ("R", "K", "rho", "gradient"))
    if len(r) != initial.D:
        raise ValueError("Reference dimension differs")
    report = validate_state(r, k, rho, initial.coupling, args, cached_energy=float(state["energy"]),
                            cached_gradient=cached_gradient,
                            saved_energy=comparison.energy if comparison else None,
                            gradient_target=getattr(args, "gradient_tolerance", None))
    gradients = report.pop("gradients")
    report.update(iteration=int(state["iteration"]), optimization_target_reached=bool(run.get("converged")),
                  optimization_stop_reason=run["stop_reason"],
                  checkpoint_sha256={p.name: hashlib.sha256(p.read_bytes()).hexdigest()
                                     for p in (checkpoint, checkpoint.with_suffix(".npz"))},
                  library_sha256=hashlib.sha256(_lib.LIBRARY_PATH.read_bytes()).hexdigest())
    for row in report["evaluations"]:
        row.pop("stats", None)
    output = Path(cli.output)
    output.parent.mkdir(parents=True, exist_ok=True)
    output.write_text(json.dumps(report, indent=2) + "\n")
    np.savez(output.with_suffix(".npz"), R=r, K=k, rho=rho, **gradients)
    if not report["passed"]:
        raise RuntimeError("Final GPU accuracy refinement failed; inspect the saved report")
    final = report["evaluations"][-1]
    refined = final["controls"]
    reached = bool(final["gradient_target_reached"])
    export = output.parent / "optimized_state"
    write_portable(export, StateRecord(
        D=len(r), model="phi4", coupling=initial.coupling, R=r, K=k, rho=rho, gradient=gradients[final["name"]],
        energy=final["energy"], gradient_norm=final["gradient_norm"], phi=final["phi"],
        symmetry=report["symmetry"], validation_passed=True,
        integration=Integration(refined["quadrature"], refined["window"], refined["atol"], refined["rtol"]),
        manifold=Manifold(float(getattr(args, "metric_reg", 1e-3)), float(state["precond_reg"])),
        producer="rcmps_b200 validate", source=f"{checkpoint.name} iteration {report['iteration']}, "
                                               f"evaluation {final['name']}",
        info=f"FP64 B200 validation at D={len(r)}; energy and gradient of the refined evaluation; "
             f"gradient target {report['gradient_target']} reached: {reached}"),
        extra=dict(gradient_target=report["gradient_target"], gradient_target_reached=reached))
    print(f"Validated portable state: {export}", flush=True)
    return report


if __name__ == "__main__":
    main()
