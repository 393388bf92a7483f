"""L-BFGS controller of rcmps_gpu's optimizer around the B200 objective.

Mirrors gpu/src/rcmps_gpu/optimizer/runtime/optimizer.py (the controller that follows
RcmpsCore/OptimKit 0.5): the metric <x, y> = 2 Re tr(x^dag y (rho + reg I)), the canonical
retraction of (R, K), the rho-preconditioner, the first direction of fixed metric norm, the
two-loop L-BFGS direction rescaled to the latest secant pair, cautious history updates and
bounded Armijo backtracking. It yields the same trial / accepted / stopped events with the same
resumable state, so the reference's drivers and checkpoint code consume it unchanged.

The GPU does the evaluation: every trial's stationary density comes from the library
(stationary_state, or with warm_stationary=True the correction started from the last accepted
density, stationary_correction.py:19-96) and objective_callable is normally
rcmps_b200.objective.objective. The L-BFGS algebra is on D x D host matrices.
"""
from __future__ import annotations

from dataclasses import dataclass, fields
from time import perf_counter

import numpy as np

from .objective import SolverFailure, metric, stationary_state, stationary_state_correction

__all__ = ["OptimizationControls", "retract", "precondition", "optimize"]


@dataclass(frozen=True)
class OptimizationControls:
    """The reference's controls (optimizer.py:24-41), same names and defaults."""
    max_iterations: int = 3000
    gradient_tol: float = 3e-5
    max_seconds: float | None = None
    history: int = 100
    metric_reg: float = 1e-3
    stationary_tolerance: float = 1e-13
    initial_precond_reg: float = 1e-4
    precond_prefactor: float = 1e-2
    initial_step: float = 1.0
    initial_direction_norm: float = 0.01
    warm_start_line_search: bool = False
    max_relative_step: float = 0.5
    line_search_trials: int = 30
    armijo_c1: float = 1e-4
    shrink: float = 0.5
    energy_atol: float = 0.0
    refresh_curvatures: bool = False


_ALIASES = {"iterations": "max_iterations", "gradtol": "gradient_tol", "gradient_tolerance": "gradient_tol",
            "lbfgs_history": "history", "max_trials": "line_search_trials", "armijo_energy_atol": "energy_atol"}


def _controls(controls):
    """OptimizationControls from a dataclass, dict or namespace (aliases of optimizer.py:44-70)."""
    if isinstance(controls, OptimizationControls):
        c = controls
    else:
        values = dict(controls) if isinstance(controls, dict) else dict(vars(controls))
        for alias, name in _ALIASES.items():
            if alias in values and name not in values:
                values[name] = values[alias]
        names = {f.name for f in fields(OptimizationControls)}
        c = OptimizationControls(**{key: value for key, value in values.items() if key in names})
    positive = (c.gradient_tol, c.stationary_tolerance, c.initial_precond_reg, c.precond_prefactor, c.initial_step,
                c.initial_direction_norm, c.max_relative_step)
    ok = (c.max_iterations >= 0 and c.history >= 1 and c.line_search_trials >= 1 and
          all(np.isfinite(x) and x > 0 for x in positive) and
          np.isfinite(c.metric_reg) and c.metric_reg >= 0 and 0 < c.armijo_c1 < 1 and 0 < c.shrink < 1 and
          np.isfinite(c.energy_atol) and c.energy_atol >= 0 and
          (c.max_seconds is None or (np.isfinite(c.max_seconds) and c.max_seconds > 0)))
    if not ok:
        raise ValueError("invalid optimization controls")
    return c


def retract(r, k, direction, alpha):
    """The canonical retraction (numerics.py:133-136): R + alpha X, and K moved so that
    Q = -iK - R^dag R / 2 stays left-canonical to first order, then made Hermitian."""
    rr = r + alpha * direction
    kk = k + 0.5j * alpha * (direction.conj().T @ r - r.conj().T @ direction)
    return rr, 0.5 * (kk + kk.conj().T)


def precondition(rho, gradient, metric_reg=1e-3, precond_reg=1e-4):
    """(rho + precond_reg I)^-1 applied from the right to G (rho + metric_reg I)
    (numerics.py:139-142)."""
    eye = np.eye(len(rho))
    lhs = (gradient @ (rho + metric_reg * eye)).conj().T
    return np.linalg.solve(rho + precond_reg * eye, lhs).conj().T


def _norm(rho, x, reg):
    sq = metric(rho, x, x, reg)
    if not np.isfinite(sq) or sq < 0:
        raise SolverFailure(f"invalid tangent metric norm squared: {sq}")
    return float(np.sqrt(sq))


def _first_direction(rho, gradient, reg, preg, length):
    p = precondition(rho, gradient, reg, preg)
    n = _norm(rho, p, reg)
    if n == 0:
        raise SolverFailure("preconditioned direction vanished before convergence")
    return -(length / n) * p


def _two_loop(rho, gradient, pairs, reg, preg):
    """L-BFGS direction from normalized pairs (s, y, 1/<s, y>), the preconditioner rescaled by
    <s, y> / <y, P y> of the newest pair (optimizer.py:88-107). (None, gamma) if that scale is
    not positive."""
    q = gradient.copy()
    alphas = []
    for s, y, rs in reversed(pairs):
        a = rs * metric(rho, s, q, reg)
        alphas.append(a)
        q -= a * y
    s, y, _ = pairs[-1]
    py = precondition(rho, y, reg, preg)
    num, den = metric(rho, s, y, reg), metric(rho, y, py, reg)
    gamma = num / den if den > 0 else np.nan
    if not np.isfinite(gamma) or gamma <= 0:
        return None, gamma
    z = gamma * precondition(rho, q, reg, preg)
    for (s, y, rs), a in zip(pairs, reversed(alphas)):
        z += s * (a - rs * metric(rho, y, z, reg))
    return -z, float(gamma)


def optimize(r, k, rho, energy, gradient, objective_callable, controls, resume_state=None, *,
             warm_stationary=False):
    """Yield trial, accepted and stopped events from an evaluated initial state
    (optimizer.py:110-259). objective_callable(r, k, rho) -> (energy, gradient, stats). Accepted
    and stopped events carry `state` (R, K, rho, gradient, energy, pairs, precond_reg, next_step,
    iteration, evaluations, elapsed_seconds) from which resume_state continues exactly.
    warm_stationary: each trial's density is corrected from the last accepted one instead of
    solved cold (the reference's plain controller solves cold)."""
    p = _controls(controls)
    res = resume_state or {}
    as_c = lambda x: np.array(x, dtype=np.complex128, copy=True)
    r = as_c(res.get("R", res.get("r", r)))
    k = as_c(res.get("K", res.get("k", k)))
    rho = as_c(res.get("rho", rho))
    gradient = as_c(res.get("gradient", res.get("g", gradient)))
    energy = float(res.get("energy", energy))
    if (r.ndim != 2 or r.shape[0] != r.shape[1] or any(x.shape != r.shape for x in (k, rho, gradient)) or
            not np.isfinite(energy) or not all(np.isfinite(x).all() for x in (r, k, rho, gradient))):
        raise ValueError("invalid accepted optimization state")
    pairs = [(as_c(s), as_c(y), float(rs)) for s, y, rs in res.get("pairs", [])][-p.history:]
    if any(s.shape != r.shape or y.shape != r.shape or not np.isfinite(rs) or rs <= 0 or
           not np.isfinite(s).all() or not np.isfinite(y).all() for s, y, rs in pairs):
        raise ValueError("invalid resumed LBFGS history")
    iteration = int(res.get("iteration", 0))
    evaluations = int(res.get("evaluations", 0))
    precond_reg = float(res.get("precond_reg", p.initial_precond_reg))
    next_step = float(res.get("next_step", p.initial_step))
    elapsed_before = float(res.get("elapsed_seconds", 0.0))
    if (iteration < 0 or evaluations < 0 or not np.isfinite(precond_reg) or precond_reg <= 0 or
            not np.isfinite(next_step) or next_step <= 0 or not np.isfinite(elapsed_before) or elapsed_before < 0):
        raise ValueError("invalid resumed optimizer controls or counters")
    last_stats = res.get("stats")
    t0 = perf_counter()
    reg = p.metric_reg

    def snapshot():
        return dict(R=r, K=k, rho=rho, gradient=gradient, g=gradient, energy=energy, pairs=list(pairs),
                    precond_reg=precond_reg, next_step=next_step, iteration=iteration, evaluations=evaluations,
                    elapsed_seconds=elapsed_before + perf_counter() - t0,
                    gradient_norm=_norm(rho, gradient, reg), stats=last_stats)

    def stop(reason, converged=False, **extra):
        return dict(type="stopped", event="stopped", reason=reason, converged=converged, state=snapshot(), **extra)

    def out_of_time():
        return p.max_seconds is not None and perf_counter() - t0 >= p.max_seconds

    while True:
        gn = _norm(rho, gradient, reg)
        if gn <= p.gradient_tol:
            yield stop("gradient tolerance reached", converged=True)
            return
        if iteration >= p.max_iterations:
            yield stop("requested iteration limit reached")
            return
        if out_of_time():
            yield stop("optimization time budget reached")
            return
        it0 = perf_counter()
        if p.refresh_curvatures:
            kept = []
            for s, y, _ in pairs:
                sy, ss = metric(rho, s, y, reg), metric(rho, s, s, reg)
                if ss > 0 and sy / ss > gn / 10000:
                    kept.append((s, y, 1 / sy))
            pairs = kept
        gamma = None
        if pairs:
            direction, gamma = _two_loop(rho, gradient, pairs, reg, precond_reg)
        else:
            direction = _first_direction(rho, gradient, reg, precond_reg, p.initial_direction_norm)
        slope = metric(rho, gradient, direction, reg) if direction is not None else np.nan
        if not np.isfinite(slope) or slope >= 0:   # not a descent direction: restart the history
            pairs = []
            direction = _first_direction(rho, gradient, reg, precond_reg, p.initial_direction_norm)
            slope = metric(rho, gradient, direction, reg)
        if not np.isfinite(slope) or slope >= 0:
            raise SolverFailure("preconditioned direction is not a descent direction")
        alpha = min(next_step, p.max_relative_step * max(1.0, np.linalg.norm(r)) /
                    max(np.linalg.norm(direction), np.finfo(float).eps))
        accepted = False
        failures = []
        for trial in range(1, p.line_search_trials + 1):
            if out_of_time():
                yield stop("optimization time budget reached during line search", numerical_failures=failures)
                return
            rr, kk = retract(r, k, direction, alpha)
            qq = -1j * kk - rr.conj().T @ rr / 2
            try:
                if warm_stationary:
                    rhonew, sstats = stationary_state_correction(qq, rr, rho, tolerance=p.stationary_tolerance)
                else:
                    rhonew, sstats = stationary_state(qq, rr, tolerance=p.stationary_tolerance)
                evaluations += 1
                enew, gnew, newstats = objective_callable(rr, kk, rhonew)
                enew = float(enew)
                gnew = np.asarray(gnew, dtype=np.complex128)
                if not np.isfinite(enew) or not np.isfinite(gnew).all() or gnew.shape != r.shape:
                    raise SolverFailure("trial returned nonfinite or invalid objective/gradient")
                bound = energy + p.armijo_c1 * alpha * slope + p.energy_atol
                accepted = bool(enew <= bound)
                yield dict(type="trial", event="trial", iteration=iteration + 1, trial=trial, alpha=float(alpha),
                           energy=enew, armijo_bound=float(bound), accepted=accepted, stats=newstats,
                           stationary=sstats, evaluations=evaluations)
                if accepted:
                    break
            except (SolverFailure, RuntimeError) as err:
                failures.append(str(err))
                yield dict(type="trial", event="trial", iteration=iteration + 1, trial=trial, alpha=float(alpha),
                           accepted=False, error=str(err), evaluations=evaluations)
            alpha *= p.shrink
        if not accepted:
            yield stop("Armijo line search exhausted; last accepted state retained", numerical_failures=failures)
            return
        step, change = alpha * direction, gnew - gradient
        new_gn = _norm(rhonew, gnew, reg)
        sy, ss = metric(rhonew, step, change, reg), metric(rhonew, step, step, reg)
        cautious = bool(np.isfinite(sy) and np.isfinite(ss) and ss > 0 and sy / ss > new_gn / 10000)
        if cautious:
            length = np.sqrt(ss)
            pairs = (pairs + [(step / length, change / length, ss / sy)])[-p.history:]
        r, k, rho, energy, gradient = rr, kk, rhonew, enew, gnew
        last_stats = newstats
        iteration += 1
        next_step = min(1.0, 2 * alpha) if p.warm_start_line_search else p.initial_step
        precond_reg = max(10 * np.finfo(float).eps, p.precond_prefactor * min(new_gn * new_gn, 1.0))
        yield dict(type="accepted", event="accepted", state=snapshot(), iteration=iteration, energy=energy,
                   gradient_norm=new_gn, alpha=float(alpha), trials=trial, seconds=perf_counter() - it0,
                   stats=newstats, stationary=sstats, gamma=gamma, cautious_update=cautious,
                   history_size=len(pairs), evaluations=evaluations)
