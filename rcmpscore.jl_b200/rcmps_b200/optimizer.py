"""L-BFGS optimizer of an RCMPS around the B200 objective.

The interface is that of rcmps_gpu's controller (gpu/src/rcmps_gpu/optimizer/runtime/
optimizer.py:24-259, which follows RcmpsCore/OptimKit 0.5): the same controls and aliases, the
same "trial", "accepted" and "stopped" events, and a resumable state with the same fields, so
the reference's sweep drivers and checkpoint code consume this module unchanged. The algorithm
it implements, stated here in full:

  * tangent vectors are D x D matrices X (the variation of R; K follows from the retraction),
    with the metric <X, Y> = 2 Re tr(X^dag Y M), M = rho + metric_reg I;
  * the preconditioner is P(X) = (N^-1 (X M)^dag)^dag, N = rho + precond_reg I; precond_reg
    starts at initial_precond_reg and becomes max(10 eps, precond_prefactor min(|g|^2, 1)) after
    every accepted step;
  * with no curvature pairs the direction is -P(g) scaled to metric norm initial_direction_norm;
    otherwise the two-loop recursion over the pairs (s_j, y_j, 1/<s_j, y_j>), with the middle
    preconditioner scaled by gamma = <s, y> / <y, P(y)> of the newest pair (no direction when
    gamma is not positive); a direction that is not a descent direction clears the history and
    falls back to the first kind;
  * bounded Armijo backtracking along the canonical retraction R + a X,
    K + i a/2 (X^dag R - R^dag X) (Hermitized), from a = min(next step, max_relative_step
    max(1, |R|) / |X|), shrinking by `shrink`, at most line_search_trials trials; every trial
    solves its stationary density first (on the GPU) and then calls the objective;
  * after an accepted step the pair (s, y) = (a X, g_new - g) is kept only when the cautious
    test <s, y> / <s, s> > |g_new| / 10^4 holds (norms in the new state's metric), normalized by
    |s|, in a history of at most `history` pairs.

Every trial's stationary density comes from the library: rcmps_stationary_state_batch, or with
warm_stationary=True the correction started from the last accepted density
(rcmps_stationary_correction_batch). objective_callable is normally
rcmps_b200.objective.objective. With device_algebra=True the directions and retractions are
formed on the GPU too (rcmps_lbfgs_direction, rcmps_retract).
"""
from __future__ import annotations

from collections import deque
from dataclasses import dataclass, fields
from time import perf_counter

import numpy as np

from .objective import SolverFailure, stationary_state, stationary_state_correction

__all__ = ["OptimizationControls", "retract", "precondition", "optimize"]

_EPS = np.finfo(float).eps


@dataclass(frozen=True)
class OptimizationControls:
    """Controls of the optimizer; names and defaults are the reference's (optimizer.py:24-41)."""
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

    def validated(self):
        """Self, or ValueError naming the first control outside its domain."""
        finite = lambda v: v is not None and np.isfinite(v)
        rules = (("max_iterations", self.max_iterations >= 0), ("history", self.history >= 1),
                 ("line_search_trials", self.line_search_trials >= 1),
                 ("gradient_tol", finite(self.gradient_tol) and self.gradient_tol > 0),
                 ("metric_reg", finite(self.metric_reg) and self.metric_reg >= 0),
                 ("stationary_tolerance", finite(self.stationary_tolerance) and self.stationary_tolerance > 0),
                 ("initial_precond_reg", finite(self.initial_precond_reg) and self.initial_precond_reg > 0),
                 ("precond_prefactor", finite(self.precond_prefactor) and self.precond_prefactor > 0),
                 ("initial_step", finite(self.initial_step) and self.initial_step > 0),
                 ("initial_direction_norm", finite(self.initial_direction_norm) and self.initial_direction_norm > 0),
                 ("max_relative_step", finite(self.max_relative_step) and self.max_relative_step > 0),
                 ("armijo_c1", 0 < self.armijo_c1 < 1), ("shrink", 0 < self.shrink < 1),
                 ("energy_atol", finite(self.energy_atol) and self.energy_atol >= 0),
                 ("max_seconds", self.max_seconds is None or (finite(self.max_seconds) and self.max_seconds > 0)))
        bad = [name for name, ok in rules if not ok]
        if bad:
            raise ValueError(f"invalid optimization controls: {', '.join(bad)}")
        return self


# Alternative spellings that drivers pass (the reference's aliases, optimizer.py:48-53).
CONTROL_ALIASES = {"iterations": "max_iterations", "gradtol": "gradient_tol", "gradient_tolerance": "gradient_tol",
                   "lbfgs_history": "history", "max_trials": "line_search_trials",
                   "armijo_energy_atol": "energy_atol"}


def _controls(controls):
    """OptimizationControls from a dataclass, a dict or a namespace; unknown names are ignored."""
    if isinstance(controls, OptimizationControls):
        return controls.validated()
    given = dict(controls) if isinstance(controls, dict) else dict(vars(controls))
    names = {f.name for f in fields(OptimizationControls)}
    chosen = {}
    for key, value in given.items():
        target = key if key in names else CONTROL_ALIASES.get(key)
        if target is not None and (target == key or target not in given):
            chosen[target] = value
    return OptimizationControls(**chosen).validated()


def retract(r, k, direction, alpha):
    """The canonical retraction of (R, K) along the tangent `direction` by `alpha`
    (numerics.py:133-136): R' = R + a X, K' = Herm(K + i a/2 (X^dag R - R^dag X))."""
    x = np.asarray(direction)
    r_new = r + alpha * x
    k_new = k + 0.5j * alpha * (x.conj().T @ r - r.conj().T @ x)
    return r_new, 0.5 * (k_new + k_new.conj().T)


def precondition(rho, gradient, metric_reg=1e-3, precond_reg=1e-4):
    """P(X) = (N^-1 (X M)^dag)^dag with M = rho + metric_reg I and N = rho + precond_reg I
    (numerics.py:139-142)."""
    eye = np.eye(len(rho))
    rhs = (gradient @ (rho + metric_reg * eye)).conj().T
    return np.linalg.solve(rho + precond_reg * eye, rhs).conj().T


class _Tangent:
    """The metric of the tangent space at one state (its density rho)."""

    def __init__(self, rho, metric_reg):
        self.rho, self.reg = rho, metric_reg
        self.m = rho + metric_reg * np.eye(len(rho))

    def inner(self, x, y):
        return float(2.0 * np.real(np.vdot(x, y @ self.m)))

    def norm(self, x):
        sq = self.inner(x, x)
        if not (np.isfinite(sq) and sq >= 0):
            raise SolverFailure(f"the metric norm of a tangent vector is invalid (squared {sq})")
        return float(np.sqrt(sq))

    def precondition(self, x, precond_reg):
        return precondition(self.rho, x, self.reg, precond_reg)


class _History:
    """Curvature pairs (s, y, 1/<s, y>) with |s| = 1, at most `size` of them (oldest dropped)."""

    def __init__(self, size, pairs=()):
        self.pairs = deque(pairs, maxlen=size)

    def __len__(self):
        return len(self.pairs)

    def clear(self):
        self.pairs.clear()

    def push(self, s, y, inv_sy):
        self.pairs.append((s, y, inv_sy))

    def refresh(self, tangent, gnorm):
        """Recompute every pair's curvature in the current metric and drop those that fail the
        cautious test."""
        kept = []
        for s, y, _ in self.pairs:
            sy, ss = tangent.inner(s, y), tangent.inner(s, s)
            if ss > 0 and sy / ss > gnorm / 1e4:
                kept.append((s, y, 1.0 / sy))
        self.pairs = deque(kept, maxlen=self.pairs.maxlen)

    def direction(self, tangent, gradient, precond_reg):
        """(-H g, gamma) by the two-loop recursion; (None, gamma) when the scaling of the
        newest pair is not positive."""
        q = gradient.copy()
        alphas = []
        for s, y, inv in reversed(self.pairs):
            a = inv * tangent.inner(s, q)
            alphas.append(a)
            q = q - a * y
        s_new, y_new, _ = self.pairs[-1]
        denom = tangent.inner(y_new, tangent.precondition(y_new, precond_reg))
        gamma = tangent.inner(s_new, y_new) / denom if denom > 0 else np.nan
        if not (np.isfinite(gamma) and gamma > 0):
            return None, gamma
        z = gamma * tangent.precondition(q, precond_reg)
        for (s, y, inv), a in zip(self.pairs, reversed(alphas)):
            z = z + (a - inv * tangent.inner(y, z)) * s
        return -z, float(gamma)


class _DeviceAlgebra:
    """The L-BFGS algebra of one state on the GPU (rcmps_lbfgs_direction, rcmps_retract). The
    matrices and history pairs go up per call (a few D x D matrices, small next to one objective
    evaluation); only the direction and its scalars come back."""

    def __init__(self, d):
        from .objective import context
        self.ctx = context()
        self.d = d

    @staticmethod
    def _dev(arrays):
        import torch
        if not arrays:
            return torch.zeros(1, dtype=torch.complex128, device="cuda")
        flat = np.concatenate([np.ascontiguousarray(a, dtype=np.complex128).ravel() for a in arrays])
        return torch.from_numpy(flat).cuda()

    def direction(self, rho, gradient, pairs, metric_reg, precond_reg, first_norm):
        """(direction, gamma, slope): with pairs, the two-loop direction and its gamma (direction
        None when gamma is not positive); without, the first direction and gamma None."""
        import torch
        from .objective import _stream
        d, m = self.d, len(pairs)
        drho, dg = self._dev([rho]), self._dev([gradient])
        dS, dY = self._dev([p[0] for p in pairs]), self._dev([p[1] for p in pairs])
        dinv = torch.tensor([float(p[2]) for p in pairs] or [0.0], dtype=torch.float64, device="cuda")
        out = torch.zeros(d * d, dtype=torch.complex128, device="cuda")
        work = torch.zeros(8 * d * d + max(m, 1), dtype=torch.float64, device="cuda")
        scal = torch.zeros(3, dtype=torch.float64, device="cuda")
        ctx = self.ctx
        rc = ctx.lib.rcmps_lbfgs_direction(ctx.handle, d, m, drho.data_ptr(), dg.data_ptr(), dS.data_ptr(),
                                           dY.data_ptr(), dinv.data_ptr(), float(metric_reg), float(precond_reg),
                                           float(first_norm), out.data_ptr(), work.data_ptr(), scal.data_ptr(),
                                           _stream())
        if rc:
            raise SolverFailure(f"L-BFGS direction on the device: {ctx.error()}")
        gamma, slope, status = scal.cpu().numpy()
        if status:
            raise SolverFailure("rho + precond_reg I is not positive definite")
        if m == 0:
            return out.cpu().numpy().reshape(d, d), None, float(slope)
        if not (np.isfinite(gamma) and gamma > 0):
            return None, float(gamma), float("nan")
        return out.cpu().numpy().reshape(d, d), float(gamma), float(slope)

    def retract(self, r, k, x, alpha):
        import torch
        from .objective import _stream
        d, ctx = self.d, self.ctx
        dR, dK, dX = self._dev([r]), self._dev([k]), self._dev([x])
        Rn, Kn = torch.empty_like(dR), torch.empty_like(dK)
        rc = ctx.lib.rcmps_retract(ctx.handle, d, dR.data_ptr(), dK.data_ptr(), dX.data_ptr(), float(alpha),
                                   Rn.data_ptr(), Kn.data_ptr(), _stream())
        if rc:
            raise SolverFailure(f"retraction on the device: {ctx.error()}")
        return Rn.cpu().numpy().reshape(d, d), Kn.cpu().numpy().reshape(d, d)


def _first_direction(tangent, gradient, precond_reg, length):
    pg = tangent.precondition(gradient, precond_reg)
    n = tangent.norm(pg)
    if n == 0.0:
        raise SolverFailure("the preconditioned gradient vanished before convergence")
    return -(length / n) * pg


class _Run:
    """One invocation of the optimizer: the accepted state, its history and counters."""

    def __init__(self, r, k, rho, energy, gradient, objective_callable, controls, resume_state, warm,
                 device_algebra=False):
        self.c = _controls(controls)
        self.objective = objective_callable
        self.warm = bool(warm)
        res = resume_state or {}
        pick = lambda *names_and_default: next((res[n] for n in names_and_default[:-1] if n in res),
                                               names_and_default[-1])
        as_c = lambda a: np.array(a, dtype=np.complex128, copy=True)
        self.r, self.k = as_c(pick("R", "r", r)), as_c(pick("K", "k", k))
        self.rho, self.g = as_c(pick("rho", rho)), as_c(pick("gradient", "g", gradient))
        self.energy = float(pick("energy", energy))
        shape = self.r.shape
        if (self.r.ndim != 2 or shape[0] != shape[1] or any(a.shape != shape for a in (self.k, self.rho, self.g))
                or not np.isfinite(self.energy) or not all(np.isfinite(a).all() for a in (self.r, self.k, self.rho, self.g))):
            raise ValueError("the accepted state to optimize from is invalid (shapes or nonfinite values)")
        pairs = [(as_c(s), as_c(y), float(inv)) for s, y, inv in res.get("pairs", [])][-self.c.history:]
        for s, y, inv in pairs:
            if s.shape != shape or y.shape != shape or not (np.isfinite(inv) and inv > 0) \
                    or not (np.isfinite(s).all() and np.isfinite(y).all()):
                raise ValueError("the resumed L-BFGS history is invalid")
        self.history = _History(self.c.history, pairs)
        self.iteration = int(res.get("iteration", 0))
        self.evaluations = int(res.get("evaluations", 0))
        self.precond_reg = float(res.get("precond_reg", self.c.initial_precond_reg))
        self.next_step = float(res.get("next_step", self.c.initial_step))
        self.elapsed_before = float(res.get("elapsed_seconds", 0.0))
        if (min(self.iteration, self.evaluations) < 0 or not (np.isfinite(self.precond_reg) and self.precond_reg > 0)
                or not (np.isfinite(self.next_step) and self.next_step > 0)
                or not (np.isfinite(self.elapsed_before) and self.elapsed_before >= 0)):
            raise ValueError("the resumed optimizer counters or controls are invalid")
        self.last_stats = res.get("stats")
        self.device = _DeviceAlgebra(shape[0]) if device_algebra else None
        self.start = perf_counter()

    # ---------------------------------------------------------------- state and events
    def tangent(self):
        return _Tangent(self.rho, self.c.metric_reg)

    def state(self):
        return dict(R=self.r, K=self.k, rho=self.rho, gradient=self.g, g=self.g, energy=self.energy,
                    pairs=list(self.history.pairs), precond_reg=self.precond_reg, next_step=self.next_step,
                    iteration=self.iteration, evaluations=self.evaluations,
                    elapsed_seconds=self.elapsed_before + perf_counter() - self.start,
                    gradient_norm=self.tangent().norm(self.g), stats=self.last_stats)

    def stopped(self, reason, converged=False, **extra):
        return dict(type="stopped", event="stopped", reason=reason, converged=converged, state=self.state(), **extra)

    def out_of_time(self):
        return self.c.max_seconds is not None and perf_counter() - self.start >= self.c.max_seconds

    # ---------------------------------------------------------------- one iteration
    def search_direction(self, tangent, gnorm):
        if self.c.refresh_curvatures:
            self.history.refresh(tangent, gnorm)
        if self.device is not None:
            return self.device_direction()
        gamma = None
        direction = None
        if len(self.history):
            direction, gamma = self.history.direction(tangent, self.g, self.precond_reg)
        else:
            direction = _first_direction(tangent, self.g, self.precond_reg, self.c.initial_direction_norm)
        slope = tangent.inner(self.g, direction) if direction is not None else np.nan
        if not (np.isfinite(slope) and slope < 0):
            self.history.clear()
            direction = _first_direction(tangent, self.g, self.precond_reg, self.c.initial_direction_norm)
            slope = tangent.inner(self.g, direction)
            if not (np.isfinite(slope) and slope < 0):
                raise SolverFailure("the preconditioned direction does not descend")
        return direction, slope, gamma

    def device_direction(self):
        """search_direction's decisions with the algebra on the GPU."""
        c, dev = self.c, self.device
        direction, gamma, slope = dev.direction(self.rho, self.g, list(self.history.pairs), c.metric_reg,
                                                self.precond_reg, c.initial_direction_norm)
        if direction is None or not (np.isfinite(slope) and slope < 0):
            self.history.clear()
            direction, _, slope = dev.direction(self.rho, self.g, [], c.metric_reg, self.precond_reg,
                                                c.initial_direction_norm)
            if not (np.isfinite(slope) and slope < 0):
                raise SolverFailure("the preconditioned direction does not descend")
        return direction, slope, gamma

    def trial_density(self, r, q):
        if self.warm:
            return stationary_state_correction(q, r, self.rho, tolerance=self.c.stationary_tolerance)
        return stationary_state(q, r, tolerance=self.c.stationary_tolerance)

    def evaluate(self, r, k):
        q = -1j * k - r.conj().T @ r / 2
        rho, stationary = self.trial_density(r, q)
        self.evaluations += 1
        e, g, stats = self.objective(r, k, rho)
        e, g = float(e), np.asarray(g, dtype=np.complex128)
        if not np.isfinite(e) or g.shape != self.r.shape or not np.isfinite(g).all():
            raise SolverFailure("the objective returned a nonfinite or misshapen energy or gradient")
        return rho, e, g, stats, stationary

    def accept(self, alpha, direction, r, k, rho, e, g, stats):
        step, change = alpha * direction, g - self.g
        new = _Tangent(rho, self.c.metric_reg)
        gnorm = new.norm(g)
        sy, ss = new.inner(step, change), new.inner(step, step)
        cautious = bool(np.isfinite(sy) and np.isfinite(ss) and ss > 0 and sy / ss > gnorm / 1e4)
        if cautious:
            length = np.sqrt(ss)
            self.history.push(step / length, change / length, ss / sy)
        self.r, self.k, self.rho, self.energy, self.g = r, k, rho, e, g
        self.last_stats = stats
        self.iteration += 1
        self.next_step = min(1.0, 2.0 * alpha) if self.c.warm_start_line_search else self.c.initial_step
        self.precond_reg = max(10 * _EPS, self.c.precond_prefactor * min(gnorm * gnorm, 1.0))
        return gnorm, cautious

    def events(self):
        c = self.c
        while True:
            tangent = self.tangent()
            gnorm = tangent.norm(self.g)
            if gnorm <= c.gradient_tol:
                yield self.stopped("gradient tolerance reached", converged=True)
                return
            if self.iteration >= c.max_iterations:
                yield self.stopped("requested iteration limit reached")
                return
            if self.out_of_time():
                yield self.stopped("optimization time budget reached")
                return
            began = perf_counter()
            direction, slope, gamma = self.search_direction(tangent, gnorm)
            alpha = min(self.next_step,
                        c.max_relative_step * max(1.0, np.linalg.norm(self.r)) / max(np.linalg.norm(direction), _EPS))
            failures, found = [], None
            for trial in range(1, c.line_search_trials + 1):
                if self.out_of_time():
                    yield self.stopped("optimization time budget reached during line search",
                                       numerical_failures=failures)
                    return
                r_t, k_t = (self.device.retract(self.r, self.k, direction, alpha) if self.device is not None
                            else retract(self.r, self.k, direction, alpha))
                try:
                    rho_t, e_t, g_t, stats_t, stationary_t = self.evaluate(r_t, k_t)
                except (SolverFailure, RuntimeError) as err:
                    failures.append(str(err))
                    yield dict(type="trial", event="trial", iteration=self.iteration + 1, trial=trial,
                               alpha=float(alpha), accepted=False, error=str(err), evaluations=self.evaluations)
                else:
                    bound = self.energy + c.armijo_c1 * alpha * slope + c.energy_atol
                    ok = bool(e_t <= bound)
                    yield dict(type="trial", event="trial", iteration=self.iteration + 1, trial=trial,
                               alpha=float(alpha), energy=e_t, armijo_bound=float(bound), accepted=ok,
                               stats=stats_t, stationary=stationary_t, evaluations=self.evaluations)
                    if ok:
                        found = (trial, r_t, k_t, rho_t, e_t, g_t, stats_t, stationary_t)
                        break
                alpha *= c.shrink
            if found is None:
                yield self.stopped("Armijo line search exhausted; last accepted state retained",
                                   numerical_failures=failures)
                return
            trial, r_t, k_t, rho_t, e_t, g_t, stats_t, stationary_t = found
            gnorm_new, cautious = self.accept(alpha, direction, r_t, k_t, rho_t, e_t, g_t, stats_t)
            yield dict(type="accepted", event="accepted", state=self.state(), iteration=self.iteration,
                       energy=self.energy, gradient_norm=gnorm_new, alpha=float(alpha), trials=trial,
                       seconds=perf_counter() - began, stats=stats_t, stationary=stationary_t, gamma=gamma,
                       cautious_update=cautious, history_size=len(self.history), evaluations=self.evaluations)


def optimize(r, k, rho, energy, gradient, objective_callable, controls, resume_state=None, *, warm_stationary=False,
             device_algebra=False):
    """Yield the optimizer's events from an accepted, already evaluated state (r, k, rho,
    energy, gradient). objective_callable(r, k, rho) -> (energy, gradient, stats).

    "trial" events report each line-search evaluation; "accepted" events carry the complete
    resumable `state` (R, K, rho, gradient, energy, the normalized pairs, precond_reg,
    next_step, iteration, evaluations, elapsed_seconds); the single "stopped" event ends the
    stream with its reason. resume_state continues a run from such a state without a new
    initial evaluation; max_iterations counts accepted iterations across resumes, max_seconds
    this invocation only. warm_stationary=True starts each trial's stationary solve from the
    last accepted density. device_algebra=True forms every search direction (two-loop recursion,
    preconditioner, scaling) and every retraction on the GPU (rcmps_lbfgs_direction,
    rcmps_retract); the host keeps the line-search decisions."""
    return _Run(r, k, rho, energy, gradient, objective_callable, controls, resume_state, warm_stationary,
                device_algebra).events()
