"""Drop-in objective of rcmps_gpu's optimizer and its components, on the B200 library.

Mirrors (same names, argument meaning, return values and exceptions):
  * objective(r, k, rho, coupling, args, xp) -> (energy, gradient, stats)
      gpu/src/rcmps_gpu/optimizer/runtime/sweep_driver.py:78-119 and the GPU coordinator
      OverlapObjective.__call__ (runtime/overlap_sweep_driver.py:132-212);
  * evaluate_quartic_persistent_trajectory(R, Q, rho, g, ...) -> dict
      (runtime/persistent_trajectory_backend.py:439-461);
  * evaluate_phi4(R, Q, rho, g, ...) -> dict, every term by ODEs (runtime/ode_backend.py:851-858);
  * kinetic_raw(q, r, rho, nodes, ...) -> dict (runtime/kinetic_backend.py:499-592);
  * finish_gradient(q, r, rho, covector, environment, ...) -> (gradient, stats)
      (runtime/numerics.py:120-126);
  * stationary_state(q, r, tolerance) -> (rho, stats) (runtime/numerics.py:74-100);
  * SolverFailure, KineticFailure, DeviceControlFailure, OverlapFailure.
plus fg_phi4_batch for many states of uneven D in one call.

Every number of the evaluation is computed by librcmps_b200.so on the GPU; this module only
moves arrays and turns status codes into exceptions. Components that take Q (as the reference
does) pass the library K = i (Q + R^dag R / 2), from which it rebuilds Q = -i K - R^dag R / 2.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
from types import SimpleNamespace

import numpy as np

from . import _lib

__all__ = ["SolverFailure", "KineticFailure", "DeviceControlFailure", "OverlapFailure", "Settings",
           "settings_from_args", "fg_phi4_batch", "objective", "OverlapObjective",
           "evaluate_quartic_persistent_trajectory", "evaluate_phi4", "evaluate_phi4_batch", "kinetic_raw",
           "finish_gradient",
           "stationary_state", "stationary_state_correction",
           "metric", "context"]


class SolverFailure(RuntimeError):
    """A numerical requirement of a solve was not met (numerics.py:13)."""


class KineticFailure(RuntimeError):
    """A kinetic Krylov requirement was not met (kinetic_backend.py:28)."""


class DeviceControlFailure(RuntimeError):
    """The device DOP853 controller stopped with a nonzero status (device_control_backend.py:410)."""

    def __init__(self, diagnostics):
        self.diagnostics = diagnostics
        super().__init__(f"device DOP853 failed: {diagnostics}")


class OverlapFailure(RuntimeError):
    """A coordinator requirement failed (overlap_benchmark.py:31)."""


Settings = _lib.Settings
_contexts = {}
_ctx_lock = threading.Lock()


def context(device=None):
    """The library context of a CUDA device (created once per process)."""
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("rcmps_b200 needs a CUDA device; there is no host fallback")
    device = torch.cuda.current_device() if device is None else int(device)
    with _ctx_lock:
        if device not in _contexts:
            _contexts[device] = _lib.Context(device)
        return _contexts[device]


def settings_from_args(args=None, **overrides):
    """Settings from an argparse namespace of the reference's optimizer (window, quadrature,
    atol, rtol, max_steps, nodes, krylov_tolerance, maxdim, metric_reg; packed_z2 or reduced
    selects the quartic route, sweep_driver.py:48-50, 100-101)."""
    s = _lib.default_settings()
    if args is not None:
        mapping = dict(window="half_window", quadrature="n_quad", atol="atol", rtol="rtol",
                       max_steps="max_steps", nodes="kinetic_nodes", krylov_tolerance="krylov_tolerance",
                       maxdim="krylov_maxdim", metric_reg="metric_reg")
        for src, dst in mapping.items():
            if getattr(args, src, None) is not None:
                setattr(s, dst, type(getattr(s, dst))(getattr(args, src)))
        packed, reduced = bool(getattr(args, "packed_z2", False)), bool(getattr(args, "reduced", False))
        if packed and reduced:
            raise ValueError("the quartic route takes one of --packed-z2, --reduced")
        s.symmetry = SYMMETRY_Z2 if packed else SYMMETRY_NONE
    for key, value in overrides.items():
        if not hasattr(s, key):
            raise KeyError(f"unknown setting {key}")
        setattr(s, key, value)
    return s


# Quartic routes of the library (rcmps_settings.symmetry): the unpacked channels, the packed Z2
# route (states without the exact Z2 block structure raise ValueError), or packed where possible.
SYMMETRY_NONE, SYMMETRY_Z2, SYMMETRY_AUTO = 0, 1, 2


def _check_matrices(*mats):
    d = None
    for m in mats:
        m = np.asarray(m)
        if m.ndim != 2 or m.shape[0] != m.shape[1] or m.shape[0] == 0:
            raise ValueError("matrices must be nonempty and square")
        if d is None:
            d = m.shape[0]
        if m.shape != (d, d):
            raise ValueError("matrices must be equally shaped")
        if not np.isfinite(m).all():
            raise ValueError("matrices must be finite")
    return d


def _device(arrays):
    """Pack host complex128 matrices into one device tensor (row-major, one after another)."""
    import torch
    flat = np.concatenate([np.ascontiguousarray(a, dtype=np.complex128).ravel() for a in arrays])
    return torch.from_numpy(flat).to("cuda", non_blocking=False)


def _unpack(t, dims):
    host = t.cpu().numpy()
    out, o = [], 0
    for d in dims:
        out.append(host[o:o + d * d].reshape(d, d).copy())
        o += d * d
    return out


# CUDA's handle of the legacy default stream (cudaStreamLegacy). torch reports its default stream
# as handle 0, which the library reads as "the context's own stream"; the explicit handle keeps the
# library's kernels ordered with torch's work on that stream (an entry that returns before its
# kernels finish would otherwise race with torch freeing and reusing its tensors).
_LEGACY_STREAM = 0x1


def _stream():
    import torch
    handle = torch.cuda.current_stream().cuda_stream
    return C.c_void_p(handle if handle else _LEGACY_STREAM)


def _raise_for(status, ctx, stats, what):
    if status == 0:
        return
    name = _lib.STATUS_NAMES.get(status, "unknown")
    detail = ctx.error()
    comp = stats.as_dict()["failed_component"] if stats is not None else None
    msg = f"{what}: {name} ({detail})" if detail else f"{what}: {name}"
    if status == 20:
        raise ValueError(msg)
    if comp == "trajectory" or (comp is None and status in range(1, 8)):
        raise DeviceControlFailure(dict(stats.as_dict() if stats is not None else {}, status_name=name,
                                        message=msg))
    if comp == "kinetic" or status == 8:
        raise KineticFailure(msg)
    raise SolverFailure(msg)


def fg_phi4_batch(R, K, rho, couplings, settings=None, *, device=None, return_parts=False, tolerances=None):
    """phi^4 energies and finished gradients of a batch of states (lists of D_i x D_i matrices,
    uneven D allowed). Returns (energies [n], gradients [n matrices], stats [n dicts]); with
    return_parts also the raw covectors and environments. `tolerances`: optional per-state
    (atol, rtol) pairs of the quartic trajectories (rcmps_fg_phi4_batch_controls), so that states
    with mixed tolerance pairs share one launch."""
    import torch
    n = len(R)
    if not (len(K) == len(rho) == len(couplings) == n):
        raise ValueError("R, K, rho and couplings must have the same length")
    if tolerances is not None and len(tolerances) != n:
        raise ValueError("tolerances must hold one (atol, rtol) pair per state")
    dims = [_check_matrices(R[i], K[i], rho[i]) for i in range(n)]
    ctx = context(device)
    s = settings if settings is not None else _lib.default_settings()
    dR, dK, dP = _device(R), _device(K), _device(rho)
    total = sum(d * d for d in dims)
    energy = torch.zeros(n, dtype=torch.float64, device="cuda")
    grad = torch.zeros(total, dtype=torch.complex128, device="cuda")
    cov = torch.zeros(total, dtype=torch.complex128, device="cuda") if return_parts else None
    env = torch.zeros(total, dtype=torch.complex128, device="cuda") if return_parts else None
    stats = (_lib.StateStats * n)()
    controls = None
    if tolerances is not None:
        controls = (_lib.StateControls * n)(*(_lib.StateControls(float(a), float(r)) for a, r in tolerances))
    rc = ctx.lib.rcmps_fg_phi4_batch_controls(ctx.handle, n, (C.c_int * n)(*dims),
                                              (C.c_double * n)(*map(float, couplings)), dR.data_ptr(), dK.data_ptr(),
                                              dP.data_ptr(), C.byref(s), controls, energy.data_ptr(),
                                              grad.data_ptr(), cov.data_ptr() if cov is not None else None,
                                              env.data_ptr() if env is not None else None, stats, _stream())
    if rc:
        bad = next((i for i in range(n) if stats[i].status), 0)
        _raise_for(rc, ctx, stats[bad], "fg_phi4")
    out = (energy.cpu().numpy(), _unpack(grad, dims), [stats[i].as_dict() for i in range(n)])
    if return_parts:
        out = out + (_unpack(cov, dims), _unpack(env, dims))
    return out


def objective(r, k, rho, coupling, args=None, xp=None):
    """(energy, gradient, stats) of one state, the callable the reference's L-BFGS controllers
    evaluate once per trial. r, k, rho: finite complex128 D x D; args: the optimizer's namespace.
    args.mode == "ode" evaluates every term by ODEs (sweep_driver.py:90-92), otherwise the
    kinetic resolvents plus the quartic trajectory."""
    mats = (r, k, rho)
    if any(np.asarray(x).dtype != np.complex128 for x in mats):
        raise SolverFailure("objective requires equally shaped finite complex128 matrices")
    try:
        _check_matrices(*mats)
    except ValueError as err:
        raise SolverFailure(f"objective requires equally shaped finite complex128 matrices: {err}") from None
    original = tuple(np.array(x, copy=True) for x in mats)
    if getattr(args, "mode", None) == "ode":
        s = settings_from_args(args)
        q = -1j * np.asarray(k) - np.asarray(r).conj().T @ np.asarray(r) / 2
        raw = evaluate_phi4(r, q, rho, coupling, half_window=s.half_window, n_quad=s.n_quad, atol=s.atol,
                            rtol=s.rtol, max_steps=s.max_steps)
        gradient, boundary = finish_gradient(q, r, rho, raw["covector"], raw["environment"], metric_reg=s.metric_reg)
        if any(not np.array_equal(a, b) for a, b in zip(original, mats)):
            raise OverlapFailure("a component mutated immutable R/K/rho inputs")
        return float(raw["value"]), gradient, dict(ode=raw["stats"], boundary=boundary)
    energies, grads, stats = fg_phi4_batch([r], [k], [rho], [coupling], settings_from_args(args))
    if any(not np.array_equal(a, b) for a, b in zip(original, mats)):
        raise OverlapFailure("a component mutated immutable R/K/rho inputs")
    gradient = grads[0]
    if not np.isfinite(gradient).all() or not math.isfinite(float(energies[0])):
        raise SolverFailure("finished metric gradient requires finite complex128")
    return float(energies[0]), gradient, stats[0]


class OverlapObjective:
    """Run-owned coordinator with the reference's call signature: one state per call, guarded
    against concurrent calls (overlap_sweep_driver.py:108-231). The library overlaps the kinetic
    and quartic terms on two streams of its own."""

    def __init__(self, device=None):
        self.device = device
        self.closed = False
        self._lock = threading.Lock()

    def __call__(self, r, k, rho, coupling, args=None, xp=None):
        if not self._lock.acquire(blocking=False):
            raise OverlapFailure("one objective coordinator cannot evaluate concurrent states")
        try:
            if self.closed:
                raise OverlapFailure("objective coordinator is closed")
            return objective(r, k, rho, coupling, args, xp)
        finally:
            self._lock.release()

    def close(self):
        with self._lock:
            self.closed = True

    def __enter__(self):
        return self

    def __exit__(self, *errors):
        self.close()


def _k_from_q(q, r):
    q, r = np.asarray(q, dtype=np.complex128), np.asarray(r, dtype=np.complex128)
    return 1j * (q + r.conj().T @ r / 2)


def evaluate_quartic_persistent_trajectory(R, Q, rho, g=1.0, *, xp=None, half_window=30.0, n_quad=512,
                                           atol=1e-13, rtol=1e-12, initial_step=None, max_steps=1_000_000,
                                           max_device_seconds=30.0, return_samples=False, unpacked=False,
                                           precision=0, **ignored):
    """g times the quartic value, raw covector and environment:
    dict(value, energy, covector, environment, stats[, samples]). As the reference
    (persistent_trajectory_backend.py:439-461), the packed Z2 route is the default and a state
    without the exact Z2 block structure raises ValueError; unpacked=True takes the seven
    unpacked channels (any state). Packed samples have 10 (D/2)^2 + 1 entries per point.
    precision=1 runs the trajectory products of a padded-64 state on the split-precision
    tensor-core engine (rcmps_settings.precision)."""
    import torch
    d = _check_matrices(R, Q, rho)
    ctx = context()
    s = _lib.default_settings(half_window=float(half_window), n_quad=int(n_quad), atol=float(atol), rtol=float(rtol),
                              max_steps=int(max_steps), max_device_seconds=float(max_device_seconds),
                              symmetry=SYMMETRY_NONE if unpacked else SYMMETRY_Z2, precision=int(precision))
    if initial_step is not None:
        s.initial_step = float(initial_step)
    K = _k_from_q(Q, R)
    dR, dK, dP = _device([R]), _device([K]), _device([rho])
    value = torch.zeros(1, dtype=torch.float64, device="cuda")
    cov = torch.zeros(d * d, dtype=torch.complex128, device="cuda")
    env = torch.zeros_like(cov)
    stats = (_lib.StateStats * 1)()
    rc = ctx.lib.rcmps_quartic_batch(ctx.handle, 1, (C.c_int * 1)(d), (C.c_double * 1)(float(g)), dR.data_ptr(),
                                     dK.data_ptr(), dP.data_ptr(), C.byref(s), value.data_ptr(), cov.data_ptr(),
                                     env.data_ptr(), stats, _stream())
    _raise_for(rc, ctx, stats[0], "quartic trajectory")
    st = stats[0].as_dict()
    st.update(accepted_steps=st["accepted"], rejected_steps=st["rejected"], persistent_trajectory=True,
              trajectory_kernel_launches=1, host_step_synchronizations=0, implicit_fallbacks=0,
              device_milliseconds=ctx.timings()[0], packed_z2=not unpacked,
              matrix_dimension=d if unpacked else d // 2)
    v = float(value.cpu().item())
    out = dict(value=v, energy=v, covector=_unpack(cov, [d])[0], environment=_unpack(env, [d])[0], stats=st)
    if return_samples:
        samples = torch.zeros((2 * int(n_quad) + 1, 7 * d * d + 1), dtype=torch.complex128, device="cuda")
        st2 = _lib.StateStats()
        rc = ctx.lib.rcmps_quartic_samples(ctx.handle, d, dR.data_ptr(), dK.data_ptr(), dP.data_ptr(), C.byref(s),
                                           samples.data_ptr(), C.byref(st2), _stream())
        _raise_for(rc, ctx, st2, "quartic samples")
        out["samples"] = samples.cpu().numpy() if unpacked else pack_z2_samples(samples.cpu().numpy(), d)
    return out


def pack_z2_samples(samples, d):
    """Dense seven-channel samples [points][7 d^2 + 1] of a Z2 state -> the packed layout
    [points][10 (d/2)^2 + 1] of the reference (ode_backend.py:262-275): per channel the upper
    off-diagonal block (F1, F3, A2, A4) or the two diagonal blocks (F2, A1, A3), then the scalar."""
    n = d // 2
    mats = samples[:, :-1].reshape(len(samples), 7, d, d)
    blocks = []
    for c in range(7):
        if c % 2 == 0:
            blocks.append(mats[:, c, :n, n:])
        else:
            blocks += [mats[:, c, :n, :n], mats[:, c, n:, n:]]
    out = np.empty((len(samples), 10 * n * n + 1), dtype=np.complex128)
    out[:, :-1] = np.stack(blocks, axis=1).reshape(len(samples), -1)
    out[:, -1] = samples[:, -1]
    return out


def evaluate_phi4(R, Q, rho, g, *, xp=None, half_window=20.0, n_quad=192, atol=1e-13, rtol=1e-12,
                  initial_step=None, max_steps=1_000_000, max_device_seconds=60.0, **ignored):
    """kinetic1 + kinetic2 + g phi^4, every term by ODEs (26 channels): dict(value, covector,
    environment, stats), as ode_backend.evaluate_phi4 (ode_backend.py:851-858) returns them."""
    import torch
    d = _check_matrices(R, Q, rho)
    ctx = context()
    s = _lib.default_settings(half_window=float(half_window), n_quad=int(n_quad), atol=float(atol), rtol=float(rtol),
                              max_steps=int(max_steps), max_device_seconds=float(max_device_seconds))
    if initial_step is not None:
        s.initial_step = float(initial_step)
    K = _k_from_q(Q, R)
    dR, dK, dP = _device([R]), _device([K]), _device([rho])
    value = torch.zeros(1, dtype=torch.float64, device="cuda")
    cov = torch.zeros(d * d, dtype=torch.complex128, device="cuda")
    env = torch.zeros_like(cov)
    stats = (_lib.StateStats * 1)()
    rc = ctx.lib.rcmps_phi4_ode_batch(ctx.handle, 1, (C.c_int * 1)(d), (C.c_double * 1)(float(g)), dR.data_ptr(),
                                      dK.data_ptr(), dP.data_ptr(), C.byref(s), value.data_ptr(), cov.data_ptr(),
                                      env.data_ptr(), stats, _stream())
    _raise_for(rc, ctx, stats[0], "ODE route")
    st = stats[0].as_dict()
    st.update(accepted_steps=st["accepted"], rejected_steps=st["rejected"], reduced_channels=False,
              device_milliseconds=ctx.timings()[0])
    return dict(value=float(value.cpu().item()), covector=_unpack(cov, [d])[0], environment=_unpack(env, [d])[0],
                stats=st)


def evaluate_phi4_batch(R, K, rho, couplings, settings=None, *, device=None):
    """The all-ODE route for a batch of states (lists of D_i x D_i matrices, uneven D allowed):
    (values [n], covectors, environments, stats) before the boundary/metric finish."""
    import torch
    n = len(R)
    if not (len(K) == len(rho) == len(couplings) == n):
        raise ValueError("R, K, rho and couplings must have the same length")
    dims = [_check_matrices(R[i], K[i], rho[i]) for i in range(n)]
    ctx = context(device)
    s = settings if settings is not None else _lib.default_settings(half_window=20.0, n_quad=192)
    dR, dK, dP = _device(R), _device(K), _device(rho)
    total = sum(d * d for d in dims)
    value = torch.zeros(n, dtype=torch.float64, device="cuda")
    cov = torch.zeros(total, dtype=torch.complex128, device="cuda")
    env = torch.zeros(total, dtype=torch.complex128, device="cuda")
    stats = (_lib.StateStats * n)()
    rc = ctx.lib.rcmps_phi4_ode_batch(ctx.handle, n, (C.c_int * n)(*dims), (C.c_double * n)(*map(float, couplings)),
                                      dR.data_ptr(), dK.data_ptr(), dP.data_ptr(), C.byref(s), value.data_ptr(),
                                      cov.data_ptr(), env.data_ptr(), stats, _stream())
    if rc:
        bad = next((i for i in range(n) if stats[i].status), 0)
        _raise_for(rc, ctx, stats[bad], "ODE route")
    return value.cpu().numpy(), _unpack(cov, dims), _unpack(env, dims), [stats[i].as_dict() for i in range(n)]


def kinetic_raw(q, r, rho, nodes=128, *, xp=None, tolerance=1e-12, initialdim=16, maxdim=1024, gradient=True,
                **ignored):
    """Both kinetic terms with unit coefficients: dict(value, energy, covector, environment, stats)."""
    import torch
    d = _check_matrices(q, r, rho)
    if not isinstance(nodes, (int, np.integer)) or nodes < 2:
        raise ValueError("angular node count must be an integer >= 2")
    ctx = context()
    s = _lib.default_settings(kinetic_nodes=int(nodes), krylov_tolerance=float(tolerance),
                              krylov_initialdim=int(initialdim), krylov_maxdim=int(maxdim))
    K = _k_from_q(q, r)
    dR, dK, dP = _device([r]), _device([K]), _device([rho])
    value = torch.zeros(1, dtype=torch.float64, device="cuda")
    cov = torch.zeros(d * d, dtype=torch.complex128, device="cuda")
    env = torch.zeros_like(cov)
    stats = (_lib.StateStats * 1)()
    rc = ctx.lib.rcmps_kinetic_batch(ctx.handle, 1, (C.c_int * 1)(d), dR.data_ptr(), dK.data_ptr(), dP.data_ptr(),
                                     C.byref(s), value.data_ptr(), cov.data_ptr(), env.data_ptr(), stats, _stream())
    if rc:
        raise KineticFailure(f"kinetic: {_lib.STATUS_NAMES.get(rc, rc)} ({ctx.error()})")
    st = stats[0].as_dict()
    labels = ("R_forward", "R_adjoint", "commutator_forward", "commutator_adjoint")
    st.update(nodes=int(nodes), solves={lab: dict(basis_size=b, fallback_used=False)
                                        for lab, b in zip(labels, st["krylov_basis"])},
              fallback_solves=0, maximum_relative_residual=st["krylov_residual"])
    v = float(value.cpu().item())
    return dict(value=v, energy=v, covector=_unpack(cov, [d])[0] if gradient else None,
                environment=_unpack(env, [d])[0] if gradient else None, stats=st, context=None)


def finish_gradient(q, r, rho, covector, environment, *, metric_reg=1e-3, tolerance=1e-13):
    """Boundary Poisson correction and metric solve: (gradient, stats)."""
    import torch
    d = _check_matrices(q, r, rho, covector, environment)
    ctx = context()
    s = _lib.default_settings(metric_reg=float(metric_reg), boundary_tolerance=float(tolerance))
    K = _k_from_q(q, r)
    dR, dK, dP, dC, dE = (_device([x]) for x in (r, K, rho, covector, environment))
    grad = torch.zeros(d * d, dtype=torch.complex128, device="cuda")
    stats = (_lib.StateStats * 1)()
    rc = ctx.lib.rcmps_finish_gradient_batch(ctx.handle, 1, (C.c_int * 1)(d), dR.data_ptr(), dK.data_ptr(),
                                             dP.data_ptr(), dC.data_ptr(), dE.data_ptr(), C.byref(s),
                                             grad.data_ptr(), stats, _stream())
    if rc:
        raise SolverFailure(f"Poisson GMRES failed: {_lib.STATUS_NAMES.get(rc, rc)} ({ctx.error()}), "
                            f"residual={stats[0].boundary_residual:.3e}")
    return _unpack(grad, [d])[0], {"matvecs": stats[0].gmres_iterations, "residual": stats[0].boundary_residual}


def boundary_environment_batch(R, K, rho, environments, *, tolerance=1e-13, x0=None, network=None, device=None,
                               preconditioner="nojump"):
    """The boundary Poisson solutions H_i, (-L*(H) + tr(rho H) I) = E - tr(rho E) I, of one
    environment E_i per entry (lists of D_i x D_i matrices; an entry may repeat a state with
    different environments), by restarted GMRES on the GPU (rcmps_boundary_environment_batch).
    preconditioner: "nojump" (the reference's right preconditioner, numerics.py:37-71, restart
    min(40, d^2)) or None (GMRES(64) unpreconditioned); x0: optional initial guesses (a warm
    start); network: a learned right preconditioner (rcmps_b200.warmstart.WarmStartNet, every
    state of its d) applied in flexible GMRES instead. Returns (H list, stats list) with
    stats[i] = dict(matvecs, iterations, residual): matvecs counted as the reference's GMRES
    counts them (Arnoldi steps plus one residual per restart cycle), as in boundary_environment
    (numerics.py:103-117)."""
    if preconditioner not in ("nojump", None):
        raise ValueError("preconditioner is 'nojump' or None")
    import torch
    n = len(R)
    if not (len(K) == len(rho) == len(environments) == n) or (x0 is not None and len(x0) != n):
        raise ValueError("R, K, rho, environments (and x0) must have the same length")
    dims = [_check_matrices(R[i], K[i], rho[i], environments[i]) for i in range(n)]
    ctx = context(device)
    s = _lib.default_settings(boundary_tolerance=float(tolerance),
                              boundary_preconditioner=1 if preconditioner == "nojump" else 0)
    dR, dK, dP, dE = _device(R), _device(K), _device(rho), _device(environments)
    dX = _device(x0) if x0 is not None else None
    H = torch.zeros(sum(d * d for d in dims), dtype=torch.complex128, device="cuda")
    stats = (_lib.StateStats * n)()
    rc = ctx.lib.rcmps_boundary_environment_batch(ctx.handle, n, (C.c_int * n)(*dims), dR.data_ptr(), dK.data_ptr(),
                                                  dP.data_ptr(), dE.data_ptr(),
                                                  dX.data_ptr() if dX is not None else None,
                                                  C.byref(network.c_struct()) if network is not None else None,
                                                  C.byref(s), H.data_ptr(), stats, _stream())
    if rc:
        raise SolverFailure(f"Poisson GMRES failed: {_lib.STATUS_NAMES.get(rc, rc)} ({ctx.error()})")
    return _unpack(H, dims), [{"matvecs": stats[i].gmres_matvecs, "iterations": stats[i].gmres_iterations,
                               "residual": stats[i].boundary_residual} for i in range(n)]


def boundary_environment(q, r, rho, environment, *, tolerance=1e-13, x0=None, preconditioner="nojump"):
    """(H, stats) of one state: the reference's boundary_environment (numerics.py:103-117)."""
    H, st = boundary_environment_batch([r], [_k_from_q(q, r)], [rho], [environment], tolerance=tolerance,
                                       x0=None if x0 is None else [x0], preconditioner=preconditioner)
    return H[0], st[0]


def stationary_state(q, r, *, tolerance=1e-11):
    """Stationary density of (Q, R): (rho, stats)."""
    import torch
    d = _check_matrices(q, r)
    ctx = context()
    K = _k_from_q(q, r)
    dR, dK = _device([r]), _device([K])
    rho = torch.zeros(d * d, dtype=torch.complex128, device="cuda")
    stats = (_lib.StateStats * 1)()
    rc = ctx.lib.rcmps_stationary_state_batch(ctx.handle, 1, (C.c_int * 1)(d), dR.data_ptr(), dK.data_ptr(),
                                              C.c_double(float(tolerance)), rho.data_ptr(), stats, _stream())
    if rc:
        raise SolverFailure(f"Invalid stationary density: {_lib.STATUS_NAMES.get(rc, rc)} ({ctx.error()})")
    return _unpack(rho, [d])[0], {"matvecs": stats[0].gmres_iterations, "stationary_residual": stats[0].boundary_residual}


def stationary_state_correction(q, r, rho_previous, *, tolerance=1e-11, maxiter=200):
    """Stationary density of (Q, R) started from a nearby density rho_previous, the previous
    accepted state of an optimizer: GMRES on the GPU solves for the correction to an absolute
    residual of `tolerance`, then the same checks as stationary_state apply
    (stationary_correction.py:19-96). rho_previous must be finite, normalized, Hermitian and
    positive (ValueError otherwise). The GPU solve restarts every 64 iterations, at most 200
    times; maxiter is accepted for the reference's signature. Returns (rho, stats)."""
    import torch
    q, r, prev = (np.asarray(x) for x in (q, r, rho_previous))
    if q.ndim != 2 or q.shape[0] != q.shape[1] or q.shape != r.shape or q.shape != prev.shape:
        raise ValueError("q, r and rho_previous must be equally sized square matrices")
    if any(x.dtype != np.complex128 for x in (q, r, prev)):
        raise ValueError("stationary correction requires complex128 inputs")
    if any(not np.isfinite(x).all() for x in (q, r, prev)):
        raise ValueError("stationary correction inputs must be finite")
    if not np.isfinite(tolerance) or tolerance <= 0 or maxiter < 1:
        raise ValueError("tolerance and maxiter must be positive")
    if abs(np.trace(prev) - 1) > 100 * tolerance or np.linalg.norm(prev - prev.conj().T) > 100 * tolerance:
        raise ValueError("rho_previous must be normalized and Hermitian")
    if np.linalg.eigvalsh(prev).min() < -10 * tolerance:
        raise ValueError("rho_previous must be positive within the existing tolerance")
    d = len(q)
    ctx = context()
    K = _k_from_q(q, r)
    dR, dK, dP = _device([r]), _device([K]), _device([prev])
    rho = torch.zeros(d * d, dtype=torch.complex128, device="cuda")
    stats = (_lib.StateStats * 1)()
    rc = ctx.lib.rcmps_stationary_correction_batch(ctx.handle, 1, (C.c_int * 1)(d), dR.data_ptr(), dK.data_ptr(),
                                                   dP.data_ptr(), C.c_double(float(tolerance)), rho.data_ptr(),
                                                   stats, _stream())
    if rc:
        raise SolverFailure(f"Invalid stationary density: {_lib.STATUS_NAMES.get(rc, rc)} ({ctx.error()})")
    return _unpack(rho, [d])[0], {"matvecs": stats[0].gmres_iterations,
                                  "stationary_residual": stats[0].boundary_residual,
                                  "warm_start": True, "fallback_used": False}


def metric(rho, x, y, metric_reg=1e-3):
    """The Riemannian metric <x, y> = 2 Re tr(x^dag y (rho + reg I)) (numerics.py:129-130): a D x D
    helper for callers (line searches, gradient norms); not part of the evaluation."""
    rho = np.asarray(rho)
    return float(2.0 * np.vdot(x, np.asarray(y) @ (rho + metric_reg * np.eye(len(rho)))).real)


def default_args(**overrides):
    """The reference optimizer's defaults (optimizer/cli.py:39-42) as a namespace."""
    a = SimpleNamespace(window=30.0, quadrature=512, atol=1e-13, rtol=1e-12, max_steps=1_000_000, nodes=512,
                        krylov_tolerance=1e-12, maxdim=1024, metric_reg=1e-3)
    for k, v in overrides.items():
        setattr(a, k, v)
    return a
