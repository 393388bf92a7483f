"""Learned warm start of the boundary Poisson GMRES (the solve behind every finished gradient).

The boundary solve (-L*(H) + tr(rho H) I) = b, b = E - tr(rho E) I, is linear in b: its solution
map is the inverse of a d^2 x d^2 operator that changes slowly along an optimizer run. Restarted
GMRES spends most of its iterations on the few slowly converging directions of that operator.
WarmStartNet learns them: a small network y = W2 (W1 x) (two linear layers, x the 2 d^2 real
entries of b scaled to unit norm, rank r hidden units) is trained on (state, right-hand side,
solution) triples that the plain GPU solver emits for the states an optimizer visits, and then
proposes the initial guess H0 = |b| W2 W1 (b / |b|) of a later solve. Its training and
inference run on the GPU through the library's own kernels (rcmps_warmstart_forward / _backward
/ _adam: FP32 tiled GEMMs, the mean-squared-error gradient, Adam); the gradients are checked
against a NumPy restatement (oracle/warmstart_oracle.py).

The GMRES residual judges every answer: a warm-started solve stops at the same target,
|b - A H| <= tol max(1, |b|), as the cold one, and unpreconditioned GMRES from zero remains the
fallback (a guess worse than zero only costs iterations, never accuracy).

No counterpart in the reference (its solves are preconditioned by the no-jump inverse,
numerics.py:37-71, and start from zero).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from .objective import _stream, boundary_environment_batch, context

__all__ = ["WarmStartNet", "random_environments", "solve_triples", "gmres_gain"]


def random_environments(rho, count, rng):
    """`count` right-hand sides of the boundary solve for a state with density rho: i.i.d.
    standard complex Gaussian d x d matrices, projected so that tr(rho E) = 0 (then b = E)."""
    d = len(rho)
    out = []
    for _ in range(count):
        g = (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / math.sqrt(2.0)
        out.append(g - np.trace(rho @ g) * np.eye(d))
    return out


def solve_triples(R, K, rho, environments, *, tolerance=1e-13):
    """(b, H) pairs of one state by the library's solver (GMRES from zero, no-jump preconditioned):
    the training data."""
    H, stats = boundary_environment_batch([R] * len(environments), [K] * len(environments),
                                          [rho] * len(environments), environments, tolerance=tolerance)
    eye = np.eye(len(rho))
    return [np.asarray(e) - np.trace(rho @ e) * eye for e in environments], H, stats


def _to_real(mats):
    """Samples as columns: (n = 2 d^2, count) float32, each column (Re, Im) interleaved."""
    return np.ascontiguousarray(np.stack([np.asarray(m, np.complex128).view(np.float64).ravel() for m in mats],
                                         axis=1).astype(np.float32))


def _from_real(cols, d):
    cols = np.asarray(cols, np.float64)
    return [cols[:, j].copy().view(np.complex128).reshape(d, d) for j in range(cols.shape[1])]


class WarmStartNet:
    """Two linear layers, W1 (rank x n) and W2 (n x rank), FP32 on the GPU; n = 2 d^2."""

    def __init__(self, d, rank=128, seed=0, device=None):
        import torch
        self.d, self.rank, self.n = int(d), int(rank), 2 * int(d) * int(d)
        self.ctx = context(device)
        g = np.random.default_rng(seed)
        w1 = g.standard_normal((self.rank, self.n)) / math.sqrt(self.n)
        w2 = g.standard_normal((self.n, self.rank)) * (0.1 / math.sqrt(self.rank))
        self.W1 = torch.from_numpy(w1.astype(np.float32)).cuda()
        self.W2 = torch.from_numpy(w2.astype(np.float32)).cuda()
        self._m = [torch.zeros_like(self.W1), torch.zeros_like(self.W2)]
        self._v = [torch.zeros_like(self.W1), torch.zeros_like(self.W2)]
        self.step = 0

    def c_struct(self, identity=None):
        """The network as the library's right preconditioner (rcmps_gmres_network): M v = W2 W1 v
        (+ v when the rank is below n, so that M stays invertible on the complement)."""
        if identity is None:
            identity = 0.0 if self.rank >= self.n else 1.0
        self._cs = _lib.GmresNetwork(self.W1.data_ptr(), self.W2.data_ptr(), self.n, self.rank, float(identity))
        return self._cs

    def _check(self, rc, what):
        if rc:
            raise RuntimeError(f"{what}: {_lib.STATUS_NAMES.get(rc, rc)} ({self.ctx.error()})")

    def forward_device(self, X):
        """H = W1 X, Y = W2 H for device float32 X of shape (n, batch)."""
        import torch
        batch = X.shape[1]
        H = torch.empty((self.rank, batch), dtype=torch.float32, device="cuda")
        Y = torch.empty((self.n, batch), dtype=torch.float32, device="cuda")
        self._check(self.ctx.lib.rcmps_warmstart_forward(self.ctx.handle, self.n, self.rank, batch,
                                                         self.W1.data_ptr(), self.W2.data_ptr(), X.data_ptr(),
                                                         H.data_ptr(), Y.data_ptr(), _stream()), "forward")
        return H, Y

    def loss_and_grads(self, X, T):
        """(loss, dW1, dW2) of loss = sum (Y - T)^2 / batch on device float32 samples."""
        import torch
        batch = X.shape[1]
        H, Y = self.forward_device(X)
        dY = torch.empty_like(Y)
        dH = torch.empty_like(H)
        dW1 = torch.empty_like(self.W1)
        dW2 = torch.empty_like(self.W2)
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        self._check(self.ctx.lib.rcmps_warmstart_backward(self.ctx.handle, self.n, self.rank, batch,
                                                          self.W2.data_ptr(), X.data_ptr(), H.data_ptr(),
                                                          Y.data_ptr(), T.data_ptr(), dY.data_ptr(), dH.data_ptr(),
                                                          dW1.data_ptr(), dW2.data_ptr(), loss.data_ptr(),
                                                          _stream()), "backward")
        return float(loss.item()), dW1, dW2

    def _adam(self, grads, lr):
        self.step += 1
        for p, g, m, v in zip((self.W1, self.W2), grads, self._m, self._v):
            self._check(self.ctx.lib.rcmps_warmstart_adam(self.ctx.handle, p.numel(), p.data_ptr(), g.data_ptr(),
                                                          m.data_ptr(), v.data_ptr(), C.c_float(lr),
                                                          C.c_float(0.9), C.c_float(0.999), C.c_float(1e-8),
                                                          self.step, _stream()), "adam")

    def fit(self, rhs, solutions, *, epochs=200, batch=128, lr=2e-3, seed=0):
        """Train on (b, H) pairs (lists of d x d complex matrices): each pair scaled by 1/|b| (the
        map is linear), Adam on the mean squared error. Returns the loss of every epoch."""
        import torch
        scale = np.array([np.linalg.norm(b) for b in rhs])
        X = torch.from_numpy(_to_real([b / s for b, s in zip(rhs, scale)])).cuda()
        T = torch.from_numpy(_to_real([h / s for h, s in zip(solutions, scale)])).cuda()
        count = X.shape[1]
        g = np.random.default_rng(seed)
        losses = []
        for _ in range(epochs):
            order = torch.from_numpy(g.permutation(count)).cuda()
            total = 0.0
            for s0 in range(0, count, batch):
                idx = order[s0:s0 + batch]
                xb, tb = X[:, idx].contiguous(), T[:, idx].contiguous()
                loss, dW1, dW2 = self.loss_and_grads(xb, tb)
                self._adam((dW1, dW2), lr)
                total += loss * xb.shape[1]
            losses.append(total / count)
        return losses

    def predict(self, rhs):
        """Initial guesses |b| W2 W1 (b / |b|) for a list of right-hand sides."""
        import torch
        scale = np.array([max(np.linalg.norm(b), 1e-300) for b in rhs])
        X = torch.from_numpy(_to_real([b / s for b, s in zip(rhs, scale)])).cuda()
        _, Y = self.forward_device(X)
        return [h * s for h, s in zip(_from_real(Y.cpu().numpy(), self.d), scale)]


def gmres_gain(net, R, K, rho, environments, *, tolerance=1e-13):
    """GMRES matrix-vector products and residuals of the same solves by the fallback (GMRES from
    zero, unpreconditioned), from the network's warm start, and with the network as the right
    preconditioner of flexible GMRES (its coarse correction applied at every step):
    dict(cold, warm, preconditioned, *_residual, target, *_difference)."""
    rhs = [e - np.trace(rho @ e) * np.eye(len(rho)) for e in environments]
    n = len(environments)
    H0, st0 = boundary_environment_batch([R] * n, [K] * n, [rho] * n, environments, tolerance=tolerance,
                                         preconditioner=None)
    H1, st1 = boundary_environment_batch([R] * n, [K] * n, [rho] * n, environments, tolerance=tolerance,
                                         x0=net.predict(rhs), preconditioner=None)
    H2, st2 = boundary_environment_batch([R] * n, [K] * n, [rho] * n, environments, tolerance=tolerance,
                                         network=net)
    diff = lambda A, B: max(np.abs(a - b).max() / max(1.0, np.abs(a).max()) for a, b in zip(A, B))
    return {"cold": [s["matvecs"] for s in st0], "warm": [s["matvecs"] for s in st1],
            "preconditioned": [s["matvecs"] for s in st2],
            "cold_residual": [s["residual"] for s in st0], "warm_residual": [s["residual"] for s in st1],
            "preconditioned_residual": [s["residual"] for s in st2],
            "target": [tolerance * max(1.0, float(np.linalg.norm(b))) for b in rhs],
            "solution_difference": diff(H0, H1), "preconditioned_difference": diff(H0, H2)}


def path_states(d, seed, count, step):
    """A seeded optimizer-like path of `count` states: each the canonical retraction of the previous
    one along a random tangent direction of relative size `step` (the stand-in for the states an
    L-BFGS run visits), with its stationary density by the library's solve."""
    from .batch import random_state
    from .objective import stationary_state
    from .optimizer import retract
    rng = np.random.default_rng(seed)
    R, K = random_state(d, seed)
    out = []
    for _ in range(count):
        Q = -1j * K - R.conj().T @ R / 2
        rho, _ = stationary_state(Q, R, tolerance=1e-13)
        out.append((R, K, rho))
        X = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
        R, K = retract(R, K, X, step * np.linalg.norm(R) / np.linalg.norm(X))
    return out


def path_experiment(d, *, train_states=8, rhs_per_state=512, test_rhs=64, rank=None, epochs=100, lr=1e-3,
                    step=1e-2, seed=161, tolerance=1e-13):
    """Train on the plain solver's triples of the first `train_states` states of a path and solve
    `test_rhs` new right-hand sides of the next (held-out) state by the fallback, from the warm
    start and with the learned preconditioner. Returns the matrix-vector products, the device
    milliseconds of each batched solve (CUDA events), the training time and the final loss."""
    import time
    import torch
    states = path_states(d, seed, train_states + 1, step)
    rng = np.random.default_rng(seed + 1)
    B, H = [], []
    t0 = time.perf_counter()
    for R, K, rho in states[:train_states]:
        b, h, _ = solve_triples(R, K, rho, random_environments(rho, rhs_per_state, rng), tolerance=tolerance)
        B += b
        H += h
    t_data = time.perf_counter() - t0
    net = WarmStartNet(d, rank=rank or min(2 * d * d, len(B)), seed=seed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = net.fit(B, H, epochs=epochs, batch=128, lr=lr)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    R, K, rho = states[train_states]
    envs = random_environments(rho, test_rhs, np.random.default_rng(seed + 2))
    n = len(envs)

    def timed(**kw):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        Hs, st = boundary_environment_batch([R] * n, [K] * n, [rho] * n, envs, tolerance=tolerance, **kw)
        ev1.record()
        torch.cuda.synchronize()
        return Hs, st, ev0.elapsed_time(ev1)

    timed(preconditioner=None)                     # warm-up (graph capture of the cycles)
    H0, st0, ms0 = timed(preconditioner=None)
    timed(network=net)
    H2, st2, ms2 = timed(network=net)
    rhs = [e - np.trace(rho @ e) * np.eye(d) for e in envs]
    H1, st1, ms1 = timed(x0=net.predict(rhs), preconditioner=None)
    timed()
    H3, st3, ms3 = timed()                         # the no-jump preconditioner (the default solve)
    diff = lambda A, Bm: max(np.abs(a - b).max() / max(1.0, np.abs(a).max()) for a, b in zip(A, Bm))
    return {"d": d, "train_triples": len(B), "rank": net.rank, "epochs": epochs, "loss_first": losses[0],
            "loss_last": losses[-1], "data_seconds": t_data, "train_seconds": t_train,
            "matvecs_cold": float(np.mean([s["matvecs"] for s in st0])),
            "matvecs_warm": float(np.mean([s["matvecs"] for s in st1])),
            "matvecs_preconditioned": float(np.mean([s["matvecs"] for s in st2])),
            "matvecs_nojump": float(np.mean([s["matvecs"] for s in st3])),
            "ms_cold": ms0, "ms_warm": ms1, "ms_preconditioned": ms2, "ms_nojump": ms3,
            "max_residual_over_target": max(s["residual"] / (tolerance * max(1.0, float(np.linalg.norm(b))))
                                            for st in (st0, st1, st2, st3) for s, b in zip(st, rhs)),
            "solution_difference": max(diff(H0, H1), diff(H0, H2), diff(H0, H3))}
