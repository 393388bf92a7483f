"""The learned warm start of the boundary GMRES (rcmps_b200.warmstart): the library's training
kernels against the NumPy oracle (oracle/warmstart_oracle.py), the boundary-solve entry against
the reference's boundary_environment, and what a trained network gains over GMRES from zero on
held-out states of an optimizer-like path.

Tolerances: FP32 kernels against the FP64 oracle to 1e-4 relative; every solve, warm or cold, to
the library's GMRES target |b - A H| <= 1e-13 max(1, |b|); warm and cold solutions equal to 1e-10.
"""
import math

import numpy as np
import pytest

from conftest import load_records
from oracle import fg_phi4_oracle as O
from oracle import warmstart_oracle as WO

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(1e-30, np.abs(b).max()))


def test_network_gradients_match_oracle(gpu_context):
    import torch
    from rcmps_b200.warmstart import WarmStartNet
    rng = np.random.default_rng(7)
    d, rank, batch = 8, 16, 40          # n = 128: tiles with partial edges in every GEMM
    net = WarmStartNet(d, rank=rank, seed=3)
    X = rng.standard_normal((net.n, batch)).astype(np.float32)
    T = rng.standard_normal((net.n, batch)).astype(np.float32)
    loss, dW1, dW2 = net.loss_and_grads(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
    W1, W2 = net.W1.cpu().numpy(), net.W2.cpu().numpy()
    ref_loss, ref1, ref2 = WO.loss_and_grads(W1, W2, X, T)
    assert abs(loss - ref_loss) <= 1e-5 * ref_loss
    assert _rel(dW1.cpu().numpy(), ref1) <= 1e-4
    assert _rel(dW2.cpu().numpy(), ref2) <= 1e-4
    _, Y = net.forward_device(torch.from_numpy(X).cuda())
    assert _rel(Y.cpu().numpy(), WO.forward(W1, W2, X)[1]) <= 1e-4
    # one Adam step of W1 against the oracle's
    p_ref, _, _ = WO.adam_step(W1.astype(np.float64), ref1, np.zeros_like(ref1), np.zeros_like(ref1), 1e-3, 1)
    net._adam((dW1, dW2), 1e-3)
    assert _rel(net.W1.cpu().numpy(), p_ref) <= 1e-5


def test_boundary_environment_matches_reference(gpu_context):
    """H of the reference's preconditioned boundary solve (finish.npz records the gradient it
    yields; H is recovered from it on the CPU) and the library's GMRES from zero and from a guess."""
    from rcmps_b200 import objective
    rec = load_records("finish.npz")[1]
    R, K, rho, env = rec["R"], rec["K"], rec["rho"], rec["environment"]
    Q = O.left_canonical_q(R, K)
    h_ref, _ = O.boundary_environment_preconditioned(Q, R, rho, env)
    H, st = objective.boundary_environment(Q, R, rho, env)
    assert np.abs(H - h_ref).max() <= 1e-10 * max(1.0, np.abs(h_ref).max())
    H2, st2 = objective.boundary_environment(Q, R, rho, env, x0=h_ref + 1e-6)
    assert np.abs(H2 - h_ref).max() <= 1e-10 * max(1.0, np.abs(h_ref).max())
    assert st2["matvecs"] < st["matvecs"]


def _path_states(d, seed, count, step):
    """A seeded optimizer-like path: each state the canonical retraction of the previous one along
    a random tangent direction of relative size `step`."""
    from rcmps_b200 import objective, optimizer
    from rcmps_b200.batch import random_state
    rng = np.random.default_rng(seed)
    R, K = random_state(d, seed)
    out = []
    for _ in range(count):
        Q = O.left_canonical_q(R, K)
        rho, _ = objective.stationary_state(Q, R, tolerance=1e-13)
        out.append((R, K, rho))
        X = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
        R, K = optimizer.retract(R, K, X, step * np.linalg.norm(R) / np.linalg.norm(X))
    return out


def test_learned_network_cuts_gmres_iterations(gpu_context):
    """Train a full-rank network (D = 16: n = 512) on triples of five states of a path (256
    right-hand sides each) and solve 64 new right-hand sides of the sixth, held-out state three
    ways: the fallback (GMRES from zero, unpreconditioned), from the network's warm start, and
    with the network as the right preconditioner of flexible GMRES. Every solve meets the same
    residual target and they agree to 1e-10; the warm start saves a little (its gain is
    logarithmic in the guess's accuracy at a 1e-13 target), the preconditioned solves take at
    most a third of the fallback's matrix-vector products."""
    from rcmps_b200.warmstart import WarmStartNet, gmres_gain, random_environments, solve_triples
    d = 16
    states = _path_states(d, 161, 6, 1e-2)
    rng = np.random.default_rng(5)
    B, H = [], []
    for R, K, rho in states[:5]:
        b, h, _ = solve_triples(R, K, rho, random_environments(rho, 256, rng))
        B += b
        H += h
    net = WarmStartNet(d, rank=2 * d * d, seed=1)
    losses = net.fit(B, H, epochs=300, batch=128, lr=2e-3)
    assert losses[-1] < 0.01 * losses[0]
    R, K, rho = states[5]
    gain = gmres_gain(net, R, K, rho, random_environments(rho, 64, np.random.default_rng(6)))
    cold, warm, pre = np.mean(gain["cold"]), np.mean(gain["warm"]), np.mean(gain["preconditioned"])
    print(f"GMRES matvecs: cold {cold:.1f}, warm {warm:.1f}, preconditioned {pre:.1f}; "
          f"final loss {losses[-1]:.3e} (first {losses[0]:.3e})")
    assert warm < cold
    assert pre <= cold / 3
    for key in ("warm_residual", "preconditioned_residual"):
        assert all(r <= t for r, t in zip(gain[key], gain["target"]))
    assert gain["solution_difference"] <= 1e-10 and gain["preconditioned_difference"] <= 1e-10
