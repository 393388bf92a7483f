"""The no-jump preconditioner of the boundary Poisson GMRES on the device (the default solve):
against the reference's own preconditioned solve (numerics.py:55-71 with NoJumpInverse; the
oracle's boundary_environment_preconditioned restates it and reproduces the reference's matvec
counts stored in tests/golden/finish.npz).

Tolerances: the GPU's operator applications within +-1 of the reference's count (35, 59, 53:
the Arnoldi steps plus one true residual per restart cycle, as SciPy's GMRES counts them; the
orthogonalisation and the eigenbasis form of the inverse change rounding only); H equal to 1e-10
relative; the unpreconditioned solve reaches the same H."""
import numpy as np
import pytest

from conftest import load_records
from oracle import fg_phi4_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("index", [0, 1, 2])
def test_matvec_counts_match_reference(gpu_context, index):
    from rcmps_b200 import objective
    rec = load_records("finish.npz")[index]
    R, K, rho, env = rec["R"], rec["K"], rec["rho"], rec["environment"]
    Q = O.left_canonical_q(R, K)
    h_ref, count_ref = O.boundary_environment_preconditioned(Q, R, rho, env)
    assert count_ref == int(rec["matvecs"])
    H, st = objective.boundary_environment(Q, R, rho, env)
    print(f"state {index}: D={len(R)} matvecs GPU {st['matvecs']} reference {count_ref}")
    assert abs(st["matvecs"] - count_ref) <= 1
    scale = max(1.0, np.abs(h_ref).max())
    assert np.abs(H - h_ref).max() <= 1e-10 * scale
    H0, st0 = objective.boundary_environment(Q, R, rho, env, preconditioner=None)
    assert np.abs(H0 - h_ref).max() <= 1e-10 * scale
    assert st0["matvecs"] > st["matvecs"]


def test_bench_states_take_the_references_iterations(gpu_context):
    """Two D = 64 states of the benchmark workload (random seed 0, Z2 seed 100): the preconditioned
    GPU solve against the oracle's restatement of the reference's solve, with one environment each."""
    from rcmps_b200 import objective
    recs = load_records("bench.npz")
    rng = np.random.default_rng(17)
    for rec in (recs[0], recs[2]):
        R, K, rho = rec["R"], rec["K"], rec["rho"]
        Q = O.left_canonical_q(R, K)
        d = len(R)
        env = (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / np.sqrt(2.0)
        h_ref, count_ref = O.boundary_environment_preconditioned(Q, R, rho, env)
        H, st = objective.boundary_environment(Q, R, rho, env)
        print(f"D=64 matvecs GPU {st['matvecs']} reference {count_ref}")
        assert abs(st["matvecs"] - count_ref) <= 2
        assert np.abs(H - h_ref).max() <= 1e-10 * max(1.0, np.abs(h_ref).max())


def test_batched_solve_with_mixed_dimensions(gpu_context):
    """One call over states of padded dimensions 16, 48 and 96 (padding stays exact zeros)."""
    from rcmps_b200 import objective
    from rcmps_b200.batch import random_state
    rng = np.random.default_rng(3)
    R, K, P, E = [], [], [], []
    for d in (12, 40, 90):
        r, k = random_state(d, 50 + d)
        rho, _ = objective.stationary_state(O.left_canonical_q(r, k), r, tolerance=1e-13)
        R.append(r)
        K.append(k)
        P.append(rho)
        E.append((rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / np.sqrt(2.0))
    H, st = objective.boundary_environment_batch(R, K, P, E)
    H0, st0 = objective.boundary_environment_batch(R, K, P, E, preconditioner=None)
    for i in range(3):
        assert np.abs(H[i] - H0[i]).max() <= 1e-10 * max(1.0, np.abs(H0[i]).max())
        assert st[i]["matvecs"] < st0[i]["matvecs"]
