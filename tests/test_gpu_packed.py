"""The packed Z2 route on the GPU against the reference's packed route and the oracle.

Z2-symmetric states (R odd, K and rho even) take the reference's default quartic route
(persistent_trajectory_backend.py:439-461 with unpacked=False): the DOP853 error norm over the
10 (D/2)^2 + 1 packed entries. The library keeps the dense layout and applies that norm; the
step counts must equal the reference's, the values agree to the parity tolerances.
"""
from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import load_records
from oracle import fg_phi4_oracle as O

pytestmark = pytest.mark.gpu

ENERGY_TOL = 1e-10
GRAD_TOL = 1e-8


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(1.0, np.abs(b).max()))


def _metric_norm(rho, x):
    return math.sqrt(max(0.0, O.metric(rho, x, x)))


@pytest.mark.parametrize("index", range(4))
def test_packed_quartic_matches_reference(gpu_context, index):
    from rcmps_b200 import objective
    rec = load_records("packed.npz")[index]
    R, K, rho, g = rec["R"], rec["K"], rec["rho"], rec["g"]
    Q = O.left_canonical_q(R, K)
    q = objective.evaluate_quartic_persistent_trajectory(R, Q, rho, g, half_window=rec["window"],
                                                         n_quad=int(rec["n_quad"]))
    assert q["stats"]["packed_z2"] and q["stats"]["matrix_dimension"] == len(R) // 2
    assert (q["stats"]["accepted"], q["stats"]["rejected"]) == (rec["accepted"], rec["rejected"])
    assert abs(q["value"] - rec["quartic_value"]) <= 1e-12 * max(1.0, abs(rec["quartic_value"]))
    assert _rel(q["covector"], rec["quartic_covector"]) < 1e-11
    assert _rel(q["environment"], rec["quartic_environment"]) < 1e-11


def test_packed_samples_match_reference(gpu_context):
    from rcmps_b200 import objective
    rec = load_records("packed.npz")[4]
    R, K, rho = rec["R"], rec["K"], rec["rho"]
    Q = O.left_canonical_q(R, K)
    out = objective.evaluate_quartic_persistent_trajectory(R, Q, rho, 1.0, half_window=float(rec["window"]),
                                                           n_quad=int(rec["n_quad"]), return_samples=True)
    assert (out["stats"]["accepted"], out["stats"]["rejected"]) == (rec["accepted"], rec["rejected"])
    ref, got = rec["samples"], out["samples"]
    assert got.shape == ref.shape
    assert np.abs(got[:, :-1] - ref[:, :-1]).max() <= 1e-12 * np.abs(ref).max()
    assert abs(got[-1, -1].real - ref[-1, -1].real) <= 1e-14


def test_packed_objective_d32_matches_reference(gpu_context):
    """The whole objective with args.packed_z2 (sweep_driver.py:100-101) at the optimizer defaults."""
    from rcmps_b200 import objective
    rec = load_records("packed.npz")[3]
    args = SimpleNamespace(window=30.0, quadrature=512, nodes=512, packed_z2=True, reduced=False)
    energy, grad, stats = objective.objective(rec["R"], rec["K"], rec["rho"], rec["g"], args)
    assert (stats["accepted"], stats["rejected"]) == (rec["accepted"], rec["rejected"])
    assert abs(energy - rec["energy"]) <= ENERGY_TOL * abs(rec["energy"])
    assert _metric_norm(rec["rho"], grad - rec["gradient"]) <= GRAD_TOL * max(1.0, _metric_norm(rec["rho"], grad))


def test_packed_bench_state_d64_matches_reference(gpu_context):
    """The first two Z2 states of the 32-state bench workload (D = 64, seeds 100, 101), quartic term
    at W = 30, n_quad = 512, against the reference's packed route run on the reference's own
    stationary density (bench.npz): exact step counts."""
    from rcmps_b200 import objective
    for rec in load_records("bench.npz")[2:]:
        R, K, rho = rec["R"], rec["K"], rec["rho"]
        Q = O.left_canonical_q(R, K)
        q = objective.evaluate_quartic_persistent_trajectory(R, Q, rho, rec["g"])
        assert (q["stats"]["accepted"], q["stats"]["rejected"]) == (rec["accepted"], rec["rejected"])
        assert abs(q["value"] - rec["quartic_value"]) <= ENERGY_TOL * abs(rec["quartic_value"])
        assert _rel(q["covector"], rec["quartic_covector"]) < 1e-10
        assert _rel(q["environment"], rec["quartic_environment"]) < 1e-10


def test_auto_route_mixed_batch(gpu_context):
    """symmetry 2: packed for the Z2 state, unpacked for the random one, in one batched call."""
    from rcmps_b200 import objective
    z2 = load_records("packed.npz")[1]
    rnd = load_records("small.npz")[2]
    s = objective.settings_from_args(None, half_window=30.0, n_quad=64, kinetic_nodes=128,
                                     symmetry=objective.SYMMETRY_AUTO)
    E, G, stats = objective.fg_phi4_batch([rnd["R"], z2["R"]], [rnd["K"], z2["K"]], [rnd["rho"], z2["rho"]],
                                          [rnd["g"], z2["g"]], s)
    assert (stats[0]["accepted"], stats[0]["rejected"]) == (rnd["accepted"], rnd["rejected"])
    assert (stats[1]["accepted"], stats[1]["rejected"]) == (z2["accepted"], z2["rejected"])
    assert abs(E[0] - rnd["energy"]) <= ENERGY_TOL * abs(rnd["energy"])
    Q = O.left_canonical_q(z2["R"], z2["K"])
    kin = O.kinetic_raw(Q, z2["R"], z2["rho"], 128)
    assert abs(E[1] - (z2["quartic_value"] + kin["value"])) <= ENERGY_TOL * abs(z2["quartic_value"] + kin["value"])


def test_packed_route_refuses_states_without_z2_structure(gpu_context):
    from rcmps_b200 import objective
    R, K = O.phi4_state(8, 3)
    Q = O.left_canonical_q(R, K)
    rho = O.stationary_state(Q, R)
    with pytest.raises(ValueError, match="packed Z2"):
        objective.evaluate_quartic_persistent_trajectory(R, Q, rho, 1.0, n_quad=16)
    z2 = load_records("packed.npz")[1]
    s = objective.settings_from_args(None, n_quad=16, kinetic_nodes=64, symmetry=objective.SYMMETRY_Z2)
    with pytest.raises(ValueError, match="state 1"):
        objective.fg_phi4_batch([z2["R"], R], [z2["K"], K], [z2["rho"], rho], [1.0, 1.0], s)
    # the context stays usable, and the same states pass on the unpacked route
    out = objective.evaluate_quartic_persistent_trajectory(R, Q, rho, 1.0, n_quad=16, unpacked=True)
    assert out["stats"]["status"] == 0


@pytest.mark.parametrize("d", [96, 128])
def test_packed_quartic_large_d_matches_oracle(gpu_context, d):
    """The skipped structural zeros at the other unpadded sizes with 16-row halves (dp 96, 128)."""
    from rcmps_b200 import objective
    from rcmps_b200.batch import z2_state
    R, K = z2_state(d, 9100 + d)
    Q = O.left_canonical_q(R, K)
    rho = O.stationary_state(Q, R, tolerance=1e-13, method="krylov")
    n = d // 2
    rho[:n, n:] = 0.0
    rho[n:, :n] = 0.0
    rho = 0.5 * (rho + rho.conj().T)
    q = objective.evaluate_quartic_persistent_trajectory(R, Q, rho, 2.0, half_window=1.0, n_quad=8)
    ref = O.evaluate_quartic(R, Q, rho, 2.0, half_window=1.0, n_quad=8, packed_z2=True)
    assert (q["stats"]["accepted"], q["stats"]["rejected"]) == (ref["stats"]["accepted"], ref["stats"]["rejected"])
    assert abs(q["value"] - ref["value"]) <= ENERGY_TOL * max(1.0, abs(ref["value"]))
    assert _rel(q["covector"], ref["covector"]) < 1e-10
    assert _rel(q["environment"], ref["environment"]) < 1e-10


def test_auto_route_d64_pair_in_one_launch(gpu_context):
    """A random and a Z2 state of the bench workload in one launch: the random state takes the
    unpacked route as when it runs alone, the Z2 state the packed one (structural zeros skipped)."""
    from rcmps_b200 import objective
    from rcmps_b200.batch import random_state, z2_state
    states = [random_state(64, 0), z2_state(64, 100)]
    rhos = []
    for R, K in states:
        Q = O.left_canonical_q(R, K)
        rho, _ = objective.stationary_state(Q, R, tolerance=1e-13)
        rhos.append(rho)
    s = objective.settings_from_args(None, half_window=2.0, n_quad=32, kinetic_nodes=64,
                                     symmetry=objective.SYMMETRY_AUTO)
    E, G, st = objective.fg_phi4_batch([x[0] for x in states], [x[1] for x in states], rhos, [2.0, 2.0], s)
    assert (st[0]["packed_z2"], st[1]["packed_z2"]) == (0, 1)
    s0 = objective.settings_from_args(None, half_window=2.0, n_quad=32, kinetic_nodes=64)
    E0, G0, st0 = objective.fg_phi4_batch([states[0][0]], [states[0][1]], [rhos[0]], [2.0], s0)
    assert (st[0]["accepted"], st[0]["rejected"]) == (st0[0]["accepted"], st0[0]["rejected"])
    assert abs(E[0] - E0[0]) <= 1e-12 * abs(E0[0])
    R, K = states[1]
    Q = O.left_canonical_q(R, K)
    ref = O.evaluate_quartic(R, Q, rhos[1], 2.0, half_window=2.0, n_quad=32, packed_z2=True)
    assert (st[1]["accepted"], st[1]["rejected"]) == (ref["stats"]["accepted"], ref["stats"]["rejected"])
    assert abs(st[1]["quartic_value"] - ref["value"]) <= ENERGY_TOL * abs(ref["value"])
