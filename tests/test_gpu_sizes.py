"""Every padded dimension of the library (dp = 16, 32, 48, 64, 96, 128) against the oracle.

The golden vectors cover dp = 16 and 64; these cases reach the kernel instantiations of the other
sizes: the full evaluation at D = 20 (dp 32) and 40 (dp 48), the quartic trajectory and the kinetic
term at D = 72 (dp 96) and 100 (dp 128), the all-ODE route at D = 40, 72 and 100, and the
stationary state at D = 100. Short windows keep the oracle's share of the run to seconds.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import fg_phi4_oracle as O

pytestmark = pytest.mark.gpu

ENERGY_TOL = 1e-10
GRAD_TOL = 1e-8


def _state(d, seed):
    from rcmps_b200.batch import random_state
    R, K = random_state(d, seed)
    Q = O.left_canonical_q(R, K)
    rho = O.stationary_state(Q, R, tolerance=1e-13, method="krylov")
    return R, K, Q, rho


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(1.0, np.abs(b).max()))


def _metric_norm(rho, x):
    return math.sqrt(max(0.0, O.metric(rho, x, x)))


def test_fg_batch_dp32_dp48(gpu_context):
    """One batched evaluation of D = 20 and D = 40 (two padded groups) against the oracle."""
    from rcmps_b200 import objective
    states = [_state(20, 2020), _state(40, 4040)]
    g = [1.5, 2.5]
    s = objective.settings_from_args(None, half_window=4.0, n_quad=32, kinetic_nodes=64)
    E, G, stats = objective.fg_phi4_batch([x[0] for x in states], [x[1] for x in states], [x[3] for x in states], g, s)
    for i, (R, K, Q, rho) in enumerate(states):
        energy, grad, parts = O.fg_phi4(R, K, rho, g[i], half_window=4.0, n_quad=32, nodes=64, method="krylov")
        assert stats[i]["status"] == 0
        assert stats[i]["accepted"] == parts["quartic"]["stats"]["accepted"]
        assert abs(E[i] - energy) <= ENERGY_TOL * abs(energy)
        assert _metric_norm(rho, G[i] - grad) <= GRAD_TOL * max(1.0, _metric_norm(rho, grad))


@pytest.mark.parametrize("d", [72, 100])
def test_quartic_and_kinetic_dp96_dp128(gpu_context, d):
    from rcmps_b200 import objective
    R, K, Q, rho = _state(d, 7000 + d)
    q = objective.evaluate_quartic_persistent_trajectory(R, Q, rho, 2.0, half_window=1.0, n_quad=8, unpacked=True)
    ref = O.evaluate_quartic(R, Q, rho, 2.0, half_window=1.0, n_quad=8)
    assert (q["stats"]["accepted"], q["stats"]["rejected"]) == (ref["stats"]["accepted"], ref["stats"]["rejected"])
    assert abs(q["value"] - ref["value"]) <= ENERGY_TOL * max(1.0, abs(ref["value"]))
    assert _rel(q["covector"], ref["covector"]) < 1e-10
    assert _rel(q["environment"], ref["environment"]) < 1e-10
    k = objective.kinetic_raw(Q, R, rho, 16)
    kref = O.kinetic_raw(Q, R, rho, 16)
    assert abs(k["value"] - kref["value"]) <= ENERGY_TOL * max(1.0, abs(kref["value"]))
    assert _rel(k["covector"], kref["covector"]) < 1e-10
    assert k["stats"]["maximum_relative_residual"] <= 1e-12


@pytest.mark.parametrize("d", [40, 72, 100])
def test_ode_route_dp48_dp96_dp128(gpu_context, d):
    """The 26-channel system at the other padded sizes (three ring stages at dp = 128)."""
    from rcmps_b200 import objective
    R, K, Q, rho = _state(d, 9000 + d)
    out = objective.evaluate_phi4(R, Q, rho, 1.5, half_window=0.5, n_quad=8)
    ref = O.evaluate_phi4(R, Q, rho, 1.5, half_window=0.5, n_quad=8)
    assert (out["stats"]["accepted"], out["stats"]["rejected"]) == (ref["stats"]["accepted"], ref["stats"]["rejected"])
    assert abs(out["value"] - ref["value"]) <= ENERGY_TOL * max(1.0, abs(ref["value"]))
    assert _rel(out["covector"], ref["covector"]) < 1e-10
    assert _rel(out["environment"], ref["environment"]) < 1e-10


def test_stationary_dp128(gpu_context):
    from rcmps_b200 import objective
    from rcmps_b200.batch import random_state
    R, K = random_state(100, 101)
    Q = O.left_canonical_q(R, K)
    rho, st = objective.stationary_state(Q, R, tolerance=1e-12)
    ref = O.stationary_state(Q, R, tolerance=1e-12, method="krylov")
    assert np.abs(rho - ref).max() < 1e-11
