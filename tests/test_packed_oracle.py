"""The packed Z2 route of the oracle against the reference's own packed route (tests/golden/packed.npz).

The reference evaluates Z2-symmetric states on ten (D/2)^2 blocks by default
(persistent_trajectory_backend.py:439-461 with unpacked=False; ode_backend.py:236-473, 700-716).
Its DOP853 error norm runs over the 10 (D/2)^2 + 1 packed entries, so its step sequence differs
from the dense seven-channel route; these tests pin the step counts, the values and the
trajectory samples of the oracle's restatement.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_records
from oracle import fg_phi4_oracle as O


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1.0, np.max(np.abs(b))))


def _metric_norm(rho, x):
    return math.sqrt(max(0.0, O.metric(rho, x, x)))


@pytest.mark.parametrize("index", range(3))
def test_packed_quartic_matches_reference(index):
    rec = load_records("packed.npz")[index]
    R, K, rho, g = rec["R"], rec["K"], rec["rho"], rec["g"]
    Q = O.left_canonical_q(R, K)
    out = O.evaluate_quartic(R, Q, rho, g, half_window=rec["window"], n_quad=int(rec["n_quad"]), packed_z2=True)
    assert (out["stats"]["accepted"], out["stats"]["rejected"]) == (rec["accepted"], rec["rejected"])
    assert abs(out["value"] - rec["quartic_value"]) <= 1e-12 * max(1.0, abs(rec["quartic_value"]))
    assert rel(out["covector"], rec["quartic_covector"]) < 1e-11
    assert rel(out["environment"], rec["quartic_environment"]) < 1e-11


def test_packed_fg_d32_matches_reference():
    """The whole objective with the packed quartic route at the optimizer defaults, D = 32."""
    rec = load_records("packed.npz")[3]
    energy, grad, parts = O.fg_phi4(rec["R"], rec["K"], rec["rho"], rec["g"], method="krylov", packed_z2=True)
    assert (parts["quartic"]["stats"]["accepted"], parts["quartic"]["stats"]["rejected"]) == \
        (rec["accepted"], rec["rejected"])
    assert abs(energy - rec["energy"]) <= 1e-12 * abs(rec["energy"])
    assert _metric_norm(rec["rho"], grad - rec["gradient"]) < 1e-10 * max(1.0, _metric_norm(rec["rho"], grad))


def test_packed_samples_match_reference():
    rec = load_records("packed.npz")[4]
    Q = O.left_canonical_q(rec["R"], rec["K"])
    system = O.PackedZ2System(Q, rec["R"], rec["rho"])
    points, _ = O.quadrature(float(rec["window"]), int(rec["n_quad"]))
    samples, stats = O.integrate(system, np.r_[points, math.sqrt(float(rec["window"]))])
    ref = rec["samples"]
    assert samples.shape == ref.shape == (2 * int(rec["n_quad"]) + 1, 10 * 2 * 2 + 1)
    assert (stats["accepted"], stats["rejected"]) == (rec["accepted"], rec["rejected"])
    assert np.abs(samples[:, :-1] - ref[:, :-1]).max() < 1e-13 * np.abs(ref).max()
    assert abs(samples[-1, -1].real - ref[-1, -1].real) < 1e-14


def test_packed_and_dense_routes_agree_on_values():
    """Same equations, different error norms: the values agree to the integration tolerance,
    the step counts do not have to."""
    rec = load_records("packed.npz")[1]
    R, K, rho, g = rec["R"], rec["K"], rec["rho"], rec["g"]
    Q = O.left_canonical_q(R, K)
    dense = O.evaluate_quartic(R, Q, rho, g, half_window=rec["window"], n_quad=int(rec["n_quad"]))
    assert abs(dense["value"] - rec["quartic_value"]) <= 1e-9 * abs(rec["quartic_value"])
    assert rel(dense["covector"], rec["quartic_covector"]) < 1e-9


def test_packed_route_requires_exact_z2_structure():
    R, K = O.phi4_state(8, 3)
    Q = O.left_canonical_q(R, K)
    rho = O.stationary_state(Q, R)
    with pytest.raises(ValueError):
        O.evaluate_quartic(R, Q, rho, 1.0, half_window=1.0, n_quad=8, packed_z2=True)
    rec = load_records("packed.npz")[1]
    R = rec["R"].copy()
    R[0, 0] = 1e-300          # one structurally zero entry that is not exactly zero
    Q = O.left_canonical_q(R, rec["K"])
    assert not O.z2_structure_ok(R, Q, rec["rho"])
    R = rec["R"]
    Q = O.left_canonical_q(R, rec["K"])
    assert O.z2_structure_ok(R, Q, rec["rho"])
    assert not O.z2_structure_ok(R[:7, :7], Q[:7, :7], rec["rho"][:7, :7])   # odd D


@pytest.mark.parametrize("index", range(3))
def test_phi_expectation_and_ode_match_reference(index):
    """<phi> of the validation report (validate_sweep.py:23-32, 140-145; ode_backend.py:782-797):
    the closed form and the ODE of the first monomial, against the reference's own routes."""
    rec = load_records("phi.npz")[index]
    phi = O.phi_expectation(rec["R"], rec["rho"], rec["window"])
    assert abs(phi - rec["phi"]) <= 1e-13 * max(1.0, abs(rec["phi"]))
    value, stats = O.phi_by_ode(rec["R"], rec["K"], rec["rho"], half_window=rec["window"], n_quad=int(rec["n_quad"]),
                                atol=rec["atol"], rtol=rec["rtol"])
    assert (stats["accepted"], stats["rejected"]) == (rec["accepted"], rec["rejected"])
    assert abs(value - rec["phi_ode"]) <= 1e-12 * max(1.0, abs(rec["phi_ode"]))
    assert abs(value - phi) <= 1e-9 * max(1.0, abs(phi))
