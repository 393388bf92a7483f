"""The oracle (oracle/fg_phi4_oracle.py) pinned to the reference: golden vectors produced by
RcmpsCore.jl's own NumPy path (tests/golden/make_golden.py) and the Julia fixture
test/fixtures/phi4_g2_D16_z2_portable. CPU only."""
import math

import numpy as np
import pytest

from conftest import GOLDEN, julia_fixture, load_records
from oracle import fg_phi4_oracle as O


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1.0, np.max(np.abs(b))))


@pytest.mark.parametrize("index", range(4))
def test_oracle_matches_reference_small_states(index):
    rec = load_records("small.npz")[index]
    R, K, rho, g = rec["R"], rec["K"], rec["rho"], rec["g"]
    Q = O.left_canonical_q(R, K)
    quartic = O.evaluate_quartic(R, Q, rho, g, half_window=rec["window"], n_quad=int(rec["n_quad"]))
    assert quartic["stats"]["accepted"] == rec["accepted"]
    assert quartic["stats"]["rejected"] == rec["rejected"]
    assert abs(quartic["value"] - rec["quartic_value"]) <= 1e-12 * max(1.0, abs(rec["quartic_value"]))
    assert rel(quartic["covector"], rec["quartic_covector"]) < 1e-11
    assert rel(quartic["environment"], rec["quartic_environment"]) < 1e-11
    kinetic = O.kinetic_raw(Q, R, rho, int(rec["nodes"]))
    assert abs(kinetic["value"] - rec["kinetic_value"]) <= 1e-12 * max(1.0, abs(rec["kinetic_value"]))
    assert rel(kinetic["covector"], rec["kinetic_covector"]) < 1e-11
    assert rel(kinetic["environment"], rec["kinetic_environment"]) < 1e-11
    cov = quartic["covector"] + kinetic["covector"]
    env = quartic["environment"] + kinetic["environment"]
    grad = O.finish_gradient(Q, R, rho, cov, env)
    diff = grad - rec["gradient"]
    assert math.sqrt(max(0.0, O.metric(rho, diff, diff))) < 1e-10 * max(1.0, math.sqrt(O.metric(rho, grad, grad)))


def test_oracle_stationary_state_matches_reference():
    for rec in load_records("small.npz"):
        Q = O.left_canonical_q(rec["R"], rec["K"])
        rho = O.stationary_state(Q, rec["R"], tolerance=1e-13)
        assert np.abs(rho - rec["rho"]).max() < 1e-12


def test_oracle_d16_full_settings():
    rec = load_records("d16.npz")[0]
    energy, grad, parts = O.fg_phi4(rec["R"], rec["K"], rec["rho"], rec["g"])
    assert abs(energy - rec["energy"]) <= 1e-12 * abs(rec["energy"])
    diff = grad - rec["gradient"]
    assert math.sqrt(max(0.0, O.metric(rec["rho"], diff, diff))) < 1e-10
    assert parts["quartic"]["stats"]["accepted"] == rec["accepted"]


def test_oracle_trajectory_samples_match_reference():
    data = np.load(GOLDEN / "samples_d5.npz")
    Q = O.left_canonical_q(data["R"], data["K"])
    system = O.QuarticSystem(Q, data["R"], data["rho"])
    points, _ = O.quadrature(float(data["window"]), int(data["n_quad"]))
    samples, stats = O.integrate(system, np.r_[points, math.sqrt(float(data["window"]))])
    ref = data["samples"]
    assert stats["accepted"] == int(data["accepted"]) and stats["rejected"] == int(data["rejected"])
    assert np.abs(samples[:, :-1] - ref[:, :-1]).max() < 1e-13 * np.abs(ref).max()
    assert abs(samples[-1, -1].real - ref[-1, -1].real) < 1e-14


def test_oracle_matches_julia_fixture():
    """Julia energy -0.15648780475169466 at W = 20, n_quad = 192 (the fixture's own settings);
    the reference's NumPy route reproduces it to 1e-13 and its gradient to 1.7e-9 in the metric
    norm (the state is near a minimum: |g| = 2.7e-6, so the Vern7/DOP853 difference dominates)."""
    fx = julia_fixture()
    energy, grad, _ = O.fg_phi4(fx["R"], fx["K"], fx["rho"], fx["meta"]["coupling"], half_window=20.0, n_quad=192)
    assert abs(energy - fx["meta"]["energy"]) < 1e-12
    diff = grad - fx["gradient"]
    assert math.sqrt(max(0.0, O.metric(fx["rho"], diff, diff))) < 5e-9


@pytest.mark.parametrize("index", range(4))
def test_oracle_ode_route_matches_reference(index):
    """The all-ODE route (26 channels: kinetic1, kinetic2 and g phi^4) against the reference's
    evaluate_phi4 + finish_gradient (ode_backend.py:851-858)."""
    rec = load_records("ode.npz")[index]
    R, K, rho, g = rec["R"], rec["K"], rec["rho"], rec["g"]
    Q = O.left_canonical_q(R, K)
    out = O.evaluate_phi4(R, Q, rho, g, half_window=rec["window"], n_quad=int(rec["n_quad"]))
    assert (out["stats"]["accepted"], out["stats"]["rejected"]) == (rec["accepted"], rec["rejected"])
    assert abs(out["value"] - rec["value"]) <= 1e-12 * max(1.0, abs(rec["value"]))
    assert rel(out["covector"], rec["covector"]) < 1e-11
    assert rel(out["environment"], rec["environment"]) < 1e-11
    grad = O.finish_gradient(Q, R, rho, out["covector"], out["environment"])
    diff = grad - rec["gradient"]
    assert math.sqrt(max(0.0, O.metric(rho, diff, diff))) < 1e-10 * max(1.0, math.sqrt(O.metric(rho, grad, grad)))


def test_oracle_ode_route_matches_julia_fixture():
    """Julia's default evaluation is this all-ODE route (Vern7 there, DOP853 here) at the
    fixture's settings: energy -0.15648780475169466 to 1e-12, gradient to 5e-9 (metric norm)."""
    fx = julia_fixture()
    R, K, rho = fx["R"], fx["K"], fx["rho"]
    Q = O.left_canonical_q(R, K)
    out = O.evaluate_phi4(R, Q, rho, fx["meta"]["coupling"], half_window=20.0, n_quad=192)
    assert abs(out["value"] - fx["meta"]["energy"]) < 1e-12
    grad = O.finish_gradient(Q, R, rho, out["covector"], out["environment"])
    diff = grad - fx["gradient"]
    assert math.sqrt(max(0.0, O.metric(rho, diff, diff))) < 5e-9


def test_source_and_quadrature():
    assert abs(O.source(0.0) - 1 / math.sqrt(math.pi)) < 1e-16
    assert abs(O.source(1e-9) - O.source(0.0)) < 1e-8
    x, w = O.quadrature(30.0, 512)
    assert np.all(np.diff(x) > 0) and abs(np.sum(w) - 2 * math.sqrt(30.0)) < 1e-12
    c, wa = O.angular_grid(512)
    assert np.all((c >= 0) & (c <= 1)) and abs(np.sum(wa) - 1.0) < 1e-13


def test_coherent_state_known_answers():
    """R = alpha I, K = 0 (a coherent state, D = 1 embedded in D = 2): <phi^n> = (sqrt2 Re alpha)^n
    up to the window tail, kinetic1 = |alpha|^2... only the field moments are checked here: the
    quartic value equals (sqrt(2) Re alpha)^4 times int J over the window (test/runtests.jl:90-104)."""
    a = 0.3
    R = a * np.eye(2, dtype=complex)
    K = np.zeros((2, 2), complex)
    Q = O.left_canonical_q(R, K)
    rho = np.eye(2, dtype=complex) / 2
    quartic = O.evaluate_quartic(R, Q, rho, 1.0, half_window=30.0, n_quad=64)
    assert abs(quartic["value"] - (math.sqrt(2) * a) ** 4) < 1e-10


@pytest.mark.parametrize("index", range(3))
def test_oracle_preconditioned_boundary_solve_matches_reference(index):
    """The reference's boundary solve itself (numerics.py:55-126): the no-jump preconditioned
    GMRES takes the same number of matrix-vector products, and the finished gradient agrees. The
    unpreconditioned solves (the oracle's others, and the library's) need several times more."""
    rec = load_records("finish.npz")[index]
    R, K, rho = rec["R"], rec["K"], rec["rho"]
    Q = O.left_canonical_q(R, K)
    h, matvecs = O.boundary_environment_preconditioned(Q, R, rho, rec["environment"])
    assert matvecs == int(rec["matvecs"])
    grad = O.finish_gradient(Q, R, rho, rec["covector"], rec["environment"], method="preconditioned")
    diff = grad - rec["gradient"]
    assert math.sqrt(max(0.0, O.metric(rho, diff, diff))) < 1e-10 * max(1.0, math.sqrt(O.metric(rho, grad, grad)))
    dense = O.finish_gradient(Q, R, rho, rec["covector"], rec["environment"], method="dense")
    diff = dense - grad
    assert math.sqrt(max(0.0, O.metric(rho, diff, diff))) < 1e-9 * max(1.0, math.sqrt(O.metric(rho, grad, grad)))
