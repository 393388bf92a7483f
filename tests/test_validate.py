"""The validation run of an optimized state (rcmps_b200.validate) and its <phi> against the
reference (validate_sweep.py:23-32, 84-145; ode_backend.py:782-797; tests/golden/phi.npz)."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from conftest import load_records


@pytest.mark.parametrize("index", range(3))
def test_phi_expectation_matches_reference(index):
    from rcmps_b200 import validate
    rec = load_records("phi.npz")[index]
    phi = validate.phi_expectation(rec["R"], rec["rho"], rec["window"])
    assert abs(phi - rec["phi"]) <= 1e-13 * max(1.0, abs(rec["phi"]))


@pytest.mark.gpu
@pytest.mark.parametrize("index", range(3))
def test_phi_by_ode_matches_reference(gpu_context, index):
    from rcmps_b200 import validate
    rec = load_records("phi.npz")[index]
    controls = SimpleNamespace(window=rec["window"], quadrature=int(rec["n_quad"]), atol=rec["atol"],
                               rtol=rec["rtol"], max_steps=1_000_000)
    value, stats = validate.phi_by_ode(rec["R"], rec["K"], rec["rho"], controls)
    # the library's count minus the reference's, pinned exactly per record: the long-window
    # records (W = 20 and the refined W = 40) take one or two more accepted steps, for the reason
    # given at ODE_STEP_OFFSETS in test_gpu_parity.py; the value then differs by the integration
    # error, within the energy parity bar
    da = {0: 0, 1: 1, 2: 2}[index]
    assert (stats["accepted_steps"], stats["rejected_steps"]) == (rec["accepted"] + da, rec["rejected"])
    tol = 1e-12 if da == 0 else 1e-10
    assert abs(value - rec["phi_ode"]) <= tol * max(1.0, abs(rec["phi_ode"]))


@pytest.mark.gpu
def test_validation_rows_of_a_z2_state(gpu_context):
    """Five rows and <phi> of the D = 8 Z2 fixture on the packed route; the oracle's energy at the
    run's controls stands in for the cached one of a checkpoint."""
    from oracle import fg_phi4_oracle as O
    from rcmps_b200 import objective, validate
    rec = load_records("packed.npz")[1]
    R, K, rho = rec["R"], rec["K"], rec["rho"]
    args = objective.default_args(window=30.0, quadrature=64, nodes=128, packed_z2=True, reduced=False,
                                  gradient_tolerance=1e-6)
    energy, grad, _ = O.fg_phi4(R, K, rho, rec["g"], n_quad=64, nodes=128, method="krylov", packed_z2=True)
    report = validate.validate_state(R, K, rho, rec["g"], args, cached_energy=energy, cached_gradient=grad)
    assert [row["name"] for row in report["evaluations"]] == [name for name, _ in validate.ROWS]
    assert report["passed"], [(r["name"], r["energy_difference_cached"], r["gradient_metric_difference_cached"])
                              for r in report["evaluations"]]
    refined = report["evaluations"][-1]
    assert refined["controls"] == dict(nodes=1024, window=40.0, quadrature=1024, atol=1e-14, rtol=1e-13)
    assert report["symmetry"] == "Z2"
    assert report["phi_ode_difference"] <= 1e-9 * max(1.0, abs(report["phi"]))
    assert report["evaluations"][1]["energy_difference_standard"] <= 1e-14 * abs(refined["energy"])
