"""Host-side logic of the Python layer that needs no GPU: the packed Z2 sample layout and the
quartic route chosen from the optimizer's arguments (sweep_driver.py:48-50)."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from conftest import load_records
from oracle import fg_phi4_oracle as O


def test_pack_z2_samples_inverts_the_dense_layout():
    from rcmps_b200 import objective
    rec = load_records("packed.npz")[4]
    Q = O.left_canonical_q(rec["R"], rec["K"])
    system = O.PackedZ2System(Q, rec["R"], rec["rho"])
    packed = rec["samples"]
    dense = np.stack([system.unpack(x) for x in packed])
    assert dense.shape[1] == 7 * 4 * 4 + 1
    np.testing.assert_array_equal(objective.pack_z2_samples(dense, 4), packed)


def test_route_from_optimizer_arguments():
    from rcmps_b200 import objective
    assert objective.settings_from_args(SimpleNamespace(packed_z2=True, reduced=False)).symmetry == objective.SYMMETRY_Z2
    assert objective.settings_from_args(SimpleNamespace(packed_z2=False, reduced=True)).symmetry == objective.SYMMETRY_NONE
    assert objective.settings_from_args(SimpleNamespace(window=20.0)).symmetry == objective.SYMMETRY_NONE
    with pytest.raises(ValueError):
        objective.settings_from_args(SimpleNamespace(packed_z2=True, reduced=True))
    s = objective.settings_from_args(None, symmetry=objective.SYMMETRY_AUTO)
    assert s.symmetry == 2


def test_validation_rows_and_refined_controls():
    from rcmps_b200 import validate
    assert [name for name, _ in validate.ROWS] == ["standard_cold", "standard_warm_1", "standard_warm_2",
                                                    "refined_512", "refined_1024"]
    assert validate.REFINED == dict(window=40.0, quadrature=1024, atol=1e-14, rtol=1e-13)
    with pytest.raises(ValueError):
        validate.source_integral(0.0)
