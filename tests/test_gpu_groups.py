"""Channel groups of the FP64 trajectory kernel (rcmps_settings.trajectory_groups): a state's
rows AND channels split over dp/16 x {1, 2, 4} CTAs of one cluster. Every layout integrates the
same equations with the same products; only the summation order of the error norm and of the
scalar channel changes, so results agree to rounding and the DOP853 step counts are equal.

Tolerances: |dE/E| <= 1e-13 and gradient <= 1e-11 relative in the metric norm between layouts;
the automatic layout spreads a lone D = 64 state over 2 or 4 groups and keeps one CTA per row
block for the 32-state workload."""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import load_records
from oracle import fg_phi4_oracle as O

pytestmark = pytest.mark.gpu


def _metric_norm(rho, x):
    return math.sqrt(max(0.0, O.metric(rho, x, x)))


def _groups(ctx, dp):
    g = C.c_int(0)
    assert ctx.lib.rcmps_trajectory_groups(ctx.handle, 0, dp, C.byref(g)) == 0
    return g.value


@pytest.mark.parametrize("d", [16, 40, 64, 96])
def test_layouts_agree(gpu_context, d):
    from rcmps_b200 import objective
    from rcmps_b200.batch import random_state
    R, K = random_state(d, 300 + d)
    rho, _ = objective.stationary_state(O.left_canonical_q(R, K), R, tolerance=1e-13)
    out = {}
    for groups in (1, 2, 4):
        s = objective.settings_from_args(None, half_window=6.0, n_quad=48, kinetic_nodes=64,
                                         symmetry=objective.SYMMETRY_NONE, trajectory_groups=groups)
        E, G, st = objective.fg_phi4_batch([R], [K], [rho], [1.5], s)
        assert st[0]["status"] == 0
        dp = ((d + 15) // 16) * 16 if d <= 64 else (96 if d <= 96 else 128)
        taken = _groups(gpu_context, dp)
        assert taken == (groups if dp // 16 * groups <= 16 else 2)
        out[groups] = (E[0], G[0], st[0]["accepted"], st[0]["rejected"])
    e1, g1, a1, r1 = out[1]
    for groups in (2, 4):
        e, g, a, r = out[groups]
        assert (a, r) == (a1, r1)
        assert abs(e - e1) <= 1e-13 * abs(e1)
        assert _metric_norm(rho, g - g1) <= 1e-11 * max(1.0, _metric_norm(rho, g1))


def test_packed_z2_state_in_groups(gpu_context):
    """The packed Z2 route (structural zeros skipped) in four groups against one."""
    from rcmps_b200 import objective
    rec = load_records("bench.npz")[2]
    res = []
    for groups in (1, 4):
        s = objective.settings_from_args(None, half_window=6.0, n_quad=48, kinetic_nodes=64,
                                         symmetry=objective.SYMMETRY_Z2, trajectory_groups=groups)
        E, G, st = objective.fg_phi4_batch([rec["R"]], [rec["K"]], [rec["rho"]], [rec["g"]], s)
        assert st[0]["packed_z2"] == 1 and st[0]["status"] == 0
        res.append((E[0], G[0], st[0]["accepted"], st[0]["rejected"]))
    assert res[0][2:] == res[1][2:]
    assert abs(res[0][0] - res[1][0]) <= 1e-13 * abs(res[0][0])
    assert _metric_norm(rec["rho"], res[0][1] - res[1][1]) <= 1e-11 * max(1.0, _metric_norm(rec["rho"], res[0][1]))


def test_automatic_layout(gpu_context):
    """A lone D = 64 state spreads over more than one group; 32 states keep one CTA per row block."""
    from rcmps_b200 import objective
    from rcmps_b200.batch import random_state
    R, K = random_state(64, 5)
    rho, _ = objective.stationary_state(O.left_canonical_q(R, K), R, tolerance=1e-13)
    s = objective.settings_from_args(None, half_window=2.0, n_quad=16, kinetic_nodes=32,
                                     symmetry=objective.SYMMETRY_NONE)
    objective.fg_phi4_batch([R], [K], [rho], [2.0], s)
    assert _groups(gpu_context, 64) in (2, 4)
    objective.fg_phi4_batch([R] * 32, [K] * 32, [rho] * 32, [2.0] * 32, s)
    assert _groups(gpu_context, 64) == 1
    with pytest.raises(ValueError):
        objective.fg_phi4_batch([R], [K], [rho], [2.0],
                                objective.settings_from_args(None, trajectory_groups=3))
