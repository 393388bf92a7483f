"""Parity of the benchmark-shaped workloads, each in ONE batched launch, against golden vectors
that the reference's own NumPy path wrote (tests/golden/make_golden.py):

  * the 64-state D = 32 batch (random seeds 0..63, g ~ U[0.5, 3]): states 0..7 against
    d32batch.npz, every state's status;
  * four states of the 32-state D = 64 benchmark workload (random seeds 0, 1 on the unpacked
    route; Z2 seeds 100, 101 on the packed route with the reference's own stationary density)
    against bench.npz;
  * the first 20 states of the uneven workload (D in {16 .. 128}, per-state atol/rtol pairs in
    one launch through rcmps_fg_phi4_batch_controls): the pinned states against uneven.npz, and
    every state against its own single-state evaluation at its own tolerances.

Tolerances: DOP853 accepted/rejected step counts exactly; energy |dE/E| <= 1e-10; gradient
<= 1e-8 relative in the metric norm with max(|g|, 1) as the scale.
"""
import math

import numpy as np
import pytest

from conftest import load_records
from oracle import fg_phi4_oracle as O

pytestmark = pytest.mark.gpu

ENERGY_TOL = 1e-10
GRAD_TOL = 1e-8


def metric_norm(rho, x):
    return math.sqrt(max(0.0, O.metric(rho, x, x)))


def check_record(rec, energy, grad, st):
    assert st["status"] == 0, st
    assert (st["accepted"], st["rejected"]) == (int(rec["accepted"]), int(rec["rejected"]))
    assert abs(energy - rec["energy"]) <= ENERGY_TOL * abs(rec["energy"])
    assert metric_norm(rec["rho"], grad - rec["gradient"]) <= GRAD_TOL * max(1.0, metric_norm(rec["rho"], rec["gradient"]))


def _rho_batch(R, K):
    from rcmps_b200 import objective
    return [objective.stationary_state(O.left_canonical_q(r, k), r, tolerance=1e-13)[0] for r, k in zip(R, K)]


def test_d32_batch_of_64_in_one_launch(gpu_context):
    from rcmps_b200 import objective
    from rcmps_b200.batch import config_states
    R, K, g, _ = config_states("d32_batch")
    golden = load_records("d32batch.npz")
    rho = [rec["rho"] for rec in golden] + _rho_batch(R[len(golden):], K[len(golden):])
    s = objective.settings_from_args(None, symmetry=objective.SYMMETRY_NONE)
    E, G, stats = objective.fg_phi4_batch(R, K, rho, g, s)
    assert all(st["status"] == 0 for st in stats)
    assert all(np.isfinite(E)) and all(np.isfinite(x).all() for x in G)
    for i, rec in enumerate(golden):
        assert abs(g[i] - rec["g"]) == 0.0
        check_record(rec, E[i], G[i], stats[i])


def test_bench_states_match_reference(gpu_context):
    """Random seeds 0, 1 (unpacked) and Z2 seeds 100, 101 (packed, the reference's density) in
    one launch with the route chosen per state (symmetry 2), as the benchmark runs them."""
    from rcmps_b200 import objective
    recs = load_records("bench.npz")
    s = objective.settings_from_args(None, symmetry=objective.SYMMETRY_AUTO)
    E, G, stats = objective.fg_phi4_batch([r["R"] for r in recs], [r["K"] for r in recs], [r["rho"] for r in recs],
                                          [r["g"] for r in recs], s)
    assert [st["packed_z2"] for st in stats] == [0, 0, 1, 1]
    for i, rec in enumerate(recs):
        check_record(rec, E[i], G[i], stats[i])


def test_uneven_batch_with_per_state_tolerances(gpu_context):
    from rcmps_b200 import objective
    from rcmps_b200.batch import uneven_states
    R, K, g, tol = uneven_states(20)
    pinned = {int(rec["index"]): rec for rec in load_records("uneven.npz")}
    rho = [pinned[i]["rho"] if i in pinned else None for i in range(20)]
    rest = [i for i in range(20) if rho[i] is None]
    for i, p in zip(rest, _rho_batch([R[i] for i in rest], [K[i] for i in rest])):
        rho[i] = p
    s = objective.settings_from_args(None, symmetry=objective.SYMMETRY_NONE)
    E, G, stats = objective.fg_phi4_batch(R, K, rho, g, s, tolerances=tol)
    for i, rec in pinned.items():
        assert (rec["atol"], rec["rtol"]) == tol[i]
        check_record(rec, E[i], G[i], stats[i])
    # every state of the mixed launch equals its own evaluation at its own tolerance pair
    for i in range(20):
        one = objective.settings_from_args(None, symmetry=objective.SYMMETRY_NONE, atol=tol[i][0], rtol=tol[i][1])
        e1, g1, st1 = objective.fg_phi4_batch([R[i]], [K[i]], [rho[i]], [g[i]], one)
        assert (st1[0]["accepted"], st1[0]["rejected"]) == (stats[i]["accepted"], stats[i]["rejected"])
        assert abs(e1[0] - E[i]) <= 1e-13 * abs(E[i])
        assert metric_norm(rho[i], g1[0] - G[i]) <= 1e-10 * max(1.0, metric_norm(rho[i], G[i]))


def test_controls_are_checked(gpu_context):
    from rcmps_b200 import objective
    rec = load_records("small.npz")[0]
    with pytest.raises(ValueError, match="controls"):
        objective.fg_phi4_batch([rec["R"]], [rec["K"]], [rec["rho"]], [1.0],
                                objective.settings_from_args(None, n_quad=32, kinetic_nodes=64),
                                tolerances=[(1e-12, 1e-17)])


def test_trajectory_tile_autotuner_records_its_choice(gpu_context):
    """The first three D = 64 evaluations of a layout take the ring depths 4, 2, 3 (results are
    identical) and record their device time per 1000 right-hand sides; the context then holds the
    chosen depth: the default 4 unless another was faster by more than 2%."""
    import ctypes as C
    from rcmps_b200 import objective
    rec = load_records("bench.npz")[0]
    s = objective.settings_from_args(None, half_window=2.0, n_quad=16, kinetic_nodes=32, trajectory_groups=1)
    results = [objective.fg_phi4_batch([rec["R"]], [rec["K"]], [rec["rho"]], [rec["g"]], s) for _ in range(3)]
    for E, G, _ in results[1:]:
        assert E[0] == results[0][0][0] and np.array_equal(G[0], results[0][1][0])
    ctx = gpu_context
    ring, ms = C.c_int(0), (C.c_float * 3)()
    assert ctx.lib.rcmps_trajectory_tuning(ctx.handle, 0, 64, C.byref(ring), ms) == 0
    ms = list(ms)
    assert ring.value in (2, 3, 4) and all(x > 0 for x in ms)
    if ring.value == 4:
        assert min(ms[:2]) >= 0.98 * ms[2]
    else:
        assert ms[ring.value - 2] == min(ms) and ms[ring.value - 2] < 0.98 * ms[2]
