"""The split-precision tensor-core engine (tcgen05, BF16 slices, FP32 accumulation in TMEM)
against FP64 products and against a NumPy restatement of the same slicing.

The engine cuts every row of A and every column of B, scaled by a power of two, into seven 7-bit
slices (nearest-integer remainders), keeps the slice pairs i + l <= 6 and recombines the group
sums in FP64. Its error per element is about 2^-50 s_m t_n per term of the K-sum (s_m, t_n the
row and column scales), unbiased; the restatement (exact group sums in FP64) agrees with it to
the FP64 rounding of the result (the groups s <= 4 are exact, and the FP32 rounding of the
shared accumulator of the groups s >= 5 stays far below), within 2^-48 of the scales.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def pow2_above(x):
    m, e = np.frexp(x)
    return np.where(x > 0, np.ldexp(1.0, e), 1.0)


def split_reference(A, B, slices=7, bits=7):
    """C = A B by the engine's slicing, with every group sum exact."""
    sa = pow2_above(np.maximum(np.abs(A.real), np.abs(A.imag)).max(axis=1))
    sb = pow2_above(np.maximum(np.abs(B.real), np.abs(B.imag)).max(axis=0))

    def cut(v):
        out, r = [], v.copy()
        for i in range(slices):
            r = r * 2.0 ** bits
            t = np.rint(r)
            r = r - t
            out.append(t * 2.0 ** (-bits * i))
        return out
    An, Bn = A / sa[:, None], B / sb[None, :]
    ar, ai, br, bi = cut(An.real), cut(An.imag), cut(Bn.real), cut(Bn.imag)
    total = np.zeros((A.shape[0], B.shape[1]), complex)
    for s in range(slices):
        for i in range(s + 1):
            l = s - i
            total += (ar[i] @ br[l] - ai[i] @ bi[l]) + 1j * (ar[i] @ bi[l] + ai[i] @ br[l])
    return total * 2.0 ** -14 * sa[:, None] * sb[None, :], sa, sb


def _run(ctx, A, B):
    import torch
    n, d = A.shape[0], A.shape[1]
    dA = torch.from_numpy(np.ascontiguousarray(A).ravel()).to("cuda")
    dB = torch.from_numpy(np.ascontiguousarray(B).ravel()).to("cuda")
    dC = torch.full((n * d * d,), float("nan"), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    rc = ctx.lib.rcmps_split_product_batch(ctx.handle, n, d, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), None)
    assert rc == 0, ctx.error()
    return dC.cpu().numpy().reshape(n, d, d)


@pytest.mark.parametrize("d", [64, 40, 7])
def test_split_products_match_fp64(gpu_context, d):
    rng = np.random.default_rng(100 + d)
    n = 6
    A = rng.standard_normal((n, d, d)) + 1j * rng.standard_normal((n, d, d))
    B = rng.standard_normal((n, d, d)) + 1j * rng.standard_normal((n, d, d))
    # rows and columns spanning many orders of magnitude, and one all-zero row and column
    A *= 10.0 ** rng.uniform(-8, 2, (n, d, 1))
    B *= 10.0 ** rng.uniform(-8, 2, (n, 1, d))
    A[:, 0, :] = 0.0
    B[:, :, -1] = 0.0
    got = _run(gpu_context, A, B)
    for b in range(n):
        ref = A[b] @ B[b]
        emu, sa, sb = split_reference(A[b], B[b])
        scale = sa[:, None] * sb[None, :]
        err = np.abs(got[b] - ref) / scale
        assert err.max() <= 2.0 ** -40, err.max()
        assert np.sqrt(np.mean(err ** 2)) <= 2.0 ** -44
        assert (np.abs(got[b] - emu) / scale).max() <= 2.0 ** -48
        assert np.all(got[b][0, :] == 0) and np.all(got[b][:, -1] == 0)


def test_split_product_rejects_sizes(gpu_context):
    ctx = gpu_context
    rc = ctx.lib.rcmps_split_product_batch(ctx.handle, 1, 65, None, None, None, None)
    assert rc == 20 and "d <= 64" in ctx.error()


# ----------------------------------------------------------------------------- the trajectory
ENERGY_TOL = 1e-10
GRAD_TOL = 1e-8


def _metric_norm(rho, x):
    from oracle import fg_phi4_oracle as O
    return float(np.sqrt(max(0.0, O.metric(rho, x, x))))


def test_split_fg_phi4_bench_states_match_reference(gpu_context):
    """Energy and finished gradient of four states of the 32-state D = 64 benchmark workload
    (random seeds 0, 1 unpacked; Z2 seeds 100, 101 on the packed route) with the split-precision
    trajectory products, against the reference's FP64 NumPy path (bench.npz): |dE/E| <= 1e-10
    and gradient <= 1e-8 in the metric norm. The step counts may differ from the FP64 ones by
    the products' rounding (about 2^-43 of the scales)."""
    from conftest import load_records
    from rcmps_b200 import objective
    recs = load_records("bench.npz")
    s = objective.settings_from_args(None, symmetry=objective.SYMMETRY_AUTO, precision=1)
    E, G, stats = objective.fg_phi4_batch([r["R"] for r in recs], [r["K"] for r in recs], [r["rho"] for r in recs],
                                          [r["g"] for r in recs], s)
    for i, rec in enumerate(recs):
        assert stats[i]["status"] == 0, stats[i]
        assert abs(E[i] - rec["energy"]) <= ENERGY_TOL * abs(rec["energy"]), (i, E[i], rec["energy"])
        scale = max(1.0, _metric_norm(rec["rho"], rec["gradient"]))
        assert _metric_norm(rec["rho"], G[i] - rec["gradient"]) <= GRAD_TOL * scale, i
        assert abs(stats[i]["accepted"] - rec["accepted"]) <= 0.05 * rec["accepted"]


def test_split_quartic_d64_against_fp64(gpu_context):
    """The quartic term of the seed-42 D = 64 state (d64.npz, the reference's own values) with
    both engines: the split value within 1e-11 relative of the reference's, covector and
    environment within 1e-9 of their largest entries."""
    from conftest import load_records
    from oracle import fg_phi4_oracle as O
    from rcmps_b200 import _lib, objective
    rec = load_records("d64.npz")[0]
    R, K, rho, g = rec["R"], rec["K"], rec["rho"], rec["g"]
    Q = O.left_canonical_q(R, K)
    out = objective.evaluate_quartic_persistent_trajectory(R, Q, rho, g, unpacked=True, precision=1)
    assert out["stats"]["status"] == 0
    assert abs(out["value"] - rec["quartic_value"]) <= 1e-11 * abs(rec["quartic_value"])
    for key in ("covector", "environment"):
        ref = rec[f"quartic_{key}"]
        assert np.abs(out[key] - ref).max() <= 1e-9 * np.abs(ref).max(), key
