"""The allocation-free finish entry (rcmps_finish_gradient_noalloc) against the batched one.

Both are called through the C ABI on the same device inputs; the no-alloc entry is called twice
in a row (its fixed device scratch is reused, so the second call checks that nothing carries
over). It is also checked directly against the reference's own finished gradients
(tests/golden/finish.npz: numerics.finish_gradient, metric_reg 1e-3, tolerance 1e-13). This
file is collected last so that it also runs after every other entry has used the device.

Every call runs on a dedicated non-default stream, and the device is synchronized after the
inputs and outputs are created, so no fill kernel on torch's stream can land after a library
write.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

from conftest import load_records
from oracle import fg_phi4_oracle as O

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-8


def _metric_norm(rho, x):
    return math.sqrt(max(0.0, O.metric(rho, x, x)))


def _cases():
    """(name, R, K, rho, covector, environment): golden records and a d = 32 state."""
    out = []
    for i, rec in enumerate(load_records("small.npz")):
        out.append((f"small{i}_d{len(rec['R'])}", rec["R"], rec["K"], rec["rho"],
                    rec["quartic_covector"] + rec["kinetic_covector"],
                    rec["quartic_environment"] + rec["kinetic_environment"]))
    rec = load_records("d16.npz")[0]
    out.append(("d16", rec["R"], rec["K"], rec["rho"], rec["quartic_covector"] + rec["kinetic_covector"],
                rec["quartic_environment"] + rec["kinetic_environment"]))
    rng = np.random.default_rng(32)
    d = 32
    R = 0.2 * (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / math.sqrt(2.0)
    A = 0.2 * (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / math.sqrt(2.0)
    K = (A + A.conj().T) / 2
    rho = O.stationary_state(O.left_canonical_q(R, K), R)
    cov = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    env = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    out.append(("d32", R, K, rho, cov, 0.5 * (env + env.conj().T)))
    return out


def _dev(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.complex128).ravel()).to("cuda")


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_noalloc_matches_batched_twice(gpu_context, case):
    import torch
    from rcmps_b200 import _lib
    _, R, K, rho, cov, env = case
    d = len(R)
    ctx = gpu_context
    lib = ctx.lib
    # the no-alloc entry's boundary solve is unpreconditioned: the batched entry takes the same
    s = _lib.default_settings(metric_reg=1e-3, boundary_tolerance=1e-13, boundary_preconditioner=0)
    dR, dK, dP, dC, dE = (_dev(torch, x) for x in (R, K, rho, cov, env))
    side = torch.cuda.Stream()
    stream = C.c_void_p(side.cuda_stream)

    ref = torch.zeros(d * d, dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    st_ref = (_lib.StateStats * 1)()
    rc = lib.rcmps_finish_gradient_batch(ctx.handle, 1, (C.c_int * 1)(d), dR.data_ptr(), dK.data_ptr(),
                                         dP.data_ptr(), dC.data_ptr(), dE.data_ptr(), C.byref(s), ref.data_ptr(),
                                         st_ref, stream)
    assert rc == 0, ctx.error()
    ref_h = ref.cpu().numpy().reshape(d, d)
    scale = max(1.0, _metric_norm(rho, ref_h))
    for call in range(2):
        got = torch.full((d * d,), float("nan"), dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        st = _lib.StateStats()
        rc = lib.rcmps_finish_gradient_noalloc(ctx.handle, d, dR.data_ptr(), dK.data_ptr(), dP.data_ptr(),
                                               dC.data_ptr(), dE.data_ptr(), C.byref(s), got.data_ptr(),
                                               C.byref(st), stream)
        assert rc == 0 and st.status == 0, (call, rc, ctx.error())
        got_h = got.cpu().numpy().reshape(d, d)
        assert _metric_norm(rho, got_h - ref_h) <= GRAD_TOL * scale, call
        assert st.gmres_iterations == st_ref[0].gmres_iterations
        assert abs(st.boundary_residual - st_ref[0].boundary_residual) <= 1e-3 * st_ref[0].boundary_residual + 1e-300


@pytest.mark.parametrize("index", range(3))
def test_noalloc_matches_reference_finish(gpu_context, index):
    """The reference's finished gradient (numerics.finish_gradient: the no-jump preconditioned
    boundary GMRES and the metric solve) on random states D = 8, 16 and a Z2 state D = 16, twice
    in a row."""
    import torch
    from rcmps_b200 import _lib
    rec = load_records("finish.npz")[index]
    R, K, rho = rec["R"], rec["K"], rec["rho"]
    d = len(R)
    ctx = gpu_context
    s = _lib.default_settings(metric_reg=1e-3, boundary_tolerance=1e-13)
    dR, dK, dP, dC, dE = (_dev(torch, x) for x in (R, K, rho, rec["covector"], rec["environment"]))
    side = torch.cuda.Stream()
    scale = max(1.0, _metric_norm(rho, rec["gradient"]))
    for call in range(2):
        got = torch.full((d * d,), float("nan"), dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        st = _lib.StateStats()
        rc = ctx.lib.rcmps_finish_gradient_noalloc(ctx.handle, d, dR.data_ptr(), dK.data_ptr(), dP.data_ptr(),
                                                   dC.data_ptr(), dE.data_ptr(), C.byref(s), got.data_ptr(),
                                                   C.byref(st), C.c_void_p(side.cuda_stream))
        assert rc == 0 and st.status == 0, (call, rc, ctx.error())
        got_h = got.cpu().numpy().reshape(d, d)
        assert _metric_norm(rho, got_h - rec["gradient"]) <= GRAD_TOL * scale, call


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu_context):
    import torch
    from rcmps_b200 import _lib
    ctx = gpu_context
    s = _lib.default_settings()
    d = 33
    buf = torch.zeros(d * d, dtype=torch.complex128, device="cuda")
    st = _lib.StateStats()
    p = buf.data_ptr()
    rc = ctx.lib.rcmps_finish_gradient_noalloc(ctx.handle, d, p, p, p, p, p, C.byref(s), p, C.byref(st), None)
    assert rc == 20   # RCMPS_INVALID_ARGUMENT
    assert "d <= 32" in ctx.error() and "2 MiB" in ctx.error()
