"""ctypes binding of librcmps_b200.so (include/rcmps_b200.h).

The library is built in-tree (rcmpscore.jl_b200/Makefile). Loading fails loudly when it is
missing: there is no host fallback for any computation of the fg_phi4 path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIBRARY_PATH = _HERE / "librcmps_b200.so"

STATUS_NAMES = {
    0: "success", 1: "max_steps", 2: "step_underflow", 3: "nonfinite_error", 4: "source_domain",
    5: "missing_samples", 6: "device_clock_timeout", 7: "wait_limit", 8: "krylov_failure",
    9: "solve_failure", 10: "nonfinite_result", 20: "invalid_argument", 21: "cuda_error",
    22: "out_of_memory",
}
COMPONENTS = {0: None, 1: "trajectory", 2: "pullback", 3: "kinetic", 4: "boundary", 5: "stationary"}


class Settings(C.Structure):
    _fields_ = [
        ("half_window", C.c_double), ("n_quad", C.c_int), ("atol", C.c_double), ("rtol", C.c_double),
        ("initial_step", C.c_double), ("max_steps", C.c_longlong), ("max_device_seconds", C.c_double),
        ("kinetic_nodes", C.c_int), ("krylov_tolerance", C.c_double), ("krylov_initialdim", C.c_int),
        ("krylov_maxdim", C.c_int), ("metric_reg", C.c_double), ("boundary_tolerance", C.c_double),
        ("symmetry", C.c_int), ("precision", C.c_int), ("trajectory_groups", C.c_int),
        ("boundary_preconditioner", C.c_int),
    ]


class StateControls(C.Structure):
    """Per-state DOP853 tolerances (rcmps_state_controls); a value <= 0 takes the settings'."""
    _fields_ = [("atol", C.c_double), ("rtol", C.c_double)]


class GmresNetwork(C.Structure):
    """A learned right preconditioner of the boundary GMRES (rcmps_gmres_network)."""
    _fields_ = [("W1", C.c_void_p), ("W2", C.c_void_p), ("n", C.c_int), ("rank", C.c_int), ("identity", C.c_float)]


class StateStats(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("failed_component", C.c_int),
        ("attempts", C.c_longlong), ("accepted", C.c_longlong), ("rejected", C.c_longlong),
        ("dense_steps", C.c_longlong), ("rhs_calls", C.c_longlong),
        ("t_end", C.c_double), ("last_step", C.c_double), ("min_step", C.c_double), ("max_step", C.c_double),
        ("quartic_value", C.c_double), ("kinetic_value", C.c_double),
        ("krylov_basis", C.c_int * 4), ("krylov_residual", C.c_double),
        ("gmres_iterations", C.c_int), ("boundary_residual", C.c_double), ("packed_z2", C.c_int),
        ("gmres_matvecs", C.c_int),
    ]

    def as_dict(self):
        out = {name: getattr(self, name) for name, _ in self._fields_}
        out["krylov_basis"] = list(self.krylov_basis)
        out["status_name"] = STATUS_NAMES.get(self.status, "unknown")
        out["failed_component"] = COMPONENTS.get(self.failed_component)
        return out


# Exported symbols and their signatures (checked by tests/test_library.py against the header).
_P = C.c_void_p
_I = C.c_int
_D = C.c_double
SIGNATURES = {
    "rcmps_default_settings": (None, [C.POINTER(Settings)]),
    "rcmps_context_create": (_I, [_I, C.POINTER(_P)]),
    "rcmps_context_destroy": (_I, [_P]),
    "rcmps_context_error": (C.c_char_p, [_P]),
    "rcmps_status_name": (C.c_char_p, [_I]),
    "rcmps_last_timings": (_I, [_P, C.POINTER(C.c_float), _I]),
    "rcmps_workspace_bytes": (C.c_longlong, [_P, _I, C.POINTER(_I), C.POINTER(Settings)]),
    "rcmps_fg_phi4_batch": (_I, [_P, _I, C.POINTER(_I), C.POINTER(_D), _P, _P, _P, C.POINTER(Settings),
                                 _P, _P, _P, _P, C.POINTER(StateStats), _P]),
    "rcmps_fg_phi4_batch_controls": (_I, [_P, _I, C.POINTER(_I), C.POINTER(_D), _P, _P, _P, C.POINTER(Settings),
                                          C.POINTER(StateControls), _P, _P, _P, _P, C.POINTER(StateStats), _P]),
    "rcmps_fg_phi4_batch_host": (_I, [_P, _I, C.POINTER(_I), C.POINTER(_D), _P, _P, _P, C.POINTER(Settings),
                                      _P, _P, _P, _P, C.POINTER(StateStats)]),
    "rcmps_quartic_batch": (_I, [_P, _I, C.POINTER(_I), C.POINTER(_D), _P, _P, _P, C.POINTER(Settings),
                                 _P, _P, _P, C.POINTER(StateStats), _P]),
    "rcmps_phi4_ode_batch": (_I, [_P, _I, C.POINTER(_I), C.POINTER(_D), _P, _P, _P, C.POINTER(Settings),
                                  _P, _P, _P, C.POINTER(StateStats), _P]),
    "rcmps_phi_ode_batch": (_I, [_P, _I, C.POINTER(_I), _P, _P, _P, C.POINTER(Settings), _P,
                                 C.POINTER(StateStats), _P]),
    "rcmps_quartic_samples": (_I, [_P, _I, _P, _P, _P, C.POINTER(Settings), _P, C.POINTER(StateStats), _P]),
    "rcmps_kinetic_batch": (_I, [_P, _I, C.POINTER(_I), _P, _P, _P, C.POINTER(Settings), _P, _P, _P,
                                 C.POINTER(StateStats), _P]),
    "rcmps_finish_gradient_batch": (_I, [_P, _I, C.POINTER(_I), _P, _P, _P, _P, _P, C.POINTER(Settings), _P,
                                         C.POINTER(StateStats), _P]),
    "rcmps_boundary_environment_batch": (_I, [_P, _I, C.POINTER(_I), _P, _P, _P, _P, _P, C.POINTER(GmresNetwork),
                                              C.POINTER(Settings), _P, C.POINTER(StateStats), _P]),
    "rcmps_finish_gradient_noalloc": (_I, [_P, _I, _P, _P, _P, _P, _P, C.POINTER(Settings), _P,
                                           C.POINTER(StateStats), _P]),
    "rcmps_stationary_state_batch": (_I, [_P, _I, C.POINTER(_I), _P, _P, _D, _P, C.POINTER(StateStats), _P]),
    "rcmps_stationary_correction_batch": (_I, [_P, _I, C.POINTER(_I), _P, _P, _P, _D, _P, C.POINTER(StateStats),
                                               _P]),
    "rcmps_split_product_batch": (_I, [_P, _I, _I, _P, _P, _P, _P]),
    "rcmps_warmstart_forward": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P]),
    "rcmps_warmstart_backward": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "rcmps_warmstart_adam": (_I, [_P, C.c_longlong, _P, _P, _P, _P, C.c_float, C.c_float, C.c_float, C.c_float, _I,
                                  _P]),
    "rcmps_lbfgs_direction": (_I, [_P, _I, _I, _P, _P, _P, _P, _P, _D, _D, _D, _P, _P, _P, _P]),
    "rcmps_retract": (_I, [_P, _I, _P, _P, _P, _D, _P, _P, _P]),
    "rcmps_trajectory_tuning": (_I, [_P, _I, _I, C.POINTER(_I), C.POINTER(C.c_float)]),
    "rcmps_trajectory_groups": (_I, [_P, _I, _I, C.POINTER(_I)]),
    "rcmps_fp64_peak_tflops": (_D, [_P]),
    "rcmps_launch_count": (C.c_longlong, []),
}

_lib = None
MISSING = []   # exported symbols of SIGNATURES absent from the loaded library


def library():
    """Load librcmps_b200.so (once). Raises if it is missing or incomplete."""
    global _lib
    if _lib is None:
        if not LIBRARY_PATH.exists():
            raise RuntimeError(f"{LIBRARY_PATH} is missing: build it with `make -C rcmpscore.jl_b200` "
                               "(or __graft_entry__.build()); there is no host fallback")
        lib = C.CDLL(os.fspath(LIBRARY_PATH))
        for name, (restype, argtypes) in SIGNATURES.items():
            try:
                fn = getattr(lib, name)
            except AttributeError:
                MISSING.append(name)
                continue
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


def default_settings(**overrides):
    s = Settings()
    library().rcmps_default_settings(C.byref(s))
    for key, value in overrides.items():
        if not hasattr(s, key):
            raise KeyError(f"unknown setting {key}")
        setattr(s, key, value)
    return s


class Context:
    """One library context on a CUDA device (streams, events, device workspace)."""

    def __init__(self, device=0):
        self.lib = library()
        handle = C.c_void_p()
        rc = self.lib.rcmps_context_create(int(device), C.byref(handle))
        if rc != 0:
            raise RuntimeError(f"rcmps_context_create failed: {STATUS_NAMES.get(rc, rc)}")
        self.handle = handle
        self.device = int(device)

    def error(self):
        return (self.lib.rcmps_context_error(self.handle) or b"").decode()

    def timings(self):
        buf = (C.c_float * 8)()
        self.lib.rcmps_last_timings(self.handle, buf, 8)
        return list(buf)

    def close(self):
        if self.handle:
            self.lib.rcmps_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
