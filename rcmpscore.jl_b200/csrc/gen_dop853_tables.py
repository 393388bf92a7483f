"""Generate csrc/dop853_tables.h from SciPy's DOP853 tables (scipy.integrate._ivp.dop853_coefficients,
BSD-3; Hairer, Norsett and Wanner's DOP853 with its order-7 dense output). The reference integrator
reads the same tables at run time (gpu/src/rcmps_gpu/optimizer/runtime/ode_backend.py:23).
Run: python gen_dop853_tables.py > dop853_tables.h
"""
import numpy as np
from scipy.integrate._ivp import dop853_coefficients as dop


def emit(name, values):
    flat = np.asarray(values, dtype=np.float64).ravel()
    print(f"static const double {name}[{flat.size}] = {{")
    for i in range(0, flat.size, 4):
        print("  " + ", ".join(repr(float(x)) for x in flat[i:i + 4]) + ",")
    print("};")


print("// Generated by gen_dop853_tables.py from scipy.integrate._ivp.dop853_coefficients; do not edit.")
print("#pragma once")
print(f"#define RCMPS_DOP_STAGES {dop.N_STAGES}")
print(f"#define RCMPS_DOP_STAGES_EXTENDED {dop.N_STAGES_EXTENDED}")
a = np.zeros((16, 16)); a[:dop.A.shape[0], :dop.A.shape[1]] = dop.A
b = np.zeros(16); b[:dop.B.size] = dop.B
e5 = np.zeros(16); e5[:dop.E5.size] = dop.E5
e3 = np.zeros(16); e3[:dop.E3.size] = dop.E3
dd = np.zeros((4, 16)); dd[:, :dop.D.shape[1]] = dop.D
emit("rcmps_dop_a", a)
emit("rcmps_dop_b", b)
emit("rcmps_dop_c", dop.C)
emit("rcmps_dop_e5", e5)
emit("rcmps_dop_e3", e3)
emit("rcmps_dop_d", dd)
# Stages the order-7 interpolation reads: k0 and k12 and every column of the dense matrix D with
# a nonzero entry.
dense = (1 << 0) | (1 << 12) | sum(1 << j for j in range(16) if np.any(dd[:, j] != 0.0))
print(f"constexpr unsigned rcmps_dop_dense_mask = 0x{dense:04x}u;")
