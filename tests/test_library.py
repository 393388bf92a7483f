"""The C ABI: the in-tree library loads and exports every entry point declared in
include/rcmps_b200.h, with the structure layouts of the header. No GPU work is done."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT
from rcmps_b200 import _lib

HEADER = ROOT / "include" / "rcmps_b200.h"


def declared():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(rcmps_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = _lib.library()
    names = declared()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), f"{name} is declared in the header but not exported"
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"
    assert _lib.MISSING == []


def test_status_names_and_defaults():
    lib = _lib.library()
    assert lib.rcmps_status_name(0) == b"success"
    assert lib.rcmps_status_name(6) == b"device_clock_timeout"
    s = _lib.default_settings()
    assert (s.half_window, s.n_quad, s.atol, s.rtol, s.kinetic_nodes) == (30.0, 512, 1e-13, 1e-12, 512)
    assert (s.krylov_tolerance, s.krylov_maxdim, s.metric_reg) == (1e-12, 1024, 1e-3)


def test_structure_layouts_match_the_header(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text(f'#include "{HEADER}"\n#include <stdio.h>\n#include <stddef.h>\n'
                   "int main(void){printf(\"%zu %zu %zu %zu\\n\", sizeof(rcmps_settings), sizeof(rcmps_state_stats),"
                   " offsetof(rcmps_state_stats, krylov_basis), offsetof(rcmps_state_stats, boundary_residual));"
                   "return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    sizes = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()))
    assert sizes == [C.sizeof(_lib.Settings), C.sizeof(_lib.StateStats),
                     _lib.StateStats.krylov_basis.offset, _lib.StateStats.boundary_residual.offset]


def test_no_host_fallback_without_a_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from rcmps_b200 import objective
    import numpy as np
    with pytest.raises(RuntimeError, match="CUDA"):
        objective.fg_phi4_batch([np.eye(2, dtype=complex)], [np.zeros((2, 2), complex)],
                                [np.eye(2, dtype=complex) / 2], [1.0])
