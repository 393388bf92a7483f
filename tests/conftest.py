"""Shared test set-up: the package path, the gpu marker and fixtures of the golden vectors."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "rcmpscore.jl_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def load_records(name):
    """Records of a golden .npz written by tests/golden/make_golden.py."""
    data = np.load(GOLDEN / name)
    out = []
    for i in range(int(data["count"])):
        prefix = f"s{i}_"
        out.append({k[len(prefix):]: (data[k].item() if data[k].ndim == 0 else data[k])
                    for k in data.files if k.startswith(prefix)})
    return out


def julia_fixture():
    """The Julia-exported D = 16 Z2 state (R, K, rho, gradient, metadata)."""
    import tomllib
    d = GOLDEN / "phi4_g2_D16_z2_portable"
    meta = tomllib.load(open(d / "metadata.toml", "rb"))
    n = meta["D"]
    read = lambda name: np.fromfile(d / f"{name}.bin", dtype="<c16").reshape(n, n, order="F")
    return dict(R=read("R"), K=read("K"), rho=read("rho"), gradient=read("gradient"), meta=meta)


@pytest.fixture(scope="session")
def gpu_context():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rcmps_b200 import objective
    return objective.context(0)
