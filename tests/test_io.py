"""The portable state format (rcmps_b200.io): the Julia fixture, round trips and refusals."""
import numpy as np
import pytest

from conftest import GOLDEN
from rcmps_b200 import io


def test_reads_the_julia_fixture():
    rec = io.read_portable(GOLDEN / "phi4_g2_D16_z2_portable")
    assert (rec.D, rec.model, rec.coupling, rec.mass, rec.origin) == (16, "phi4", 2.0, 1.0, "portable")
    assert rec.energy == -0.15648780475169466
    assert rec.integration == io.Integration(192, 20.0, 1e-13, 1e-12, 1000000)
    assert rec.manifold.metric_reg == 1e-3
    for m in (rec.R, rec.K, rec.rho, rec.gradient):
        assert m.shape == (16, 16) and m.dtype == np.complex128 and m.flags.c_contiguous
    assert np.abs(rec.K - rec.K.conj().T).max() < 1e-14
    head = io.read_portable(GOLDEN / "phi4_g2_D16_z2_portable", arrays=False)
    assert head.R is None and "R.bin" in head.files


def test_round_trip(tmp_path):
    rec = io.read_portable(GOLDEN / "phi4_g2_D16_z2_portable")
    out = io.write_portable(tmp_path / "state", rec, extra={"note": "x"}, extra_matrices={"saved_gradient": rec.gradient})
    back = io.read_portable(out)
    for name in ("R", "K", "rho", "gradient"):
        assert np.array_equal(getattr(back, name), getattr(rec, name))
    assert back.energy == rec.energy and back.integration == rec.integration and back.metadata["note"] == "x"
    with pytest.raises(FileExistsError):
        io.write_portable(tmp_path / "state", rec)


def test_refusals(tmp_path):
    rec = io.read_portable(GOLDEN / "phi4_g2_D16_z2_portable")
    bad = io.StateRecord(D=16, model="phi4", coupling=2.0, R=rec.R, K=rec.K, mass=2.0)
    with pytest.raises(ValueError, match="mass"):
        io.write_portable(tmp_path / "a", bad)
    d = io.write_portable(tmp_path / "b", io.StateRecord(D=16, model="phi4", coupling=2.0, R=rec.R, K=rec.K))
    (d / "metadata.toml").write_text((d / "metadata.toml").read_text().replace("format_version = 1", "format_version = 2"))
    with pytest.raises(ValueError, match="format_version"):
        io.read_portable(d)
    d = io.write_portable(tmp_path / "c", io.StateRecord(D=16, model="phi4", coupling=2.0, R=rec.R, K=rec.K))
    (d / "R.bin").write_bytes(b"\0" * 16)
    with pytest.raises(ValueError, match="bytes"):
        io.read_portable(d)


def test_legacy_dialect(tmp_path):
    rec = io.read_portable(GOLDEN / "phi4_g2_D16_z2_portable")
    d = tmp_path / "legacy"
    d.mkdir()
    for name in ("R", "K", "rho"):
        getattr(rec, name).ravel(order="F").astype("<c16").tofile(d / f"{name}.bin")
    rec.gradient.ravel(order="F").astype("<c16").tofile(d / "saved_gradient.bin")
    (d / "metadata.toml").write_text("D = 16\ncoupling = 2.0\nsaved_energy = -0.15\nwindow = 30.0\nquadrature = 512\n"
                                     "atol = 1e-13\nrtol = 1e-12\n")
    back = io.read_portable(d)
    assert back.origin == "portable-legacy" and back.energy == -0.15 and back.integration is None
    assert np.array_equal(back.gradient, rec.gradient)


def _record_strategy():
    from hypothesis import strategies as st

    def build(d, seed, coupling, symmetry, energy, phi, passed, text, integ, man):
        rng = np.random.default_rng(seed)
        mat = lambda: rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
        a = mat()
        return io.StateRecord(D=d, model="phi4", coupling=coupling, R=mat(), K=(a + a.conj().T) / 2,
                              rho=mat() if seed % 2 else None, gradient=mat() if seed % 3 else None,
                              energy=energy, gradient_norm=abs(energy) if energy is not None else None,
                              symmetry=symmetry, phi=phi, validation_passed=passed, producer=text, source=text,
                              info=text, integration=integ, manifold=man)

    real = st.floats(allow_nan=False, allow_infinity=False, width=64)
    pos = st.floats(min_value=1e-300, max_value=1e300)
    integ = st.none() | st.builds(io.Integration, st.integers(1, 4096), pos, pos, pos, st.none() | st.integers(1, 10**9))
    man = st.none() | st.builds(io.Manifold, st.floats(0, 1e3), st.floats(0, 1e3), st.none() | st.floats(0, 1e3))
    return st.builds(build, st.integers(1, 9), st.integers(0, 2**32 - 1), real, st.none() | st.sampled_from(io.SYMMETRIES),
                     st.none() | real, st.none() | real, st.none() | st.booleans(), st.none() | st.text(max_size=20),
                     integ, man)


def test_round_trip_property(tmp_path_factory):
    """Any record that write_portable accepts reads back bit for bit: matrices, scalars, strings
    (control characters and quotes included) and both tables."""
    from hypothesis import given, settings

    @settings(max_examples=60, deadline=None)
    @given(_record_strategy())
    def check(rec):
        out = io.write_portable(tmp_path_factory.mktemp("rt") / "s", rec)
        back = io.read_portable(out)
        for name in ("R", "K", "rho", "gradient"):
            a, b = getattr(rec, name), getattr(back, name)
            assert (a is None and b is None) or np.array_equal(a, b)
        for name in ("D", "model", "coupling", "mass", "energy", "gradient_norm", "symmetry", "phi",
                     "validation_passed", "producer", "source", "info", "integration", "manifold"):
            assert getattr(back, name) == getattr(rec, name), name
        assert back.origin == "portable"

    check()


def test_column_major_bytes(tmp_path):
    """The .bin layout is Julia's: element (i, j) at byte offset 16 (i + j D), little-endian."""
    d = 3
    R = np.arange(d * d).reshape(d, d) + 1j * np.arange(d * d).reshape(d, d) / 10
    out = io.write_portable(tmp_path / "s", io.StateRecord(D=d, model="phi4", coupling=1.0, R=R, K=np.eye(d)))
    raw = np.fromfile(out / "R.bin", dtype="<c16")
    for i in range(d):
        for j in range(d):
            assert raw[i + j * d] == R[i, j]
