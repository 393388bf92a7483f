"""State files shared with RcmpsCore.jl: the portable directory format and JLD2 checkpoints.

Same API and semantics as rcmps_gpu.io (gpu/src/rcmps_gpu/io.py:94-471 of RcmpsCore.jl):
StateRecord, Integration, Manifold, read_portable, write_portable, read_jld2.

Portable state directory, "rcmps-portable-state" format 1:
    metadata.toml   format, format_version = 1, D, model, coupling (required); mass, symmetry
                    ("Z2" | "none"), energy, gradient_norm, phi, validation_passed, producer,
                    source, info (optional); [integration] n_quad, max_point, atol, rtol,
                    maxiters; [manifold] metric_reg, precond_reg, precond_reg_prefactor
    R.bin, K.bin    required; rho.bin, gradient.bin optional
Every .bin is a headerless D x D complex128 matrix, little-endian, column-major (16 D^2 bytes).
Readers ignore unknown keys and files. Research directories without `format` (the GPU
optimizer's initial/ and optimized_state/, the Julia exports) are read too: they describe phi4
with mass 1; energy, gradient and gradient norm fall back to the saved_* keys (their settings to
[saved_integration]).

JLD2 schema 1 (RcmpsCore's rcmps_store): read with h5py, which this environment may lack; the
reader then raises ImportError. Matrices are stored column-major, so the HDF5 view is transposed.
"""
from __future__ import annotations

import math
import os
import re
import tomllib
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

__all__ = ["FORMAT", "FORMAT_VERSION", "SYMMETRIES", "Integration", "Manifold", "StateRecord",
           "read_jld2", "read_portable", "write_portable"]

FORMAT = "rcmps-portable-state"
FORMAT_VERSION = 1
SYMMETRIES = ("Z2", "none")
MATRICES = ("R", "K", "rho", "gradient")
# top-level keys of format 1, in written order
KEYS = ("format", "format_version", "D", "model", "coupling", "mass", "symmetry", "energy",
        "gradient_norm", "phi", "validation_passed", "producer", "source", "info", "integration", "manifold")


@dataclass(frozen=True)
class Integration:
    """IntegratorParameters: max_point is the physical half-window, n_quad the nodes per half."""
    n_quad: int
    max_point: float
    atol: float
    rtol: float
    maxiters: int | None = None


@dataclass(frozen=True)
class Manifold:
    """ManifoldParameters."""
    metric_reg: float
    precond_reg: float
    precond_reg_prefactor: float | None = None


@dataclass(frozen=True, eq=False)
class StateRecord:
    """A state as stored; matrices are C-ordered complex128 (D, D) arrays or None."""
    D: int
    model: str
    coupling: float
    R: np.ndarray | None = None
    K: np.ndarray | None = None
    mass: float = 1.0
    rho: np.ndarray | None = None
    gradient: np.ndarray | None = None
    energy: float | None = None
    gradient_norm: float | None = None
    symmetry: str | None = None
    phi: float | None = None
    validation_passed: bool | None = None
    integration: Integration | None = None
    manifold: Manifold | None = None
    producer: str | None = None
    source: str | None = None
    info: str | None = None
    origin: str = ""
    files: tuple[str, ...] = ()
    metadata: dict = field(default_factory=dict)


# ---------------------------------------------------------------------------- value checks

def _int(v, name, minimum=1):
    if isinstance(v, (bool, np.bool_)) or not isinstance(v, (int, np.integer)) or v < minimum:
        raise ValueError(f"{name} must be an integer >= {minimum}, not {v!r}")
    return int(v)


def _real(v, name, *, positive=False, nonnegative=False):
    if isinstance(v, (bool, np.bool_)) or not isinstance(v, (int, float, np.integer, np.floating)):
        raise ValueError(f"{name} must be a real number, not {v!r}")
    v = float(v)
    if not math.isfinite(v) or (positive and v <= 0) or (nonnegative and v < 0):
        qual = " and positive" if positive else " and nonnegative" if nonnegative else ""
        raise ValueError(f"{name} must be finite{qual}, not {v!r}")
    return v


def _str(v, name):
    if not isinstance(v, str):
        raise ValueError(f"{name} must be a string, not {v!r}")
    return v


def _bool(v, name):
    if not isinstance(v, (bool, np.bool_)):
        raise ValueError(f"{name} must be true or false, not {v!r}")
    return bool(v)


def _sym(v, name):
    if v not in SYMMETRIES:
        raise ValueError(f"{name} must be one of {SYMMETRIES}, not {v!r}")
    return v


def _opt(conv, v, name, **kw):
    return None if v is None else conv(v, name, **kw)


def _model_check(model, mass):
    if not model:
        raise ValueError("the model name is empty")
    if model == "phi4" and mass != 1.0:
        raise ValueError(f"model phi4 has no mass parameter (its normal-ordering mass is 1); mass = {mass!r} refused")


def _integration(t, name):
    if not isinstance(t, dict):
        raise ValueError(f"{name} must be a table")
    try:
        return Integration(_int(t["n_quad"], f"{name}.n_quad"),
                           _real(t["max_point"], f"{name}.max_point", positive=True),
                           _real(t["atol"], f"{name}.atol", positive=True),
                           _real(t["rtol"], f"{name}.rtol", positive=True),
                           _opt(_int, t.get("maxiters"), f"{name}.maxiters"))
    except KeyError as err:
        raise ValueError(f"{name} has no {err.args[0]}") from None


def _manifold(t, name):
    if not isinstance(t, dict):
        raise ValueError(f"{name} must be a table")
    try:
        return Manifold(_real(t["metric_reg"], f"{name}.metric_reg", nonnegative=True),
                        _real(t["precond_reg"], f"{name}.precond_reg", nonnegative=True),
                        _opt(_real, t.get("precond_reg_prefactor"), f"{name}.precond_reg_prefactor",
                             nonnegative=True))
    except KeyError as err:
        raise ValueError(f"{name} has no {err.args[0]}") from None


def _matrix(v, name, d):
    x = np.asarray(v)
    if x.shape != (d, d) or not np.issubdtype(x.dtype, np.number):
        raise ValueError(f"{name} must be a {d}x{d} matrix, not of shape {x.shape} and type {x.dtype}")
    x = np.ascontiguousarray(x, dtype=np.complex128)
    if not np.isfinite(x).all():
        raise ValueError(f"{name} holds nonfinite values")
    return x


# ---------------------------------------------------------------------------- JLD2

def _jld2_complex(ds):
    raw = ds[()]
    out = np.empty(np.shape(raw), dtype=np.complex128)
    out.real, out.imag = raw["re"], raw["im"]
    return out


def _jld2_string(f, name):
    try:
        v = f[name][()]
    except (KeyError, OSError):
        if name not in f:
            raise
        return ""
    return v.decode() if isinstance(v, (bytes, np.bytes_)) else str(v)


def read_jld2(path):
    """Read an rcmps_store checkpoint (JLD2 schema 1). rho is not stored (None)."""
    import h5py   # optional dependency

    with h5py.File(path, "r") as f:
        if int(f["schema_version"][()]) != 1:
            raise ValueError("unsupported schema")
        R, K = _jld2_complex(f["R"]).T, _jld2_complex(f["K"]).T
        coupling = _jld2_complex(f["coupling"])
        model = _jld2_string(f, "model")
        mass = float(f["mass"][()]) if "mass" in f else 1.0
        e0 = float(f["e0"][()])
        grad = _jld2_complex(f["grad"]).T if "grad" in f else None
        info = _jld2_string(f, "info") if "info" in f else None
        row = f["integration"][()]
        integ = Integration(int(row["n_quad"]), float(row["max_point"]), float(row["atol"]), float(row["rtol"]),
                            int(row["maxiters"]) if "maxiters" in row.dtype.names else None)
        mrow = f["manifold"][()] if "manifold" in f else None
        man = None if mrow is None else Manifold(
            float(mrow["metric_reg"]), float(mrow["precond_reg"]),
            float(mrow["precond_reg_prefactor"]) if "precond_reg_prefactor" in mrow.dtype.names else None)
    if coupling.imag != 0:
        raise ValueError("model coupling must be real")
    _model_check(model, mass)
    if R.ndim != 2 or R.shape[0] != R.shape[1] or R.shape[0] == 0:
        raise ValueError("R must be nonempty and square")
    d = R.shape[0]
    evaluated = math.isfinite(e0)
    return StateRecord(D=d, model=model, coupling=float(coupling.real), R=_matrix(R, "R", d), K=_matrix(K, "K", d),
                       mass=mass, gradient=_matrix(grad, "grad", d) if evaluated and grad is not None else None,
                       energy=e0 if evaluated else None, integration=integ, manifold=man, info=info, origin="jld2")


# ---------------------------------------------------------------------------- portable

def _fields_format1(md):
    if md["format"] != FORMAT:
        raise ValueError(f"metadata.toml: format {md['format']!r} is not {FORMAT!r}")
    ver = md.get("format_version")
    if type(ver) is not int or ver != FORMAT_VERSION:
        raise ValueError(f"metadata.toml: unsupported {FORMAT} format_version {ver!r} (this reader knows {FORMAT_VERSION})")
    for key in ("D", "model", "coupling"):
        if key not in md:
            raise ValueError(f"metadata.toml: required key {key} is missing")
    g = md.get
    return dict(
        D=_int(g("D"), "D"), model=_str(g("model"), "model"), coupling=_real(g("coupling"), "coupling"),
        mass=_real(g("mass", 1.0), "mass"), energy=_opt(_real, g("energy"), "energy"),
        gradient_norm=_opt(_real, g("gradient_norm"), "gradient_norm", nonnegative=True),
        symmetry=_opt(_sym, g("symmetry"), "symmetry"), phi=_opt(_real, g("phi"), "phi"),
        validation_passed=_opt(_bool, g("validation_passed"), "validation_passed"),
        producer=_opt(_str, g("producer"), "producer"), source=_opt(_str, g("source"), "source"),
        info=_opt(_str, g("info"), "info"),
        integration=_opt(_integration, g("integration"), "[integration]"),
        manifold=_opt(_manifold, g("manifold"), "[manifold]"), origin="portable"), "gradient.bin"


def _fields_legacy(md, directory):
    g = md.get
    for key in ("D", "coupling"):
        if key not in md:
            raise ValueError(f"metadata.toml: required key {key} is missing")
    from_saved = False

    def available(flag, default=True):
        return g(flag, default) is not False

    energy = g("energy")
    if energy is None and "saved_energy" in md and available("saved_energy_available"):
        energy, from_saved = g("saved_energy"), True
    gname = "gradient.bin"
    if not (directory / gname).exists():
        gname = "saved_gradient.bin"
        if (directory / gname).exists() and available("saved_gradient_available"):
            from_saved = True
        else:
            gname = None
    norm = g("gradient_norm")
    if norm is None and "saved_gradient_norm" in md and available(
            "saved_gradient_norm_available", available("saved_gradient_available")):
        norm, from_saved = g("saved_gradient_norm"), True
    if from_saved:
        integ = _integration(g("saved_integration"), "[saved_integration]") if "saved_integration" in md else None
    else:
        n_quad = g("quadrature", g("n_quad"))
        max_point = g("window", g("half_window", g("max_point")))
        integ = None if n_quad is None and max_point is None else _integration(
            dict(n_quad=n_quad, max_point=max_point, atol=g("atol"), rtol=g("rtol"), maxiters=g("maxiters")),
            "metadata.toml (integration keys)")
    man = (_manifold(md, "metadata.toml (metric_reg, precond_reg)")
           if "metric_reg" in md and "precond_reg" in md else None)
    return dict(D=_int(g("D"), "D"), model="phi4", coupling=_real(g("coupling"), "coupling"), mass=1.0,
                energy=_opt(_real, energy, "energy"),
                gradient_norm=_opt(_real, norm, "gradient_norm", nonnegative=True),
                validation_passed=_opt(_bool, g("validation_passed"), "validation_passed"),
                source=_opt(_str, g("source"), "source"), integration=integ, manifold=man,
                origin="portable-legacy"), gname


def _read_bin(path, d):
    size = path.stat().st_size
    if size != 16 * d * d:
        raise ValueError(f"{path.name} has {size} bytes, not the {16 * d * d} of a {d}x{d} complex128 matrix")
    return _matrix(np.fromfile(path, dtype="<c16").reshape((d, d), order="F"), path.name, d)


def read_portable(directory, *, arrays=True):
    """Read a portable state directory (format 1 or a research dialect). With arrays=False only
    metadata.toml is read and checked."""
    directory = Path(directory)
    with (directory / "metadata.toml").open("rb") as stream:
        md = tomllib.load(stream)
    fields, gname = _fields_format1(md) if "format" in md else _fields_legacy(md, directory)
    _model_check(fields["model"], fields["mass"])
    names = dict(R="R.bin", K="K.bin", rho="rho.bin", gradient=gname)
    names = {k: v for k, v in names.items() if v is not None and (k in ("R", "K") or (directory / v).exists())}
    files = ("metadata.toml", *names.values())
    if arrays:
        fields.update({k: _read_bin(directory / v, fields["D"]) for k, v in names.items()})
    return StateRecord(**fields, files=files, metadata=md)


def _toml_str(text):
    esc = {'"': '\\"', "\\": "\\\\", "\b": "\\b", "\t": "\\t", "\n": "\\n", "\f": "\\f", "\r": "\\r"}
    return '"' + "".join(esc.get(c, f"\\u{ord(c):04X}" if ord(c) < 0x20 or ord(c) == 0x7F else c) for c in text) + '"'


def _toml_val(v, name):
    if isinstance(v, (bool, np.bool_)):
        return "true" if v else "false"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        return repr(_real(v, name))
    if isinstance(v, str):
        return _toml_str(v)
    raise TypeError(f"{name}: a metadata value must be a string, boolean, integer or real, not {v!r}")


def _toml_table(name, values):
    rows = [f"{k} = {_toml_val(v, f'{name}.{k}')}" for k, v in values.items() if v is not None]
    return f"\n[{name}]\n" + "".join(r + "\n" for r in rows)


def write_portable(directory, record, *, extra=None, extra_matrices=None):
    """Write `record` as a new format-1 directory (refused if it exists); .bin files first,
    metadata.toml last by rename. Returns the directory."""
    directory = Path(directory)
    d = _int(record.D, "D")
    if record.R is None or record.K is None:
        raise ValueError("R and K are required")
    mats = {n: _matrix(getattr(record, n), n, d) for n in MATRICES if getattr(record, n) is not None}
    for n, m in (extra_matrices or {}).items():
        if n in MATRICES or not re.fullmatch(r"[A-Za-z0-9_]+", n):
            raise ValueError(f"extra matrix name {n!r} is not allowed")
        mats[n] = _matrix(m, n, d)
    model, mass = _str(record.model, "model"), _real(record.mass, "mass")
    _model_check(model, mass)
    head = dict(format=FORMAT, format_version=FORMAT_VERSION, D=d, model=model,
                coupling=_real(record.coupling, "coupling"), mass=mass,
                symmetry=_opt(_sym, record.symmetry, "symmetry"), energy=_opt(_real, record.energy, "energy"),
                gradient_norm=_opt(_real, record.gradient_norm, "gradient_norm", nonnegative=True),
                phi=_opt(_real, record.phi, "phi"),
                validation_passed=_opt(_bool, record.validation_passed, "validation_passed"),
                producer=_opt(_str, record.producer, "producer"), source=_opt(_str, record.source, "source"),
                info=_opt(_str, record.info, "info"))
    for key in extra or {}:
        if key in KEYS or not re.fullmatch(r"[A-Za-z0-9_-]+", key):
            raise ValueError(f"extra metadata key {key!r} is not allowed")
    text = "".join(f"{k} = {_toml_val(v, k)}\n" for k, v in {**head, **(extra or {})}.items() if v is not None)
    if record.integration is not None:
        i = record.integration
        text += _toml_table("integration", dict(
            n_quad=_int(i.n_quad, "integration.n_quad"),
            max_point=_real(i.max_point, "integration.max_point", positive=True),
            atol=_real(i.atol, "integration.atol", positive=True),
            rtol=_real(i.rtol, "integration.rtol", positive=True),
            maxiters=_opt(_int, i.maxiters, "integration.maxiters")))
    if record.manifold is not None:
        m = record.manifold
        text += _toml_table("manifold", dict(
            metric_reg=_real(m.metric_reg, "manifold.metric_reg", nonnegative=True),
            precond_reg=_real(m.precond_reg, "manifold.precond_reg", nonnegative=True),
            precond_reg_prefactor=_opt(_real, m.precond_reg_prefactor, "manifold.precond_reg_prefactor",
                                       nonnegative=True)))
    tomllib.loads(text)
    directory.mkdir(parents=True, exist_ok=False)
    for n, m in mats.items():
        m.ravel(order="F").astype("<c16").tofile(directory / f"{n}.bin")
    tmp = directory / ".metadata.toml.tmp"
    tmp.write_bytes(text.encode("utf-8"))
    os.replace(tmp, directory / "metadata.toml")
    return directory
