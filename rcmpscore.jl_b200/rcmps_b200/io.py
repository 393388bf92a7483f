"""State files exchanged with RcmpsCore.jl: portable directories and JLD2 checkpoints.

Public names follow rcmps_gpu.io (gpu/src/rcmps_gpu/io.py of RcmpsCore.jl): StateRecord,
Integration, Manifold, read_portable, write_portable, read_jld2, FORMAT, FORMAT_VERSION,
SYMMETRIES. The implementation here is table-driven: every metadata key of the format is one
row of a schema (`_FORMAT1`), and reading, checking and writing all walk that table.

The on-disk format ("rcmps-portable-state", format 1; the format description of
gpu/src/rcmps_gpu/io.py:15-61 and gpu/julia/portable.jl:141-260):
  * metadata.toml: required format, format_version (= 1), D, model, coupling; optional mass
    (1.0 when absent; phi4 only admits 1.0), symmetry ("Z2" or "none"), energy, gradient_norm,
    phi, validation_passed, producer, source, info, a table [integration] (n_quad, max_point,
    atol, rtol, optional maxiters) and a table [manifold] (metric_reg, precond_reg, optional
    precond_reg_prefactor). Unknown keys are kept in StateRecord.metadata and otherwise ignored.
  * R.bin and K.bin (required), rho.bin and gradient.bin (optional): each a headerless D x D
    complex128 matrix, little-endian, column-major (Julia's memory order), exactly 16 D^2 bytes.
    In memory every matrix is a C-ordered (D, D) complex128 array.
Research directories without a `format` key (the earlier GPU optimizer's initial/ and
optimized_state/, Julia exports of the research tree) are read as the "legacy" dialect: they
describe phi4 with mass 1, and a value missing under its format-1 name is taken from its saved_*
counterpart unless the matching saved_*_available flag is false; the integration settings of
such saved values are [saved_integration], and otherwise come from the top-level window /
quadrature style keys.

JLD2 checkpoints (RcmpsCore's rcmps_store, schema_version 1) are read with h5py, which is an
optional dependency: without it read_jld2 raises ImportError. JLD2 stores column-major matrices,
so their HDF5 view is the transpose.
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
_BIN = "<c16"                       # element type of every .bin file
_NAME = re.compile(r"[A-Za-z0-9_]+\Z")


@dataclass(frozen=True)
class Integration:
    """RcmpsCore IntegratorParameters: Gauss nodes per half window and the half window x_max."""
    n_quad: int
    max_point: float
    atol: float
    rtol: float
    maxiters: int | None = None


@dataclass(frozen=True)
class Manifold:
    """RcmpsCore ManifoldParameters."""
    metric_reg: float
    precond_reg: float
    precond_reg_prefactor: float | None = None


@dataclass(frozen=True, eq=False)
class StateRecord:
    """One stored state. Matrices are C-ordered complex128 (D, D) arrays, or None when absent
    (or not read). `origin` says what was read ("portable", "portable-legacy", "jld2"), `files`
    which files of the directory hold the record, `metadata` the raw TOML table."""
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


# ------------------------------------------------------------------------------- value kinds
# A kind turns a TOML value into its Python value or raises ValueError naming `where`.

def _is_bool(v):
    return isinstance(v, (bool, np.bool_))


def _kind_count(v, where):
    """A positive integer (booleans are not integers here)."""
    if _is_bool(v) or not isinstance(v, (int, np.integer)) or v <= 0:
        raise ValueError(f"{where}: expected a positive integer, got {v!r}")
    return int(v)


def _finite(v, where):
    if _is_bool(v) or not isinstance(v, (int, float, np.integer, np.floating)) or not math.isfinite(float(v)):
        raise ValueError(f"{where}: expected a finite real number, got {v!r}")
    return float(v)


def _kind_real(v, where):
    return _finite(v, where)


def _kind_positive(v, where):
    x = _finite(v, where)
    if x <= 0.0:
        raise ValueError(f"{where}: expected a real number > 0, got {v!r}")
    return x


def _kind_nonneg(v, where):
    x = _finite(v, where)
    if x < 0.0:
        raise ValueError(f"{where}: expected a real number >= 0, got {v!r}")
    return x


def _kind_text(v, where):
    if not isinstance(v, str):
        raise ValueError(f"{where}: expected a string, got {v!r}")
    return v


def _kind_flag(v, where):
    if not _is_bool(v):
        raise ValueError(f"{where}: expected true or false, got {v!r}")
    return bool(v)


def _kind_symmetry(v, where):
    if v not in SYMMETRIES:
        raise ValueError(f"{where}: expected one of {', '.join(SYMMETRIES)}, got {v!r}")
    return v


# ------------------------------------------------------------------------------- the schema
# (key, kind, required); the order is the order in which write_portable writes the keys.
_INTEGRATION = (("n_quad", _kind_count, True), ("max_point", _kind_positive, True),
                ("atol", _kind_positive, True), ("rtol", _kind_positive, True),
                ("maxiters", _kind_count, False))
_MANIFOLD = (("metric_reg", _kind_nonneg, True), ("precond_reg", _kind_nonneg, True),
             ("precond_reg_prefactor", _kind_nonneg, False))
_FORMAT1 = (("D", _kind_count, True), ("model", _kind_text, True), ("coupling", _kind_real, True),
            ("mass", _kind_real, False), ("symmetry", _kind_symmetry, False), ("energy", _kind_real, False),
            ("gradient_norm", _kind_nonneg, False), ("phi", _kind_real, False),
            ("validation_passed", _kind_flag, False), ("producer", _kind_text, False),
            ("source", _kind_text, False), ("info", _kind_text, False))
_TABLES = {"integration": (_INTEGRATION, Integration), "manifold": (_MANIFOLD, Manifold)}
_RESERVED = {"format", "format_version", *(k for k, _, _ in _FORMAT1), *_TABLES}


def _parse(schema, table, where):
    """Checked values of `schema`'s keys found in `table` (absent optional keys are None)."""
    if not isinstance(table, dict):
        raise ValueError(f"{where}: expected a table")
    out = {}
    for key, kind, required in schema:
        if key in table:
            out[key] = kind(table[key], f"{where} {key}")
        elif required:
            raise ValueError(f"{where}: the required key {key!r} is absent")
        else:
            out[key] = None
    return out


def _parse_table(name, table, where):
    schema, cls = _TABLES[name]
    return cls(**_parse(schema, table, where))


def _check_model(model, mass):
    if not model:
        raise ValueError("model: the name is empty")
    if model == "phi4" and mass != 1.0:
        raise ValueError(f"mass: model phi4 is normal-ordered at mass 1 and takes no other mass (got {mass!r})")


def _square(m, where, d):
    """A finite (d, d) complex128 C-ordered copy of `m`."""
    a = np.asarray(m)
    if a.shape != (d, d) or not (np.issubdtype(a.dtype, np.number) and not np.issubdtype(a.dtype, np.bool_)):
        raise ValueError(f"{where}: expected a numeric {d}x{d} matrix, got shape {a.shape} of {a.dtype}")
    a = np.ascontiguousarray(a, dtype=np.complex128)
    if not np.isfinite(a).all():
        raise ValueError(f"{where}: contains a NaN or infinite entry")
    return a


# ------------------------------------------------------------------------------- .bin files

def _load_bin(path, d):
    expect = 16 * d * d
    have = path.stat().st_size
    if have != expect:
        raise ValueError(f"{path.name}: a {d}x{d} complex128 matrix takes {expect} bytes, the file has {have} bytes")
    return _square(np.fromfile(path, dtype=_BIN).reshape(d, d, order="F"), path.name, d)


def _store_bin(path, m):
    np.asfortranarray(m).ravel(order="K").astype(_BIN).tofile(path)


# ------------------------------------------------------------------------------- dialects

def _format1(md, directory):
    """Fields of a format-1 metadata table, and the name of its gradient file."""
    if md.get("format") != FORMAT:
        raise ValueError(f"metadata.toml: format is {md.get('format')!r}; this reader reads {FORMAT!r}")
    version = md.get("format_version")
    if type(version) is not int or version != FORMAT_VERSION:
        raise ValueError(f"metadata.toml: format_version {version!r} is not supported "
                         f"(known: {FORMAT_VERSION})")
    fields = _parse(_FORMAT1, md, "metadata.toml")
    if fields["mass"] is None:
        fields["mass"] = 1.0
    for name in _TABLES:
        fields[name] = _parse_table(name, md[name], f"[{name}]") if name in md else None
    fields["origin"] = "portable"
    return fields, "gradient.bin"


class _Legacy:
    """The research dialect: metadata without `format`. A value is read under its format-1 name
    first; otherwise, when a saved_* copy exists and its availability flag is not false, the
    saved copy is used and the record's integration settings become [saved_integration]."""

    def __init__(self, md, directory):
        self.md, self.dir, self.saved = md, directory, False

    def _available(self, flag, default=True):
        return self.md.get(flag, default) is not False

    def _scalar(self, name, flag, flag_default=True):
        if name in self.md:
            return self.md[name]
        if f"saved_{name}" in self.md and self._available(flag, flag_default):
            self.saved = True
            return self.md[f"saved_{name}"]
        return None

    def _gradient_file(self):
        if (self.dir / "gradient.bin").exists():
            return "gradient.bin"
        if (self.dir / "saved_gradient.bin").exists() and self._available("saved_gradient_available"):
            self.saved = True
            return "saved_gradient.bin"
        return None

    def _integration(self):
        md = self.md
        if self.saved:
            return _parse_table("integration", md["saved_integration"], "[saved_integration]") \
                if "saved_integration" in md else None
        n_quad = next((md[k] for k in ("quadrature", "n_quad") if k in md), None)
        window = next((md[k] for k in ("window", "half_window", "max_point") if k in md), None)
        if n_quad is None and window is None:
            return None
        table = {"n_quad": n_quad, "max_point": window, **{k: md[k] for k in ("atol", "rtol", "maxiters") if k in md}}
        return _parse_table("integration", {k: v for k, v in table.items() if v is not None},
                            "metadata.toml integration keys")

    def fields(self):
        md = self.md
        for key in ("D", "coupling"):
            if key not in md:
                raise ValueError(f"metadata.toml: the required key {key!r} is absent")
        energy = self._scalar("energy", "saved_energy_available")
        gradient_file = self._gradient_file()
        norm = self._scalar("gradient_norm", "saved_gradient_norm_available",
                            self._available("saved_gradient_available"))
        manifold = (_parse_table("manifold", md, "metadata.toml manifold keys")
                    if "metric_reg" in md and "precond_reg" in md else None)
        opt = lambda kind, v, where: None if v is None else kind(v, where)
        fields = dict(D=_kind_count(md["D"], "metadata.toml D"), model="phi4",
                      coupling=_kind_real(md["coupling"], "metadata.toml coupling"), mass=1.0,
                      energy=opt(_kind_real, energy, "metadata.toml energy"),
                      gradient_norm=opt(_kind_nonneg, norm, "metadata.toml gradient_norm"),
                      validation_passed=opt(_kind_flag, md.get("validation_passed"), "metadata.toml validation_passed"),
                      source=opt(_kind_text, md.get("source"), "metadata.toml source"),
                      integration=self._integration(), manifold=manifold, origin="portable-legacy")
        return fields, gradient_file


def read_portable(directory, *, arrays=True):
    """Read a portable state directory (format 1, or the research dialect when metadata.toml
    has no `format`). With arrays=False only metadata.toml is read and checked, and the
    matrices stay None."""
    directory = Path(directory)
    with open(directory / "metadata.toml", "rb") as fh:
        md = tomllib.load(fh)
    fields, gradient_file = _format1(md, directory) if "format" in md else _Legacy(md, directory).fields()
    _check_model(fields["model"], fields["mass"])
    matrix_files = {"R": "R.bin", "K": "K.bin"}
    for name, fname in (("rho", "rho.bin"), ("gradient", gradient_file)):
        if fname is not None and (directory / fname).exists():
            matrix_files[name] = fname
    if arrays:
        for name, fname in matrix_files.items():
            fields[name] = _load_bin(directory / fname, fields["D"])
    return StateRecord(**fields, files=("metadata.toml", *matrix_files.values()), metadata=md)


# ------------------------------------------------------------------------------- writing

def _toml_scalar(v, where):
    if _is_bool(v):
        return "true" if v else "false"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        return repr(_kind_real(v, where))
    if isinstance(v, str):
        out = ['"']
        for ch in v:
            if ch in '"\\':
                out.append("\\" + ch)
            elif ord(ch) < 0x20 or ord(ch) == 0x7F:
                out.append({"\n": "\\n", "\t": "\\t", "\r": "\\r"}.get(ch, f"\\u{ord(ch):04X}"))
            else:
                out.append(ch)
        return "".join(out) + '"'
    raise TypeError(f"{where}: metadata values are strings, booleans, integers or reals, not {type(v).__name__}")


def _render(schema, values, where):
    """`key = value` lines of the non-None values, checked by the schema's kinds."""
    lines = []
    for key, kind, required in schema:
        v = values.get(key)
        if v is None:
            if required:
                raise ValueError(f"{where}: {key} is required")
            continue
        lines.append(f"{key} = {_toml_scalar(kind(v, f'{where} {key}'), f'{where} {key}')}")
    return lines


def write_portable(directory, record, *, extra=None, extra_matrices=None):
    """Write `record` as a new format-1 directory; an existing directory is refused
    (FileExistsError). `extra` adds top-level keys and `extra_matrices` further D x D .bin
    files. The .bin files are written first and metadata.toml last, by an atomic rename, so a
    reader never sees a metadata file without its matrices. Returns the directory."""
    directory = Path(directory)
    d = _kind_count(record.D, "D")
    if record.R is None or record.K is None:
        raise ValueError("write_portable: R and K are required")
    matrices = {}
    for name in ("R", "K", "rho", "gradient"):
        if getattr(record, name) is not None:
            matrices[name] = _square(getattr(record, name), name, d)
    for name, m in (extra_matrices or {}).items():
        if name in matrices or name in ("R", "K", "rho", "gradient") or not _NAME.match(name):
            raise ValueError(f"write_portable: {name!r} cannot name an extra matrix")
        matrices[name] = _square(m, name, d)
    values = {key: getattr(record, key) for key, _, _ in _FORMAT1}
    values["mass"] = 1.0 if record.mass is None else record.mass
    _check_model(_kind_text(values["model"], "model"), _kind_real(values["mass"], "mass"))
    lines = [f'format = "{FORMAT}"', f"format_version = {FORMAT_VERSION}"]
    lines += _render(_FORMAT1, values, "metadata")
    for key, v in (extra or {}).items():
        if key in _RESERVED or not re.fullmatch(r"[A-Za-z0-9_-]+", key):
            raise ValueError(f"write_portable: {key!r} cannot be an extra metadata key")
        lines.append(f"{key} = {_toml_scalar(v, key)}")
    for name, (schema, _) in _TABLES.items():
        obj = getattr(record, name)
        if obj is not None:
            lines += ["", f"[{name}]"] + _render(schema, obj.__dict__, f"[{name}]")
    text = "\n".join(lines) + "\n"
    tomllib.loads(text)                     # what is written must read back
    directory.mkdir(parents=True, exist_ok=False)
    for name, m in matrices.items():
        _store_bin(directory / f"{name}.bin", m)
    staging = directory / ".metadata.toml.partial"
    staging.write_text(text, encoding="utf-8")
    os.replace(staging, directory / "metadata.toml")
    return directory


# ------------------------------------------------------------------------------- JLD2

def read_jld2(path):
    """Read an rcmps_store checkpoint (JLD2 schema_version 1) with h5py. rho is not stored
    (rcmps_load recomputes it), so the record's rho is None; energy and gradient are None for a
    state that was never evaluated (e0 not finite)."""
    import h5py                             # optional dependency

    def cplx(node):
        raw = node[()]
        return np.asarray(raw["re"]) + 1j * np.asarray(raw["im"])

    def text(f, key):
        if key not in f:
            return None
        raw = f[key][()]
        return raw.decode() if isinstance(raw, (bytes, np.bytes_)) else str(raw)

    def row_table(raw, schema, cls):
        names = raw.dtype.names
        return cls(**{key: (None if key not in names else
                            int(raw[key]) if kind is _kind_count else float(raw[key]))
                      for key, kind, _ in schema})

    with h5py.File(path, "r") as f:
        if int(f["schema_version"][()]) != 1:
            raise ValueError(f"{path}: only schema_version 1 checkpoints are read")
        R, K = cplx(f["R"]).T, cplx(f["K"]).T
        coupling = complex(cplx(f["coupling"]))
        model = text(f, "model") or ""
        mass = float(f["mass"][()]) if "mass" in f else 1.0
        e0 = float(f["e0"][()])
        grad = cplx(f["grad"]).T if "grad" in f else None
        info = text(f, "info")
        integration = row_table(f["integration"][()], _INTEGRATION, Integration)
        manifold = row_table(f["manifold"][()], _MANIFOLD, Manifold) if "manifold" in f else None
    if coupling.imag != 0.0:
        raise ValueError(f"{path}: the coupling is not real ({coupling})")
    _check_model(model, mass)
    if R.ndim != 2 or R.shape[0] != R.shape[1] or R.shape[0] == 0:
        raise ValueError(f"{path}: R is not a nonempty square matrix")
    d = R.shape[0]
    evaluated = math.isfinite(e0)
    return StateRecord(D=d, model=model, coupling=coupling.real, R=_square(R, "R", d), K=_square(K, "K", d), mass=mass,
                       gradient=_square(grad, "grad", d) if evaluated and grad is not None else None,
                       energy=e0 if evaluated else None, integration=integration, manifold=manifold, info=info,
                       origin="jld2")
