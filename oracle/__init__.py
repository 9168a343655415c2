"""ORACLE — test infrastructure only; never imported by the product.

Python access to the two CPU checkers for the photon walk:

* ``run`` calls ``liboracle.so``, this repository's restatement of TissueMC's CPU engine
  (``oracle/oracle.cpp``), which adds the 2-D tallies A(r,z), R_d(r,a), T_t(r,a) that TissueMC does
  not have. It follows the reference files listed at the top of ``oracle.cpp``.
* ``run_reference`` runs ``oracle/_ref/tissuemc``, the reference's own CPU engine and CLI compiled
  from its sources by ``oracle/Makefile``, and returns its JSON result (``{"runs": [...]}``'s first
  run), exactly as ``python/tissuemc_analysis/validate.py:63-89`` of the reference reads it.

Only ``tests/``, the smoke check in ``__graft_entry__.py`` and the CPU-baseline leg of ``bench.py``
may use this module.
"""

from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_BIN = HERE / "_ref" / "tissuemc"

MAX_LAYERS = 16


class _Layer(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("n", "mua", "mus", "g", "d")]


class _Spec(ctypes.Structure):
    _fields_ = [
        ("dz", ctypes.c_double),
        ("dr", ctypes.c_double),
        ("nz", ctypes.c_int32),
        ("nr", ctypes.c_int32),
        ("na", ctypes.c_int32),
        ("n_above", ctypes.c_double),
        ("n_below", ctypes.c_double),
        ("num_layers", ctypes.c_int32),
        ("layers", _Layer * MAX_LAYERS),
    ]


_P = ctypes.POINTER
_fd, _fu = _P(ctypes.c_double), _P(ctypes.c_uint64)


class _Out(ctypes.Structure):
    _fields_ = [
        ("rd", _fd), ("tt", _fd), ("absorbed", _fd), ("events", _fu), ("anomalies", _fu),
        ("a_z", _fd), ("rd_r", _fd), ("a_rz", _fd), ("rd_ra", _fd), ("tt_ra", _fd),
        ("n_a_rz", _fu), ("n_rd_ra", _fu), ("n_tt_ra", _fu),
        ("b_a_rz", _fd), ("b_rd_ra", _fd), ("b_tt_ra", _fd), ("boundary_steps", _fu),
        ("specular", ctypes.c_double), ("wall_seconds", ctypes.c_double),
        ("threads_used", ctypes.c_int32), ("error", ctypes.c_char * 256),
    ]  # fmt: skip


@dataclass
class Spec:
    """One .mci run: layers are (n, mua, mus, g, d) tuples."""

    layers: list[tuple[float, float, float, float, float]]
    dz: float = 0.01
    dr: float = 0.01
    nz: int = 1
    nr: int = 1
    na: int = 1
    n_above: float = 1.0
    n_below: float = 1.0
    photons: int = 1000
    name: str = "run.mco"

    def to_c(self) -> _Spec:
        s = _Spec()
        s.dz, s.dr, s.nz, s.nr, s.na = self.dz, self.dr, self.nz, self.nr, self.na
        s.n_above, s.n_below = self.n_above, self.n_below
        s.num_layers = len(self.layers)
        for i, lay in enumerate(self.layers):
            s.layers[i] = _Layer(*lay)
        return s

    def to_mci(self) -> str:
        lines = ["1.0", "1", f"{self.name} A", str(self.photons), f"{self.dz!r} {self.dr!r}",
                 f"{self.nz} {self.nr} {self.na}", str(len(self.layers)), repr(self.n_above)]
        lines += [" ".join(repr(float(v)) for v in lay) for lay in self.layers]
        lines.append(repr(self.n_below))
        return "\n".join(lines) + "\n"


@dataclass
class Result:
    """Oracle output; arrays are numpy. 2-D arrays are (nr, nz) and (nr, na)."""

    rd: np.ndarray
    tt: np.ndarray
    absorbed: np.ndarray  # (B, L)
    events: np.ndarray
    anomalies: np.ndarray
    a_z: np.ndarray
    rd_r: np.ndarray
    a_rz: np.ndarray
    rd_ra: np.ndarray
    tt_ra: np.ndarray
    photons: np.ndarray  # per batch
    specular: float
    wall_seconds: float
    threads: int
    n_a_rz: np.ndarray | None = None
    n_rd_ra: np.ndarray | None = None
    n_tt_ra: np.ndarray | None = None
    b_a_rz: np.ndarray | None = None
    b_rd_ra: np.ndarray | None = None
    b_tt_ra: np.ndarray | None = None
    boundary_steps: np.ndarray | None = None
    extra: dict = field(default_factory=dict)


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), str(LIB_PATH)], check=True)
        _lib = ctypes.CDLL(str(LIB_PATH))
        _lib.oracle_run.restype = ctypes.c_int
        _lib.oracle_run.argtypes = [_P(_Spec), ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint64,
                                    ctypes.c_int32, ctypes.c_int32, _P(_Out)]
        _lib.oracle_philox.argtypes = [_P(ctypes.c_uint32), _P(ctypes.c_uint32), _P(ctypes.c_uint32)]
        _lib.oracle_stream.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                       _P(ctypes.c_uint32)]
        _lib.oracle_fresnel.restype = ctypes.c_double
        _lib.oracle_fresnel.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, _P(ctypes.c_double)]
    return _lib


def _ptr(a: np.ndarray | None, ctype):
    if a is None:
        return ctypes.cast(None, _P(ctype))
    return a.ctypes.data_as(_P(ctype))


def batch_sizes(photons: int, batches: int) -> np.ndarray:
    """Photons per batch (include/tissuemc/batching.hpp:11-29): the first `extra` get one more."""
    base, extra = divmod(photons, batches)
    return np.array([base + (1 if b < extra else 0) for b in range(batches)], dtype=np.uint64)


def run(spec: Spec, photons: int, batches: int = 10, seed: int = 1, precision: int = 64,
        threads: int = 0, counts: bool = False, per_batch_bins: bool = False) -> Result:
    lib = _load()
    L, nz, nr, na = len(spec.layers), spec.nz, spec.nr, spec.na
    f = lambda *shape: np.zeros(shape, dtype=np.float64)  # noqa: E731
    u = lambda *shape: np.zeros(shape, dtype=np.uint64)  # noqa: E731
    res = Result(boundary_steps=u(batches), rd=f(batches), tt=f(batches), absorbed=f(batches, L), events=u(batches),
                 anomalies=u(batches), a_z=f(nz), rd_r=f(nr), a_rz=f(nr, nz), rd_ra=f(nr, na),
                 tt_ra=f(nr, na), photons=batch_sizes(photons, batches), specular=0.0,
                 wall_seconds=0.0, threads=0)
    if counts:
        res.n_a_rz, res.n_rd_ra, res.n_tt_ra = u(nr, nz), u(nr, na), u(nr, na)
    if per_batch_bins:
        res.b_a_rz, res.b_rd_ra, res.b_tt_ra = f(batches, nr, nz), f(batches, nr, na), f(batches, nr, na)
    out = _Out()
    out.rd, out.tt, out.absorbed = _ptr(res.rd, ctypes.c_double), _ptr(res.tt, ctypes.c_double), \
        _ptr(res.absorbed, ctypes.c_double)
    out.events, out.anomalies = _ptr(res.events, ctypes.c_uint64), _ptr(res.anomalies, ctypes.c_uint64)
    for k in ("a_z", "rd_r", "a_rz", "rd_ra", "tt_ra", "b_a_rz", "b_rd_ra", "b_tt_ra"):
        setattr(out, k, _ptr(getattr(res, k), ctypes.c_double))
    for k in ("n_a_rz", "n_rd_ra", "n_tt_ra", "boundary_steps"):
        setattr(out, k, _ptr(getattr(res, k), ctypes.c_uint64))
    c_spec = spec.to_c()
    rc = lib.oracle_run(ctypes.byref(c_spec), photons, batches, seed, precision, threads,
                        ctypes.byref(out))
    if rc != 0:
        raise ValueError(out.error.decode())
    res.specular, res.wall_seconds, res.threads = out.specular, out.wall_seconds, out.threads_used
    return res


def philox(ctr, key) -> list[int]:
    lib = _load()
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib.oracle_philox(c, k, o)
    return list(o)


def stream(seed: int, photon_id: int, n: int) -> np.ndarray:
    lib = _load()
    out = np.zeros(n, dtype=np.uint32)
    lib.oracle_stream(seed, photon_id, n, out.ctypes.data_as(_P(ctypes.c_uint32)))
    return out


def fresnel(n1: float, n2: float, cos_i: float, precision: int = 64) -> tuple[float, float]:
    lib = _load()
    ca2 = ctypes.c_double(0.0)
    r = lib.oracle_fresnel(precision, n1, n2, cos_i, ctypes.byref(ca2))
    return r, ca2.value


def reference_available() -> bool:
    return REF_BIN.exists() and os.access(REF_BIN, os.X_OK)


def run_reference(mci_text: str, photons: int, batches: int, seed: int = 1, precision: str = "float64",
                  threads: int = 1, binary: Path = REF_BIN, extra_args: list[str] | None = None) -> dict:
    """Run the reference's own CLI (`tissuemc run`) on an .mci text and return its first run."""
    with tempfile.TemporaryDirectory() as tmp:
        cfg = Path(tmp) / "in.mci"
        cfg.write_text(mci_text)
        out = Path(tmp) / "out.json"
        cmd = [str(binary), "run", str(cfg), "--photons", str(photons), "--batches", str(batches),
               "--seed", str(seed), "--threads", str(threads), "--precision", precision,
               "--output", str(out)] + (extra_args or [])
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode not in (0, 1):
            raise RuntimeError(f"reference engine failed ({proc.returncode}): {proc.stderr.strip()}")
        return json.loads(out.read_text())["runs"][0]
