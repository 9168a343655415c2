"""tissuemc_b200 — a B200 (sm_100a) engine for TissueMC's MCML photon walk.

Python access to the engine's C ABI (include/tissuemc_b200.h) through ctypes. The CUDA kernels,
the C ABI and the C++ host code (the .mci reader, the run_cuda drop-in, the JSON writer and the
`tissuemc` CLI) are all in the in-tree library ``libtissuemc_b200.so``; this module only marshals
arguments. There is no fallback: if the library is missing or no GPU is present, the calls raise.

    import tissuemc_b200 as tmc
    spec = tmc.parse_mci("tissuemc_b200/configs/slab_n14.mci")[0]
    res = tmc.run(spec, photons=10**6, batches=10, seed=1)
    print(res.summary())
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libtissuemc_b200.so"
CLI_PATH = PKG / "bin" / "tissuemc"
CONFIGS = PKG / "configs"
MAX_LAYERS = 16
FIXED_SCALE = 2.0**32

# status codes (tmc_status_code)
OK, BAD_CONFIG, NO_DEVICE, CUDA_ERROR, DEVICE_TIMEOUT, BAD_ARGUMENT = range(6)


class ConfigError(ValueError):
    """An invalid run description or options (the reference's tissuemc::ConfigError)."""


class EngineError(RuntimeError):
    """No usable device, a CUDA failure or a device-side timeout."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


# ---------------------------------------------------------------------------------- C structs
class Layer(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("n", "mua", "mus", "g", "d")]


class CRunSpec(ctypes.Structure):
    _fields_ = [
        ("photons", ctypes.c_uint64),
        ("dz", ctypes.c_double),
        ("dr", ctypes.c_double),
        ("nz", ctypes.c_int32),
        ("nr", ctypes.c_int32),
        ("na", ctypes.c_int32),
        ("n_above", ctypes.c_double),
        ("n_below", ctypes.c_double),
        ("num_layers", ctypes.c_int32),
        ("layers", Layer * MAX_LAYERS),
    ]


class COptions(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("batches", ctypes.c_int32),
        ("photons", ctypes.c_uint64),
        ("rung", ctypes.c_int32),
        ("profiles", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("fast_math", ctypes.c_int32),
        ("threads_per_block", ctypes.c_int32),
        ("blocks_per_sm", ctypes.c_int32),
        ("smem_budget", ctypes.c_int32),
        ("step_cap", ctypes.c_uint32),
        ("tile_tz", ctypes.c_int32),
        ("tile_ra_rows", ctypes.c_int32),
        ("tile_cross", ctypes.c_int32),
    ]


class CSizes(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in
                ("batches", "layers", "nz", "nr", "na", "absorbed", "a_rz", "ra", "tally_words", "device_words")]


_pd, _pu = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint64)


class CResult(ctypes.Structure):
    _fields_ = [
        ("first_photon", _pu), ("photons", _pu), ("rd", _pd), ("tt", _pd), ("absorbed", _pd),
        ("events", _pu), ("anomalies", _pu), ("a_z", _pd), ("rd_r", _pd), ("tt_r", _pd),
        ("a_rz", _pd), ("rd_ra", _pd), ("tt_ra", _pd), ("raw", _pu),
        ("specular", ctypes.c_double), ("kernel_seconds", ctypes.c_double),
        ("wall_seconds", ctypes.c_double), ("device", ctypes.c_char * 128),
    ]  # fmt: skip


class CStatus(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int32), ("message", ctypes.c_char * 512)]


class CPlan(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in
                ("threads", "blocks_per_sm", "grid", "tr_a", "tz_a", "cross", "tr_rd", "tr_tt",
                 "batch_smem", "smem_bytes")]


class CSweepConfig(ctypes.Structure):
    _fields_ = [
        ("photons", ctypes.c_uint64),
        ("seed", ctypes.c_uint64),
        ("n_above", ctypes.c_double),
        ("n_below", ctypes.c_double),
        ("num_layers", ctypes.c_int32),
        ("layers", Layer * MAX_LAYERS),
    ]


class CAdamTensor(ctypes.Structure):
    """tmc_adam_tensor: one parameter tensor of a many-tensor Adam step (device pointers)."""

    _fields_ = [("w", ctypes.c_void_p), ("g", ctypes.c_void_p), ("m", ctypes.c_void_p), ("v", ctypes.c_void_p),
                ("wb", ctypes.c_void_p), ("wt", ctypes.c_void_p), ("avg", ctypes.c_void_p),
                ("rows", ctypes.c_int32), ("cols", ctypes.c_int32), ("weight_decay", ctypes.c_float),
                ("first_block", ctypes.c_int32)]


class CSweepOptions(ctypes.Structure):
    _fields_ = [("dz", ctypes.c_double), ("dr", ctypes.c_double)] + [
        (k, ctypes.c_int32) for k in ("nz", "nr", "na", "batches", "fast_math", "profiles", "device",
                                      "threads_per_block", "item_photons", "tile_r", "tile_z")]


class CSweepSizes(ctypes.Structure):
    _fields_ = [("words_per_config", ctypes.c_uint64), ("summary_per_config", ctypes.c_uint64),
                ("max_layers", ctypes.c_int32)]


# Every entry point include/tissuemc_b200.h declares: name -> (restype, argtypes)
_P = ctypes.POINTER
PROTOTYPES = {
    "tmc_b200_available": (ctypes.c_int, []),
    "tmc_b200_abi_version": (ctypes.c_int, []),
    "tmc_b200_version": (ctypes.c_char_p, []),
    "tmc_b200_default_options": (None, [_P(COptions)]),
    "tmc_b200_query_sizes": (ctypes.c_int, [_P(CRunSpec), _P(COptions), _P(CSizes), _P(CStatus)]),
    "tmc_b200_run": (ctypes.c_int, [_P(CRunSpec), _P(COptions), _P(CResult), _P(CStatus)]),
    "tmc_b200_run_device": (ctypes.c_int, [_P(CRunSpec), _P(COptions), ctypes.c_void_p,
                                           ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_decode": (ctypes.c_int, [_P(CRunSpec), _P(COptions), _pu, _P(CResult), _P(CStatus)]),
    "tmc_b200_parse_mci": (ctypes.c_int, [ctypes.c_char_p, _P(CRunSpec), ctypes.c_int32,
                                          _P(ctypes.c_int32), _P(CStatus)]),
    "tmc_b200_run_static": (ctypes.c_int, [_P(CRunSpec), _P(COptions), _P(CResult), _P(CStatus)]),
    "tmc_b200_run_device_range": (ctypes.c_int, [_P(CRunSpec), _P(COptions), ctypes.c_uint64, ctypes.c_uint64,
                                                  ctypes.c_void_p, ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_probe_physics": (ctypes.c_int, [ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                                              ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32,
                                              _P(ctypes.c_double), _P(CStatus)]),
    "tmc_b200_write_mco": (ctypes.c_int, [_P(CRunSpec), _P(COptions), _P(CResult), ctypes.c_char_p, _P(CStatus)]),
    "tmc_b200_sweep_default_options": (None, [_P(CSweepOptions)]),
    "tmc_b200_sweep_sample": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_int32, _P(CSweepConfig), _P(CStatus)]),
    "tmc_b200_sweep_costs": (ctypes.c_int, [_P(CSweepConfig), ctypes.c_int32, _P(ctypes.c_double), _P(CStatus)]),
    "tmc_b200_sweep_sizes": (ctypes.c_int, [_P(CSweepConfig), ctypes.c_int32, _P(CSweepOptions),
                                            _P(CSweepSizes), _P(CStatus)]),
    "tmc_b200_sweep_run": (ctypes.c_int, [_P(CSweepConfig), ctypes.c_int32, _P(CSweepOptions), _pu, _pd, _pd,
                                          _P(CStatus)]),
    "tmc_b200_sweep_run_loop": (ctypes.c_int, [_P(CSweepConfig), ctypes.c_int32, _P(CSweepOptions), _pu, _pd,
                                               _P(CStatus)]),
    "tmc_b200_sweep_autotune": (ctypes.c_int, [_P(CSweepConfig), ctypes.c_int32, _P(CSweepOptions), _pd,
                                               _P(CStatus)]),
    "tmc_b200_probe_wait_timeout": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint32, _P(CStatus)]),
    "tmc_b200_gemm_bf16": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                          _P(CStatus)]),
    "tmc_b200_nn_linear": (ctypes.c_int, [ctypes.c_void_p] * 6 + [ctypes.c_int32] * 4 + [ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_nn_backward_data": (ctypes.c_int, [ctypes.c_void_p] * 5 + [ctypes.c_int32] * 3 +
                                  [ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_nn_matmul_f32": (ctypes.c_int, [ctypes.c_void_p] * 3 + [ctypes.c_int32] * 3 + [ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_nn_matmul_f32_splitk": (ctypes.c_int, [ctypes.c_void_p] * 4 + [ctypes.c_int32] * 4 +
                                      [ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_nn_transpose": (ctypes.c_int, [ctypes.c_void_p] * 2 + [ctypes.c_int32] * 2 + [ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_nn_colsum": (ctypes.c_int, [ctypes.c_void_p] * 2 + [ctypes.c_int32] * 2 +
                           [ctypes.c_void_p, ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_nn_colsum_work": (ctypes.c_int32, [ctypes.c_int32]),
    "tmc_b200_nn_mse": (ctypes.c_int, [ctypes.c_void_p] * 4 + [ctypes.c_int32] * 3 + [ctypes.c_float, ctypes.c_void_p,
                                                                                        _P(CStatus)]),
    "tmc_b200_nn_adam": (ctypes.c_int, [ctypes.c_void_p] * 4 + [ctypes.c_int32] * 2 +
                         [ctypes.c_float, ctypes.c_void_p] + [ctypes.c_float] * 4 + [ctypes.c_void_p] * 3 +
                         [ctypes.c_float, ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_nn_status": (ctypes.c_int, [ctypes.c_int32]),
    "tmc_b200_nn_adam_plan": (ctypes.c_int32, [_P(CAdamTensor), ctypes.c_int32]),
    "tmc_b200_nn_adam_multi": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                                              ctypes.c_void_p] + [ctypes.c_float] * 4 + [ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_nn_ema": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_float,
                                       ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_nn_to_bf16": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_nn_encode": (ctypes.c_int, [ctypes.c_void_p] * 4 + [ctypes.c_int32] * 3 + [ctypes.c_void_p, _P(CStatus)]),
    "tmc_b200_nn_gate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32] +
                         [ctypes.c_void_p] * 3 + [ctypes.c_int32, ctypes.c_int32, ctypes.c_float] +
                         [ctypes.c_void_p] * 4 + [_P(CStatus)]),
    "tmc_b200_nn_packed_bytes": (ctypes.c_int64, [ctypes.c_int32]),
    "tmc_b200_nn_pack": (ctypes.c_int, [_P(ctypes.c_void_p), ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                        _P(CStatus)]),
    "tmc_b200_nn_ensemble_infer": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                                  ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_int32, ctypes.c_float] + [ctypes.c_void_p] * 5 +
                                   [_P(CStatus)]),
    "tmc_b200_autotune": (ctypes.c_int, [_P(CRunSpec), _P(COptions), ctypes.c_uint64, _P(CPlan), _pd, _pd,
                                         _P(CStatus)]),
    "tmc_b200_plan": (ctypes.c_int, [_P(CRunSpec), _P(COptions), ctypes.c_int32, ctypes.c_int64,
                                     ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, _P(CPlan),
                                     _P(CStatus)]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded engine library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m tissuemc_b200.build` "
                "(there is no CPU fallback)"
            )
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def _check(rc: int, st: CStatus) -> None:
    if rc == OK:
        return
    msg = st.message.decode(errors="replace")
    if rc == BAD_CONFIG:
        raise ConfigError(msg)
    raise EngineError(rc, msg)


# ---------------------------------------------------------------------------------- Python API
@dataclass
class RunSpec:
    """One MCML run (the reference's RunSpec): layers are (n, mua, mus, g, d) tuples."""

    layers: list[tuple[float, float, float, float, float]]
    photons: int = 1000
    dz: float = 0.01
    dr: float = 0.01
    nz: int = 1
    nr: int = 1
    na: int = 1
    n_above: float = 1.0
    n_below: float = 1.0
    output_name: str = "run.mco"

    def to_c(self) -> CRunSpec:
        s = CRunSpec()
        s.photons, s.dz, s.dr = self.photons, self.dz, self.dr
        s.nz, s.nr, s.na = self.nz, self.nr, self.na
        s.n_above, s.n_below = self.n_above, self.n_below
        s.num_layers = len(self.layers)
        for i, lay in enumerate(self.layers[:MAX_LAYERS]):
            s.layers[i] = Layer(*map(float, lay))
        return s

    @staticmethod
    def from_c(c: CRunSpec, name: str = "run.mco") -> RunSpec:
        layers = [(c.layers[i].n, c.layers[i].mua, c.layers[i].mus, c.layers[i].g, c.layers[i].d)
                  for i in range(c.num_layers)]
        return RunSpec(layers=layers, photons=c.photons, dz=c.dz, dr=c.dr, nz=c.nz, nr=c.nr,
                       na=c.na, n_above=c.n_above, n_below=c.n_below, output_name=name)

    def to_mci(self) -> str:
        rows = ["1.0", "1", f"{self.output_name} A", str(self.photons), f"{self.dz!r} {self.dr!r}",
                f"{self.nz} {self.nr} {self.na}", str(len(self.layers)), repr(float(self.n_above))]
        rows += [" ".join(repr(float(v)) for v in lay) for lay in self.layers]
        rows.append(repr(float(self.n_below)))
        return "\n".join(rows) + "\n"


def options(seed: int = 1, batches: int = 10, photons: int = 0, rung: int = 0, profiles: bool = True,
            device: int = 0, fast_math: bool = True, threads_per_block: int = 0, blocks_per_sm: int = 0,
            smem_budget: int = 0, step_cap: int = 0, tile_tz: int = 0, tile_ra_rows: int = 0,
            tile_cross: int = 0) -> COptions:
    o = COptions()
    lib().tmc_b200_default_options(ctypes.byref(o))
    o.seed, o.batches, o.photons, o.rung = seed, batches, photons, rung
    o.profiles, o.device, o.fast_math = int(profiles), device, int(fast_math)
    o.threads_per_block, o.blocks_per_sm, o.smem_budget = threads_per_block, blocks_per_sm, smem_budget
    o.step_cap = step_cap
    o.tile_tz, o.tile_ra_rows, o.tile_cross = tile_tz, tile_ra_rows, tile_cross
    return o


def plan_dict(p: CPlan) -> dict:
    return {k: int(getattr(p, k)) for k, _ in CPlan._fields_}


def autotune(spec: RunSpec, opt: COptions, sample_photons: int = 20_000_000) -> tuple[COptions, dict, float, float]:
    """Autotune the walk's launch and tally-tile plan on a sample of this run (tmc_b200_autotune):
    returns the tuned options (a copy), the chosen plan, and the sample's kernel seconds with the
    planner's default plan and with the chosen one."""
    o = COptions.from_buffer_copy(opt)
    plan, st = CPlan(), CStatus()
    t0, t1 = ctypes.c_double(), ctypes.c_double()
    c = spec.to_c()
    _check(lib().tmc_b200_autotune(ctypes.byref(c), ctypes.byref(o), sample_photons, ctypes.byref(plan),
                                   ctypes.byref(t0), ctypes.byref(t1), ctypes.byref(st)), st)
    return o, plan_dict(plan), t0.value, t1.value


@dataclass
class Estimate:
    mean: float
    se: float


def batch_estimate(sums, photons) -> Estimate:
    """Per-photon mean and its standard error from per-batch sums (src/io/json_out.cpp:37-64)."""
    sums = np.asarray(sums, dtype=np.float64)
    photons = np.asarray(photons, dtype=np.float64)
    mean = float(math.fsum(sums) / photons.sum())
    n = len(sums)
    if n < 2:
        return Estimate(mean, math.nan)
    per = sums / photons
    centre = math.fsum(per) / n
    ss = math.fsum((per - centre) ** 2)
    return Estimate(mean, math.sqrt(ss / (n - 1) / n))


@dataclass
class RunResult:
    """Output of one run, in the reference's layout plus the 2-D tallies (numpy arrays)."""

    spec: RunSpec
    seed: int
    first_photon: np.ndarray
    photons: np.ndarray
    rd: np.ndarray
    tt: np.ndarray
    absorbed: np.ndarray  # (batches, layers)
    events: np.ndarray
    anomalies: np.ndarray
    a_z: np.ndarray
    rd_r: np.ndarray
    tt_r: np.ndarray
    a_rz: np.ndarray  # (nr, nz)
    rd_ra: np.ndarray  # (nr, na)
    tt_ra: np.ndarray  # (nr, na)
    raw: np.ndarray
    specular: float
    kernel_seconds: float
    wall_seconds: float
    device: str
    rung: int = 0
    profiles: bool = True
    extra: dict = field(default_factory=dict)

    def estimate(self, key: str) -> Estimate:
        if key == "absorbed":
            return batch_estimate(self.absorbed.sum(axis=1), self.photons)
        if key == "conservation_residual":
            e = batch_estimate(self.rd + self.tt + self.absorbed.sum(axis=1), self.photons)
            return Estimate(e.mean + self.specular - 1.0, e.se)
        return batch_estimate(getattr(self, key), self.photons)

    def summary(self) -> dict:
        return {k: self.estimate(k).__dict__ for k in ("rd", "tt", "absorbed", "conservation_residual")}

    def to_json(self) -> dict:
        """The result as the reference's JSON run object (src/io/json_out.cpp:164-306) plus the
        2-D arrays."""
        s = self.spec
        return {
            "tissuemc_version": "0.1.0", "engine": "cuda", "precision": "float32", "seed": self.seed,
            "threads": 1, "photons": int(self.photons.sum()), "output_name": s.output_name,
            "n_above": s.n_above, "n_below": s.n_below,
            "layers": [dict(zip(("n", "mua", "mus", "g", "d"), lay, strict=True)) for lay in s.layers],
            "grid": {"dz": s.dz, "dr": s.dr, "nz": s.nz, "nr": s.nr, "na": s.na},
            "specular": self.specular, "wall_seconds": self.wall_seconds,
            "kernel_seconds": self.kernel_seconds, "device": self.device,
            "tally_precision": "fixed64", "rung": self.rung, "profiles": self.profiles,
            "events": int(self.events.sum()), "anomalies": int(self.anomalies.sum()),
            "summary": self.summary(),
            "batches": [
                {"first_photon": int(self.first_photon[b]), "photons": int(self.photons[b]),
                 "rd": float(self.rd[b]), "tt": float(self.tt[b]),
                 "absorbed": [float(v) for v in self.absorbed[b]], "events": int(self.events[b]),
                 "anomalies": int(self.anomalies[b])}
                for b in range(len(self.rd))
            ],
            "a_z": self.a_z.tolist(), "rd_r": self.rd_r.tolist(), "tt_r": self.tt_r.tolist(),
            "a_rz": self.a_rz.tolist(), "rd_ra": self.rd_ra.tolist(), "tt_ra": self.tt_ra.tolist(),
        }  # fmt: skip


def available() -> bool:
    return bool(lib().tmc_b200_available())


def query_sizes(spec: RunSpec, opt: COptions) -> CSizes:
    sz, st = CSizes(), CStatus()
    c = spec.to_c()
    _check(lib().tmc_b200_query_sizes(ctypes.byref(c), ctypes.byref(opt), ctypes.byref(sz), ctypes.byref(st)), st)
    return sz


def _alloc_result(sz: CSizes):
    b, nz, nr, na = int(sz.batches), int(sz.nz), int(sz.nr), int(sz.na)
    arrs = {
        "first_photon": np.zeros(b, np.uint64), "photons": np.zeros(b, np.uint64),
        "rd": np.zeros(b), "tt": np.zeros(b), "absorbed": np.zeros((b, int(sz.layers))),
        "events": np.zeros(b, np.uint64), "anomalies": np.zeros(b, np.uint64),
        "a_z": np.zeros(nz), "rd_r": np.zeros(nr), "tt_r": np.zeros(nr),
        "a_rz": np.zeros((nr, nz)), "rd_ra": np.zeros((nr, na)), "tt_ra": np.zeros((nr, na)),
        "raw": np.zeros(int(sz.tally_words), np.uint64),
    }  # fmt: skip
    res = CResult()
    for k, a in arrs.items():
        ct = ctypes.c_uint64 if a.dtype == np.uint64 else ctypes.c_double
        setattr(res, k, a.ctypes.data_as(ctypes.POINTER(ct)))
    return arrs, res


def run(spec: RunSpec, opt: COptions | None = None, **kw) -> RunResult:
    """Run the photon walk on the GPU (the reference's run_cuda). Keyword arguments build the
    options when `opt` is not given (see `options`)."""
    if opt is None:
        opt = options(**kw)
    sz = query_sizes(spec, opt)
    arrs, res = _alloc_result(sz)
    st = CStatus()
    c = spec.to_c()
    _check(lib().tmc_b200_run(ctypes.byref(c), ctypes.byref(opt), ctypes.byref(res), ctypes.byref(st)), st)
    return RunResult(spec=spec, seed=opt.seed, specular=res.specular, kernel_seconds=res.kernel_seconds,
                     wall_seconds=res.wall_seconds, device=res.device.decode(), rung=opt.rung,
                     profiles=bool(opt.profiles), **arrs)


STATIC_SCRATCH_WORDS = 65536


def run_static(spec: RunSpec, opt: COptions | None = None, **kw) -> RunResult:
    """Run the walk through the allocation-free entry point (tmc_b200_run_static): the library
    allocates nothing; its scratch is a static device array of STATIC_SCRATCH_WORDS tally words."""
    if opt is None:
        opt = options(**kw)
    sz = query_sizes(spec, opt)
    arrs, res = _alloc_result(sz)
    st = CStatus()
    c = spec.to_c()
    _check(lib().tmc_b200_run_static(ctypes.byref(c), ctypes.byref(opt), ctypes.byref(res), ctypes.byref(st)), st)
    return RunResult(spec=spec, seed=opt.seed, specular=res.specular, kernel_seconds=res.kernel_seconds,
                     wall_seconds=res.wall_seconds, device=res.device.decode(), rung=opt.rung,
                     profiles=bool(opt.profiles), **arrs)


def decode(spec: RunSpec, opt: COptions, raw: np.ndarray) -> RunResult:
    """Decode a raw fixed-point tally buffer (from run_device) into a RunResult."""
    sz = query_sizes(spec, opt)
    arrs, res = _alloc_result(sz)
    raw = np.ascontiguousarray(raw, dtype=np.uint64)
    st = CStatus()
    c = spec.to_c()
    _check(lib().tmc_b200_decode(ctypes.byref(c), ctypes.byref(opt),
                                 raw.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                 ctypes.byref(res), ctypes.byref(st)), st)
    return RunResult(spec=spec, seed=opt.seed, specular=res.specular, kernel_seconds=0.0,
                     wall_seconds=0.0, device="", rung=opt.rung, profiles=bool(opt.profiles), **arrs)


def run_device(spec: RunSpec, opt: COptions, d_tally_ptr: int, stream_ptr: int = 0) -> None:
    """Launch the walk into a device buffer of query_sizes(...).device_words words (the tallies,
    then the launch's claim counter) on a stream, without synchronising."""
    st = CStatus()
    c = spec.to_c()
    _check(lib().tmc_b200_run_device(ctypes.byref(c), ctypes.byref(opt), ctypes.c_void_p(d_tally_ptr),
                                     ctypes.c_void_p(stream_ptr), ctypes.byref(st)), st)


def run_device_range(spec: RunSpec, opt: COptions, first_photon: int, count: int, d_tally_ptr: int,
                     stream_ptr: int = 0) -> None:
    """Launch one shard of a run (photons [first_photon, first_photon + count)) into a device buffer
    of device_words words on a stream, without synchronising; the shards of a partition add up to
    the run (their first tally_words words)."""
    st = CStatus()
    c = spec.to_c()
    _check(lib().tmc_b200_run_device_range(ctypes.byref(c), ctypes.byref(opt), first_photon, count,
                                           ctypes.c_void_p(d_tally_ptr), ctypes.c_void_p(stream_ptr),
                                           ctypes.byref(st)), st)


def probe_wait_timeout(wait_limit: int = 4096, device: int = 0) -> tuple[int, str]:
    """Make the tensor-core GEMM kernel's bounded wait run out on purpose (its producer issues no
    loads) and return (status code, message): DEVICE_TIMEOUT when the kernel reported the give-up."""
    st = CStatus()
    rc = lib().tmc_b200_probe_wait_timeout(device, wait_limit, ctypes.byref(st))
    return rc, st.message.decode(errors="replace")


def probe_physics(what: str, g: float, mu_t: float = 10.0, samples: int = 1_000_000, seed: int = 7,
                  fast_math: bool = True, device: int = 0) -> dict:
    """Run the walk's device physics in isolation (tmc_b200_probe_physics): what = "hg"
    (Henyey-Greenstein cosines), "rotate" (consecutive rotations of one direction) or "step"
    (free paths). Returns the sums, extremes and sample count."""
    out = (ctypes.c_double * 5)()
    st = CStatus()
    code = {"hg": 0, "rotate": 1, "step": 2}[what]
    _check(lib().tmc_b200_probe_physics(code, g, mu_t, samples, seed, int(fast_math), device, out,
                                        ctypes.byref(st)), st)
    n = out[4]
    if code == 1:
        return {"worst_norm_error": out[0], "samples": n}
    r = {"mean": out[0] / n, "mean_square": out[1] / n, "samples": n}
    if code == 0:
        r["min"], r["max"] = out[2], out[3]
    return r


def shard_range(photons: int, rank: int, world: int) -> tuple[int, int]:
    """(first photon, count) of rank's contiguous share of a run's photons."""
    first = photons * rank // world
    return first, photons * (rank + 1) // world - first


def plan(spec: RunSpec, opt: COptions, sms: int = 148, smem_sm: int = 233472,
         smem_block_optin: int = 232448, reserved: int = 1024, regs_blocks_per_sm: int = 4) -> CPlan:
    """The launch and shared-memory tile plan the engine would use on a device with these limits
    (pure host code)."""
    p, st = CPlan(), CStatus()
    c = spec.to_c()
    _check(lib().tmc_b200_plan(ctypes.byref(c), ctypes.byref(opt), sms, smem_sm, smem_block_optin,
                               reserved, regs_blocks_per_sm, ctypes.byref(p), ctypes.byref(st)), st)
    return p


def parse_mci(path: str | Path) -> list[RunSpec]:
    """Read an MCML .mci file with the engine's C++ reader (errors carry line numbers)."""
    runs = (CRunSpec * 64)()
    n = ctypes.c_int32(0)
    st = CStatus()
    _check(lib().tmc_b200_parse_mci(str(path).encode(), runs, 64, ctypes.byref(n), ctypes.byref(st)), st)
    if n.value > 64:
        raise ConfigError(f"{path}: more than 64 runs")
    return [RunSpec.from_c(runs[i], name=Path(path).stem + ".mco") for i in range(n.value)]


def write_mco(result: RunResult, path: str | Path) -> None:
    """Write a run as an MCML output file (.mco) with the engine's C++ writer; `read_mco` in
    tissuemc_b200.mco reads it back."""
    opt = options(seed=result.seed, batches=len(result.photons))
    res = CResult()
    keep = {}
    for k in ("first_photon", "photons", "rd", "tt", "absorbed", "events", "anomalies", "a_z", "rd_r", "tt_r",
              "a_rz", "rd_ra", "tt_ra"):
        a = getattr(result, k)
        a = keep[k] = np.ascontiguousarray(a, dtype=np.uint64 if a.dtype == np.uint64 else np.float64)
        ct = ctypes.c_uint64 if a.dtype == np.uint64 else ctypes.c_double
        setattr(res, k, a.ctypes.data_as(ctypes.POINTER(ct)))
    res.specular = result.specular
    res.kernel_seconds = result.kernel_seconds
    res.device = result.device.encode()[:127]
    st = CStatus()
    c = result.spec.to_c()
    _check(lib().tmc_b200_write_mco(ctypes.byref(c), ctypes.byref(opt), ctypes.byref(res), str(path).encode(),
                                    ctypes.byref(st)), st)


def workload(name: str) -> RunSpec:
    """A bundled workload: 'slab_n14' (one slab, 1e6 photons) or 'skin5' (five layers, 1e8)."""
    return parse_mci(CONFIGS / f"{name}.mci")[0]


# ---------------------------------------------------------------------------------- batched sweep
def sweep_options(**kw) -> CSweepOptions:
    """Sweep options (grid shared by every configuration); defaults: nr = nz = 64, dr = dz = 0.01 cm,
    na = 1, 10 batches, fast math, 256 threads, 256 photons per work item."""
    o = CSweepOptions()
    lib().tmc_b200_sweep_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def sweep_sample(master_seed: int, n: int):
    """n configurations of the sweep distribution (1-3 layers, log-uniform optics, 1e4-1e6
    photons, one seed each), as a ctypes array of CSweepConfig."""
    arr = (CSweepConfig * n)()
    st = CStatus()
    _check(lib().tmc_b200_sweep_sample(master_seed, n, arr, ctypes.byref(st)), st)
    return arr



def sweep_costs(cfgs) -> np.ndarray:
    """The estimated steps per photon of each configuration, by which a sweep orders them inside
    its launch (largest first)."""
    arr = cfgs if isinstance(cfgs, ctypes.Array) else (CSweepConfig * len(cfgs))(*cfgs)
    out = np.zeros(len(arr), dtype=np.float64)
    st = CStatus()
    _check(lib().tmc_b200_sweep_costs(arr, len(arr), out.ctypes.data_as(_P(ctypes.c_double)), ctypes.byref(st)), st)
    return out


def sweep_config(spec: RunSpec, photons: int, seed: int) -> CSweepConfig:
    c = CSweepConfig()
    c.photons, c.seed, c.n_above, c.n_below = photons, seed, spec.n_above, spec.n_below
    c.num_layers = len(spec.layers)
    for i, lay in enumerate(spec.layers[:MAX_LAYERS]):
        c.layers[i] = Layer(*map(float, lay))
    return c


def config_spec(c: CSweepConfig, opt: CSweepOptions) -> RunSpec:
    """A sweep configuration as a single run on the sweep's grid."""
    layers = [(c.layers[i].n, c.layers[i].mua, c.layers[i].mus, c.layers[i].g, c.layers[i].d)
              for i in range(c.num_layers)]
    return RunSpec(layers=layers, photons=int(c.photons), dz=opt.dz, dr=opt.dr, nz=opt.nz, nr=opt.nr, na=opt.na,
                   n_above=c.n_above, n_below=c.n_below)


def sweep_sizes(cfgs, opt: CSweepOptions) -> CSweepSizes:
    sz, st = CSweepSizes(), CStatus()
    _check(lib().tmc_b200_sweep_sizes(cfgs, len(cfgs), ctypes.byref(opt), ctypes.byref(sz), ctypes.byref(st)), st)
    return sz


@dataclass
class SweepResult:
    summary: np.ndarray  # (n, nr + 3): R_d(r) per photon, then R_d, T_t, A per photon
    raw: np.ndarray | None  # (n, words_per_config) fixed-point tallies
    seconds: float  # device time of the sweep kernel (or of the whole loop for run_loop)


def sweep_run(cfgs, opt: CSweepOptions | None = None, raw: bool = False) -> SweepResult:
    """Run every configuration in one graph-captured persistent launch."""
    opt = opt or sweep_options()
    sz = sweep_sizes(cfgs, opt)
    n = len(cfgs)
    summary = np.zeros((n, int(sz.summary_per_config)))
    raw_arr = np.zeros((n, int(sz.words_per_config)), np.uint64) if raw else None
    secs = ctypes.c_double(0.0)
    st = CStatus()
    rc = lib().tmc_b200_sweep_run(cfgs, n, ctypes.byref(opt),
                                  raw_arr.ctypes.data_as(_pu) if raw else ctypes.cast(None, _pu),
                                  summary.ctypes.data_as(_pd), ctypes.byref(secs), ctypes.byref(st))
    _check(rc, st)
    return SweepResult(summary, raw_arr, secs.value)


def sweep_run_loop(cfgs, opt: CSweepOptions | None = None, raw: bool = False) -> SweepResult:
    """The baseline: one single-run launch per configuration, back to back on one stream."""
    opt = opt or sweep_options()
    sz = sweep_sizes(cfgs, opt)
    n = len(cfgs)
    raw_arr = np.zeros((n, int(sz.words_per_config)), np.uint64) if raw else None
    secs = ctypes.c_double(0.0)
    st = CStatus()
    rc = lib().tmc_b200_sweep_run_loop(cfgs, n, ctypes.byref(opt),
                                       raw_arr.ctypes.data_as(_pu) if raw else ctypes.cast(None, _pu),
                                       ctypes.byref(secs), ctypes.byref(st))
    _check(rc, st)
    return SweepResult(np.zeros((0, 0)), raw_arr, secs.value)


def sweep_autotune(cfgs, opt: CSweepOptions | None = None) -> tuple[CSweepOptions, float]:
    """Pick the sweep's block size, work-item size and per-warp tile of A(r,z) by timing candidates
    on these configurations."""
    opt = opt or sweep_options()
    best = ctypes.c_double(0.0)
    st = CStatus()
    _check(lib().tmc_b200_sweep_autotune(cfgs, len(cfgs), ctypes.byref(opt), ctypes.byref(best), ctypes.byref(st)), st)
    return opt, best.value


def gemm_bf16(A, B, bias=None, out=None):
    """D = A @ B.T (+ bias) on the tcgen05 tensor cores for torch CUDA tensors (A: M x K bf16,
    B: N x K bf16, K a multiple of 64); returns a float32 tensor."""
    import torch

    M, K = A.shape
    N = B.shape[0]
    assert A.dtype == torch.bfloat16 and B.dtype == torch.bfloat16 and B.shape[1] == K
    A, B = A.contiguous(), B.contiguous()
    D = out if out is not None else torch.empty((M, N), dtype=torch.float32, device=A.device)
    st = CStatus()
    rc = lib().tmc_b200_gemm_bf16(A.data_ptr(), B.data_ptr(), bias.data_ptr() if bias is not None else None,
                                  D.data_ptr(), M, N, K, torch.cuda.current_stream().cuda_stream, ctypes.byref(st))
    _check(rc, st)
    return D
