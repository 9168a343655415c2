"""Build the B200 engine in-tree: libtissuemc_b200.so (CUDA kernels + C ABI + C++ host code) and
the `tissuemc` CLI, both for sm_100a only.

    python -m tissuemc_b200.build          # or: python tissuemc_b200/build.py

Objects go to tissuemc_b200/_build/; the library to tissuemc_b200/libtissuemc_b200.so and the CLI
to tissuemc_b200/bin/tissuemc (linked with an $ORIGIN rpath). Rebuilds only what changed.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libtissuemc_b200.so"
CLI = PKG / "bin" / "tissuemc"
DIGEST = PKG / "bin" / "ncu_digest"  # Nsight Compute CSV digest (host tool, no CUDA)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr", *ARCH]
CXX_FLAGS = ["-std=c++17", "-O3", "-fPIC", "-Wall", "-Wextra", "-fvisibility=hidden"]

# The shared library: kernels, C ABI and the C++ it needs (exports only the C ABI).
CUDA_SOURCES = ["engine.cu", "sweep.cu", "mlp.cu", "probe.cu"]
HOST_SOURCES = ["host/engine_host.cpp", "host/mci.cpp", "host/abi_mci.cpp", "host/mco.cpp"]
# The CLI: the reference-shaped C++ host code, linked against the library's C ABI.
CLI_SOURCES = ["host/cli.cpp", "host/run_cuda.cpp", "host/result.cpp", "host/mci.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the B200 engine needs the CUDA toolkit to build")


def _headers() -> list[Path]:
    return sorted(CSRC.rglob("*.cuh")) + sorted(CSRC.rglob("*.hpp")) + [ROOT / "include" / "tissuemc_b200.h"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")


def build(verbose: bool = False) -> Path:
    nvcc = _nvcc()
    cxx = os.environ.get("CXX", "g++")
    BUILD.mkdir(exist_ok=True)
    CLI.parent.mkdir(exist_ok=True)
    hdrs = _headers()
    objs: list[Path] = []
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = BUILD / (Path(src).stem + "_cu.o")
        if _stale(o, [s, *hdrs]):
            if verbose:
                print("nvcc", src)
            _run([nvcc, *NVCC_FLAGS, "-c", str(s), "-o", str(o)])
        objs.append(o)
    for src in HOST_SOURCES:
        s = CSRC / src
        o = BUILD / (Path(src).stem + ".o")
        if _stale(o, [s, *hdrs]):
            if verbose:
                print("c++", src)
            _run([cxx, *CXX_FLAGS, "-c", str(s), "-o", str(o)])
        objs.append(o)
    if _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-Xlinker", "-soname=libtissuemc_b200.so"])
    cli_srcs = [CSRC / s for s in CLI_SOURCES]
    if _stale(CLI, [*cli_srcs, LIB, *hdrs]):
        _run([cxx, *[f for f in CXX_FLAGS if f != "-fvisibility=hidden"], *map(str, cli_srcs), "-o", str(CLI),
              f"-L{PKG}", "-ltissuemc_b200", "-Wl,-rpath,$ORIGIN/..", "-pthread"])
    dsrc = CSRC / "host" / "ncu_digest.cpp"
    if _stale(DIGEST, [dsrc]):
        _run([cxx, *[f for f in CXX_FLAGS if f != "-fvisibility=hidden"], str(dsrc), "-o", str(DIGEST)])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
