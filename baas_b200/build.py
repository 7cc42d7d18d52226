"""In-tree build of the CUDA library (sm_100a) and of the oracle checkers.

``python -m baas_b200.build`` compiles ``baas_b200/_lib/libbaas_b200.so`` with nvcc (cross
compilation works without a GPU). The oracle libraries (``oracle/_lib``, ``oracle/_ref``) are
built by ``oracle/Makefile``; the reference one only when the reference tree is present.
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
LIB_DIR = PKG / "_lib"
LIB = LIB_DIR / "libbaas_b200.so"
# the bounds-checked variant (-DBAAS_DEBUG_BOUNDS): kernels record an out-of-range index in the
# status word instead of touching memory outside an array; loaded when BAAS_LIB=bounds
LIB_BOUNDS = LIB_DIR / "libbaas_b200_bounds.so"
SOURCES = ["capi.cu", "analysis.cu", "schedule.cpp", "mtx.cpp"]
HEADERS = ["kernels.cuh", "part_kernels.cuh", "staged.cuh", "fetch.cuh", "batched.cuh", "small.cuh", "device_common.cuh",
           "schedule.hpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> list[str]:
    # the system g++ (an environment CXX wrapper may lack parts of the toolchain)
    return ["-ccbin", "/usr/bin/g++"] if Path("/usr/bin/g++").exists() else []


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_lib(force: bool = False, verbose: bool = False, bounds: bool = False) -> Path:
    target = LIB_BOUNDS if bounds else LIB
    deps = [CSRC / s for s in SOURCES] + [CSRC / h for h in HEADERS] + [ROOT / "include" / "baas_b200.h"]
    if not force and not _stale(target, deps):
        return target
    LIB_DIR.mkdir(exist_ok=True)
    cmd = [_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-ffp-contract=off", *_host_cxx(), "-o", str(target)]
    if bounds:
        cmd.append("-DBAAS_DEBUG_BOUNDS")
    cmd += [str(CSRC / s) for s in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return target


def reference_tree():
    """The reference's source tree: $BAAS_REFERENCE, else a `reference` directory beside this
    repository; None when neither exists (the reference-built checker is then skipped)."""
    cand = os.environ.get("BAAS_REFERENCE") or str(ROOT.parent / "reference")
    return Path(cand) if Path(cand).is_dir() else None


def build_oracle(verbose: bool = False) -> None:
    mk = ["make", "-s", "-C", str(ROOT / "oracle")]
    subprocess.run(mk + ["oracle"], check=True)
    ref = reference_tree()
    if ref is not None:
        subprocess.run(mk + ["ref", f"REF={ref}"], check=True)


if __name__ == "__main__":
    if "--debug-bounds" in sys.argv:
        print(build_lib(force="--force" in sys.argv, verbose="-v" in sys.argv, bounds=True))
    else:
        build_lib(force="--force" in sys.argv, verbose="-v" in sys.argv)
        build_oracle()
        print(LIB)
