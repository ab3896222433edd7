"""Build recipe for the native parts of the package.

* ``lib/libcufhe_client.so`` -- CPU client library (key generation,
  encryption, decryption) in C.
* ``lib/libcufhe_b200.so``   -- the gate engine: the C-ABI of
  ``include/cufhe_b200.h`` over hand-written sm_100a CUDA kernels.

Both are built in-tree so that they travel with the repository.  nvcc
cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]

ENGINE_SOURCES = [
    "engine.cu",
    "keyswitch.cu",
    "iks_tc.cu",
    "br_fp64.cu",
    "br_int8.cu",
    "gates_misc.cu",
    "peaks.cu",
    "noalloc.cu",
    "br_fp64_lvl02.cu",
    "cb.cu",
    "br_int8_lvl02.cu",
]


def _run(cmd: list[str], cwd: Path | None = None) -> None:
    proc = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if os.environ.get("CUFHE_BUILD_VERBOSE"):
        sys.stderr.write(proc.stdout + proc.stderr)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_client(force: bool = False) -> Path:
    LIB.mkdir(exist_ok=True)
    out = LIB / "libcufhe_client.so"
    src = CSRC / "client" / "tfhe_client.c"
    if force or _stale(out, [src, CSRC / "params.h"]):
        _run(["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-std=c11",
              "-Wall", "-shared", "-o", str(out), str(src), "-lm"])
    return out


def build_engine(force: bool = False, extra: list[str] | None = None) -> Path:
    LIB.mkdir(exist_ok=True)
    out = LIB / "libcufhe_b200.so"
    srcs = [CSRC / s for s in ENGINE_SOURCES]
    deps = srcs + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [
        ROOT / "include" / "cufhe_b200.h"]
    if not (force or _stale(out, deps)):
        return out
    objdir = LIB / "_obj"
    objdir.mkdir(exist_ok=True)
    common = [NVCC, *GENCODE, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-I", str(CSRC), "-I", str(ROOT / "include"), "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"] + (extra or [])
    objs = []
    for s in srcs:
        o = objdir / (s.stem + ".o")
        _run(common + ["-c", str(s), "-o", str(o)])
        objs.append(str(o))
    _run([NVCC, *GENCODE, "-shared", "-cudart", "static", "-o", str(out), *objs])
    return out


def ptxas_report(src: str) -> str:
    """Registers / spills / shared memory of one engine source (-Xptxas -v)."""
    proc = subprocess.run(
        [NVCC, *GENCODE, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(CSRC), "-I",
         str(ROOT / "include"), "--expt-relaxed-constexpr", "-Xptxas", "-v", "-c",
         str(CSRC / src), "-o", os.devnull], capture_output=True, text=True)
    return proc.stdout + proc.stderr


def build_all(force: bool = False) -> None:
    build_client(force)
    build_engine(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", LIB)
