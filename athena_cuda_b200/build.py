"""Build libathena_b200.so in-tree for sm_100a (B200).

Device code is compiled with ``--fmad=false`` so that no multiply-add is fused:
every FP64 ``+ - * /`` and ``sqrt`` is one correctly rounded IEEE-754 operation,
which is what makes the GPU step bit-identical to the reference CPU path.

Usage: ``python -m athena_cuda_b200.build [--force] [--verbose]``
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libathena_b200.so"
EXE = PKG / "athena_b200"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_HOME = Path(NVCC).resolve().parent.parent
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
    "-Xptxas", "-O3", f"-I{ROOT / 'include'}",
]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", f"-I{ROOT / 'include'}",
             f"-I{CUDA_HOME / 'include'}"]

CU_SOURCES = ["athb_core.cu", "athb_dropin.cu", "athb_batch.cu", "athb_noalloc.cu", "athb_output.cu", "athb_adjoint.cu",
              "athb_problems_dev.cu", "athb_slab.cu"]
CPP_SOURCES = ["athinput.cpp", "problems.cpp"]
HEADERS = ["dual.cuh", "mhd_physics.cuh", "step_types.cuh", "step_kernels.cuh", "athb_internal.h", "mhd_adjoint.cuh",
           "step_generic.cuh", "step_adjoint.cuh", "adjoint_driver.cuh"]


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    return r.stdout + r.stderr


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False,
          defines: list[str] = (), lib: Path | None = None, obj: Path | None = None) -> Path:
    global OBJ
    lib = lib or LIB
    OBJ = obj or OBJ
    OBJ.mkdir(exist_ok=True, parents=True)
    hdrs = [CSRC / h for h in HEADERS] + [ROOT / "include" / "athena_b200.h", Path(__file__)]
    objs = []
    for src in CU_SOURCES:
        o = OBJ / (src + ".o")
        if force or ptxas_info or _stale(o, [CSRC / src] + hdrs):
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            out = _run([NVCC, *NVCC_FLAGS, *[f"-D{d}" for d in defines], *extra, "-c", str(CSRC / src),
                        "-o", str(o)], verbose)
            if ptxas_info:
                print(out)
        objs.append(o)
    for src in CPP_SOURCES:
        o = OBJ / (src + ".o")
        if force or _stale(o, [CSRC / src] + hdrs):
            _run(["g++", *CXX_FLAGS, "-c", str(CSRC / src), "-o", str(o)], verbose)
        objs.append(o)
    if force or _stale(lib, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-lcudart"], verbose)
    if lib == LIB:  # the command-line driver, next to the library it links
        if force or _stale(EXE, [CSRC / "athena_main.cpp", lib] + hdrs):
            _run(["g++", *CXX_FLAGS, "-o", str(EXE), str(CSRC / "athena_main.cpp"), f"-L{PKG}", "-lathena_b200",
                  "-Wl,-rpath,$ORIGIN"], verbose)
    return lib


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills per kernel")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas_info))


if __name__ == "__main__":
    main()
