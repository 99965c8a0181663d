"""Build the host-CPU checks of the adjoint (TEST INFRASTRUCTURE): the
per-function dot-product program and the ctypes library that runs the
generic step, the tangent-linear model and the adjoint of the main loop on
the CPU.  Outputs go to tests/_build/ (git-ignored)."""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
OUT = ROOT / "tests" / "_build"
CSRC = ROOT / "athena_cuda_b200" / "csrc"
# ATHB_HOST_BOUNDS: every plane access of the step / adjoint items is checked
# to stay inside its plane, so the kernels' index ranges are verified here
FLAGS = ["-O2", "-std=c++17", "-ffp-contract=off", "-Wall", "-Wno-unused-function", "-Wno-unknown-pragmas",
         "-DATHB_HOST_BOUNDS"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _deps(src: Path):
    return [src, *sorted(CSRC.glob("*.cuh")), ROOT / "include" / "athena_b200.h", Path(__file__)]


def build() -> dict:
    OUT.mkdir(parents=True, exist_ok=True)
    pieces = OUT / "adjoint_pieces"
    src = HERE / "adjoint_pieces.cpp"
    if _stale(pieces, _deps(src)):
        subprocess.run(["g++", *FLAGS, "-o", str(pieces), str(src)], check=True)
    lib = OUT / "libathb_hostcheck.so"
    src = HERE / "adjoint_host.cpp"
    if _stale(lib, _deps(src)):
        subprocess.run(["g++", *FLAGS, "-shared", "-fPIC", "-o", str(lib), str(src)], check=True)
    return {"pieces": pieces, "lib": lib}


if __name__ == "__main__":
    print(build())
