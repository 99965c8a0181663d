"""Build the C++ restatement of the oracle (oracle/mhd_oracle.cpp) into
oracle/_build/libmhd_oracle.so -- TEST INFRASTRUCTURE ONLY.

Flags: -O2 -ffp-contract=off (no FMA contraction), so every FP64 operation is
one IEEE-754 operation, as in the reference build.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "mhd_oracle.cpp"
LIB = HERE / "_build" / "libmhd_oracle.so"


def build(force: bool = False) -> Path:
    LIB.parent.mkdir(exist_ok=True)
    if force or not LIB.exists() or LIB.stat().st_mtime < max(SRC.stat().st_mtime, Path(__file__).stat().st_mtime):
        subprocess.run(["g++", "-O2", "-ffp-contract=off", "-std=c++17", "-fPIC", "-shared", "-o", str(LIB),
                        str(SRC)], check=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
