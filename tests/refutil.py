"""Helpers shared by the tests: the raw state format written by the oracle
drivers, and running the reference CPU path built in oracle/_ref/."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
REF_DIR = ROOT / "oracle" / "_ref"
RAW_MAGIC = 0x41544842


def read_raw(path) -> dict:
    """Read a raw state file (format in oracle/ref_harness.c)."""
    b = Path(path).read_bytes()
    hdr = np.frombuffer(b, dtype="<i4", count=6)
    assert hdr[0] == RAW_MAGIC, "bad magic"
    nx1, nx2, ng, nstep = (int(x) for x in hdr[2:6])
    dh = np.frombuffer(b, dtype="<f8", count=6, offset=24)
    sx, sy = nx1 + 2 * ng, nx2 + 2 * ng
    planes = np.frombuffer(b, dtype="<f8", offset=72, count=11 * sx * sy).reshape(11, sy, sx).copy()
    return {"nx1": nx1, "nx2": nx2, "nstep": nstep, "dt": float(dh[0]), "time": float(dh[1]),
            "dx1": float(dh[2]), "dx2": float(dh[3]), "planes": planes}


def write_raw(path, planes: np.ndarray, nstep=0, dt=0.0, time=0.0, dx=(0.0, 0.0), x0=(0.0, 0.0)) -> Path:
    """Write a raw state file (used to feed an arbitrary initial state to the
    reference's 'file' problem build)."""
    _, sy, sx = planes.shape
    hdr = np.array([RAW_MAGIC, 1, sx - 8, sy - 8, 4, nstep], dtype="<i4")
    dh = np.array([dt, time, dx[0], dx[1], x0[0], x0[1]], dtype="<f8")
    Path(path).write_bytes(hdr.tobytes() + dh.tobytes() + np.ascontiguousarray(planes, "<f8").tobytes())
    return Path(path)


def reference_root() -> Path | None:
    """The reference source tree ($ATHENA_REF, else ``reference`` beside the
    repository), or None where it is absent (CPU-side checks only)."""
    import os
    env = os.environ.get("ATHENA_REF")
    p = Path(env) if env else ROOT.parent / "reference"
    return p if p.is_dir() else None


def ref_binary(problem: str, flux: str = "roe") -> Path:
    return REF_DIR / f"athref_{problem}_{flux}"


def have_ref(problem: str = "blast", flux: str = "roe") -> bool:
    return ref_binary(problem, flux).exists()


def run_ref(problem: str, flux: str, athinput, workdir, steps: int | None = None,
            init=None, exe: Path | None = None, extra=()) -> dict:
    """Run the reference CPU path and return its final raw state."""
    exe = exe or ref_binary(problem, flux)
    out = Path(workdir) / f"ref_{problem}_{flux}.bin"
    cmd = [str(exe), "-i", str(athinput), "--dump", str(out), *extra]
    if steps is not None:
        cmd += ["--steps", str(steps)]
    if init is not None:
        cmd += ["--init", str(init)]
    subprocess.run(cmd, check=True, capture_output=True, cwd=workdir)
    return read_raw(out)


def mismatch_report(a: np.ndarray, b: np.ndarray, names) -> str:
    """First differing cells per plane (for assertion messages)."""
    lines = []
    for k in range(a.shape[0]):
        bad = np.argwhere(~((a[k] == b[k]) | (np.isnan(a[k]) & np.isnan(b[k]))))
        if len(bad):
            j, i = bad[0]
            lines.append(f"{names[k]}: {len(bad)} cells differ, first (j={j}, i={i}) "
                         f"{a[k][j, i]!r} vs {b[k][j, i]!r}")
    return "\n".join(lines)


def random_state(rng, nx1, nx2, smooth: bool) -> np.ndarray:
    """A random, divergence-free, positive state (periodic) in the raw layout."""
    sx, sy = nx1 + 8, nx2 + 8
    P = np.zeros((11, sy, sx))

    def field(lo, hi):
        x = rng.uniform(lo, hi, size=(sy, sx))
        if smooth:
            for _ in range(4):
                x = 0.25 * (np.roll(x, 1, 0) + np.roll(x, -1, 0) + np.roll(x, 1, 1) + np.roll(x, -1, 1))
        return x

    d = field(0.3, 2.0)
    v1, v2, v3 = field(-1.5, 1.5), field(-1.5, 1.5), field(-0.5, 0.5)
    p = field(0.02, 1.0)
    # face fields from a vector potential so that div B = 0 to round-off
    az = field(-0.05, 0.05)
    b1i = np.zeros((sy, sx)); b2i = np.zeros((sy, sx))
    b1i[:-1, :] = (az[1:, :] - az[:-1, :]) * 20.0
    b2i[:, :-1] = -(az[:, 1:] - az[:, :-1]) * 20.0
    b3i = field(-0.3, 0.3)
    b1c = np.zeros((sy, sx)); b2c = np.zeros((sy, sx))
    b1c[:, :-1] = 0.5 * (b1i[:, :-1] + b1i[:, 1:])
    b2c[:-1, :] = 0.5 * (b2i[:-1, :] + b2i[1:, :])
    from athena_cuda_b200 import configs

    g1 = configs.GAMMA - 1.0
    e = p / g1 + 0.5 * d * (v1 * v1 + v2 * v2 + v3 * v3) + 0.5 * (b1c * b1c + b2c * b2c + b3i * b3i)
    for k, a in enumerate([d, d * v1, d * v2, d * v3, e, b1c, b2c, b3i, b1i, b2i, b3i]):
        P[k] = a
    return P
