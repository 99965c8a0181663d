"""Build recipe for oracle/_ref/ -- TEST INFRASTRUCTURE ONLY.

Compiles the reference's own CPU path, unmodified, from the sources where they
lie (``<reference>/src``) together with ``oracle/ref_harness.c`` (a replacement
for src/main.c only).  Nothing is copied out of the reference tree; objects and
binaries go to ``oracle/_ref/`` (git-ignored; it still travels to GPU boxes).

Builds, per problem generator and flux:

* ``athref_{blast,field_loop,cpaw2d,file,userbc}_{roe,hlle}``: the reference CPU
  step (``userbc``: oracle/userbc_problem.c, a user boundary condition set
  through ``set_bvals_fun``).
  ``roe`` is the reference as shipped (``__integrate_2d__.c`` always calls
  ``flux_roe``, ``__integrate_2d__.c:178,238,444,461``); ``hlle`` recompiles
  ``__integrate_2d__.c`` alone with ``-Dflux_roe=flux_hlle``.
* ``athdrop_{blast,field_loop,cpaw2d,file}``: the same harness and the
  reference's host-side files (``init_grid.c``, ``par.c``, the problem file)
  linked against ``libathena_b200.so`` instead of the reference's integrator,
  boundary and dt sources -- the drop-in test (only when the library exists).
* ``palettes.txt``: the colour tables of ``src/palette.h`` as text, written by
  ``oracle/palette_dump.c`` (the palette file of the ppm parity tests).
* ``athmain_{blast,field_loop,cpaw2d}``: the reference's own ``src/main.c``
  with its output code (``output.c``, ``dump_binary.c``, ``dump_tab.c`` ...),
  the program whose output files the command-line driver must reproduce;
  ``oracle/ref_stubs.c`` supplies ``dt_destruct``, which ``main.c`` calls and
  only the reference's CUDA engine defines.

Flags: ``-O2 -ffp-contract=off`` (no FMA contraction, so every ``+ - * /`` and
``sqrt`` is one IEEE-754 binary64 operation).  The reference's own Debug flags
are ``-O0 -mpc64`` (src/Debug/subdir.mk:130); ``-mpc64`` only affects x87 and
x86-64 uses SSE2 for double, so results are identical; ``-O0`` is ~3x slower.

Usage: ``python oracle/build_ref.py [--ref <reference root>] [--force]``; the
reference root defaults to ``$ATHENA_REF``, else ``../reference`` beside the
repository.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"


def default_reference() -> Path:
    """The reference checkout: $ATHENA_REF, else a ``reference`` directory
    beside this repository."""
    env = os.environ.get("ATHENA_REF")
    return Path(env) if env else HERE.parent.parent / "reference"


DEFAULT_REF = default_reference()

# Reference CPU sources on the step path (plus host glue they need to link).
CORE = [
    "ath_array.c", "ath_log.c", "cc_pos.c", "convert_var.c", "esystem_prim.c",
    "esystem_roe.c", "flux_hlle.c", "flux_roe.c", "init_grid.c",
    "lr_states_plm.c", "new_dt.c", "par.c", "set_bvals.c", "utils.c",
]
# Host-side files kept by the drop-in build (the integrator, boundary and dt
# sources are replaced by libathena_b200.so).
DROPIN_HOST = ["ath_array.c", "ath_log.c", "cc_pos.c", "init_grid.c", "par.c", "utils.c"]
PROBLEMS = {
    "blast": ("blast.c", ["-DBLAST_PROBLEM"]),
    "field_loop": ("field_loop.c", []),  # FIELD_LOOP is defined by debug_tools_cuda.h:73
    "cpaw2d": ("cpaw2d.c", ["-DCPAW2D"]),
    "file": (None, ["-DHARNESS_FILE_PROBLEM"]),
    # a user boundary condition registered through set_bvals_fun (test problem
    # of this directory, not a reference file)
    "userbc": (HERE / "userbc_problem.c", []),
}
# The reference's main program and its output path (athmain_*).
MAIN_EXTRA = [
    "main.c", "ath_files.c", "debug_tools_cuda.c", "dump_binary.c", "dump_tab.c", "output.c",
    "output_ppm.c", "output_tab.c", "show_config.c", "utils_cu.c",
]
# ath_array.c:calloc_*_array_cu call cudaMalloc (never reached on this path),
# so the CUDA runtime is linked only to resolve those symbols.
LDCUDA = ["-L/usr/local/cuda/lib64", "-Wl,-rpath,/usr/local/cuda/lib64", "-lcudart"]
CFLAGS = ["-O2", "-ffp-contract=off", "-DONLY_HOST", "-w", "-std=gnu99"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"command failed: {cmd[0]} ... ({r.returncode})")


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(d.stat().st_mtime <= t for d in deps if d.exists())


def _cc(src: Path, obj: Path, extra: list[str], inc: list[str], force: bool) -> Path:
    if force or not _newer(obj, [src, HERE / "build_ref.py"]):
        _run(["gcc", *CFLAGS, *extra, *inc, "-c", str(src), "-o", str(obj)])
    return obj


def build(ref_root: Path = DEFAULT_REF, force: bool = False, lib: Path | None = None) -> list[Path]:
    src = ref_root / "src"
    if not (src / "__integrate_2d__.c").exists():
        raise FileNotFoundError(f"reference sources not found under {src}")
    OUT.mkdir(exist_ok=True)
    obj = OUT / "obj"
    obj.mkdir(exist_ok=True)
    inc = [f"-I{src}", "-I/usr/local/cuda/include"]
    core = [_cc(src / f, obj / (f[:-2] + ".o"), [], inc, force) for f in CORE]
    integ = {
        "roe": _cc(src / "__integrate_2d__.c", obj / "integrate_roe.o", [], inc, force),
        "hlle": _cc(src / "__integrate_2d__.c", obj / "integrate_hlle.o",
                    ["-Dflux_roe=flux_hlle"], inc, force),
    }
    built = []
    pal = OUT / "palettes.txt"
    pexe = obj / "palette_dump"
    if force or not _newer(pal, [HERE / "palette_dump.c", src / "palette.h", HERE / "build_ref.py"]):
        _run(["gcc", *CFLAGS, *inc, str(HERE / "palette_dump.c"), "-o", str(pexe)])
        r = subprocess.run([str(pexe)], capture_output=True, text=True, check=True)
        pal.write_text(r.stdout)
    built.append(pal)
    for prob, (pfile, pdefs) in PROBLEMS.items():
        harness = _cc(HERE / "ref_harness.c", obj / f"harness_{prob}.o", pdefs, inc, force)
        pobj = [] if pfile is None else [_cc(src / pfile, obj / f"prob_{prob}.o", pdefs, inc, force)]  # src / absolute = absolute
        for flux, iobj in integ.items():
            exe = OUT / f"athref_{prob}_{flux}"
            deps = [harness, iobj, *core, *pobj]
            if force or not _newer(exe, deps):
                _run(["gcc", "-o", str(exe), *map(str, deps), *LDCUDA, "-lm"])
            built.append(exe)
        if pfile is not None and not Path(pfile).is_absolute():
            mobj = [_cc(src / f, obj / f"main_{prob}_{f[:-2]}.o", pdefs, inc, force) for f in MAIN_EXTRA]
            stub = _cc(HERE / "ref_stubs.c", obj / "ref_stubs.o", [], inc, force)
            exe = OUT / f"athmain_{prob}"
            deps = [*mobj, stub, integ["roe"], *core, *pobj]
            if force or not _newer(exe, deps):
                _run(["gcc", "-o", str(exe), *map(str, deps), *LDCUDA, "-lm"])
            built.append(exe)
        if lib is not None and lib.exists():
            host = [obj / (f[:-2] + ".o") for f in DROPIN_HOST]
            exe = OUT / f"athdrop_{prob}"
            deps = [harness, *host, *pobj]
            if force or not _newer(exe, deps + [lib]):
                _run(["gcc", "-o", str(exe), *map(str, deps), str(lib),
                      f"-Wl,-rpath,{lib.parent}", *LDCUDA, "-lm"])
            built.append(exe)
    return built


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=str(DEFAULT_REF))
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--lib", default=str(HERE.parent / "athena_cuda_b200" / "libathena_b200.so"))
    a = ap.parse_args()
    for p in build(Path(a.ref), a.force, Path(a.lib)):
        print(p)


if __name__ == "__main__":
    main()
