"""The command-line driver against the reference's own main program
(src/main.c with its output code, built into oracle/_ref/athmain_*): the same
athinput file and command-line overrides must give the same cycle lines and
byte-identical bin and tab dumps (src/dump_binary.c, src/dump_tab.c) and ppm
images of single-variable expressions (src/output_ppm.c, src/output.c), with
the per-cycle loop and with the device loop that stops only for outputs (-q).
The ppm palettes come from oracle/_ref/palettes.txt (the reference's
palette.h tables as text)."""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

import pytest

import refutil
from athena_cuda_b200 import configs, write_athinput

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "athena_cuda_b200" / "athena_b200"


def _outputs(blocks: dict, specs: list[dict]) -> dict:
    blocks["job"]["maxout"] = len(specs)
    for n, spec in enumerate(specs, 1):
        blocks[f"output{n}"] = dict(spec)
    return blocks


CASES = [
    # output intervals shorter than a step fall behind by one per step, as in
    # the reference; two tab outputs write the same file name in block order
    ("field_loop", configs.field_loop(32, 16, tlim=0.06),
     [{"out_fmt": "bin", "dt": 0.01}, {"out_fmt": "tab", "dt": 0.02},
      {"out_fmt": "tab", "dt": 0.001, "dat_fmt": "%14.6e"}], ["time/tlim=0.05"]),
    ("blast", configs.blast(40, 60, tlim=0.02, bc=(2, 2, 1, 1)),
     [{"out_fmt": "bin", "dt": 0.004, "time": 0.002}, {"out_fmt": "tab", "dt": 0.005, "num": 3}], []),
    ("cpaw2d", configs.cpaw2d(32, 16, tlim=0.1),
     [{"out_fmt": "tab", "dt": 0.03}, {"out_fmt": "bin", "dt": 0.05}], ["grid/Nx1=24"]),
]


def _files(d: Path) -> dict:
    return {p.name: p.read_bytes() for p in sorted(d.iterdir()) if p.suffix in (".bin", ".tab", ".ppm")}


def _cycles(text: str) -> list[str]:
    return [l for l in text.splitlines() if l.startswith("cycle=")]


PALETTES = refutil.REF_DIR / "palettes.txt"


def _run_both(problem, ath, overrides, tmp_path, rc=0) -> dict:
    ref_exe = refutil.REF_DIR / f"athmain_{problem}"
    if not ref_exe.exists() or not PALETTES.exists():
        pytest.skip("reference main program not built (python oracle/build_ref.py)")
    env = dict(os.environ, ATHB_PALETTES=str(PALETTES))
    runs = {}
    for name, cmd in {
        "ref": [str(ref_exe), "-i", str(ath), *overrides],
        "ours": [str(EXE), "-i", str(ath), "-p", problem, *overrides],
        "ours_q": [str(EXE), "-i", str(ath), "-p", problem, "-q", *overrides],
    }.items():
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=300, env=env)
        assert (r.returncode == 0) == (rc == 0), (name, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
        runs[name] = (r.stdout, _files(d), r.stderr)
    return runs


@pytest.mark.parametrize("problem,blocks,outputs,overrides", CASES, ids=[c[0] for c in CASES])
def test_cli_matches_reference_main(problem, blocks, outputs, overrides, tmp_path):
    ath = write_athinput(tmp_path / "athinput", _outputs(blocks, outputs))
    runs = _run_both(problem, ath, overrides, tmp_path)
    _same(runs)


def _same(runs):
    ref_out, ref_files = runs["ref"][0], runs["ref"][1]
    assert ref_files, "the reference wrote no dumps"
    assert _cycles(runs["ours"][0]) == _cycles(ref_out)
    assert _cycles(runs["ours_q"][0])[-1] == _cycles(ref_out)[-1]
    for name in ("ours", "ours_q"):
        files = runs[name][1]
        assert sorted(files) == sorted(ref_files), name
        for f, data in ref_files.items():
            assert files[f] == data, f"{name}: {f} differs from the reference's"


PPM_CASES = [
    # every expression of src/output.c and the field loop's J3 / Bp2, every
    # palette, fixed scales, a running gmin/gmax from num = 2, ids, and
    # expressions that do not parse (skipped, as in the reference)
    ("field_loop", configs.field_loop(32, 16, tlim=0.05),
     [{"out_fmt": "ppm", "out": "d", "dt": 0.01},
      {"out_fmt": "ppm", "out": "J3", "usr_expr_flag": 1, "palette": "heat", "dt": 0.015, "id": "cur"},
      {"out_fmt": "ppm", "out": "ME", "dmin": 0.0, "dmax": 1e-6, "palette": "jh_colors", "dt": 0.01},
      {"out_fmt": "ppm", "out": "S", "dt": 0.02},
      {"out_fmt": "ppm", "out": "bogus", "dt": 0.02},
      {"out_fmt": "ppm", "out": "Bp2", "usr_expr_flag": 1, "palette": "step8", "dt": 0.02, "num": 2},
      {"out_fmt": "bin", "dt": 0.02}], []),
    ("blast", configs.blast(40, 30, tlim=0.02),
     [{"out_fmt": "ppm", "out": "P", "palette": "idl1", "dt": 0.005},
      {"out_fmt": "ppm", "out": "cs2", "palette": "idl2", "dt": 0.007},
      {"out_fmt": "ppm", "out": "V1", "palette": "step32", "dmin": -0.5, "dt": 0.005},
      {"out_fmt": "ppm", "out": "J3", "usr_expr_flag": 1, "dt": 0.005},
      {"out_fmt": "ppm", "out": "M1", "dmax": 0.25, "dt": 0.01},
      {"out_fmt": "ppm", "out": "E", "dt": 0.01}], []),
    ("cpaw2d", configs.cpaw2d(32, 16, tlim=0.1),
     [{"out_fmt": "ppm", "out": "B1c", "dt": 0.03}, {"out_fmt": "ppm", "out": "B2c", "dt": 0.03},
      {"out_fmt": "ppm", "out": "B3c", "dt": 0.03}, {"out_fmt": "ppm", "out": "M2", "dt": 0.04},
      {"out_fmt": "ppm", "out": "M3", "dt": 0.04}, {"out_fmt": "ppm", "out": "V2", "dt": 0.05},
      {"out_fmt": "ppm", "out": "V3", "palette": "heat", "dt": 0.05}], ["grid/Nx2=12"]),
]


@pytest.mark.parametrize("problem,blocks,outputs,overrides", PPM_CASES, ids=[c[0] for c in PPM_CASES])
def test_cli_ppm_matches_reference_main(problem, blocks, outputs, overrides, tmp_path):
    ath = write_athinput(tmp_path / "athinput", _outputs(blocks, outputs))
    runs = _run_both(problem, ath, overrides, tmp_path)
    assert any(f.endswith(".ppm") for f in runs["ref"][1])
    _same(runs)


def test_cli_ppm_of_a_slice_fails_as_the_reference(tmp_path):
    """A slice (ix1 = 3) leaves a 1D image, which output_ppm refuses when it
    is due (the run stops there; the outputs before it are written)."""
    blocks = _outputs(configs.field_loop(16, 8, tlim=0.02),
                      [{"out_fmt": "ppm", "out": "d", "dt": 0.01},
                       {"out_fmt": "ppm", "out": "V1", "ix1": "3", "dt": 0.01}])
    ath = write_athinput(tmp_path / "athinput", blocks)
    runs = _run_both("field_loop", ath, [], tmp_path, rc=1)
    assert "Data must be 2D" in runs["ours"][2]
    assert runs["ours"][1] == runs["ref"][1] == runs["ours_q"][1] and runs["ref"][1]


def test_cli_rejects_unknown_override(tmp_path):
    ath = write_athinput(tmp_path / "athinput", configs.field_loop(16, 8))
    r = subprocess.run([str(EXE), "-i", str(ath), "-p", "field_loop", "grid/nonexistent=3"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "not found" in r.stderr


def test_cli_hlle_matches_reference_step(tmp_path):
    """job/flux = hlle selects flux_hlle everywhere; the reference's main
    program cannot (its flux is fixed at compile time), so the dumps are
    checked against the reference CPU step built with flux_hlle."""
    if not refutil.have_ref("blast", "hlle"):
        pytest.skip("reference CPU path not built")
    blocks = _outputs(configs.blast(30, 20, tlim=0.01, flux="hlle"), [{"out_fmt": "bin", "dt": 1.0}])
    ath = write_athinput(tmp_path / "athinput", blocks)
    r = subprocess.run([str(EXE), "-i", str(ath), "-p", "blast", "-q"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    ref = refutil.run_ref("blast", "hlle", ath, tmp_path)
    last = _cycles(r.stdout)[-1]
    assert last.startswith(f"cycle={ref['nstep']} ")
    assert (tmp_path / "Blast.0000.bin").exists()



def test_cli_takes_problem_from_comment_config(tmp_path):
    """Without -p the problem comes from <comment> config = --with-problem=...,
    the configure line of the reference's own athinput files."""
    blocks = {"comment": {"problem": "Blast wave", "config": "--with-problem=blast"}}
    blocks.update(_outputs(configs.blast(24, 16, tlim=0.01), [{"out_fmt": "tab", "dt": 0.005}]))
    ath = write_athinput(tmp_path / "athinput", blocks)
    outs = {}
    for name, extra in {"p": ["-p", "blast"], "comment": []}.items():
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([str(EXE), "-i", str(ath), *extra], cwd=d, capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        outs[name] = (_cycles(r.stdout), _files(d))
    assert outs["p"] == outs["comment"] and outs["p"][1]


@pytest.mark.parametrize("problem,blocks,expr,usr,palette", [
    ("blast", configs.blast(40, 30), "P", False, "jh_colors"),
    ("field_loop", configs.field_loop(32, 24), "J3", True, "heat"),
])
def test_output_ppm_api_matches_reference_main(problem, blocks, expr, usr, palette, tmp_path):
    """athb_output_ppm called through the Python binding on the initial state
    writes the file the reference main program writes at t = 0."""
    from athena_cuda_b200 import Grid, load_palette

    out = {"out_fmt": "ppm", "out": expr, "dt": 10.0, "palette": palette, "id": "img"}
    if usr:
        out["usr_expr_flag"] = 1
    blocks = _outputs(blocks, [out])
    blocks["time"]["nlim"] = 1   # the output at t = 0, written before the one step
    ath = write_athinput(tmp_path / "athinput", blocks)
    runs = _run_both(problem, ath, [], tmp_path)
    name = f"{blocks['job']['problem_id']}.0000.img.ppm"
    want = runs["ref"][1][name]
    g = Grid.from_athinput(ath, problem)
    rgb = load_palette(PALETTES, palette)
    gmin, gmax = g.output_ppm(tmp_path / "api.ppm", expr, usr_expr=usr, rgb=rgb)
    g.close()
    assert (tmp_path / "api.ppm").read_bytes() == want
    assert gmin <= gmax
