"""The command-line driver against the reference's own main program
(src/main.c with its output code, built into oracle/_ref/athmain_*): the same
athinput file and command-line overrides must give the same cycle lines and
byte-identical bin and tab dumps (src/dump_binary.c, src/dump_tab.c), with the
per-cycle loop and with the device loop that stops only for outputs (-q)."""
from __future__ import annotations

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
    return {p.name: p.read_bytes() for p in sorted(d.iterdir()) if p.suffix in (".bin", ".tab")}


def _cycles(text: str) -> list[str]:
    return [l for l in text.splitlines() if l.startswith("cycle=")]


@pytest.mark.parametrize("problem,blocks,outputs,overrides", CASES, ids=[c[0] for c in CASES])
def test_cli_matches_reference_main(problem, blocks, outputs, overrides, tmp_path):
    ref_exe = refutil.REF_DIR / f"athmain_{problem}"
    if not ref_exe.exists():
        pytest.skip("reference main program not built (python oracle/build_ref.py)")
    ath = write_athinput(tmp_path / "athinput", _outputs(blocks, outputs))
    runs = {}
    for name, cmd in {
        "ref": [str(ref_exe), "-i", str(ath), *overrides],
        "ours": [str(EXE), "-i", str(ath), "-p", problem, *overrides],
        "ours_q": [str(EXE), "-i", str(ath), "-p", problem, "-q", *overrides],
    }.items():
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (name, r.stdout[-2000:], r.stderr[-2000:])
        runs[name] = (r.stdout, _files(d))
    ref_out, ref_files = runs["ref"]
    assert ref_files, "the reference wrote no dumps"
    assert _cycles(runs["ours"][0]) == _cycles(ref_out)
    assert _cycles(runs["ours_q"][0])[-1] == _cycles(ref_out)[-1]
    for name in ("ours", "ours_q"):
        files = runs[name][1]
        assert sorted(files) == sorted(ref_files), name
        for f, data in ref_files.items():
            assert files[f] == data, f"{name}: {f} differs from the reference's"


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
