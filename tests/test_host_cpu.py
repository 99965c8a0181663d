"""CPU-only checks of libathena_b200.so: the C ABI exports every entry point
include/athena_b200.h declares, the athinput parser follows the reference
format (src/par.c), and the host-side problem generators reproduce the
reference's initial conditions bit for bit.  No kernel is launched here."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import refutil
from athena_cuda_b200 import (LIB_PATH, NGHOST, PLANES, AthbError, Params, configs, lib, load_palette, problem_state,
                              write_athinput)

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "athena_b200.h"


def declared_functions() -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("typedef"))
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in {"if", "for", "while"}))


def test_library_exports_every_declared_function():
    L = lib()
    names = declared_functions()
    assert "integrate_2d" in names and "athb_run" in names and "new_dt" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"not exported: {missing}"


def test_library_exports_reference_globals():
    L = lib()
    for g in ("Gamma", "Gamma_1", "Gamma_2", "CourNo"):
        ctypes.c_double.in_dll(L, g)


def test_athinput_format(tmp_path):
    f = tmp_path / "athinput"
    f.write_text(
        "# comment line\n<comment>\nproblem = x y z\n\n<grid>\n"
        "Nx1 = 64   # trailing comment\n  x1min=-1.0\nx1max = 1e0\nNx1 = 32\n"
        "<time>\ntlim = 0.25\n<par_end>\n<ignored>\nfoo = 1\n")
    p = Params(f, ["grid/x1max=2.5"])
    assert p.geti("grid", "Nx1") == 32          # later duplicate replaces
    assert p.getd("grid", "x1min") == -1.0
    assert p.getd("grid", "x1max") == 2.5       # command-line override
    assert p.getd("time", "tlim") == 0.25
    with pytest.raises(AthbError):
        p.getd("ignored", "foo")                # after <par_end>
    with pytest.raises(AthbError):
        Params(f, ["grid/newkey=1"])            # overrides may not add keys
    with pytest.raises(AthbError):
        Params(f, ["nosuchblock/x=1"])


def test_config_validation(tmp_path):
    ath = write_athinput(tmp_path / "a", configs.blast(3, 40))
    with pytest.raises(AthbError, match="Nx1 >= 4"):
        Params(ath).config()
    ath = write_athinput(tmp_path / "b", configs.blast(40, 40, bc=(3, 4, 4, 4)))
    with pytest.raises(AthbError, match="boundary"):
        Params(ath).config()
    ath = write_athinput(tmp_path / "c", configs.cpaw2d(32, 16, flux="hlle"))
    assert Params(ath).config().flux == 1


GEN_CASES = {
    "blast": configs.blast(40, 60),
    "field_loop": configs.field_loop(64, 32),
    "cpaw2d": configs.cpaw2d(32, 16),
}


@pytest.mark.parametrize("problem", sorted(GEN_CASES))
def test_problem_generator_matches_reference(problem, tmp_path):
    if not refutil.have_ref(problem):
        pytest.skip("oracle/_ref not built")
    ath = write_athinput(tmp_path / "athinput", GEN_CASES[problem])
    ref = refutil.run_ref(problem, "roe", ath, tmp_path, steps=0)["planes"]
    mine = problem_state(problem, Params(ath))
    ng = NGHOST
    sy, sx = mine.shape[1:]
    interior = (slice(ng, sy - ng), slice(ng, sx - ng))
    for k in range(8):  # cell-centred planes and B3i
        np.testing.assert_array_equal(mine[k][interior], ref[k][interior], err_msg=PLANES[k])
    np.testing.assert_array_equal(mine[10][interior], ref[10][interior], err_msg="B3i")
    # face fields: interior plus the outer faces B1i(ie+1) and B2i(je+1)
    np.testing.assert_array_equal(mine[8][ng:sy - ng, ng:sx - ng + 1], ref[8][ng:sy - ng, ng:sx - ng + 1])
    np.testing.assert_array_equal(mine[9][ng:sy - ng + 1, ng:sx - ng], ref[9][ng:sy - ng + 1, ng:sx - ng])


def test_palette_file_forms(tmp_path):
    """Both palette file forms the ppm output reads: the C initialisers of the
    reference's palette.h and one text line per table."""
    vals = np.linspace(0.0, 1.0, 768).astype(np.float32)
    c_form = tmp_path / "pal.h"
    c_form.write_text("static float other[256*3] = { 1.0, 2.0 };\n"
                      "static float mine[256*3] = {\n" + " , ".join(f"{v:.6e}" for v in vals) + " ,\n};\n")
    got = load_palette(c_form, "mine")
    np.testing.assert_array_equal(got, np.array([float(f"{v:.6e}") for v in vals]).astype(np.float32))
    short = load_palette(c_form, "other")   # a short initialiser: the rest is zero
    assert short[0] == 1.0 and short[1] == 2.0 and not short[2:].any()
    lines = tmp_path / "pal.txt"
    lines.write_text("mine " + " ".join(f"{v:.9g}" for v in vals) + "\n")
    np.testing.assert_array_equal(load_palette(lines, "mine"), vals)
    with pytest.raises(AthbError, match="not found"):
        load_palette(lines, "min")


def test_reference_palettes_as_text():
    """oracle/_ref/palettes.txt (written from the reference's palette.h) reads
    back as the tables the C compiler builds from palette.h itself."""
    pal = refutil.REF_DIR / "palettes.txt"
    h = refutil.reference_root() / "src" / "palette.h" if refutil.reference_root() else None
    if not pal.exists() or h is None or not h.exists():
        pytest.skip("reference palettes not available")
    for name in ("rainbow", "jh_colors", "step8", "step32", "idl1", "idl2", "heat"):
        np.testing.assert_array_equal(load_palette(pal, name), load_palette(h, name), err_msg=name)


def test_null_handles_are_rejected_without_touching_a_gpu():
    """The C ABI reports bad arguments with ATHB_ERR_ARG (1) and a message
    instead of crashing; these checks run before any CUDA call."""
    L = ctypes.CDLL(str(LIB_PATH))   # a handle of its own: no argtypes set
    P = ctypes.c_void_p
    buf = (ctypes.c_double * 16)()
    checks = {
        "athb_rect_pack": (None, 0, 4, 0, 4, ctypes.cast(buf, P)),
        "athb_rect_unpack": (None, 0, 4, 0, 4, ctypes.cast(buf, P)),
        "athb_rows_pack": (None, 0, 4, ctypes.cast(buf, P)),
        "athb_finish_step_device": (None, ctypes.cast(buf, P), 1, 1),
        "athb_max_dti_bits_device": (None, ctypes.cast(buf, P)),
        "athb_copy_async": (None, ctypes.cast(buf, P), ctypes.cast(buf, P), ctypes.c_ulonglong(8)),
        "athb_batch_set_threads": (None, 64),
        "athb_adjoint_keep_workspace": (None, 1),
        "athb_cpaw2d_errors": (None, ctypes.cast(buf, P)),
        "athb_generate_device": (None, b"blast", None),
    }
    for name, args in checks.items():
        f = getattr(L, name)
        f.restype = ctypes.c_int
        assert f(*args) == 1, name
        L.athb_last_error.restype = ctypes.c_char_p
        assert L.athb_last_error(), name
    out = np.zeros(768, dtype=np.float32)
    L.athb_palette_load.restype = ctypes.c_int
    assert L.athb_palette_load(b"/nonexistent/palette.h", b"rainbow",
                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))) == 7   # ATHB_ERR_IO
