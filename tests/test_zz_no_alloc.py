"""athb_integrate_noalloc: the integrate step for callers that cannot allocate
device memory -- code that runs while a CUDA graph is being captured, programs
that reserve the whole device memory budget up front, allocation-free
real-time loops.  Its scratch is a fixed __device__ array inside the library.
Checked, through the C ABI, against the drop-in integrate_2d (which uses the
regular, allocating context) on two consecutive steps: the results must be
identical value for value."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from athena_cuda_b200 import AthbError, Config, Grid, Params, configs, lib, write_athinput
from athena_cuda_b200.dropin import HostGrid, _setup_signatures

pytestmark = pytest.mark.gpu


def _noalloc():
    L = lib()
    f = L.athb_integrate_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(Config), C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
    return f


@pytest.mark.parametrize("nx1,nx2,bc", [
    (40, 28, (4, 4, 4, 4)),   # (40+8)*(28+8) = 1728 cells; rows of 48 doubles
    (30, 20, (2, 2, 1, 1)),   # rows of 38 doubles (not a multiple of 16), outflow / reflecting
    (64, 64, (4, 4, 4, 4)),   # the largest grid the fixed scratch holds (72*72 = 5184 cells)
])
def test_noalloc_step_matches_integrate_2d_twice(nx1, nx2, bc, tmp_path):
    import torch

    blocks = configs.blast(nx1, nx2, bc=bc)
    ath = write_athinput(tmp_path / "athinput", blocks)
    g = Grid.from_athinput(ath, "blast")  # problem, set_bvals, first new_dt
    planes, dt, _, _ = g.download()
    g.close()
    cfg = Params(ath).config()

    # the existing entry point: drop-in integrate_2d on a host Grid
    Ld = _setup_signatures()
    C.c_double.in_dll(Ld, "Gamma").value = cfg.gamma
    C.c_double.in_dll(Ld, "Gamma_1").value = cfg.gamma - 1.0
    C.c_double.in_dll(Ld, "Gamma_2").value = cfg.gamma - 2.0
    C.c_double.in_dll(Ld, "CourNo").value = cfg.cour_no
    Ld.athb_dropin_set_bc(cfg.bc_ix1, cfg.bc_ox1, cfg.bc_ix2, cfg.bc_ox2)
    hg = HostGrid(planes, (cfg.x1max - cfg.x1min) / cfg.nx1, (cfg.x2max - cfg.x2min) / cfg.nx2,
                  cfg.x1min, cfg.x2min)

    noalloc = _noalloc()
    d_in = torch.tensor(planes, device="cuda")
    d_out = d_in.clone()
    stream = torch.cuda.current_stream()
    for step_dt in (dt, 0.9 * dt):
        rc = noalloc(C.byref(cfg), d_in.data_ptr(), d_out.data_ptr(), step_dt, stream.cuda_stream)
        assert rc == 0, lib().athb_last_error().decode()
        stream.synchronize()
        hg.grid.dt = step_dt
        Ld.integrate_2d(C.byref(hg.grid))
        np.testing.assert_array_equal(d_out.cpu().numpy(), hg.planes())
        d_in, d_out = d_out, d_out.clone()
    Ld.integrate_destruct_2d()
    hg.close()


def test_noalloc_rejects_grids_beyond_its_scratch(tmp_path):
    import torch

    cfg = Params.from_blocks(configs.field_loop(80, 64)).config()  # 88*72 cells > 5184
    buf = torch.zeros(11 * 72 * 88, dtype=torch.float64, device="cuda")
    out = torch.zeros_like(buf)
    rc = _noalloc()(C.byref(cfg), buf.data_ptr(), out.data_ptr(), 1e-3, None)
    assert rc == 1 and b"5184" in lib().athb_last_error()


def test_noalloc_rejects_a_config_for_another_device(tmp_path):
    import torch

    cfg = Params.from_blocks(configs.field_loop(16, 16)).config()
    cfg.device = torch.cuda.current_device() + 1
    buf = torch.zeros(11 * 24 * 24, dtype=torch.float64, device="cuda")
    out = torch.zeros_like(buf)
    rc = _noalloc()(C.byref(cfg), buf.data_ptr(), out.data_ptr(), 1e-3, None)
    assert rc == 1 and b"current device" in lib().athb_last_error()


def test_noalloc_writes_only_the_step_cells(tmp_path):
    """Guard bands around the caller's output buffer, and every cell the step
    does not write, keep a sentinel (a memory-safety check in place of a
    sanitizer): only interior cells, B1i column ie+1 and B2i row je+1 change."""
    import torch

    blocks = configs.blast(30, 20, bc=(2, 2, 1, 1))
    ath = write_athinput(tmp_path / "athinput", blocks)
    g = Grid.from_athinput(ath, "blast")
    planes, dt, _, _ = g.download()
    g.close()
    cfg = Params(ath).config()
    guard, mark = 4096, 0x7FF4DEADBEEF0001
    d_in = torch.tensor(planes, device="cuda")
    out = torch.empty(2 * guard + planes.size, dtype=torch.float64, device="cuda")
    out.view(torch.int64).fill_(mark)
    rc = _noalloc()(C.byref(cfg), d_in.data_ptr(), out[guard:].data_ptr(), dt, None)
    assert rc == 0, lib().athb_last_error().decode()
    torch.cuda.synchronize()
    bits = out.view(torch.int64).cpu().numpy()
    assert (bits[:guard] == mark).all() and (bits[-guard:] == mark).all()
    body = bits[guard:-guard].reshape(planes.shape)
    written = np.zeros(planes.shape, dtype=bool)
    is_, ie, js, je = 4, 4 + cfg.nx1 - 1, 4, 4 + cfg.nx2 - 1
    written[:, js:je + 1, is_:ie + 1] = True
    written[8, js:je + 1, ie + 1] = True   # B1i column ie+1
    written[9, je + 1, is_:ie + 1] = True  # B2i row je+1
    assert (body[~written] == mark).all(), "the step wrote outside its cells"
    assert (body[written] != mark).all()

