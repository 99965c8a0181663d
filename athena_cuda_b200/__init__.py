"""Python access to libathena_b200.so (the sm_100a 2D ideal-MHD CTU+CT step).

A thin ctypes layer over the C ABI in ``include/athena_b200.h``; the compute
runs in the CUDA library only.  Importing this module raises if the library has
not been built (``python -m athena_cuda_b200.build``): there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libathena_b200.so"
NPLANES = 11
PLANES = ("d", "M1", "M2", "M3", "E", "B1c", "B2c", "B3c", "B1i", "B2i", "B3i")
NGHOST = 4

FLUX_ROE, FLUX_HLLE = 0, 1
BC_REFLECT, BC_OUTFLOW, BC_PERIODIC = 1, 2, 4


class AthbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"athb error {code}: {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [
        ("nx1", C.c_int), ("nx2", C.c_int),
        ("x1min", C.c_double), ("x1max", C.c_double), ("x2min", C.c_double), ("x2max", C.c_double),
        ("bc_ix1", C.c_int), ("bc_ox1", C.c_int), ("bc_ix2", C.c_int), ("bc_ox2", C.c_int),
        ("gamma", C.c_double), ("cour_no", C.c_double), ("tlim", C.c_double),
        ("nlim", C.c_int), ("flux", C.c_int), ("device", C.c_int),
    ]


class AdjointStats(C.Structure):
    _fields_ = [("steps", C.c_int), ("snapshots", C.c_int), ("advances", C.c_longlong), ("taped", C.c_longlong),
                ("workspace_bytes", C.c_longlong), ("seconds", C.c_double), ("tape_mode", C.c_int)]


class PpmOpts(C.Structure):
    _fields_ = [("expr", C.c_char_p), ("usr_expr", C.c_int), ("nx1", C.c_int), ("nx2", C.c_int),
                ("rgb", C.POINTER(C.c_float)), ("sdmin", C.c_int), ("sdmax", C.c_int),
                ("dmin", C.c_float), ("dmax", C.c_float), ("num", C.c_int)]


class GridInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nx1", "nx2", "sx", "sy", "is_", "ie", "js", "je")] + [
        (n, C.c_double) for n in ("dx1", "dx2", "x1_0", "x2_0")] + [
        ("idisp", C.c_int), ("jdisp", C.c_int)] + [
        (n, C.c_double) for n in ("gamma", "gamma_1", "gamma_2")]


_lib = None


def lib() -> C.CDLL:
    """Load libathena_b200.so (once); raise if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is not built; run `python -m athena_cuda_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        P, I, D = C.c_void_p, C.c_int, C.c_double
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        sig = {
            "athb_create": (I, [C.POINTER(Config), C.POINTER(P)]),
            "athb_destroy": (None, [P]),
            "athb_shape": (I, [P, ip, ip]),
            "athb_upload": (I, [P, dp, D, D, I]),
            "athb_download": (I, [P, dp, dp, dp, ip]),
            "athb_set_bvals": (I, [P]),
            "athb_new_dt": (I, [P, dp]),
            "athb_run": (I, [P, I, ip]),
            "athb_run_async": (I, [P, I]),
            "athb_synchronize": (I, [P]),
            "athb_status": (I, [P, dp, dp, ip, ip]),
            "athb_stream": (P, [P]),
            "athb_last_error": (C.c_char_p, []),
            "athb_error_string": (C.c_char_p, [I]),
            "athb_create_from_athinput": (I, [C.c_char_p, I, C.POINTER(C.c_char_p), C.c_char_p, C.POINTER(P)]),
            "athb_cpaw2d_errors": (I, [P, dp]),
            "athb_grid_info_of": (I, [P, C.POINTER(GridInfo)]),
            "athb_params_open": (I, [C.c_char_p, C.POINTER(P)]),
            "athb_params_override": (I, [P, C.c_char_p]),
            "athb_params_getd": (I, [P, C.c_char_p, C.c_char_p, dp]),
            "athb_params_geti": (I, [P, C.c_char_p, C.c_char_p, ip]),
            "athb_params_close": (None, [P]),
            "athb_config_from_params": (I, [P, C.POINTER(Config)]),
            "athb_problem_generate": (I, [C.c_char_p, C.POINTER(GridInfo), P, dp]),
            "athb_host_alloc": (P, [C.c_ulonglong]),
            "athb_params_from_string": (I, [C.c_char_p, C.POINTER(P)]),
            "athb_batch_create": (I, [I, C.POINTER(Config), C.POINTER(P)]),
            "athb_batch_destroy": (None, [P]),
            "athb_batch_upload": (I, [P, I, dp, D, D, I]),
            "athb_batch_download": (I, [P, I, dp, dp, dp, ip]),
            "athb_batch_prepare": (I, [P]),
            "athb_batch_run": (I, [P, I, ip]),
            "athb_batch_run_async": (I, [P, I]),
            "athb_batch_synchronize": (I, [P]),
            "athb_batch_stream": (P, [P]),
            "athb_batch_set_ly": (I, [P, I, I]),
            "athb_batch_commit": (I, [P]),
            "athb_batch_set_grid": (I, [P, I]),
            "athb_batch_set_threads": (I, [P, I]),
            "athb_batch_threads": (I, [P]),
            "athb_batch_grid": (I, [P]),
            "athb_batch_timing": (I, [P, I, dp]),
            "athb_batch_set_mode": (I, [P, I]),
            "athb_batch_mode": (I, [P]),
            "athb_batch_generate": (I, [P, I, C.c_char_p, P]),
            "athb_generate": (I, [P, C.c_char_p, P]),
            "athb_generate_device": (I, [P, C.c_char_p, P]),
            "athb_set_pause": (I, [P, D, I]),
            "athb_dump_bin": (I, [P, C.c_char_p]),
            "athb_dump_tab": (I, [P, C.c_char_p, C.c_char_p]),
            "athb_output_ppm": (I, [P, C.c_char_p, C.POINTER(PpmOpts), C.POINTER(C.c_float),
                                    C.POINTER(C.c_float)]),
            "athb_palette_load": (I, [C.c_char_p, C.c_char_p, C.POINTER(C.c_float)]),
            "athb_profile_steps": (I, [P, I, dp]),
            "athb_fp64_peak": (I, [I, dp]),
            "athb_set_ly": (I, [P, I]),
            "athb_diagnostics": (I, [P, dp]),
            "athb_get_ly": (I, [P]),
            "athb_host_free": (None, [P]),
            "athb_tlm_run": (I, [P, I, dp, dp, dp, dp]),
            "athb_adjoint_keep_workspace": (I, [P, I]),
            "athb_adjoint_vjp": (I, [P, I, C.c_longlong, dp, dp, dp, C.POINTER(AdjointStats)]),
            "athb_adjoint_gradient": (I, [P, I, C.c_longlong, dp, dp, C.POINTER(AdjointStats)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise AthbError(rc, lib().athb_last_error().decode())


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


# problem generators whose device form is bit-identical to the host one
# (athb_generate forms these on the GPU); cpaw2d also has a device form
# (athb_generate_device, athb_batch_generate) equal to a few ulp
DEVICE_PROBLEMS = ("blast", "field_loop")


class Params:
    """An athinput parameter file (reference src/par.c format)."""

    def __init__(self, path: str | os.PathLike | None, overrides: list[str] = (), text: str | None = None):
        self._h = C.c_void_p()
        if text is not None:
            _check(lib().athb_params_from_string(text.encode(), C.byref(self._h)))
        else:
            _check(lib().athb_params_open(str(path).encode(), C.byref(self._h)))
        for o in overrides:
            _check(lib().athb_params_override(self._h, o.encode()))

    @classmethod
    def from_blocks(cls, blocks: dict) -> "Params":
        return cls(None, text=athinput_text(blocks))

    def getd(self, block: str, name: str) -> float:
        v = C.c_double()
        _check(lib().athb_params_getd(self._h, block.encode(), name.encode(), C.byref(v)))
        return v.value

    def geti(self, block: str, name: str) -> int:
        v = C.c_int()
        _check(lib().athb_params_geti(self._h, block.encode(), name.encode(), C.byref(v)))
        return v.value

    def config(self) -> Config:
        c = Config()
        _check(lib().athb_config_from_params(self._h, C.byref(c)))
        return c

    def close(self) -> None:
        if self._h:
            lib().athb_params_close(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def grid_info(cfg: Config) -> GridInfo:
    """Host-side geometry of a config (reference src/init_grid.c)."""
    g = GridInfo()
    g.nx1, g.nx2 = cfg.nx1, cfg.nx2
    g.sx, g.sy = cfg.nx1 + 2 * NGHOST, cfg.nx2 + 2 * NGHOST
    g.is_, g.js = NGHOST, NGHOST
    g.ie, g.je = cfg.nx1 + NGHOST - 1, cfg.nx2 + NGHOST - 1
    g.dx1 = (cfg.x1max - cfg.x1min) / cfg.nx1
    g.dx2 = (cfg.x2max - cfg.x2min) / cfg.nx2
    g.x1_0, g.x2_0 = cfg.x1min, cfg.x2min
    g.idisp, g.jdisp = -NGHOST, -NGHOST
    g.gamma, g.gamma_1, g.gamma_2 = cfg.gamma, cfg.gamma - 1.0, cfg.gamma - 2.0
    return g


def problem_state(name: str, params: Params) -> np.ndarray:
    """Initial state of a built-in problem generator, as (11, sy, sx) planes."""
    cfg = params.config()
    g = grid_info(cfg)
    planes = np.zeros((NPLANES, g.sy, g.sx))
    _check(lib().athb_problem_generate(name.encode(), C.byref(g), params._h, _dp(planes)))
    return planes


class Grid:
    """A device-resident grid (an ``athb_ctx``)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        sx, sy = C.c_int(), C.c_int()
        _check(lib().athb_shape(self._h, C.byref(sx), C.byref(sy)))
        self.sx, self.sy = sx.value, sy.value

    @classmethod
    def create(cls, cfg: Config) -> "Grid":
        h = C.c_void_p()
        _check(lib().athb_create(C.byref(cfg), C.byref(h)))
        return cls(h)

    @classmethod
    def from_athinput(cls, path, problem: str, overrides: list[str] = ()) -> "Grid":
        h = C.c_void_p()
        arr = (C.c_char_p * max(1, len(overrides)))(*[o.encode() for o in overrides])
        _check(lib().athb_create_from_athinput(str(path).encode(), len(overrides), arr,
                                               problem.encode(), C.byref(h)))
        return cls(h)

    def upload(self, planes: np.ndarray, dt: float = 0.0, time: float = 0.0, nstep: int = 0) -> None:
        planes = np.ascontiguousarray(planes, dtype=np.float64)
        assert planes.shape == (NPLANES, self.sy, self.sx)
        _check(lib().athb_upload(self._h, _dp(planes), dt, time, nstep))

    def download(self) -> tuple[np.ndarray, float, float, int]:
        planes = np.empty((NPLANES, self.sy, self.sx))
        dt, t, n = C.c_double(), C.c_double(), C.c_int()
        _check(lib().athb_download(self._h, _dp(planes), C.byref(dt), C.byref(t), C.byref(n)))
        return planes, dt.value, t.value, n.value

    def set_bvals(self) -> None:
        _check(lib().athb_set_bvals(self._h))

    def new_dt(self) -> float:
        dt = C.c_double()
        _check(lib().athb_new_dt(self._h, C.byref(dt)))
        return dt.value

    def run(self, nsteps: int) -> int:
        done = C.c_int()
        _check(lib().athb_run(self._h, nsteps, C.byref(done)))
        return done.value

    def run_async(self, nsteps: int) -> None:
        _check(lib().athb_run_async(self._h, nsteps))

    def synchronize(self) -> None:
        _check(lib().athb_synchronize(self._h))

    def status(self) -> dict:
        t, dt, n, done = C.c_double(), C.c_double(), C.c_int(), C.c_int()
        _check(lib().athb_status(self._h, C.byref(t), C.byref(dt), C.byref(n), C.byref(done)))
        return {"time": t.value, "dt": dt.value, "nstep": n.value, "done": done.value == 1,
                "paused": done.value == 2}

    @property
    def stream(self) -> int:
        return lib().athb_stream(self._h) or 0

    @property
    def ly(self) -> int:
        return lib().athb_get_ly(self._h)

    @ly.setter
    def ly(self, v: int) -> None:
        _check(lib().athb_set_ly(self._h, v))

    def profile(self, nsteps: int = 5) -> dict:
        """Mean ms per step of each kernel (CUDA events between launches)."""
        ms = (C.c_double * 7)()
        _check(lib().athb_profile_steps(self._h, nsteps, ms))
        return dict(zip(("predict", "emf_half", "correct", "emf_full", "update_cfl", "finalize", "ghost"), ms))

    def diagnostics(self) -> dict:
        """Device-side integrals / maxima of the current state."""
        out = np.zeros(6)
        _check(lib().athb_diagnostics(self._h, _dp(out)))
        return dict(zip(("mass", "energy", "emag", "bp2", "max_divb", "max_j3"), out.tolist()))

    def tlm(self, nsteps: int, direction: np.ndarray, want_state: bool = False):
        """Tangent-linear model of nsteps main-loop iterations from the
        resident state (taken as the loop-entry state): (J, dJ[, dS^N]) for
        J = sum over interior cells of (B1c^2 + B2c^2)/2 along `direction`
        (host planes; ghost entries ignored).  The resident state is kept."""
        d = np.ascontiguousarray(direction, dtype=np.float64)
        assert d.shape == (NPLANES, self.sy, self.sx)
        J, dJ = C.c_double(), C.c_double()
        out = np.empty_like(d) if want_state else None
        _check(lib().athb_tlm_run(self._h, nsteps, _dp(d), C.byref(J), C.byref(dJ),
                                  _dp(out) if out is not None else None))
        return (J.value, dJ.value, out) if want_state else (J.value, dJ.value)

    def keep_adjoint_workspace(self, on: bool = True) -> None:
        """Keep the adjoint's device workspace between calls (a repeated
        gradient of the same size allocates nothing), or free it now."""
        _check(lib().athb_adjoint_keep_workspace(self._h, int(on)))

    def adjoint_gradient(self, nsteps: int, snapshot_bytes: int = 0):
        """Adjoint of nsteps main-loop iterations from the resident state:
        (J, dJ/d(state), stats).  snapshot_bytes bounds the device memory for
        checkpoints (0: most of the free memory)."""
        g = np.empty((NPLANES, self.sy, self.sx))
        J = C.c_double()
        st = AdjointStats()
        _check(lib().athb_adjoint_gradient(self._h, nsteps, snapshot_bytes, C.byref(J), _dp(g), C.byref(st)))
        stats = {k: getattr(st, k) for k, _ in AdjointStats._fields_}
        return J.value, g, stats

    def adjoint_vjp(self, nsteps: int, seed: np.ndarray, snapshot_bytes: int = 0):
        """Adjoint of nsteps iterations for any objective of the final state:
        seed = dJ/dS^N (state layout); returns (<seed, S^N>,
        (dS^N/dS^0)^T seed, stats)."""
        seed = np.ascontiguousarray(seed, dtype=np.float64)
        assert seed.shape == (NPLANES, self.sy, self.sx)
        g = np.empty((NPLANES, self.sy, self.sx))
        J = C.c_double()
        st = AdjointStats()
        _check(lib().athb_adjoint_vjp(self._h, nsteps, snapshot_bytes, _dp(seed), C.byref(J), _dp(g), C.byref(st)))
        stats = {k: getattr(st, k) for k, _ in AdjointStats._fields_}
        return J.value, g, stats

    def cpaw2d_errors(self) -> np.ndarray:
        err = np.zeros(9)
        _check(lib().athb_cpaw2d_errors(self._h, _dp(err)))
        return err

    def generate(self, name: str, params: "Params") -> None:
        """Replace the state with problem `name`'s initial condition (clock
        reset, no ghost fill); blast and field_loop are formed on the GPU."""
        _check(lib().athb_generate(self._h, name.encode(), params._h))

    def generate_device(self, name: str, params: "Params") -> None:
        """As generate, every built-in problem formed on the GPU (cpaw2d with
        CUDA's sin/cos: a few ulp from the host generator)."""
        _check(lib().athb_generate_device(self._h, name.encode(), params._h))

    def set_pause(self, tpause: float, on: bool = True) -> None:
        """Stop the device loop at the first step starting at time >= tpause."""
        _check(lib().athb_set_pause(self._h, tpause, int(on)))

    def dump_bin(self, path) -> None:
        """The reference's binary dump of the current state (src/dump_binary.c)."""
        _check(lib().athb_dump_bin(self._h, str(path).encode()))

    def dump_tab(self, path, dat_fmt: str | None = None) -> None:
        """The reference's table dump of the current state (src/dump_tab.c)."""
        _check(lib().athb_dump_tab(self._h, str(path).encode(), dat_fmt.encode() if dat_fmt else None))

    def output_ppm(self, path, expr: str, usr_expr: bool = False, rgb: np.ndarray | None = None,
                   dmin: float | None = None, dmax: float | None = None, num: int = 0,
                   extremes: tuple[float, float] = (0.0, 0.0)) -> tuple[float, float]:
        """The reference's ppm image of one expression (src/output_ppm.c);
        returns the running (gmin, gmax), `extremes` being the previous ones
        (ignored when num is 0)."""
        o = PpmOpts(expr=expr.encode(), usr_expr=int(usr_expr), sdmin=int(dmin is not None),
                    sdmax=int(dmax is not None), dmin=dmin or 0.0, dmax=dmax or 0.0, num=num)
        if rgb is not None:
            rgb = np.ascontiguousarray(rgb, dtype=np.float32)
            assert rgb.size == 768
            o.rgb = rgb.ctypes.data_as(C.POINTER(C.c_float))
        gmin, gmax = C.c_float(extremes[0]), C.c_float(extremes[1])
        _check(lib().athb_output_ppm(self._h, str(path).encode(), C.byref(o), C.byref(gmin), C.byref(gmax)))
        return gmin.value, gmax.value

    def close(self) -> None:
        if self._h:
            lib().athb_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_palette(path, name: str) -> np.ndarray:
    """Colour table `name` (256 x 3 floats in 0..1) from a palette file: the
    reference's palette.h, or lines "<name> v0 .. v767"."""
    rgb = np.zeros(768, dtype=np.float32)
    _check(lib().athb_palette_load(str(path).encode(), name.encode(), rgb.ctypes.data_as(C.POINTER(C.c_float))))
    return rgb


def athinput_text(blocks: dict) -> str:
    """athinput text from {block: {name: value}} (reference format)."""
    lines = []
    for b, kv in blocks.items():
        lines.append(f"<{b}>")
        for k, v in kv.items():
            lines.append(f"{k} = {v!r}" if isinstance(v, float) else f"{k} = {v}")
        lines.append("")
    return "\n".join(lines)


def write_athinput(path, blocks: dict) -> Path:
    """Write an athinput file from {block: {name: value}} (reference format)."""
    path = Path(path)
    path.write_text(athinput_text(blocks))
    return path


class Batch:
    """Independent grids advanced together, one persistent launch per step."""

    def __init__(self, cfgs: list[Config]):
        arr = (Config * len(cfgs))(*cfgs)
        self._h = C.c_void_p()
        _check(lib().athb_batch_create(len(cfgs), arr, C.byref(self._h)))
        self.n = len(cfgs)
        self.shapes = [(c.nx2 + 2 * NGHOST, c.nx1 + 2 * NGHOST) for c in cfgs]

    @classmethod
    def from_problems(cls, items: list[tuple[str, dict]]) -> "Batch":
        """items: (problem name, athinput blocks) per instance; runs each
        problem generator, set_bvals and the first new_dt."""
        params = [Params.from_blocks(b) for _, b in items]
        cfgs = [p.config() for p in params]
        b = cls(cfgs)
        for k, ((name, _), p) in enumerate(zip(items, params)):
            if name in DEVICE_PROBLEMS:
                b.generate(k, name, p)  # formed on the GPU
            else:
                b.upload(k, problem_state(name, p))
        b.prepare()
        return b

    def generate(self, k: int, name: str, params: "Params") -> None:
        """Instance k's initial condition formed on the GPU (built-in
        problems, as Grid.generate_device)."""
        _check(lib().athb_batch_generate(self._h, k, name.encode(), params._h))

    def upload(self, k: int, planes: np.ndarray, dt=0.0, time=0.0, nstep=0) -> None:
        planes = np.ascontiguousarray(planes, dtype=np.float64)
        assert planes.shape == (NPLANES, *self.shapes[k])
        _check(lib().athb_batch_upload(self._h, k, _dp(planes), dt, time, nstep))

    def download(self, k: int):
        planes = np.empty((NPLANES, *self.shapes[k]))
        dt, t, n = C.c_double(), C.c_double(), C.c_int()
        _check(lib().athb_batch_download(self._h, k, _dp(planes), C.byref(dt), C.byref(t), C.byref(n)))
        return planes, dt.value, t.value, n.value

    def prepare(self) -> None:
        _check(lib().athb_batch_prepare(self._h))

    def run(self, max_steps: int = 1_000_000) -> int:
        n = C.c_int()
        _check(lib().athb_batch_run(self._h, max_steps, C.byref(n)))
        return n.value

    def run_async(self, nsteps: int) -> None:
        _check(lib().athb_batch_run_async(self._h, nsteps))

    def synchronize(self) -> None:
        _check(lib().athb_batch_synchronize(self._h))

    @property
    def stream(self) -> int:
        return lib().athb_batch_stream(self._h) or 0

    def set_ly(self, k: int, ly: int) -> None:
        _check(lib().athb_batch_set_ly(self._h, k, ly))

    def commit(self) -> None:
        _check(lib().athb_batch_commit(self._h))

    def set_grid(self, blocks: int) -> None:
        _check(lib().athb_batch_set_grid(self._h, blocks))

    @property
    def grid(self) -> int:
        return lib().athb_batch_grid(self._h)

    @property
    def threads(self) -> int:
        """Threads per work unit of the phased launches (64, 128, 256)."""
        return lib().athb_batch_threads(self._h)

    @threads.setter
    def threads(self, nt: int) -> None:
        _check(lib().athb_batch_set_threads(self._h, nt))
        self.commit()

    PERSISTENT, PHASED = 0, 1

    @property
    def mode(self) -> int:
        """Batch.PHASED (one launch per phase, the default) or
        Batch.PERSISTENT (one cooperative launch per step); results are
        identical."""
        return lib().athb_batch_mode(self._h)

    @mode.setter
    def mode(self, m: int) -> None:
        _check(lib().athb_batch_set_mode(self._h, m))

    def timing(self, enable: int = -1) -> dict:
        """Per-phase ms (enable=1 to start recording, 0 to stop, -1 to just
        read)."""
        ms = np.zeros(6)
        _check(lib().athb_batch_timing(self._h, enable, _dp(ms)))
        return dict(zip(("predict", "emf_half", "correct", "emf_full", "update_cfl", "ghost_finalize"), ms.tolist()))

    def close(self) -> None:
        if self._h:
            lib().athb_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
