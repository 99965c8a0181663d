#!/usr/bin/env python
"""Throughput of the FP64 2D ideal-MHD CTU+CT step on B200, in zone-cycles/s.

Workload: the field-loop advection problem (reference src/field_loop.c) on
2048 x 2048 cells, [-1,1] x [-0.5,0.5], periodic, v = (2,1), gamma = 5/3, Roe
fluxes, CFL 0.8.  A "step" is one iteration of the reference main loop
(src/main.c:229-307): integrate_2d, time += dt, new_dt, set_bvals.  The state
(372 MB) and the per-step face scratch (1.9 GB) are far larger than the 126 MB
L2, so every step streams from HBM.

Arms:
  default            sm_100a kernels, device-resident state, CUDA graph; the
                     device-timed `value`, the per-kernel roofline, `e2e`
                     through the reference-named drop-in ABI on pinned host
                     buffers, and a CPU baseline (the reference's own CPU path)
  --impl reference   the reference CPU path (oracle/_ref) on all host cores

Under torchrun (N > 1) every rank runs an independent replica of the
workload (the single-grid step does not shard): weak scaling, max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "zone-cycles/s (FP64 CTU+CT step, bit-exact vs reference)"
UNIT = "zone-cycles/s"

# Algorithmic FP64 operations per zone-cycle of the reference step on the
# 2048x2048 field loop (every binary + - * / and sqrt on a Real that the
# reference performs), split by the kernel that performs them.  Counted by
# `python oracle/opcount.py --problem field_loop --nx 2048 --ny 2048 --steps 3`
# (profiles/opcount_field_loop_2048.md).  Per launch = value x nx x ny.
OPS_PER_ZC = {
    "predict": 3432.2,     # steps 1a-2e and 3 (PLM, MHD source, Roe, emf3_cc)
    "emf_half": 18.0,      # step 4 corner EMF + half-step CT
    "correct": 1378.6,     # steps 5a-8c (transverse terms, emf3_cc n+1/2, Roe)
    "emf_full": 12.0,      # step 9 corner EMF
    "update_cfl": 129.0,   # steps 9 CT, 11a, 11b, 13 (52) + new_dt (77)
}
OPS_STEP = sum(OPS_PER_ZC.values())
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# dominant kernels from single-kernel ncu captures of the 1024x1024 field loop
# (profiles/k_predict_field_loop_1024.md, k_correct_k_update_field_loop_1024.md),
# scaled to 2048x2048 by the cell ratio 4.  Applies to the 2048x2048 default
# workload.
TRAFFIC_1024 = {"predict": 508.49e6, "correct": 725.48e6, "update_cfl": 244.51e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="field_loop", choices=["field_loop", "ensemble", "cpaw", "configs", "adjoint"])
    ap.add_argument("--adj-cases", default="256x200,1024x2000",
                    help="adjoint workload: comma-separated <N>x<steps> field-loop cases")
    ap.add_argument("--adj-snapshot-gb", type=float, default=0.0,
                    help="adjoint workload: device memory for checkpoints (0: most of the free memory)")
    ap.add_argument("--ensemble-n", type=int, default=512)
    ap.add_argument("--seq-sample", type=int, default=0,
                    help="time sequential single-grid runs on every k-th instance only (0: all)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x: float, ws: int, device) -> float:
    """The slowest rank's device time (every rank takes part; all get it)."""
    if ws == 1:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_value(ws: int, cells: int, ms_step: float) -> float:
    """Whole-job zone-cycles/s of ws independent replicas of `cells` zones
    whose slowest rank took ms_step per step."""
    return ws * cells / (ms_step * 1e-3)


def config_dict(a):
    return {"workload": f"field_loop {a.nx}x{a.ny}", "problem": "field_loop", "nx1": a.nx, "nx2": a.ny,
            "flux": "roe", "precision": "fp64", "cfl": 0.8, "l2": "inputs larger than L2 (372 MB state)",
            "parallelism": "replicas" if a.gpus > 1 else "single"}


def write_input(a, d: Path, device: int = 0) -> Path:
    from athena_cuda_b200 import configs, write_athinput
    blocks = configs.field_loop(a.nx, a.ny)
    blocks["job"]["device"] = device
    return write_athinput(d / "athinput.field_loop", blocks)


# ---------------------------------------------------------------------------
# CPU reference (oracle/_ref)
# ---------------------------------------------------------------------------
def ref_exe() -> Path:
    return ROOT / "oracle" / "_ref" / "athref_field_loop_roe"


def run_ref_sample(ath: Path, steps: int, procs: int, workdir: Path, max_seconds: float = 25.0,
                   exe: Path | None = None, warmup: int = 0, warmup_seconds: float = 6.0) -> dict:
    """`procs` concurrent single-threaded reference processes, each running
    up to `warmup` untimed main-loop iterations (at most warmup_seconds of
    them), then `steps` timed ones (or fewer once its loop has run
    max_seconds); zone-cycles/s summed over processes (each process times its
    own main loop, setup and warm-up excluded)."""
    exe = exe or ref_exe()
    ps = [subprocess.Popen([str(exe), "-i", str(ath), "--steps", str(steps), "--bench",
                            "--max-seconds", str(max_seconds), "--warmup", str(warmup),
                            "--warmup-seconds", str(warmup_seconds)],
                           stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, cwd=workdir, text=True)
          for _ in range(procs)]
    outs = []
    for p in ps:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("reference run failed")
        outs.append(json.loads(out.strip().splitlines()[-1]))
    total = sum(o["zone_cycles_per_s"] for o in outs)
    return {"value": total, "per_process": [o["zone_cycles_per_s"] for o in outs],
            "seconds": max(o["seconds"] for o in outs),
            "steps_per_process": [int(o["steps"]) for o in outs],
            "warmup_per_process": [int(o.get("warmup", 0)) for o in outs],
            "ms_per_step_per_process": [1e3 * o["seconds"] / o["steps"] for o in outs if o["steps"]]}


def run_ref_instances(aths: list[Path], problem: str, workdir: Path, max_seconds: float = 20.0) -> dict:
    """One single-threaded reference process per athinput, all at once, each
    running its instance to its end time (or for max_seconds of main loop);
    zone-cycles/s summed over processes."""
    exe = ROOT / "oracle" / "_ref" / f"athref_{problem}_roe"
    ps = [subprocess.Popen([str(exe), "-i", str(ath), "--steps", "1000000000", "--bench", "--max-seconds",
                            str(max_seconds)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, cwd=workdir,
                           text=True) for ath in aths]
    outs = []
    for p in ps:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("reference run failed")
        outs.append(json.loads(out.strip().splitlines()[-1]))
    return {"value": sum(o["zone_cycles_per_s"] for o in outs), "seconds": max(o["seconds"] for o in outs)}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_arm(a) -> None:
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    if not ref_exe().exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (python oracle/build_ref.py)"}))
        return
    cores = max(1, min(os.cpu_count() or 1, 16))
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        ath = write_input(a, td)
        # one bounded sample: every process runs the timed steps (capped at
        # ~20 s of main loop); the warm-up is the page-in of the first step
        r = run_ref_sample(ath, max(1, min(a.steps, 3)), cores, td, max_seconds=20.0, warmup=a.warmup,
                           warmup_seconds=6.0)
        value = r["value"]
    # what was timed: every process ran the same number of main-loop
    # iterations (the smallest is reported) at its own per-step time (the mean
    # is reported); `value` is the sum of the processes' rates
    steps_run = min(r["steps_per_process"])
    ms_step = statistics.mean(r["ms_per_step_per_process"])
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
        "steps": steps_run, "warmup": min(r["warmup_per_process"]), "ms_per_step": ms_step,
        "steps_requested": a.steps, "warmup_requested": a.warmup, "processes": cores,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (field-loop initial condition, src/field_loop.c)",
        "config": config_dict(a),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{cores} concurrent single-threaded reference processes (-O2 "
                                   f"-ffp-contract=off), each {steps_run} timed main-loop iterations "
                                   f"(after up to {a.warmup} untimed ones, <= 6 s) of the {a.nx}x{a.ny} "
                                   f"field loop; ms_per_step is one process's step time, value the sum of "
                                   f"the processes' rates; {cpu_model()}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.proc, self.path = device, None, None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.path = Path(tempfile.mkstemp(suffix=".csv")[1])
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # the timed region can be shorter than nvidia-smi's start-up: wait
            # for its first sample so that the region is covered
            t0 = time.time()
            while time.time() - t0 < 10.0 and self.path.stat().st_size == 0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.skip = len(self.path.read_text().splitlines())
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.05)   # a sample just after the region
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict | None:
        if not self.path or not self.path.exists():
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.path.read_text().splitlines()
        # samples from the last one before the region on (the region itself
        # may be shorter than the sampling interval)
        for line in lines[max(0, getattr(self, "skip", 1) - 1):]:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        self.path.unlink(missing_ok=True)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def ours(a) -> None:
    import ctypes as C

    import torch

    import athena_cuda_b200 as ab
    from athena_cuda_b200 import Grid, lib

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    L = lib()
    L.athb_profile_steps.restype, L.athb_profile_steps.argtypes = C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
    L.athb_fp64_peak.restype, L.athb_fp64_peak.argtypes = C.c_int, [C.c_int, C.POINTER(C.c_double)]

    td = Path(tempfile.mkdtemp())
    ath = write_input(a, td, local)
    g = Grid.from_athinput(ath, "field_loop")
    g.run(a.warmup)
    st0 = g.status()
    stream = torch.cuda.ExternalStream(g.stream, device=torch.device("cuda", local))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(stream)
        g.run_async(a.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    st1 = g.status()
    assert st1["nstep"] - st0["nstep"] == a.steps and not st1["done"], "timed steps did not all run"
    ms = max_over_ranks(ms, ws, torch.device("cuda", local))
    cells = a.nx * a.ny
    ms_step = ms / a.steps
    value = replica_value(ws, cells, ms_step)

    # per-kernel event timing (same stream, outside the graph)
    kms = (C.c_double * 7)()
    rc = L.athb_profile_steps(g._h, 10, kms)
    if rc:
        raise RuntimeError(L.athb_last_error().decode())
    names = ["predict", "emf_half", "correct", "emf_full", "update_cfl", "finalize", "ghost"]
    kernel_ms = dict(zip(names, list(kms)))
    peak = C.c_double()
    rc = L.athb_fp64_peak(local, C.byref(peak))
    if rc:
        raise RuntimeError(L.athb_last_error().decode())
    top = max(("predict", "correct"), key=lambda k: kernel_ms[k])
    per_launch = OPS_PER_ZC[top] * cells
    achieved = per_launch / (kernel_ms[top] * 1e-3)
    step_ops = OPS_STEP * cells
    # the same kernel against HBM: its DRAM bytes per launch over its time
    traffic = TRAFFIC_1024[top] * cells / (1024 * 1024) if TRAFFIC_1024.get(top) else None
    hbm_peak = measured_hbm_gbs()
    hbm_view = None
    if traffic and hbm_peak:
        gbs = traffic / (kernel_ms[top] * 1e-3) / 1e9
        hbm_view = {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
                    "peak_kind": "measured copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"}
    roofline = {"bound": "fp64", "kernel": f"k_{top}", "achieved": achieved / 1e12,
                "peak": peak.value / 1e12, "unit": "TFLOP/s", "frac": achieved / peak.value,
                "peak_kind": "measured FP64 add/mul issue rate on this GPU (athb_fp64_peak, no FMA)",
                "algorithmic_ops_per_launch": per_launch,
                "traffic": traffic,
                "traffic_note": "ncu dram read+write per launch at 1024x1024, scaled by cells" if traffic else None,
                "hbm_view": hbm_view,
                "step_achieved": step_ops / (ms_step * 1e-3) / 1e12,
                "step_frac": step_ops / (ms_step * 1e-3) / peak.value,
                "kernel_ms": kernel_ms}
    g.close()

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (field-loop initial condition, src/field_loop.c)",
            "config": config_dict(a), "gpu_launches": 7 * a.steps * ws, "roofline": roofline,
            "clocks": clk.summary()}

    if not a.no_e2e:
        line["e2e"] = e2e(a, ath, local, ws, host_unchanged=True)  # every rank: a collective for N > 1
        line["e2e_default_mode"] = e2e(a, ath, local, ws, host_unchanged=False)
    if rank == 0 and ws == 1 and not a.no_cpu and ref_exe().exists():
        r = run_ref_sample(ath, a.cpu_steps, 1, td)
        line["cpu_baseline"] = {"value": r["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                                "sample": f"{a.cpu_steps} main-loop iterations of the {a.nx}x{a.ny} field loop, "
                                          f"1 reference process (-O2 -ffp-contract=off), {cpu_model()}"}
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        torch.distributed.destroy_process_group()


def e2e(a, ath: Path, device: int = 0, ws: int = 1, host_unchanged: bool = True) -> dict:
    """The same metric through the reference-named drop-in ABI: the reference
    main loop (integrate_2d, new_dt, set_bvals) on a pinned host Grid, which
    after every call holds exactly what the reference's would.
    host_unchanged: the opt-in mode for loops that do not write the Grid
    between calls (athb_dropin_set_host_unchanged): the device copy stays
    authoritative, so a step uploads nothing and downloads the cells it writes
    plus the ghost frame; otherwise every call uploads what it reads.  With ws
    ranks each runs its own replica on its GPU (collective: the whole-job
    value uses the slowest rank's time)."""
    from athena_cuda_b200 import Params, configs, problem_state
    from athena_cuda_b200.dropin import DropInLoop, HostGrid

    p = Params(ath)
    cfg = p.config()
    planes = problem_state("field_loop", p)
    dx1, dx2 = (cfg.x1max - cfg.x1min) / cfg.nx1, (cfg.x2max - cfg.x2min) / cfg.nx2
    hg = HostGrid(planes, dx1, dx2, cfg.x1min, cfg.x2min)
    loop = DropInLoop(hg, configs.GAMMA, cfg.cour_no, bc=(4, 4, 4, 4), device=device,
                      host_unchanged=host_unchanged)
    loop.steps(2)  # warm-up
    h0, d0 = loop.bytes_moved()
    t0 = time.perf_counter()
    n = loop.steps(a.e2e_steps)
    dt = time.perf_counter() - t0
    h1, d1 = loop.bytes_moved()
    loop.close()
    hg.close()
    if ws > 1:
        import torch
        dt = max_over_ranks(dt, ws, torch.device("cuda", device))
    path = "integrate_2d + new_dt + set_bvals drop-in calls on a pinned host Grid"
    if host_unchanged:
        path += (" (host-unchanged mode: the device copy is authoritative; per step the cells integrate_2d "
                 "writes and the ghost frame come down, nothing goes up)")
    return {"value": ws * a.nx * a.ny * n / dt, "unit": UNIT, "h2d_bytes_per_step": (h1 - h0) // n,
            "d2h_bytes_per_step": (d1 - d0) // n, "steps": n, "path": path}


def _time_ly(g, ly: int) -> float:
    """Predictor ms of a grid at segment length ly (grid advanced 2 steps;
    callers restore the state)."""
    g.ly = ly
    return g.profile(2)["predict"]


def _blast_big() -> dict:
    from athena_cuda_b200 import configs

    b = configs.blast(1024, 1024, tlim=10.0)
    return b


def ensemble_arm(a) -> None:
    """Batched ensemble (configs: 512 blast instances, sizes 64..512 per side,
    per-instance parameters, each to its own t = 0.1): one launch per phase
    (or one persistent cooperative launch per step) for all instances, against
    the same instances run one after another with the single-grid stepper,
    and against the ideal time: the larger of (all zone-cycles at the best
    single-grid per-cell rate, a 1024^2 blast grid) and the longest single
    instance run alone (the chain of dependent steps no batching shortens)."""
    import torch

    from athena_cuda_b200 import Batch, Grid, Params, autotune, ensemble, problem_state

    items = ensemble.instances(a.ensemble_n, seed=2024)
    ws, rank, local = dist_env()
    if ws > 1:
        ensemble_ranks(a, items, ws, rank, local)
        return
    sizes = [(b["grid"]["Nx1"], b["grid"]["Nx2"]) for _, b in items]
    runs = {}
    for mode_name, mode in (("phased", Batch.PHASED), ("persistent", Batch.PERSISTENT)):
        t0 = time.perf_counter()
        batch = Batch.from_problems(items)
        batch.mode = mode
        setup_s = time.perf_counter() - t0
        t1 = time.perf_counter()
        tune = autotune.tune_batch(batch, sizes, cache=Path(tempfile.gettempdir()) / "athb_ly_tuning.json")
        tune_s = time.perf_counter() - t1
        batch.timing(1)
        stream = torch.cuda.ExternalStream(batch.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        e0.record(stream)
        launches = batch.run(100000)
        e1.record(stream)
        torch.cuda.synchronize()
        batched_s = time.perf_counter() - w0
        phase_ms = batch.timing(0)
        finals = [batch.download(k) for k in range(batch.n)]
        zc = sum(nx1 * nx2 * f[3] for (nx1, nx2), f in zip(sizes, finals))
        assert all(f[2] == 0.1 for f in finals), "every instance ends at its t = 0.1"
        batch.close()
        if runs:
            first = next(iter(runs.values()))
            assert all(np.array_equal(f[0], g[0]) for f, g in zip(finals, first["finals"])), "modes differ"
        runs[mode_name] = {"batched_s": batched_s, "batched_device_ms": e0.elapsed_time(e1), "setup_s": setup_s,
                           "tune_s": tune_s, "launches": launches, "phase_ms": phase_ms, "ly_table": tune,
                           "finals": finals, "zc": zc}
    best_mode = min(runs, key=lambda m: runs[m]["batched_s"])
    finals, zc, batched_s = runs[best_mode]["finals"], runs[best_mode]["zc"], runs[best_mode]["batched_s"]

    # sequential single-grid runs of the same instances: (1) the CUDA-graph
    # loop (segment length tuned for an isolated grid), (2) plain launches with
    # the host reading the clock after every step, as a solver driving one
    # grid at a time from the host does
    stride = a.seq_sample if a.seq_sample > 0 else 1
    seq_s, seq_zc, checked, plain_s = 0.0, 0, 0, 0.0
    longest_s = 0.0
    iso_ly = {}
    for k in range(0, len(items), stride):
        name, blocks = items[k]
        p = Params.from_blocks(blocks)
        g = Grid.create(p.config())
        g.upload(problem_state(name, p))
        g.set_bvals()
        g.new_dt()
        if sizes[k] not in iso_ly:
            best, _ = min(((ly, _time_ly(g, ly)) for ly in (1, 2, 4, 8, 16, 32) if ly <= sizes[k][1] + 3),
                          key=lambda x: x[1])
            iso_ly[sizes[k]] = best
            g.upload(problem_state(name, p))  # the trials advanced the grid
            g.set_bvals()
            g.new_dt()
        g.ly = iso_ly[sizes[k]]
        torch.cuda.synchronize()
        w = time.perf_counter()
        g.run(100000)
        one_s = time.perf_counter() - w
        seq_s += one_s
        longest_s = max(longest_s, one_s)
        planes, dt, t, n = g.download()
        # (2) one step per call, host reads the clock every step
        g.upload(problem_state(name, p))
        g.set_bvals()
        g.new_dt()
        torch.cuda.synchronize()
        w = time.perf_counter()
        while not g.status()["done"]:
            g.run_async(1)
        plain_s += time.perf_counter() - w
        seq_zc += sizes[k][0] * sizes[k][1] * n
        if k % 64 == 0:  # bit-exact spot check against the batched result
            assert np.array_equal(planes, finals[k][0]) and n == finals[k][3]
            checked += 1
        g.close()
    scale = 1.0 if stride == 1 else zc / seq_zc
    # the best single-grid rate: a 1024^2 blast grid, best segment length,
    # 20 steps of the CUDA-graph loop timed with events
    p = Params.from_blocks(_blast_big())
    g = Grid.create(p.config())
    g.upload(problem_state("blast", p))
    g.set_bvals()
    g.new_dt()
    g.ly = min(((ly, _time_ly(g, ly)) for ly in (4, 8, 16, 32)), key=lambda x: x[1])[0]
    g.run(3)
    big_stream = torch.cuda.ExternalStream(g.stream)
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record(big_stream)
    g.run_async(20)
    b1.record(big_stream)
    b1.synchronize()
    best_rate = 1024 * 1024 * 20 / (b0.elapsed_time(b1) * 1e-3)
    g.close()
    ideal_s = max(zc / best_rate, longest_s)
    line = {"metric": "ensemble zone-cycles/s (512 blast instances to t=0.1, batched)",
            "value": zc / batched_s, "unit": UNIT, "n_gpus": 1, "dtype": "f64", "data": "synthetic (seeded blast ensemble)",
            "config": {"workload": f"blast ensemble n={len(items)} sizes 64..512 per side", "seed": 2024,
                       "batch_mode": best_mode},
            "zone_cycles": zc, "batched_s": batched_s,
            "modes": {m: {k: v for k, v in r.items() if k not in ("finals", "zc")} | {"zc_per_s": r["zc"] / r["batched_s"]}
                      for m, r in runs.items()},
            "sequential_s": seq_s * scale, "sequential_zc_per_s": seq_zc / seq_s,
            "speedup_vs_sequential": (seq_s * scale) / batched_s,
            "sequential_plain_s": plain_s * scale, "speedup_vs_sequential_plain": (plain_s * scale) / batched_s,
            "sequential_sample_stride": stride, "bit_exact_spot_checks": checked,
            "ideal": {"s": ideal_s, "best_single_grid_zc_per_s": best_rate, "work_bound_s": zc / best_rate,
                      "longest_instance_s": longest_s if stride == 1 else None,
                      "speedup_bound_vs_sequential_plain": (plain_s * scale) / ideal_s,
                      "batched_over_ideal": batched_s / ideal_s}}
    ref = ROOT / "oracle" / "_ref" / "athref_blast_roe"
    if ref.exists():
        # the reference CPU path, one process per host core (up to 16, each
        # ~10 MB per instance), on the first instances of the same ensemble
        from athena_cuda_b200 import write_athinput

        cores = max(1, min(os.cpu_count() or 1, 16))
        with tempfile.TemporaryDirectory() as td:
            aths = [write_athinput(Path(td) / f"athinput.{k}", items[k][1]) for k in range(cores)]
            r = run_ref_instances(aths, "blast", Path(td))
        line["cpu_baseline"] = {"value": r["value"], "unit": UNIT, "cores": cores, "kind": "reference",
                                "sample": f"instances 0..{cores - 1} of the ensemble, one single-threaded "
                                          f"reference process each (-O2 -ffp-contract=off), up to 20 s of "
                                          f"main loop each; {cpu_model()}"}
    print(json.dumps(line))


def run_batch(items, local: int, mode: int):
    """One Batch of `items` on GPU `local`, tuned, run to every end time;
    (wall seconds, zone-cycles, final states)."""
    import torch

    from athena_cuda_b200 import Batch, autotune

    for _, b in items:
        b["job"]["device"] = local
    sizes = [(b["grid"]["Nx1"], b["grid"]["Nx2"]) for _, b in items]
    batch = Batch.from_problems(items)
    batch.mode = mode
    autotune.tune_batch(batch, sizes, cache=Path(tempfile.gettempdir()) / f"athb_ly_tuning_{local}.json")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch.run(100000)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    finals = [batch.download(k) for k in range(batch.n)]
    batch.close()
    return wall, sum(nx1 * nx2 * f[3] for (nx1, nx2), f in zip(sizes, finals)), finals


def ensemble_ranks(a, items, ws: int, rank: int, local: int) -> None:
    """The ensemble bin-packed over ws GPUs (ensemble.partition by estimated
    work), each rank one phased Batch of its share, no communication but the
    timing: whole-job zone-cycles/s over the slowest rank's time."""
    import datetime

    import torch

    from athena_cuda_b200 import Batch, ensemble

    torch.cuda.set_device(local)
    torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                         device_id=torch.device("cuda", local))
    mine = [items[k] for k in ensemble.partition(items, ws)[rank]]
    torch.distributed.barrier()
    wall, zc, _ = run_batch(mine, local, Batch.PHASED)
    worst = max_over_ranks(wall, ws, torch.device("cuda", local))
    t = torch.tensor([float(zc)], dtype=torch.float64, device=torch.device("cuda", local))
    torch.distributed.all_reduce(t)
    if rank == 0:
        print(json.dumps({"metric": "ensemble zone-cycles/s (512 blast instances to t=0.1, batched)",
                          "value": float(t.item()) / worst, "unit": UNIT, "n_gpus": ws, "scaling": "strong",
                          "dtype": "f64", "data": "synthetic (seeded blast ensemble)",
                          "config": {"workload": f"blast ensemble n={len(items)} sizes 64..512 per side",
                                     "seed": 2024, "batch_mode": "phased", "parallelism": f"partitioned x{ws}"},
                          "zone_cycles": float(t.item()), "batched_s": worst}))
    torch.distributed.destroy_process_group()


def cpaw_arm(a) -> None:
    """The circularly polarised Alfven wave over one period (32x16 .. 512x256,
    Roe and HLLE): L1 error against the initial state (src/cpaw2d.c:222-302)
    on the GPU, its convergence order, the reference CPU path's own L1 output
    beside it (oracle/_ref, when built), and the GPU time per run."""
    import torch

    from athena_cuda_b200 import Grid, configs, write_athinput

    sizes = [(32, 16), (64, 32), (128, 64), (256, 128), (512, 256)]
    rows = []
    with tempfile.TemporaryDirectory() as td:
        for flux in ("roe", "hlle"):
            prev = None
            for nx1, nx2 in sizes:
                d = Path(td) / f"{flux}_{nx1}"
                d.mkdir()
                ath = write_athinput(d / "athinput", configs.cpaw2d(nx1, nx2, flux=flux))
                g = Grid.from_athinput(ath, "cpaw2d")
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                g.run(1_000_000)
                wall = time.perf_counter() - t0
                err = [float(x) for x in g.cpaw2d_errors()]
                n = g.status()["nstep"]
                g.close()
                row = {"flux": flux, "nx1": nx1, "nx2": nx2, "steps": n, "gpu_s": wall, "l1_rms": err[0],
                       "order": None if prev is None else math.log2(prev / err[0])}
                exe = ROOT / "oracle" / "_ref" / f"athref_cpaw2d_{flux}"
                if exe.exists():
                    subprocess.run([str(exe), "-i", str(ath), "--l1", "--quiet"], cwd=d, check=True,
                                   capture_output=True)
                    last = [l for l in (d / "cpaw2d-errors.dat").read_text().splitlines() if not l.startswith("#")][-1]
                    ref_rms = float(last.split()[2])
                    row["ref_l1_rms"] = ref_rms
                    row["same_to_6_digits"] = float(f"{err[0]:e}") == ref_rms
                rows.append(row)
                prev = err[0]
    print(json.dumps({"workload": "cpaw2d convergence, one period (t = 1/sqrt(5)), Roe and HLLE",
                      "metric": "L1 RMS error vs the initial state", "rows": rows}))


def configs_arm(a) -> None:
    """Every plain configuration of the reference's benchmark set run to its
    end time on the GPU (device-resident loop, CUDA events), beside the
    reference CPU path on one core (the whole run when it takes under ~30 s,
    else a bounded number of steps)."""
    import torch

    from athena_cuda_b200 import Grid, configs, write_athinput

    cases = [
        ("blast 200x300 to t=0.2", "blast", configs.blast(200, 300), None),
        ("field loop 1024x512 to t=1", "field_loop", configs.field_loop(1024, 512), 20),
        ("field loop 2048x2048 to t=1", "field_loop", configs.field_loop(2048, 2048), 3),
    ]
    rows = []
    with tempfile.TemporaryDirectory() as td:
        for label, problem, blocks, ref_steps in cases:
            d = Path(td) / problem
            d.mkdir(exist_ok=True)
            ath = write_athinput(d / f"athinput.{len(rows)}", blocks)
            g = Grid.from_athinput(ath, problem)
            stream = torch.cuda.ExternalStream(g.stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            g.run(10_000_000)
            e1.record(stream)
            torch.cuda.synchronize()
            st = g.status()
            g.close()
            cells = blocks["grid"]["Nx1"] * blocks["grid"]["Nx2"]
            gpu = cells * st["nstep"] / (e0.elapsed_time(e1) * 1e-3)
            row = {"config": label, "steps": st["nstep"], "time": st["time"], "gpu_s": e0.elapsed_time(e1) * 1e-3,
                   "gpu_zc_per_s": gpu}
            exe = ROOT / "oracle" / "_ref" / f"athref_{problem}_roe"
            if exe.exists():
                r = run_ref_sample(ath, ref_steps or 10_000_000, 1, d, max_seconds=30.0, exe=exe)
                row.update(ref_zc_per_s=r["value"], ref_seconds=r["seconds"],
                           ref_sample="whole run" if ref_steps is None else f"{ref_steps} steps",
                           speedup=gpu / r["value"])
            rows.append(row)
    print(json.dumps({"workload": "plain configurations to their end times, Roe, FP64", "unit": UNIT,
                      "cpu": cpu_model(), "rows": rows}))


def adjoint_arm(a) -> None:
    """Cost of the adjoint: the gradient of the field loop's final magnetic
    energy with respect to its initial density (1 + 0.01 N(0,1) smoothed by a
    4-cell Gaussian, seed 2024) over N x N cells and K steps, against a plain
    forward solve of the same K steps (the graph-captured device loop).  Both
    timed with a device synchronisation on each side (the adjoint call returns
    synchronised); ratio = adjoint / forward, lower is better.  Both warm: the
    forward is the faster of two runs, the adjoint the second of two calls
    with the workspace kept (the first call's time, which includes
    allocating the workspace, is `adjoint_cold_s`)."""
    import torch

    from athena_cuda_b200 import Grid, Params, configs, problem_state, write_athinput
    from athena_cuda_b200 import adjoint as fl

    rows = []
    with tempfile.TemporaryDirectory() as td:
        for case in a.adj_cases.split(","):
            n, k = (int(x) for x in case.split("x"))
            blocks = configs.field_loop(n, n)
            blocks["time"]["nlim"] = k
            ath = write_athinput(Path(td) / f"athinput.{n}", blocks)
            base = problem_state("field_loop", Params(ath))
            S0 = fl.density_state(base, fl.smoothed_density(n, n, 2024))
            g = Grid.from_athinput(ath, "field_loop")
            # forward solve: loop entry (set_bvals, new_dt) then K steps
            fwd = []
            for _ in range(2):
                g.upload(S0)
                g.set_bvals()
                g.new_dt()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                g.run(k)
                torch.cuda.synchronize()
                fwd.append(time.perf_counter() - t0)
            # the gradient twice with the workspace kept: the first call
            # allocates it (cold), the second reuses it (warm, the cost of
            # every further gradient, e.g. in an optimisation loop)
            g.keep_adjoint_workspace(True)
            snap = int(a.adj_snapshot_gb * 1e9)
            t_calls = []
            for _ in range(2):
                g.upload(S0)
                t0 = time.perf_counter()
                J, grad, st = g.adjoint_gradient(k, snapshot_bytes=snap)
                t_calls.append(time.perf_counter() - t0)
            g.close()
            t_adj = t_calls[1]
            grho = fl.density_gradient(base, grad)
            t_fwd = min(fwd)
            rows.append({"case": f"field loop {n}x{n}, {k} steps", "forward_s": t_fwd, "adjoint_s": t_adj,
                         "adjoint_cold_s": t_calls[0], "ratio": t_adj / t_fwd, "ratio_cold": t_calls[0] / t_fwd,
                         "J": J, "grad_rho_l2": float(np.sqrt(np.sum(grho * grho))),
                         "adjoint_zone_cycles_per_s": n * n * k / t_adj, "stats": st})
    head = rows[-1]
    print(json.dumps({"metric": "adjoint/forward cost ratio (gradient of final magnetic energy w.r.t. initial "
                                "density, field loop)", "value": head["ratio"], "unit": "x",
                      "higher_is_better": False, "n_gpus": 1, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": head["case"], "objective": "sum (B1c^2+B2c^2)/2",
                                 "checkpointing": "binomial (revolve) state snapshots in HBM"},
                      "rows": rows}))


def measured_hbm_gbs():
    """HBM copy bandwidth measured on this GPU pool (MEASURED_PEAKS.json)."""
    f = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(f.read_text())["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0  # earlier measurement on the same pool


def main():
    a = parse()
    if a.impl == "reference":
        reference_arm(a)
    elif a.workload == "ensemble":
        ensemble_arm(a)
    elif a.workload == "cpaw":
        cpaw_arm(a)
    elif a.workload == "configs":
        configs_arm(a)
    elif a.workload == "adjoint":
        adjoint_arm(a)
    else:
        ours(a)


if __name__ == "__main__":
    main()
