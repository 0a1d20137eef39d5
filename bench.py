"""Benchmark of the fused surface-flow step (one JSON line on rank 0).

Workload: the 3-hour dam-break on a 4096 x 8192 grid (33.5 M cells, dx 5 m, FP32 state with the
split bed/depth slope), seeded synthetic inputs (hydropol2d_b200.synthetic.dambreak_case).  A step
is one accepted time step of HydroPol2D_Main_While over the whole grid (rain, infiltration (off
here), local-inertial fluxes, draining limiter, continuity, outlet sink, maxima, CFL reduction and
timestep refresh) -- one fused kernel launch.

The run goes from t = 0 to the end of the 3 simulated hours, every launch timed with CUDA events
(`full_run`: cells x steps / device time over the whole simulation, with the time-averaged wet
fraction).  The headline window (`value`) is taken when the clock first passes 60 min, a third of
the way through the flood: W untimed warm-up steps, then K timed steps.  The same K steps with the
dry skips switched off give `dense_window` (every record read, stepped and written; bit-identical
results).  `roofline.achieved` counts the dense algorithmic bytes of every cell of the grid, 40 B
per cell-update (h, q_x, q_y, z and n^2 read, 20 B; h, q_x, q_y written, 12 B; the running
maximum depth read and written, 8 B), over the launch time; `bytes_still_moved` is what the
kernel's records moved after the dry skips.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --workload wet|dambreak|urban|unet|ensemble [...]   one profiling line

N > 1 runs under torchrun, one rank per GPU, each rank an independent dam-break member
(different DEM seed): ensemble members share nothing, so there is no collective on the data path
(weak scaling).  The 256-member ensemble leg is split the same way (hydropol2d_b200.sharding),
members/h is the whole job's.  Timing: CUDA events on the library's stream, barrier + synchronize
on both sides, max over ranks.  The state (~1.5 GB) is far larger than L2, so no flush is needed
between steps.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NY, NX, DX = 4096, 8192, 5.0
WORKLOAD = "dambreak_4096x8192_dx5_fp32_3h"
METRIC = "GCell-updates/s"
WINDOW_MIN = 60.0          # the headline window starts when the clock first passes this [min]
# algorithmic HBM bytes per cell-update of the step without rain and infiltration: h, q_x, q_y,
# z, n^2 read (20 B), h, q_x, q_y written (12 B), the running maximum read and written (8 B)
ALG_BYTES_PER_CELL = 40.0
# bytes the fused kernel's records move per cell on a dense step: static record {dz_x, dz_y, n^2,
# meta} 16 B + state record 16 B read, state record 16 B written
RECORD_BYTES_PER_CELL = 48.0
# Green-Ampt step (configuration 2): + soil record {I, T} read and written, 2 x 8 B
RECORD_BYTES_PER_CELL_GA = 64.0
ALG_BYTES_PER_CELL_GA = 49.0   # + I read/write 8 B + soil class 1 B
# DRAM bytes per cell of one launch in the headline window, measured with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum of k_fused_step, three launches: 240.2 MB per
# launch over 2048 x 8192 cells) on the same dam-break with 2048 rows advanced to the 60-minute
# mark (28 % wet), scaled per cell; the bench grid's window is 29 % wet
NCU_DRAM_BYTES_PER_CELL = 14.32


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            vis = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
            gid = vis[self.device] if self.device < len(vis) else str(self.device)
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={gid}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.flush()
        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[4], parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k, v in enumerate(r[4]) if v.lower() == "active"})
        loaded = [r for r in rows if r[2] > 200.0] or rows
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": max(r[1] for r in rows),
                "power_w_max": max(r[2] for r in rows), "samples": len(rows), "reasons": reasons}


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_port_gcups(budget_s: float, steps_hint: int | None = None):
    """Kernel-form CPU restatement (FP64, OpenMP over all host cores) on a row strip of
    the same dam-break workload; returns (GCUPS, sample description, cores)."""
    import oracle
    from hydropol2d_b200 import synthetic as S
    cores = cpu_cores()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    rows = 256
    case = S.dambreak_case(rows, NX, DX, seed=11)
    o = oracle.KernelFormOracle(rows, NX, DX, "fp64", **case.params)
    case.apply(o)
    o.fused_steps(2)
    t0 = time.perf_counter()
    o.fused_steps(3)
    per = (time.perf_counter() - t0) / 3
    n = steps_hint if steps_hint else max(3, int(budget_s / max(per, 1e-6)))
    t0 = time.perf_counter()
    o.fused_steps(n)
    el = time.perf_counter() - t0
    return rows * NX * n / el / 1e9, f"{rows}x{NX} strip of the dam-break grid, {n} steps, FP64", cores


def run_reference(args, rank, world):
    """Reference arm: the CPU restatement timed on the host cores, rank 0 only."""
    if rank != 0:
        return
    import oracle
    from hydropol2d_b200 import synthetic as S
    cores = cpu_cores()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    # each step is a bounded sample (a row strip of the grid) so K+W steps end in minutes
    budget = 120.0
    rows = 64
    case = S.dambreak_case(rows, NX, DX, seed=11)
    o = oracle.KernelFormOracle(rows, NX, DX, "fp64", **case.params)
    case.apply(o)
    t0 = time.perf_counter()
    o.fused_steps(2)
    per_cell = (time.perf_counter() - t0) / 2 / (rows * NX)
    rows = int(min(1024, max(8, budget / max(args.steps + args.warmup, 1) / (per_cell * NX))))
    case = S.dambreak_case(rows, NX, DX, seed=11)
    o = oracle.KernelFormOracle(rows, NX, DX, "fp64", **case.params)
    case.apply(o)
    o.fused_steps(args.warmup)
    t0 = time.perf_counter()
    o.fused_steps(args.steps)
    el = time.perf_counter() - t0
    v = rows * NX * args.steps / el / 1e9
    sample = f"{rows}x{NX} row strip of the {NY}x{NX} dam-break grid per step, FP64 kernel-form restatement"
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded dam-break, hydropol2d_b200.synthetic.dambreak_case)",
        "config": {"workload": WORKLOAD, "sample_rows": rows},
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "MATLAB/Octave are not installed: the reference's own CPU path cannot run here; "
                "this is the C++ restatement of its arithmetic (oracle/kernel_form.hpp). It updates "
                "every cell every step, so its rate does not depend on the window.",
    }
    print(json.dumps(line), flush=True)


def ensemble_leg(device: int, n_members: int = 256) -> dict | None:
    """The batched-ensemble configuration: 256 members with sides log-uniform in
    [256, 1024] (multiples of 32), rain or breach forcing, run to their own end times in one
    persistent launch per step; the launch shape is autotuned first (trial steps undone).
    With N ranks every rank runs its share of the members on its own GPU (balanced by an a
    priori cost, no collective on the data path) and the job's time is the slowest rank's.
    Returns the summary on rank 0, None elsewhere."""
    from hydropol2d_b200 import synthetic as S
    from hydropol2d_b200.sharding import run_sharded
    costs = [S.ensemble_member_cost(i) for i in range(n_members)]
    res = run_sharded(S.ensemble_member, n_members, costs=costs, device=device)
    if res is None:
        return None
    ks = [r["steps"] for r in res["results"]]
    return {"members": n_members, "ranks": res["ranks"], "members_per_rank": res["members_per_rank"],
            "members_per_h": res["members_per_h"], "seconds": res["seconds"], "gcups": res["gcups"],
            "cells": sum(r["cells"] for r in res["results"]), "launches_rank0": res["launches_rank0"],
            "rows_per_warp_rank0": res["rows_per_warp_rank0"],
            "steps_min": min(ks), "steps_max": max(ks), "steps_mean": float(np.mean(ks)),
            "breach_members": sum(S.ensemble_member_spec(i)["kind"] == "breach" for i in range(n_members)),
            "timing": "CUDA events on each rank's ensemble stream around every launch until its last "
                      "member reaches its routing_time; max over ranks"}


def accuracy_leg(device: int, n_members: int = 12) -> dict:
    """The north star's peak-depth gate (<= 1 cm against FP64) measured on ensemble members at
    256 x 256: each member run to its end time in FP32 and in FP64 (the FP64 path is bit-exact
    with the FP64 oracle), per forcing kind the largest per-member peak-depth error and the
    largest share of cells beyond 1 cm."""
    from hydropol2d_b200 import SurfaceFlow, synthetic as S
    kinds: dict = {}
    for i in range(n_members):
        spec = S.ensemble_member_spec(i, lo=256, hi=256)
        c = S.ensemble_member(i, lo=256, hi=256)
        peaks = []
        for prec in ("fp32", "fp64"):
            sf = SurfaceFlow(*c.shape, c.resolution, prec, device=device, **c.params)
            c.apply(sf)
            sf.run()
            peaks.append(sf.download("dmax") / 1000.0)
            sf.close()
        err = np.abs(peaks[0] - peaks[1])
        err = err[np.isfinite(err)]
        k = kinds.setdefault(spec["kind"], {"members": 0, "max_peak_err_m": 0.0, "max_cells_over_1cm_pct": 0.0,
                                            "members_within_1cm": 0})
        k["members"] += 1
        k["max_peak_err_m"] = max(k["max_peak_err_m"], float(err.max()))
        k["max_cells_over_1cm_pct"] = max(k["max_cells_over_1cm_pct"], 100.0 * float(np.mean(err > 0.01)))
        k["members_within_1cm"] += int(err.max() <= 0.01)
    return {"gate": "peak depth within 1 cm of FP64", "size": "256 x 256", "by_kind": kinds}


def urban_leg(device: int, n: int = 2048, peak: float | None = None) -> dict:
    """Configuration 2: urban rain-on-grid 2048 x 2048 (dx 2 m) with Green-Ampt soils and 64 x 64
    rain maps changing every 5 minutes, run over its whole 2 simulated hours (every launch timed)."""
    from hydropol2d_b200 import SurfaceFlow, synthetic as S
    case = S.urban_case(n, 2.0, seed=7, hours=2.0)
    sf = SurfaceFlow(n, n, 2.0, "fp32", device=device, **case.params)
    case.apply(sf)
    sf.fused_steps(20)
    ms_win = sf.fused_steps_timed(200)
    steps, ms = 220, ms_win
    while True:
        d = sf.diag()
        if d["t"] > case.params["routing_time"] + case.params["min_time_step"] / 60:
            break
        ms += sf.fused_steps_timed(2000)
        steps += 2000
    d = sf.diag()
    steps_done = d["k"] - 1
    sf.close()
    cells = n * n
    g_win = cells * 200 / (ms_win / 1e3) / 1e9
    out = {"workload": f"urban_{n}x{n}_dx2_green_ampt_rainmaps_2h", "window_gcups": g_win,
           "window_ms_per_step": ms_win / 200, "full_run_steps": steps_done,
           "full_run_gcups": cells * steps_done / (ms / 1e3) / 1e9, "sim_minutes": d["t"],
           "record_bytes_per_cell": RECORD_BYTES_PER_CELL_GA, "alg_bytes_per_cell": ALG_BYTES_PER_CELL_GA,
           "window_record_gbs": RECORD_BYTES_PER_CELL_GA * g_win,
           "window_alg_gbs": ALG_BYTES_PER_CELL_GA * g_win}
    if peak:
        out["window_record_hbm_frac"] = out["window_record_gbs"] / peak
    return out


def run_surrogate(args):
    """Learned screening at the configuration's size: 4096 solver runs on 256 x 256 tiles
    train three U-Nets; 1024 held-out members are screened (inference + reruns of members
    whose networks disagree by more than 5 cm) and compared with the plain batched solver
    and, on a subset, with the FP64 solver."""
    from hydropol2d_b200 import build, screening
    build.build()
    res = screening.study(n_train=4096, n_test=1024, size=256, epochs=args.surrogate_epochs,
                          batch=16, n_fp64=64, log=lambda m: print(m, file=sys.stderr, flush=True))
    line = {"metric": "ensemble members/h", "value": res["screened_members_per_h"], "unit": "members/h",
            "n_gpus": 1, "higher_is_better": True, "dtype": "bf16 network / f32 solver",
            "data": "synthetic (seeded members, hydropol2d_b200.synthetic.ensemble_member, 256 x 256)",
            "config": {"workload": "screening_4096train_1024test_256x256", "threshold_m": 0.05},
            "vs_baseline": None, "impl": "ours", "study": res}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- profiling workloads
_WL_SHAPE = [0, 0]   # profiling workloads: cells per lane and rows per warp (0: the library's)


def _apply_shape(g) -> None:
    if _WL_SHAPE[0]:
        g.set_layout(_WL_SHAPE[0])
    if _WL_SHAPE[1]:
        g.set_tuning(_WL_SHAPE[1])


def workload_wet(steps: int, tb: int = 1) -> str:
    """The V-tilted catchment geometry on 2048 x 2048 cells (dx 10 m) plus a 0.5 m random field,
    5 cm of water everywhere and 60 mm/h of rain: every cell takes the full local-inertial path
    of the fused step (no dry-row shortcuts).  tb > 1: the same without rain, in blocks of tb
    steps (temporal blocking runs without rain)."""
    from hydropol2d_b200 import SurfaceFlow, synthetic as S
    z, ch = S.vtilt_domain(2048, 2048, 10.0, 0.005, 0.002)
    z = z + 0.5 * S.gaussian_random_field(2048, 2048, -3.0, 5)
    p = dict(routing_time=600.0, alfa_min=0.7, alfa_max=0.7, outlet_type=1, slope_outlet=0.002,
             min_time_step=0.01, max_time_step=10.0)
    case = S.Case("wet2048", z, np.full(z.shape, 0.03), 10.0, np.zeros(ch.size, dtype=np.int32),
                  ch.astype(np.int32), p, np.full(z.shape, 50.0),
                  rain_uniform=None if tb > 1 else (np.array([0.0]), np.array([60.0])))
    g = SurfaceFlow(2048, 2048, 10.0, "fp32", **p)
    case.apply(g)
    _apply_shape(g)
    if tb > 1:
        g.set_temporal_blocking(tb)
    g.fused_steps(steps)
    n = 240
    ms = g.fused_steps_timed(n)
    g.close()
    return "wet 2048^2%s: %.4f ms/step, %.1f GCUPS" % (f" (blocks of {tb})" if tb > 1 else "", ms / n,
                                                       2048 * 2048 * n / ms / 1e6)


def workload_dambreak(ny: int, steps: int, advance_min: float, state: str | None, timed: int, tb: int = 1) -> str:
    """The bench's dam-break on ny x 8192 cells.  advance_min > 0 runs it to that clock first;
    --state FILE saves the state reached there (.npz) or, when FILE exists, starts from it."""
    from hydropol2d_b200 import SurfaceFlow, synthetic as S
    case = S.dambreak_case(ny, 8192, 5.0, seed=11)
    g = SurfaceFlow(ny, 8192, 5.0, "fp32", **case.params)
    case.apply(g)
    _apply_shape(g)
    if state and Path(state).exists():
        z = np.load(state)
        g.set_state(z["h"].astype(np.float64) * 1000.0,
                    np.stack([z["qx"], z["qy"]]).astype(np.float64) / 5.0 * 3.6e6)
        g.set_clock(float(z["t"]), float(z["ts"]), int(z["k"]))
    elif advance_min > 0:
        while g.diag()["t"] < advance_min:
            g.fused_steps(1000)
        if state:
            d = g.diag()
            np.savez(state, h=g.download_native("h"), qx=g.download_native("qx"), qy=g.download_native("qy"),
                     t=d["t"], ts=d["time_step"], k=d["k"])
    if tb > 1:
        g.set_temporal_blocking(tb)
    g.fused_steps(steps)
    ms = g.fused_steps_timed(timed)
    t = g.diag()["t"]
    wet = float(np.mean(g.download_native("h") > 0))
    g.close()
    return ("dambreak %dx8192 at t=%.1f min (%.1f%% wet)%s: %.4f ms/step, %.1f GCUPS"
            % (ny, t, 100 * wet, f" blocks of {tb}" if tb > 1 else "", ms / timed, ny * 8192 * timed / ms / 1e6))


def workload_urban(n: int, steps: int, timed: int) -> str:
    from hydropol2d_b200 import SurfaceFlow, synthetic as S
    case = S.urban_case(n, 2.0, seed=7, hours=2.0)
    g = SurfaceFlow(n, n, 2.0, "fp32", **case.params)
    case.apply(g)
    _apply_shape(g)
    g.fused_steps(steps)
    ms = g.fused_steps_timed(timed)
    g.close()
    return "urban %dx%d (Green-Ampt, rain maps): %.4f ms/step, %.1f GCUPS" % (n, n, ms / timed, n * n * timed / ms / 1e6)


def workload_unet(batch: int) -> str:
    import torch
    from hydropol2d_b200 import nn
    from hydropol2d_b200.surrogate import UNet, forward_flops
    net = UNet(seed=0)
    x = torch.randn(batch, 256, 256, 4, device="cuda").to(torch.bfloat16)
    for _ in range(3):
        net.predict(x)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        net.predict(x)
    e1.record()
    torch.cuda.synchronize()
    ms_f = e0.elapsed_time(e1) / 10
    f = forward_flops(256, 256) * batch
    t = torch.randn(batch * 256 * 256, 2, device="cuda")
    w = torch.ones_like(t)
    for _ in range(3):
        net.train_step(x, t, w, 1e-4)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(5):
        net.train_step(x, t, w, 1e-4)
    e1.record()
    torch.cuda.synchronize()
    ms_t = e0.elapsed_time(e1) / 5
    nn.check()
    return ("unet B=%d 256^2: forward %.3f ms (%.1f TFLOP/s), training step %.3f ms (%.1f TFLOP/s, 3x forward)"
            % (batch, ms_f, f / ms_f / 1e9, ms_t, 3 * f / ms_t / 1e9))


def workload_ensemble(members: int, launches: int) -> str:
    from hydropol2d_b200 import SurfaceFlow, synthetic as S
    from hydropol2d_b200.ensemble import Ensemble
    ens = Ensemble()
    for i in range(members):
        c = S.ensemble_member(i)
        g = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(g)
        ens.add(g)
    ens.set_tuning(64)
    ens.steps(4)
    _, ms = ens.steps_timed(launches)
    cells = ens.cells()
    ens.close()
    return "ensemble %d members: %.4f ms/launch, %.1f GCUPS" % (members, ms / launches, cells * launches / ms / 1e6)


def run_workload(args):
    from hydropol2d_b200 import build
    build.build()
    w = args.workload
    _WL_SHAPE[:] = [args.layout, args.rpw]
    if w == "wet":
        line = workload_wet(args.steps, args.tb)
    elif w == "dambreak":
        line = workload_dambreak(args.ny, args.steps, args.advance_min, args.state, args.timed, args.tb)
    elif w == "urban":
        line = workload_urban(args.nx if args.nx != NX else 2048, args.steps, args.timed)
    elif w == "unet":
        line = workload_unet(args.batch)
    else:
        line = workload_ensemble(args.members, args.launches)
    print(line, flush=True)


# ---------------------------------------------------------------- the benchmark
def pinned(a: np.ndarray) -> np.ndarray:
    """A copy of `a` in page-locked host memory (the end-to-end leg's inputs and outputs)."""
    import torch
    t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
    out = t.numpy()
    out[...] = a
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ny", type=int, default=NY)
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 256-member ensemble leg")
    ap.add_argument("--no-urban", action="store_true", help="skip the urban Green-Ampt leg")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP32-vs-FP64 peak-depth leg")
    ap.add_argument("--window-min", type=float, default=WINDOW_MIN,
                    help="clock [min] the headline window starts at")
    ap.add_argument("--hours", type=float, default=3.0, help="simulated hours of the dam-break run")
    ap.add_argument("--surrogate", action="store_true",
                    help="run the learned-screening study instead (4096 training / 1024 held-out members)")
    ap.add_argument("--surrogate-epochs", type=int, default=8)
    ap.add_argument("--workload", choices=["wet", "dambreak", "urban", "unet", "ensemble"],
                    help="print one timing line of a profiling workload instead")
    ap.add_argument("--advance-min", type=float, default=0.0)
    ap.add_argument("--state", default=None)
    ap.add_argument("--timed", type=int, default=240)
    ap.add_argument("--tb", type=int, default=1, help="profiling workloads: steps per temporal block")
    ap.add_argument("--layout", type=int, default=0, help="profiling workloads: cells per lane (1 or 2)")
    ap.add_argument("--rpw", type=int, default=0, help="profiling workloads: rows per warp")
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--launches", type=int, default=64)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_env()

    if args.workload:
        run_workload(args)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.surrogate:
        run_surrogate(args)
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from hydropol2d_b200 import SurfaceFlow, build, synthetic as S
    if rank == 0:
        build.build()
    if dist is not None:
        dist.barrier()

    ny, nx = args.ny, args.nx
    cells = ny * nx
    t_e2e0 = time.perf_counter()
    case = S.dambreak_case(ny, nx, DX, seed=11 + rank, hours=args.hours)
    t_gen = time.perf_counter() - t_e2e0
    t_end = case.params["routing_time"] + case.params["min_time_step"] / 60

    # ---- the whole simulation, every launch timed; the headline window at WINDOW_MIN --------
    sf = SurfaceFlow(ny, nx, DX, "fp32", device=local, **case.params)
    case.apply(sf)
    chunk = 1000
    run_ms, run_steps, wet_samples, trace = 0.0, 0, [], []
    win = None
    with ClockSampler(local) as clocks:
        while True:
            d = sf.diag()
            if d["t"] > t_end:
                break
            if win is None and d["t"] >= args.window_min:
                # headline window: W warm-up steps, then K timed steps (all part of the run)
                run_ms += sf.fused_steps_timed(args.warmup)
                h0_mm = sf.download("depth")
                of0 = np.stack([sf.download("qout_right"), sf.download("qout_up")])
                run_steps += args.warmup
                if dist is not None:
                    dist.barrier()
                torch.cuda.synchronize()
                d0 = sf.diag()
                ms = sf.fused_steps_timed(args.steps)
                torch.cuda.synchronize()
                d1 = sf.diag()
                run_ms += ms
                run_steps += args.steps
                if dist is not None:
                    t = torch.tensor([ms], device=f"cuda:{local}")
                    dist.all_reduce(t, op=dist.ReduceOp.MAX)
                    ms = float(t.item())
                wet_win = float(np.mean(sf.download_native("h") > 0))
                # the end-to-end leg starts from the state the window started from
                e2e_in = (d0, pinned(h0_mm), pinned(of0))
                # the same number of steps with the dry skips off: every record read and written
                sf.set_dry_skip(False)
                ms_dense = sf.fused_steps_timed(args.steps)
                sf.set_dry_skip(True)
                run_ms += ms_dense
                run_steps += args.steps
                win = {"ms": ms, "t0_min": d0["t"], "t1_min": d1["t"], "wet_fraction": wet_win,
                       "dt_s_last": d1["time_step"] * 60,
                       "write_skip": (d1["skipped_cells"] - d0["skipped_cells"]) / (cells * args.steps),
                       "read_skip": (d1["skipped_read_cells"] - d0["skipped_read_cells"]) / (cells * args.steps),
                       "ms_dense": ms_dense}
                continue
            n = chunk
            ms_c = sf.fused_steps_timed(n)
            d2 = sf.diag()
            run_ms += ms_c
            run_steps += n
            wet = float(np.mean(sf.download_native("h") > 0))
            wet_samples.append(wet)
            trace.append({"t_min": round(d2["t"], 2), "wet": round(wet, 4),
                          "gcups": round(cells * n / (ms_c / 1e3) / 1e9, 1)})
    d_end = sf.diag()
    steps_total = d_end["k"] - 1   # accepted steps of the whole run (launches after the end are no-ops)
    sf.close()
    if win is None:
        raise SystemExit(f"the run ended before the clock reached {args.window_min} min")
    ms_per_step = win["ms"] / args.steps
    value = cells * args.steps * world / (win["ms"] / 1e3) / 1e9
    full_run = {"sim_minutes": d_end["t"], "steps": steps_total, "launches": run_steps,
                "device_s": run_ms / 1e3,
                "gcups": cells * steps_total / (run_ms / 1e3) / 1e9,
                "wet_fraction_time_avg": float(np.mean(wet_samples)) if wet_samples else None,
                "timing": "CUDA events around every launch of the run, t = 0 to the end of the simulated time; "
                          "launches after the end are no-ops and their time is counted",
                "trace_every_1000_steps": trace}
    dense = {"value": cells * args.steps / (win["ms_dense"] / 1e3) / 1e9, "ms_per_step": win["ms_dense"] / args.steps,
             "record_gbs": RECORD_BYTES_PER_CELL * cells / (win["ms_dense"] / args.steps / 1e3) / 1e9,
             "alg_gbs": ALG_BYTES_PER_CELL * cells / (win["ms_dense"] / args.steps / 1e3) / 1e9}

    # ---- end to end through the C ABI with host buffers ------------------------------
    # The 60-minute state (depth and the two flux pages, as a MATLAB caller holds them) and the
    # static inputs sit in pinned host memory; timed: context creation, hp2d_upload_static and
    # hp2d_set_state / hp2d_set_clock from those arrays, K steps reading the outlet hydrograph and
    # the clock back after every step, then the depth and dmax maps back into pinned host arrays.
    dw, h_mm, of = e2e_in
    z_p, n_p = pinned(case.z), pinned(case.roughness)
    depth_out = pinned(np.empty((ny, nx)))
    dmax_out = pinned(np.empty((ny, nx)))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sf = SurfaceFlow(ny, nx, DX, "fp32", device=local, **case.params)
    ta = time.perf_counter()
    sf.upload_static(z_p, n_p, case.outlet_rows, case.outlet_cols)
    tb = time.perf_counter()
    sf.set_state(h_mm, of)
    sf.set_clock(dw["t"], dw["time_step"], dw["k"])
    t1 = time.perf_counter()
    for _ in range(args.steps):
        sf.fused_steps(1)
        sf.download_native("qo")
    t2 = time.perf_counter()
    sf.download_into("depth", depth_out)
    sf.download_into("dmax", dmax_out)
    e2e_s = time.perf_counter() - t0
    e2e_split = {"setup_s": t1 - t0, "create_s": ta - t0, "static_s": tb - ta, "state_s": t1 - tb,
                 "steps_s": t2 - t1, "readback_s": e2e_s - (t2 - t0)}
    n_out = sf.n_outlets
    # host-copy rates of the boundary: a state upload (depth + two flux pages, FP64) and a map
    # read-back (FP64), from and into page-locked and pageable host arrays (best of 3)
    host_copies = {}
    h_pg, of_pg, out_pg = np.array(h_mm), np.array(of), np.empty((ny, nx))
    for route, (hh, oo, dst) in {"page_locked": (h_mm, of, depth_out),
                                 "pageable": (h_pg, of_pg, out_pg)}.items():
        up, down = [], []
        for _ in range(3):
            a = time.perf_counter()
            sf.set_state(hh, oo)
            b = time.perf_counter()
            sf.download_into("depth", dst)
            c = time.perf_counter()
            up.append(b - a)
            down.append(c - b)
        host_copies[route] = {"state_upload_gbs": 24 * cells / min(up) / 1e9,
                              "map_readback_gbs": 8 * cells / min(down) / 1e9}
    del h_pg, of_pg, out_pg
    sf.close()
    # H2D per run: elevation and roughness (FP64) + the 4-byte meta word built on the host
    # (20 B/cell), depth and two flux pages (FP64, 24 B/cell).  D2H: the outlet hydrograph (4 B per
    # outlet) and the clock block every step, the depth and dmax maps (FP64) once.
    h2d_per_step = 44 * cells / args.steps
    d2h_per_step = n_out * 4 + 2 * 296 + 16 * cells / args.steps   # 296 B: the clock block
    e2e = cells * args.steps / e2e_s / 1e9
    if dist is not None:
        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = cells * args.steps * world / float(t.item()) / 1e9

    # ---- temporal blocking on the same window (opt-in mode; the time step is refreshed once
    # per block, so its trajectory differs from the per-step one) -----------------------------
    blocked = {}
    for kb in (2, 4):
        sb = SurfaceFlow(ny, nx, DX, "fp32", device=local, **case.params)
        sb.upload_static(case.z, case.roughness, case.outlet_rows, case.outlet_cols)
        sb.set_state(h_mm, of)
        sb.set_clock(dw["t"], dw["time_step"], dw["k"])
        sb.set_temporal_blocking(kb)
        sb.fused_steps(args.warmup)
        n_b = max(kb, (args.steps // kb) * kb)
        ms_b = sb.fused_steps_timed(n_b)
        blocked[str(kb)] = {"value": cells * n_b / (ms_b / 1e3) / 1e9, "ms_per_step": ms_b / n_b, "steps": n_b}
        sb.close()

    peak, peak_kind = load_peaks()
    dense["record_hbm_frac"] = dense["record_gbs"] / peak
    dense["alg_hbm_frac"] = dense["alg_gbs"] / peak
    achieved = ALG_BYTES_PER_CELL * cells / (ms_per_step / 1e3) / 1e9
    moved_bpc = RECORD_BYTES_PER_CELL - 32.0 * win["read_skip"] - 16.0 * win["write_skip"]

    urban = None
    if not args.no_urban:
        urban = urban_leg(local, peak=peak)
    ens = None
    if not args.no_ensemble:
        ens = ensemble_leg(local)   # every rank takes part (its share of the members)

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    acc = None if args.no_accuracy or world > 1 else accuracy_leg(local)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        v, sample, cores = cpu_port_gcups(15.0)
        cpu = {"value": v, "unit": METRIC, "cores": cores, "kind": "port", "sample": sample}

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded dam-break, hydropol2d_b200.synthetic.dambreak_case)",
        "config": {"workload": WORKLOAD, "ny": ny, "nx": nx, "dx_m": DX, "cells": cells,
                   "parallelism": f"{world} independent members (one per GPU)" if world > 1 else "single grid",
                   "l2": "state 1.5 GB per step > 126 MB L2; no flush needed",
                   "window": f"K steps after the clock first passes {args.window_min:g} min of the "
                             f"{args.hours:g} h run (W warm-up steps before them)",
                   "window_clock_min": [win["t0_min"], win["t1_min"]], "dt_s_last": win["dt_s_last"],
                   "wet_fraction": win["wet_fraction"]},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_cell": ALG_BYTES_PER_CELL,
                     "bytes_definition": "dense algorithmic bytes of every cell of the grid: state record "
                                         "read + written (h, q_x, q_y, dmax) and the static slopes and "
                                         "roughness read, over the launch time",
                     "traffic": None if NCU_DRAM_BYTES_PER_CELL is None else NCU_DRAM_BYTES_PER_CELL * cells},
        "bytes_still_moved": {"per_cell": moved_bpc, "gbs": moved_bpc * cells / (ms_per_step / 1e3) / 1e9,
                              "write_skip_fraction": win["write_skip"], "read_skip_fraction": win["read_skip"],
                              "note": "records of the fused kernel (48 B dense) less those the dry skips "
                                      "did not read (32 B) or write (16 B)"},
        "full_run": full_run,
        "dense_window": dense,
        "temporal_blocking_window": {"blocks": blocked,
                                     "note": "the same 60-minute state in blocks of K steps per launch at the "
                                             "time step of the block-start refresh (opt-in mode), dry skips off"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": h2d_per_step,
                "d2h_bytes_per_step": d2h_per_step, "steps": args.steps, **e2e_split,
                "includes": "context creation, static + 60-minute state upload from pinned host arrays, "
                            "per-step hydrograph and clock readback, final depth and dmax readback into "
                            "pinned host arrays",
                "host_copies": host_copies},
        "urban_c2": urban,
        "accuracy": acc,
        "ensemble": ens,
        "gpu_launches": args.steps,
        "clocks": clocks.summary(),
        "input_generation_s": t_gen,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
