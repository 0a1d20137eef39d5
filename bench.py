"""Benchmark of the fused surface-flow step (one JSON line on rank 0).

Workload: dam-break on a 4096 x 8192 grid (33.5 M cells, dx 5 m, FP32 state with the split
bed/depth slope), seeded synthetic inputs (hydropol2d_b200.synthetic.dambreak_case).
A step is one accepted time step of HydroPol2D_Main_While over the whole grid (rain,
infiltration (off here), local-inertial fluxes, draining limiter, continuity, outlet
sink, maxima, CFL reduction and timestep refresh) -- one fused kernel launch.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one rank per GPU, each rank an independent dam-break member
(different DEM seed): ensemble members share nothing, so there is no collective on the
data path (weak scaling).  The 256-member ensemble leg is split the same way: each rank
runs its cost-balanced share (hydropol2d_b200.sharding), members/h is the whole job's.  Timing: CUDA events on the library's stream, barrier +
synchronize on both sides, max over ranks.  The state (~1.5 GB) is far larger than L2,
so no flush is needed between steps.
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
WORKLOAD = "dambreak_4096x8192_dx5_fp32"
METRIC = "GCell-updates/s"
# algorithmic bytes per cell-update of the fused FP32 step without infiltration and rain:
# read the static record {dz_x, dz_y, n^2, meta} and the state record {h, q_x, q_y, dmax}
# (2 x 16 B), write the state record (16 B)
BYTES_PER_CELL = 48.0


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["dram_bytes_per_cell"])
        except Exception:
            return None
    return None


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
                "this is the C++ restatement of its arithmetic (oracle/kernel_form.hpp).",
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ny", type=int, default=NY)
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 256-member ensemble leg")
    ap.add_argument("--late-steps", type=int, default=10000,
                    help="steps the dam-break advances before the late-window measurement (0: skip)")
    ap.add_argument("--surrogate", action="store_true",
                    help="run the learned-screening study instead (4096 training / 1024 held-out members)")
    ap.add_argument("--surrogate-epochs", type=int, default=8)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_env()

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
    case = S.dambreak_case(ny, nx, DX, seed=11 + rank)
    t_gen = time.perf_counter() - t_e2e0

    # ---- device-resident timing of the fused step ----------------------------------
    sf = SurfaceFlow(ny, nx, DX, "fp32", device=local, **case.params)
    case.apply(sf)
    sf.fused_steps(args.warmup)
    if dist is not None:
        dist.barrier()
    d0 = sf.diag()
    skip0, skipr0 = d0["skipped_cells"], d0["skipped_read_cells"]
    with ClockSampler(local) as clocks:
        ms = sf.fused_steps_timed(args.steps)
    if dist is not None:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = cells * args.steps * world / (ms / 1e3) / 1e9
    d = sf.diag()
    # deep-dry rows whose records the output buffer already held were not stored again
    skip_frac = (d["skipped_cells"] - skip0) / (cells * args.steps)
    # ... and whole dry row blocks were neither read nor written
    skipr_frac = (d["skipped_read_cells"] - skipr0) / (cells * args.steps)
    req_bpc = BYTES_PER_CELL - 32.0 * skipr_frac - 16.0 * skip_frac
    wet_main = float(np.mean(sf.download_native("h") > 0))
    # the same window with the dry skips off, on a second context from the same inputs: every
    # row read, stepped and written (bit-identical results)
    dn = SurfaceFlow(ny, nx, DX, "fp32", device=local, **case.params)
    case.apply(dn)
    dn.set_dry_skip(False)
    dn.fused_steps(args.warmup)
    ms_dense = dn.fused_steps_timed(args.steps)
    dn.close()
    dense = {"value": cells * args.steps / (ms_dense / 1e3) / 1e9, "ms_per_step": ms_dense / args.steps,
             "achieved_gbs": BYTES_PER_CELL * cells / (ms_dense / args.steps / 1e3) / 1e9}
    late = None
    if args.late_steps > 0:
        # the same run later on, once the flood wave has spread over more of the valley
        sf.fused_steps(args.late_steps)
        ms_late = sf.fused_steps_timed(args.steps)
        h = sf.download_native("h")
        d_late = sf.diag()
        late = {"after_steps": args.warmup + args.steps + args.late_steps, "sim_clock_min": d_late["t"],
                "wet_fraction": float(np.mean(h > 0)), "ms_per_step": ms_late / args.steps,
                "value": cells * args.steps / (ms_late / 1e3) / 1e9,
                "wet_fraction_main_window": wet_main}
    sf.close()

    # ---- end to end through the C ABI with host buffers ------------------------------
    # host arrays -> hp2d_upload_static/hp2d_set_state -> K steps, reading the outlet
    # hydrograph and the clock back every step -> final depth and dmax back to the host
    e2e_steps = args.steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sf = SurfaceFlow(ny, nx, DX, "fp32", device=local, **case.params)
    case.apply(sf)
    t1 = time.perf_counter()
    q_hydro = []
    for _ in range(e2e_steps):
        sf.fused_steps(1)
        q_hydro.append(sf.download_native("qo"))
    t2 = time.perf_counter()
    d_final = sf.download("depth")
    dmax = sf.download("dmax")
    e2e_s = time.perf_counter() - t0
    e2e_split = {"setup_s": t1 - t0, "steps_s": t2 - t1, "readback_s": e2e_s - (t2 - t0)}
    n_out = sf.n_outlets
    sf.close()
    # H2D per run: the static upload (FP64 elevation and roughness and the 4-byte meta word,
    # 20 B/cell) and the state upload (FP64 depth, 8 B/cell); the context's records are built
    # and filled on the device.  D2H: outlet hydrograph (4 B per outlet) and the clock block
    # every step, then the depth and dmax components (FP32, 8 B/cell) once
    h2d_per_step = 28 * cells / e2e_steps
    d2h_per_step = n_out * 4 + 2 * 232 + 8 * cells / e2e_steps   # 232 B: the clock block
    e2e = cells * e2e_steps / e2e_s / 1e9
    if dist is not None:
        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = cells * e2e_steps * world / float(t.item()) / 1e9

    peak, peak_kind = load_peaks()
    dense["hbm_frac"] = dense["achieved_gbs"] / peak   # 48 B/cell streamed, of measured HBM
    # bytes the step must move: the dense 48 B per cell less the records it skipped
    achieved = req_bpc * cells / (ms_per_step / 1e3) / 1e9
    traffic_pc = load_traffic()

    ens = None
    if not args.no_ensemble:
        ens = ensemble_leg(local)   # every rank takes part (its share of the members)

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

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
                   "sim_clock_min_after": d["t"], "dt_s_last": d["time_step"] * 60,
                   "wet_fraction": wet_main},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_cell": req_bpc,
                     "dense_bytes_per_cell": BYTES_PER_CELL,
                     "write_skip_fraction": skip_frac, "read_skip_fraction": skipr_frac,
                     "traffic": None if traffic_pc is None else traffic_pc * cells},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": h2d_per_step,
                "d2h_bytes_per_step": d2h_per_step, "steps": e2e_steps, **e2e_split,
                "includes": "input generation excluded; static+state upload, per-step hydrograph "
                            "and clock readback, final depth and dmax readback"},
        "late_window": late,
        "dense_window": dense,
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
