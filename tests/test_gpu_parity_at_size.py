"""Parity at the configurations' own sizes.

* Configuration 3 (dam-break, 4096 x 8192 cells, dx 5 m) and configuration 2 (urban rain-on-grid
  2048 x 2048, Green-Ampt soils, 64 x 64 rain maps): the FP32 library against the FP32
  kernel-form oracle bit for bit over 40 adaptive steps on the full grids, and the same steps in
  FP64 on the GPU (itself bit-exact with the FP64 oracle in the smaller tests) for the RMS and
  maximum depth differences.
* The dry-row / dry-block skips on the bench grid: 2000 steps with and without them, bit for bit.
* Configuration 2 over its full 2 simulated hours, FP32 against FP64 on the GPU: peak depth,
  arrival time, depth at the end and the mass ledger.
* Configuration 3 over its first 2000 steps, FP32 against FP64: the horizon over which the two
  trajectories stay within 1 mm RMS.

The measured figures are printed (pytest -s) for the design notes.
"""
import json

import numpy as np
import pytest

from tests.conftest import first_mismatch, same_bits
from tests.test_gpu_parity import FIELDS, assert_same_clock

pytestmark = pytest.mark.gpu


def _pair_full(case, steps):
    import oracle
    from hydropol2d_b200 import SurfaceFlow
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    g.fused_steps(steps)
    o = oracle.KernelFormOracle(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(o)
    assert o.fused_steps(steps) == 0
    return g, o


def _fp64_gap(case, steps, g32):
    from hydropol2d_b200 import SurfaceFlow
    g64 = SurfaceFlow(*case.shape, case.resolution, "fp64", **case.params)
    case.apply(g64)
    g64.fused_steps(steps)
    a = g32.download_native("h").astype(np.float64)
    b = g64.download_native("h")
    fin = np.isfinite(a) & np.isfinite(b)
    d = (a - b)[fin]
    out = {"rms_mm": float(np.sqrt(np.mean(d * d)) * 1000), "max_mm": float(np.abs(d).max() * 1000),
           "wet_dry_mismatch": int(np.sum((a[fin] > 0) != (b[fin] > 0)))}
    g64.close()
    return out


def test_configuration3_full_grid_bit_exact(hp2d_lib, oracle_lib):
    from hydropol2d_b200 import synthetic as S
    case = S.dambreak_case(4096, 8192, 5.0, seed=11)
    g, o = _pair_full(case, 40)
    for f in FIELDS:
        a, b = g.download_native(f), o.download_native(f)
        assert same_bits(a, b), f"field {f}: first mismatch {first_mismatch(a, b)}"
    assert_same_clock(g, o)
    assert same_bits(g.download_native("qo"), o.download_native("qo"))
    gap = _fp64_gap(case, 40, g)
    print("configuration 3, 40 steps, FP32 vs FP64:", json.dumps(gap))
    assert gap["rms_mm"] < 1.0
    g.close()


def test_configuration2_full_grid_bit_exact(hp2d_lib, oracle_lib):
    from hydropol2d_b200 import synthetic as S
    case = S.urban_case(2048, 2.0, seed=7, hours=2.0)
    g, o = _pair_full(case, 40)
    for f in FIELDS + ["I", "T"]:
        a, b = g.download_native(f), o.download_native(f)
        assert same_bits(a, b), f"field {f}: first mismatch {first_mismatch(a, b)}"
    assert_same_clock(g, o)
    gap = _fp64_gap(case, 40, g)
    print("configuration 2, 40 steps, FP32 vs FP64:", json.dumps(gap))
    assert gap["rms_mm"] < 1.0
    g.close()


def test_dry_skips_bitwise_on_the_bench_grid(hp2d_lib):
    """2000 steps of the 4096 x 8192 dam-break with the skips on and off (thousands of CTAs,
    40-row blocks): every field identical, and the skips did skip."""
    from hydropol2d_b200 import SurfaceFlow, synthetic as S
    case = S.dambreak_case(4096, 8192, 5.0, seed=11)
    a = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    b = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(a)
    case.apply(b)
    b.set_dry_skip(False)
    for chunk in (1000, 1000):
        a.fused_steps(chunk)
        b.fused_steps(chunk)
        for f in FIELDS:
            assert same_bits(a.download_native(f), b.download_native(f)), f
    da, db = a.diag(), b.diag()
    assert da["t"] == db["t"] and da["k"] == db["k"] == 2001
    assert da["skipped_read_cells"] > 0.5 * 4096 * 8192 * 2000
    assert db["skipped_cells"] == 0
    a.close()
    b.close()


def _peaks(g, precision):
    return (g.download_native("dmax").astype(np.float64), g.download_native("arrival").astype(np.float64),
            g.download_native("h").astype(np.float64), g.diag())


def test_configuration2_full_run_fp32_against_fp64(hp2d_lib):
    """The whole 2 h urban run: FP32 peak depths within 1 cm of FP64 on at least 99.5 % of the
    cells, mass ledgers within 1e-5 (FP32 per-lane partial sums)."""
    from hydropol2d_b200 import SurfaceFlow, synthetic as S
    case = S.urban_case(2048, 2.0, seed=7, hours=2.0)
    res = {}
    for prec in ("fp32", "fp64"):
        g = SurfaceFlow(*case.shape, case.resolution, prec, **case.params)
        case.apply(g)
        g.run()
        res[prec] = _peaks(g, prec)
        g.close()
    (p32, a32, h32, d32), (p64, a64, h64, d64) = res["fp32"], res["fp64"]
    fin = np.isfinite(p32) & np.isfinite(p64)
    dp = np.abs(p32 - p64)[fin]
    dh = (h32 - h64)[fin]
    both = np.isfinite(a32) & np.isfinite(a64)
    stats = {"steps_fp32": d32["k"] - 1, "steps_fp64": d64["k"] - 1,
             "peak_max_mm": float(dp.max() * 1000), "peak_rms_mm": float(np.sqrt(np.mean(dp * dp)) * 1000),
             "peak_cells_over_1cm_pct": float(np.mean(dp > 0.01) * 100),
             "end_depth_rms_mm": float(np.sqrt(np.mean(dh * dh)) * 1000),
             "arrival_max_diff_min": float(np.abs(a32 - a64)[both].max() / 60) if both.any() else 0.0,
             "arrival_only_one_cells": int(np.sum(np.isfinite(a32) != np.isfinite(a64))),
             "rain_volume_rel": abs(d32["rain_volume"] / d64["rain_volume"] - 1),
             "outlet_volume_rel": abs(d32["outlet_volume"] / max(d64["outlet_volume"], 1e-9) - 1),
             "infiltration_volume_rel": abs(d32["infiltration_volume"] / d64["infiltration_volume"] - 1)}
    print("configuration 2, full 2 h, FP32 vs FP64:", json.dumps(stats))
    assert stats["peak_cells_over_1cm_pct"] < 0.5
    assert stats["rain_volume_rel"] < 1e-5


def test_configuration3_fp32_fp64_horizon(hp2d_lib):
    """Configuration 3 in FP32 and FP64 side by side over its first 2000 steps: RMS depth gap
    at checkpoints; the first 100 steps stay within 1 mm RMS."""
    from hydropol2d_b200 import SurfaceFlow, synthetic as S
    case = S.dambreak_case(4096, 8192, 5.0, seed=11)
    g32 = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    g64 = SurfaceFlow(*case.shape, case.resolution, "fp64", **case.params)
    case.apply(g32)
    case.apply(g64)
    trace = []
    for chunk in (50, 50, 100, 200, 400, 600, 600):
        g32.fused_steps(chunk)
        g64.fused_steps(chunk)
        a = g32.download_native("h").astype(np.float64)
        b = g64.download_native("h")
        d = a - b
        trace.append({"steps": g32.diag()["k"] - 1, "t32_min": g32.diag()["t"], "t64_min": g64.diag()["t"],
                      "rms_mm": float(np.sqrt(np.mean(d * d)) * 1000), "max_mm": float(np.abs(d).max() * 1000)})
    print("configuration 3, FP32 vs FP64 horizon:", json.dumps(trace))
    assert trace[1]["rms_mm"] < 1.0   # the first 100 steps
    g32.close()
    g64.close()
