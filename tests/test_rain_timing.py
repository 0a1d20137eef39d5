"""Rain timing of the loop (no GPU): a step applies the rain update_spatial_BC computed at the
end of the step before it -- the exact integral of the piecewise-constant rate over the clock
interval [t_previous, t] -- with the loop's t_previous bookkeeping
(HydroPol2D_Main_While.m:115-120, :721, :734-738, :779).

* The start-stamped integral of the library (oracle/literal.rain_depth_mm) equals the
  reference's end-stamped average (localAverageRateOverStep, update_spatial_BC.m:1131-1184,
  restated as literal.average_rate_over_step) x interval / 60 on the converted series.
* The interval sequence: [0, t1], [0, t1], [t_prev = dt2, t2], [t2, t3], [t3, t4], ...
* The kernel-form oracle keeps the same interval as the literal restatement.
* Over a whole event the delivered rain is the rate times the union of those intervals.
"""
import math

import numpy as np
import pytest

from oracle import literal as L


def _to_start_stamped(times_end, values):
    """End-stamped (value i up to times_end[i], first from times_end[0] - spacing) to the
    library's start-stamped table (rate q from t_start[q], last for ever)."""
    te = np.asarray(times_end, float)
    dt_force = te[1] - te[0] if te.size >= 2 else 0.0
    starts = np.concatenate([[te[0] - dt_force], te[:-1], [te[-1]]])
    rates = np.concatenate([values, [0.0]])
    return starts, rates


@pytest.mark.parametrize("seed", range(6))
def test_start_stamped_integral_equals_reference_average(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 9))
    spacing = float(rng.uniform(1.0, 15.0))
    te = spacing * (1 + np.arange(n)) + float(rng.uniform(0, 5))
    vals = rng.uniform(0, 150, n)
    if seed % 3 == 0:
        vals[rng.integers(0, n)] = np.nan          # a gap in the record adds nothing
    starts, rates = _to_start_stamped(te, vals)
    cfg = L.RunConfig(z=np.zeros((2, 2)), roughness=np.ones((2, 2)), resolution=1.0,
                      outlet_rows=np.array([0]), outlet_cols=np.array([0]),
                      rain_times_min=starts, rain_rates_mmh=rates)
    lo, hi = te[0] - spacing - 3.0, te[-1] + 4.0
    for _ in range(40):
        t0, t1 = np.sort(rng.uniform(lo, hi, 2))
        if rng.uniform() < 0.2:
            t1 = t0 + float(rng.uniform(0, 0.05))   # model-step sized intervals
        ref = L.average_rate_over_step(te, vals, t0, t1) * (t1 - t0) / 60.0
        got = L.rain_depth_mm(cfg, t0, t1, 2, 2)
        assert got == pytest.approx(ref, rel=1e-12, abs=1e-12), (t0, t1)
    assert L.rain_depth_mm(cfg, 5.0, 5.0, 2, 2) == 0.0
    assert L.average_rate_over_step(te, vals, 5.0, 4.0) == 0.0


def test_map_integral_blends_maps_by_overlap():
    rng = np.random.default_rng(3)
    maps = rng.uniform(0, 100, (3, 4, 4)).astype(np.float32)
    cfg = L.RunConfig(z=np.zeros((8, 8)), roughness=np.ones((8, 8)), resolution=1.0,
                      outlet_rows=np.array([0]), outlet_cols=np.array([0]),
                      rain_maps_mmh=maps, rain_map_dt_min=5.0)
    b = [L.bilinear_rain(maps[m], 8, 8) for m in range(3)]
    got = L.rain_depth_mm(cfg, 4.0, 5.5, 8, 8)          # 1 min of map 0, 0.5 min of map 1
    assert np.allclose(got, (1.0 * b[0] + 0.5 * b[1]) / 60.0, rtol=1e-12)
    assert np.all(L.rain_depth_mm(cfg, 15.0, 16.0, 8, 8) == 0.0)   # after the last map: none
    assert np.allclose(L.rain_depth_mm(cfg, 14.5, 15.5, 8, 8), 0.5 * b[2] / 60.0, rtol=1e-12)


def _rain_case(minutes=12.0, rate=80.0, dur=6.0):
    from tests.cases import small_vtilt
    case = small_vtilt(24, 24)
    p = dict(case.params, routing_time=minutes)
    cfg = L.RunConfig(z=case.z, roughness=case.roughness, resolution=case.resolution,
                      outlet_rows=case.outlet_rows, outlet_cols=case.outlet_cols,
                      outlet_type=p.get("outlet_type", 1), slope_outlet=p.get("slope_outlet", 0.005),
                      routing_time=minutes, min_time_step=p["min_time_step"], max_time_step=p["max_time_step"],
                      alfa_min=p["alfa_min"], alfa_max=p["alfa_max"],
                      rain_times_min=np.array([0.0, dur]), rain_rates_mmh=np.array([rate, 0.0]), d0=case.d0)
    return case, p, cfg


def test_interval_sequence_follows_the_loop():
    _, _, cfg = _rain_case()
    st = L.init_state(cfg)
    seq = []
    for _ in range(6):
        seq.append((st.rain_a, st.rain_b, st.t, st.time_step))
        L.step(cfg, st)
    t = [s[2] for s in seq]
    ts = [s[3] for s in seq]
    assert seq[0][:2] == (0.0, t[0])                 # before the loop, t_previous = 0
    assert seq[1][:2] == (0.0, t[0])                 # end of step 1: t_previous still 0
    assert seq[2][:2] == (ts[1], t[1])               # t_previous = the first increment
    for k in range(3, 6):
        assert seq[k][:2] == (t[k - 2], t[k - 1])    # then the previous clock interval


def test_event_rain_is_the_rate_over_the_union_of_intervals():
    case, p, cfg = _rain_case(minutes=10.0, rate=90.0, dur=4.0)
    st = L.init_state(cfg)
    ivals = []
    while st.t <= cfg.routing_time + cfg.min_time_step / 60:
        ivals.append((st.rain_a, st.rain_b))
        L.step(cfg, st)
    covered = sum(max(0.0, min(b, 4.0) - max(a, 0.0)) for a, b in ivals)
    cells = np.isfinite(case.z).sum()
    expect = 90.0 * covered / 60.0 / 1000.0 * case.resolution ** 2 * cells
    assert st.rain_volume == pytest.approx(expect, rel=1e-9)
    # the first steps' quirk: [0, t1] twice, then [dt2, dt2 + t1] -- the minutes between t1
    # and dt2 are never rained on, so the event delivers slightly less than rate x duration
    assert covered < 4.0 and covered > 4.0 - 10.0 / 60.0


def test_kernel_form_oracle_tracks_the_same_interval(oracle_lib):
    import oracle
    case, p, cfg = _rain_case()
    o = oracle.KernelFormOracle(*case.shape, case.resolution, "fp64", **p)
    case.apply(o)
    o.set_rain_uniform(np.array([0.0, 6.0]), np.array([80.0, 0.0]))
    st = L.init_state(cfg)
    for k in range(8):
        d = o.diag()
        assert (d["rain_t0"], d["rain_t1"]) == pytest.approx((st.rain_a, st.rain_b), rel=1e-12, abs=1e-15)
        assert d["t_previous"] == pytest.approx(st.t_previous, rel=1e-12, abs=1e-15)
        o.fused_steps(1)
        L.step(cfg, st)
    assert o.diag()["rain_volume"] == pytest.approx(st.rain_volume, rel=1e-9)


def test_oracle_set_clock_follows_the_loop(oracle_lib):
    import oracle
    case, p, _ = _rain_case()
    o = oracle.KernelFormOracle(*case.shape, case.resolution, "fp64", **p)
    case.apply(o)
    o.set_clock(0.5, 0.1, 1)
    d = o.diag()
    assert (d["rain_t0"], d["rain_t1"], d["t_previous"]) == (0.0, 0.5, 0.0)
    o.set_clock(0.6, 0.1, 2)                     # the loop's advance after step 1
    d = o.diag()
    assert (d["rain_t0"], d["rain_t1"], d["t_previous"]) == (0.0, 0.5, 0.1)
    o.set_clock(0.7, 0.1, 3)
    d = o.diag()
    assert (d["rain_t0"], d["rain_t1"], d["t_previous"]) == (0.1, 0.6, 0.6)
    o.set_clock(5.0, 0.25, 40)                   # a jump re-seeds with the given step
    d = o.diag()
    assert (d["rain_t0"], d["rain_t1"], d["t_previous"]) == (4.5, 4.75, 4.75)
    o.set_rain_clock(1.0, 2.0, 3.0)
    d = o.diag()
    assert (d["rain_t0"], d["rain_t1"], d["t_previous"]) == (1.0, 2.0, 3.0)
    assert math.isfinite(d["t"])


def test_idw_gauge_maps():
    """Rainfall_Interpolator / idw_function restated: a cell centred on a gauge takes its value
    (its weight is 1/eps^2), equal gauges give a uniform map, a NaN record drops the gauge for
    that interval, an interval without records is dry."""
    ny, nx, res = 12, 16, 10.0
    xg = np.array([res * 3, res * 10, res * 15])          # cell centres of columns 2, 9, 14
    yg = np.array([-res * 2, -res * 7, -res * 11])        # rows 1, 6, 10
    rates = np.array([[10.0, 40.0, 70.0], [25.0, 25.0, 25.0], [np.nan, 40.0, 70.0], [np.nan] * 3])
    maps = L.idw_rain_maps(xg, yg, rates, ny, nx, res)
    assert maps.shape == (4, ny, nx) and maps.dtype == np.float32
    assert maps[0, 1, 2] == np.float32(10.0) and maps[0, 6, 9] == np.float32(40.0)
    assert np.all((maps[0] >= 10.0) & (maps[0] <= 70.0))
    assert np.allclose(maps[1], 25.0, rtol=1e-6)
    no0 = L.idw_rain_maps(xg[1:], yg[1:], rates[2:3, 1:], ny, nx, res)
    assert np.array_equal(maps[2], no0[0])
    assert np.all(maps[3] == 0.0)
