"""Inflow hydrographs (flags.flag_inflow; update_spatial_BC.m:359-395, Hydrological_Model.m:27-28)
in the two oracles (no GPU): each step adds to a gauge's cells the integral of its rate over
the step's rain interval / 60 mm, after the infiltration; the kernel-form restatement follows
the literal one through a whole flood, and the water balance closes with the inflow volume."""
import numpy as np
import pytest

from hydropol2d_b200 import synthetic as S
from oracle import literal as L
from tests.test_oracle_crosscheck import kernel_form, literal_cfg


def test_inflow_depth_is_the_gauge_integral():
    case = S.inflow_case(24, 24)
    cfg = literal_cfg(case)
    f = case.inflow
    d = L.inflow_depth_mm(cfg, 9.25, 10.75)
    r = np.asarray(f["rates"])
    # gauge 0 over [9.25, 10.75]: 0.75 min of interval 9 and 0.75 min of interval 10
    expect0 = (r[9, 0] * 0.75 + r[10, 0] * 0.75) / 60.0
    g0 = (f["rows"][0], f["cols"][0])
    assert d[g0] == pytest.approx(expect0, rel=1e-13)
    g1 = np.nonzero(f["gauge"] == 1)[0][0]
    assert d[f["rows"][g1], f["cols"][g1]] == pytest.approx(r[9, 1] * 1.5 / 60.0, rel=1e-13)
    assert (d > 0).sum() == len(set(zip(f["rows"].tolist(), f["cols"].tolist())))
    assert L.inflow_depth_mm(cfg, 3.0, 3.0).max() == 0.0


def test_kernel_form_follows_literal_through_the_flood(oracle_lib):
    case = S.inflow_case(32, 32, minutes=25.0)
    cfg = literal_cfg(case)
    st = L.init_state(cfg)
    o = kernel_form(case)
    for k in range(300):
        if st.t > cfg.routing_time + cfg.min_time_step / 60:
            break
        L.step(cfg, st)
        o.fused_steps(1)
        d = o.diag()
        assert d["t"] == pytest.approx(st.t, rel=1e-12)
        if k % 25 == 0:
            h = o.download_native("h") * 1000
            assert np.allclose(h, st.d, rtol=1e-9, atol=1e-9), k
    assert d["inflow_volume"] == pytest.approx(st.inflow_volume, rel=1e-10)
    assert st.inflow_volume > 0
    assert np.nanmax(st.d) > 10.0   # the hydrograph has made a flood


def test_water_balance_with_inflow(oracle_lib):
    case = S.inflow_case(32, 32, minutes=12.0)
    o = kernel_form(case)
    v0 = o.stored_volume() if hasattr(o, "stored_volume") else 0.0
    o.run()
    d = o.diag()
    h = o.download_native("h")
    stored = float(np.nansum(h)) * case.resolution ** 2
    lhs = stored + d["outlet_volume"] + d["infiltration_volume"]
    rhs = v0 + d["rain_volume"] + d["inflow_volume"]
    assert d["inflow_volume"] > 0
    # the 1e-6 mm clamp (Hydrological_Model.m:49) removes the thinnest films at the wave's edge
    assert lhs == pytest.approx(rhs, rel=1e-7)
    assert lhs <= rhs


def stage_case(ny=32, nx=32, minutes=8.0):
    """The V-tilted catchment, dry, with a stage hydrograph on the channel's upstream cells
    (0.2 m from minute 0, 0.6 m from minute 2, 0.1 m from minute 5) and a second gauge on one
    plane cell that is also in the first mask (the higher gauge wins)."""
    case = S.inflow_case(ny, nx, minutes=minutes)
    case.inflow = None
    ch = case.outlet_cols
    rows = np.concatenate([np.full(ch.size, ny - 1), [ny - 1]]).astype(np.int32)
    cols = np.concatenate([ch, [ch[0]]]).astype(np.int32)
    gauge = np.concatenate([np.zeros(ch.size), [1]]).astype(np.int32)
    case.stage = dict(t_start=np.array([0.0, 2.0, 5.0]),
                      depth_m=np.array([[0.2, 0.05], [0.6, 0.3], [0.1, 0.0]]),
                      rows=rows, cols=cols, gauge=gauge)
    return case


def test_stage_kernel_form_follows_literal(oracle_lib):
    case = stage_case()
    cfg = literal_cfg(case)
    st = L.init_state(cfg)
    o = kernel_form(case)
    for k in range(400):
        if st.t > cfg.routing_time + cfg.min_time_step / 60:
            break
        L.step(cfg, st)
        o.fused_steps(1)
        if k % 40 == 0:
            h = o.download_native("h") * 1000
            assert np.allclose(h, st.d, rtol=1e-9, atol=1e-9), k
    d = o.diag()
    assert d["t"] == pytest.approx(st.t, rel=1e-12)
    assert d["stage_volume"] == pytest.approx(st.stage_volume, rel=1e-9)
    assert st.stage_volume > 0
    # the last record in force at the end (0.1 m) sits on the stage cells
    h = o.download_native("h")
    assert case.stage["cols"].size >= 3
    assert h[case.stage["rows"][1], case.stage["cols"][1]] == pytest.approx(0.1)
    # the shared cell takes gauge 1
    assert h[case.stage["rows"][-1], case.stage["cols"][-1]] == pytest.approx(0.0)
