"""van Genuchten-Mualem infiltration (flag_infiltration = 2, the single-layer branch of the
current Infiltration_Module.m) on the GPU against the literal FP64 restatement
(oracle/literal.vg_infiltration).  The closure's non-integer powers come from the CUDA math
library, so the check is to a tolerance (FP64: 1e-9 relative; FP32: 1e-4 relative, 1e-3 mm),
and the fused and unfused GPU paths, which share the device function, agree bit for bit."""
import numpy as np
import pytest

from tests.cases import random_terrain
from tests.conftest import same_bits

pytestmark = pytest.mark.gpu

FIELDS = ("h", "qx", "qy", "dmax", "I")


def vg_case(ny=40, nx=56, seed=6):
    from hydropol2d_b200 import synthetic as S
    case = random_terrain(ny, nx, seed=seed)
    case.params = dict(case.params, flag_infiltration=2)
    soil = S.vg_soil(ny, nx, case.z, seed=seed)
    rng = np.random.default_rng(seed)
    I0 = rng.uniform(0, 150, (ny, nx))
    return case, soil, I0


def make(case, soil, I0, precision):
    from hydropol2d_b200 import SurfaceFlow
    g = SurfaceFlow(*case.shape, case.resolution, precision, **case.params)
    g.upload_static(case.z, case.roughness, case.outlet_rows, case.outlet_cols)
    g.set_soil_vg(**soil)
    g.set_state(case.d0, None, I0)
    g.set_rain_uniform(*case.rain_uniform)
    return g


@pytest.mark.parametrize("precision,rtol,atol", [("fp64", 1e-9, 1e-9), ("fp32", 1e-4, 1e-3)])
def test_vg_hydrology_step_matches_literal(precision, rtol, atol):
    from oracle import literal as L
    case, soil, I0 = vg_case()
    g = make(case, soil, I0, precision)
    ts = 0.5   # minutes
    g.set_rain_clock(0.0, ts, 0.0)   # the step applies the rain of [0, ts]
    d = g.diag()
    g.hydrology_step(ts)
    h = g.download("depth")
    I = g.download("soil_storage")
    act = soil["soil_class"] != 255
    c = np.where(act, soil["soil_class"], 0)
    p = L.VGParams(theta_r=soil["theta_r"][c], theta_sat=soil["theta_sat"][c], n_vg=soil["n_vg"][c],
                   alpha_vg=soil["alpha_vg"][c], ksat=soil["ksat"][c], soil_depth=soil["soil_depth"], active=act)
    zwt = L.vg_water_table_depth(case.z, soil["soil_depth"], soil["gw_head"])
    rate = case.rain_uniform[1][0]
    dl, Il, f = L.vg_infiltration(case.d0 + rate * ts / 60, I0, ts, p, zwt, case.resolution)
    dl[dl < 1e-6] = 0
    assert np.allclose(h, dl, rtol=rtol, atol=atol), np.abs(h - dl).max()
    Ig = np.where(act, I, I0)
    assert np.allclose(Ig, Il, rtol=rtol, atol=atol), np.abs(Ig - Il).max()
    assert (f > 0).mean() > 0.3 and (Il > I0 + 1e-6).any()   # the closure is exercised
    assert d["k"] == 1
    g.close()


def test_vg_fused_equals_unfused_sequence():
    case, soil, I0 = vg_case(48, 80, seed=4)
    a = make(case, soil, I0, "fp32")
    b = make(case, soil, I0, "fp32")
    for _ in range(20):
        d = b.diag()
        t, ts, k = d["t"], d["time_step"], d["k"]
        b.hydrology_step(ts)
        b.li_step(ts)
        new_ts, _ = b.cfl_dt()
        b.track_maxima(t + ts)
        b.set_clock(new_ts + t, new_ts, k + 1)
        a.fused_steps(1)
        for fld in FIELDS:
            assert same_bits(a.download_native(fld), b.download_native(fld)), fld
        assert a.diag()["t"] == b.diag()["t"]
    a.close()
    b.close()


def test_vg_run_closes_the_water_balance():
    """FP64 run of 10 simulated minutes: stored + infiltrated + outlet volume = initial +
    rain, to round-off."""
    case, soil, I0 = vg_case(64, 64, seed=9)
    case.params = dict(case.params, routing_time=10.0)
    g = make(case, soil, I0, "fp64")
    v0 = g.stored_volume()
    g.run()
    d = g.diag()
    v1 = g.stored_volume()
    assert d["infiltration_volume"] > 0
    lhs = v1 + d["infiltration_volume"] + d["outlet_volume"]
    rhs = v0 + d["rain_volume"]
    assert abs(lhs - rhs) <= 1e-9 * rhs, (lhs, rhs)
    g.close()
