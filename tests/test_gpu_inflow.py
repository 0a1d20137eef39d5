"""Inflow hydrographs on the GPU against the kernel-form oracle, bit for bit (fused and unfused
paths, with and without Green-Ampt cells, an ensemble member), the water balance with the
inflow volume, and the C ABI's checks (outlet cells cannot be inflow cells; removing the
inflow restores the plain run)."""
import numpy as np
import pytest

from hydropol2d_b200 import synthetic as S
from tests.test_gpu_parity import FIELDS, assert_same_clock, assert_same_state, make_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_fused_inflow_bit_exact(precision, hp2d_lib, oracle_lib):
    case = S.inflow_case(48, 64, minutes=20.0)
    g, o = make_pair(case, precision)
    for chunk in (1, 3, 40, 64, 200):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS, f"after chunk {chunk}")
        assert_same_clock(g, o)
    dg, do = g.diag(), o.diag()
    rel = 1e-5 if precision == "fp32" else 1e-12
    assert dg["inflow_volume"] == pytest.approx(do["inflow_volume"], rel=rel)
    assert dg["inflow_volume"] > 0


def test_inflow_on_green_ampt_cells(hp2d_lib, oracle_lib):
    """Inflow cells on infiltrating soil: the inflow comes after the infiltration."""
    case = S.urban_case(48, 2.0, seed=4, hours=0.1)
    rng = np.random.default_rng(0)
    cells = rng.choice(case.z.size, 30, replace=False)
    rows, cols = np.divmod(cells, case.shape[1])
    keep = ~np.isin(rows * case.shape[1] + cols, case.outlet_rows * case.shape[1] + case.outlet_cols)
    rows, cols = rows[keep].astype(np.int32), cols[keep].astype(np.int32)
    gauge = (np.arange(rows.size) % 3).astype(np.int32)
    t = np.array([0.0, 1.0, 2.5])
    rates = rng.uniform(0, 400, (3, 3))
    case.inflow = dict(t_start=t, rates=rates, rows=np.concatenate([rows, rows[:5]]),
                       cols=np.concatenate([cols, cols[:5]]), gauge=np.concatenate([gauge, (gauge[:5] + 1) % 3]))
    g, o = make_pair(case, "fp32")
    for chunk in (2, 50, 100):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS + ["I"], f"after chunk {chunk}")
        assert_same_clock(g, o)


def test_unfused_sequence_with_inflow_matches_fused(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    from tests.conftest import same_bits
    case = S.inflow_case(32, 40, minutes=10.0)
    a = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    b = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(a)
    case.apply(b)
    for _ in range(40):
        d = b.diag()
        t, ts, k = d["t"], d["time_step"], d["k"]
        b.hydrology_step(ts)
        b.li_step(ts)
        new_ts, _ = b.cfl_dt()
        b.track_maxima(t + ts)
        b.set_clock(new_ts + t, new_ts, k + 1)
        a.fused_steps(1)
        for f in FIELDS:
            assert same_bits(a.download_native(f), b.download_native(f)), f
    assert a.diag()["inflow_volume"] == pytest.approx(b.diag()["inflow_volume"], rel=1e-6)


def test_water_balance_with_inflow_fp64(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    case = S.inflow_case(48, 48, minutes=15.0)
    g = SurfaceFlow(*case.shape, case.resolution, "fp64", **case.params)
    case.apply(g)
    v0 = g.stored_volume()
    g.run()
    d = g.diag()
    lhs = g.stored_volume() + d["outlet_volume"] + d["infiltration_volume"]
    rhs = v0 + d["rain_volume"] + d["inflow_volume"]
    assert d["inflow_volume"] > 0
    assert lhs == pytest.approx(rhs, rel=1e-7) and lhs <= rhs   # the 1e-6 mm clamp drops films


def test_outlet_cells_cannot_be_inflow_cells_and_removal(hp2d_lib):
    from hydropol2d_b200 import HP2DError, SurfaceFlow
    from tests.conftest import same_bits
    case = S.inflow_case(24, 24, minutes=5.0)
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    with pytest.raises(HP2DError):
        g.set_inflow([0.0], [[100.0]], case.outlet_rows[:1], case.outlet_cols[:1], [0])
    g.set_inflow([0.0], np.zeros((1, 0)), [], [], [])          # no gauges: the inflow is removed
    plain = S.inflow_case(24, 24, minutes=5.0)
    plain.inflow = None
    h = SurfaceFlow(*plain.shape, plain.resolution, "fp32", **plain.params)
    plain.apply(h)
    g.fused_steps(50)
    h.fused_steps(50)
    for f in FIELDS:
        assert same_bits(g.download_native(f), h.download_native(f)), f
    assert g.diag()["inflow_volume"] == 0.0


def test_ensemble_member_with_inflow(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    from hydropol2d_b200.ensemble import Ensemble
    from tests.conftest import same_bits
    cases = [S.inflow_case(40, 56, minutes=6.0), S.inflow_case(64, 32, minutes=6.0, peak_m3s=2.0)]
    ens = Ensemble()
    solo = []
    for c in cases:
        m = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(m)
        ens.add(m)
        s = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(s)
        solo.append(s)
    ens.run()
    for m, s in zip(ens.members, solo):
        s.run()
        for f in FIELDS:
            assert same_bits(m.download_native(f), s.download_native(f)), f
        assert m.diag()["t"] == s.diag()["t"]
    ens.close()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_stage_hydrograph_bit_exact(precision, hp2d_lib, oracle_lib):
    from tests.test_inflow import stage_case
    case = stage_case(40, 48, minutes=8.0)
    g, o = make_pair(case, precision)
    for chunk in (1, 5, 64, 300):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS, f"after chunk {chunk}")
        assert_same_clock(g, o)
    rel = 1e-5 if precision == "fp32" else 1e-12
    assert g.diag()["stage_volume"] == pytest.approx(o.diag()["stage_volume"], rel=rel)


def test_stage_and_inflow_together(hp2d_lib, oracle_lib):
    from tests.test_inflow import stage_case
    case = stage_case(40, 48, minutes=6.0)
    flood = S.inflow_case(40, 48, minutes=6.0).inflow
    keep = flood["gauge"] == 1                      # the plane block, away from the stage cells
    case.inflow = dict(t_start=flood["t_start"], rates=flood["rates"][:, 1:], rows=flood["rows"][keep],
                       cols=flood["cols"][keep], gauge=np.zeros(keep.sum(), np.int32))
    g, o = make_pair(case, "fp32")
    g.fused_steps(400)
    o.fused_steps(400)
    assert_same_state(g, o, FIELDS)
    assert_same_clock(g, o)
    assert g.diag()["inflow_volume"] > 0 and g.diag()["stage_volume"] > 0


def test_breach_hydrograph_member(hp2d_lib, oracle_lib):
    """A dam-break member fed by the breach outflow hydrograph through the inflow cells."""
    case = S.breach_inflow_case(64, 256, minutes=6.0)
    assert case.meta["inflow_cells"] >= 1
    g, o = make_pair(case, "fp32")
    for chunk in (10, 200, 400):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS, f"after chunk {chunk}")
        assert_same_clock(g, o)
    assert g.diag()["inflow_volume"] > 0
