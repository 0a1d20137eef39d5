"""Reservoir / control structures (flag_reservoir = 1) on the GPU: the fused step against the
kernel-form oracle (FP32 bit for bit; FP64 to the last bits, because the rating curve's
pow is CUDA's on the device and the C library's in the oracle), with Green-Ampt cells and with
rain maps (the transfers read the depth phase (A) of the step produces, restated for the
reservoir cells by the step before); the unfused entry points and an ensemble member against
the fused step bit for bit; the water balance; the C ABI's checks."""
import numpy as np
import pytest

from hydropol2d_b200 import synthetic as S
from tests.test_gpu_parity import FIELDS, assert_same_clock, assert_same_state, make_pair

pytestmark = pytest.mark.gpu


def _close_state(g, o, where):
    for f in FIELDS:
        a, b = g.download_native(f), o.download_native(f)
        fin = np.isfinite(b)
        assert np.array_equal(np.isfinite(a), fin), f"{where} {f}"
        assert np.allclose(a[fin], b[fin], rtol=1e-12, atol=1e-15), f"{where} {f}"
    dg, do = g.diag(), o.diag()
    assert dg["k"] == do["k"]
    for k in ("t", "time_step", "max_velocity"):
        assert dg[k] == pytest.approx(do[k], rel=1e-12), k


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("soil,maps", [(False, False), (True, False), (False, True)])
def test_fused_structures_follow_oracle(precision, soil, maps, hp2d_lib, oracle_lib):
    case = S.structures_case(40, 48, minutes=5.0, soil=soil, maps=maps)
    g, o = make_pair(case, precision)
    for chunk in (1, 2, 31, 100, 400):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        if precision == "fp32":
            assert_same_state(g, o, FIELDS + (["I"] if soil else []), f"after chunk {chunk}")
            assert_same_clock(g, o)
        else:
            _close_state(g, o, f"after chunk {chunk}")
    dg, do = g.diag(), o.diag()
    assert do["structure_volume"] > 1.0
    assert dg["structure_volume"] == pytest.approx(do["structure_volume"], rel=1e-5 if precision == "fp32" else 1e-10)


def test_unfused_sequence_with_structures_matches_fused(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    from tests.conftest import same_bits
    case = S.structures_case(32, 40, minutes=30.0, soil=True)   # the run outlasts the 60 steps
    a = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    b = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(a)
    case.apply(b)
    for _ in range(60):
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
    assert a.diag()["structure_volume"] == pytest.approx(b.diag()["structure_volume"], rel=1e-6)
    assert a.diag()["structure_volume"] > 0


def test_ensemble_member_with_structures(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    from hydropol2d_b200.ensemble import Ensemble
    from tests.conftest import same_bits
    cases = [S.structures_case(40, 56, minutes=3.0), S.structures_case(64, 32, minutes=3.0),
             S.inflow_case(48, 48, minutes=3.0)]
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
        assert m.diag()["structure_volume"] == s.diag()["structure_volume"]
    ens.close()


def test_water_balance_with_structures_fp64(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    case = S.structures_case(48, 48, minutes=6.0)
    g = SurfaceFlow(*case.shape, case.resolution, "fp64", **case.params)
    case.apply(g)
    v0 = g.stored_volume()
    g.run()
    d = g.diag()
    lhs = g.stored_volume() + d["outlet_volume"] + d["infiltration_volume"]
    rhs = v0 + d["rain_volume"] + d["structure_volume"]
    assert d["structure_volume"] > 0
    assert lhs == pytest.approx(rhs, rel=1e-9)


def test_structure_checks(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    from hydropol2d_b200._abi import HP2DError
    case = S.structures_case(24, 24, minutes=1.0)
    params = dict(case.params)
    params["flag_reservoir"] = 0
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **params)
    case.reservoirs, rs = None, case.reservoirs
    case.apply(g)
    with pytest.raises(HP2DError, match="flag_reservoir"):
        g.set_reservoirs(**rs)
    g.close()
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    bad = dict(rs, ds1_row=[-1, rs["ds1_row"][1], rs["ds1_row"][2]])
    with pytest.raises(HP2DError, match="first downstream"):
        g.set_reservoirs(**bad)
    bad = dict(rs, ds1_row=[0, rs["ds1_row"][1], rs["ds1_row"][2]],
               ds1_col=[int(case.outlet_cols[0]), rs["ds1_col"][1], rs["ds1_col"][2]])
    with pytest.raises(HP2DError, match="outlet"):
        g.set_reservoirs(**bad)
    bad = dict(rs, res_row=[99, rs["res_row"][1], rs["res_row"][2]])
    with pytest.raises(HP2DError, match="out of range"):
        g.set_reservoirs(**bad)
    # removing the structures gives the plain run
    g.set_reservoirs(**rs)
    g.set_reservoirs(*([[]] * 12))
    p = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(p)
    g.fused_steps(50)
    p.fused_steps(50)
    assert np.array_equal(g.download_native("h"), p.download_native("h"))
    assert g.diag()["structure_volume"] == 0.0
