"""The fused step leaves a deep-dry row's record unwritten when its output buffer already holds
it (the same row deep-dry two steps before): results stay bit-exact with the kernel-form oracle
through many steps, across layout changes, host state writes, an autotune and ensemble runs,
and the step reports the records it did not rewrite."""
import numpy as np
import pytest

from hydropol2d_b200 import synthetic as S
from tests.conftest import same_bits
from tests.test_gpu_parity import FIELDS, assert_same_clock, assert_same_state, make_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_long_run_bit_exact(precision, hp2d_lib, oracle_lib):
    case = S.dambreak_case(64, 256, 5.0, seed=3, hours=0.2)
    g, o = make_pair(case, precision)
    for chunk in (1, 2, 3, 5, 64, 300, 600):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS, f"after chunk {chunk}")
        assert_same_clock(g, o)
    sk = g.diag()["skipped_cells"]
    assert sk > 0.1 * case.z.size * 975   # much of the valley stays dry
    assert o.diag()["skipped_cells"] == 0


def test_layout_switches_and_host_writes(hp2d_lib, oracle_lib):
    case = S.dambreak_case(48, 320, 5.0, seed=4, hours=0.2)
    g, o = make_pair(case, "fp32")
    for step, action in enumerate(["layout1", "layout2", "state", "tuning16", "tuning5", "tuning40", "autotune",
                                   "layout1"]):
        g.fused_steps(97)
        o.fused_steps(97)
        assert_same_state(g, o, FIELDS, f"before {action}")
        if action.startswith("layout"):
            g.set_layout(int(action[-1]))
        elif action == "state":
            d = g.download("depth")
            d[:, :5] += 100.0                    # the host floods the first columns
            of = np.stack([g.download("qout_right"), g.download("qout_up")])
            g.set_state(d, of)
            o.set_state(d, of)
        elif action.startswith("tuning"):
            g.set_tuning(int(action[6:]))   # 5 rows per warp: launches without the flags
        else:
            g.autotune(3)
        g.fused_steps(33)
        o.fused_steps(33)
        assert_same_state(g, o, FIELDS, f"after {action}")
        assert_same_clock(g, o)


def test_ensemble_members_match_solo_runs(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    from hydropol2d_b200.ensemble import Ensemble
    cases = [S.dambreak_case(64, 192, 5.0, seed=7, hours=0.1), S.dambreak_case(96, 96, 5.0, seed=8, hours=0.1)]
    solo = []
    for c in cases:
        s = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(s)
        s.set_layout(1)                          # a layout other than the ensemble's
        s.fused_steps(40)
        solo.append(s)
    ens = Ensemble()
    members = []
    for c in cases:
        m = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(m)
        m.set_layout(1)
        m.fused_steps(40)
        ens.add(m)
        members.append(m)
    ens.set_layout(2)
    ens.run()
    for m, s in zip(members, solo):
        s.set_layout(2)
        s.run()
        for f in FIELDS:
            assert same_bits(m.download_native(f), s.download_native(f)), f
        assert m.diag()["skipped_cells"] > 0
    ens.close()


def test_dense_switch_gives_the_same_bits(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    case = S.dambreak_case(64, 320, 5.0, seed=9, hours=0.1)
    a = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    b = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(a)
    case.apply(b)
    b.set_dry_skip(False)
    for chunk in (5, 100, 200):
        a.fused_steps(chunk)
        b.fused_steps(chunk)
        for f in FIELDS:
            assert same_bits(a.download_native(f), b.download_native(f)), f
    assert a.diag()["skipped_read_cells"] > 0 and b.diag()["skipped_cells"] == 0
    b.set_dry_skip(True)                         # back on mid-run
    a.fused_steps(100)
    b.fused_steps(100)
    for f in FIELDS:
        assert same_bits(a.download_native(f), b.download_native(f)), f
    assert b.diag()["skipped_cells"] > 0


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_row_wet_for_one_step_between_deep_dry_steps(precision, hp2d_lib, oracle_lib):
    """Rain on every other one-second step, a little faster than the soil takes it: every row gets
    a thin film in the rainy steps and is dry again (all of it soaked up) in the next, so a row
    is deep-dry at steps s-2 and s and wet at s-1.  The record a deep-dry step would write then
    differs from the one written at s-2 (the running maximum moved at s-1): it must be written."""
    n = 72
    z = 0.05 * S.gaussian_random_field(n, n, -3.0, 2)
    steps = 40
    t_start = np.arange(steps + 2) / 60.0           # [min], one interval per one-second step
    rate = np.where(np.arange(steps + 2) % 2 == 0, 40.0, 0.0)
    tabs = S.green_ampt_soil_tables([30.0], [50.0], [0.3])
    params = dict(routing_time=30.0, alfa_min=0.5, alfa_max=0.7, outlet_type=1, slope_outlet=0.01,
                  min_time_step=1.0, max_time_step=1.0, flag_infiltration=1)
    case = S.Case("film", z, np.full((n, n), 0.03), 5.0, np.zeros(0, np.int32), np.zeros(0, np.int32), params,
                  np.zeros((n, n)), rain_uniform=(t_start, rate),
                  soil=dict(soil_class=np.zeros((n, n), np.uint8), **tabs), I0=np.full((n, n), 500.0))
    g, o = make_pair(case, precision)
    seen_wet = seen_dry = 0
    for _ in range(steps):
        g.fused_steps(1)
        o.fused_steps(1)
        h = g.download_native("h")
        seen_wet += int((h > 0).all())
        seen_dry += int((h == 0).all())
    assert seen_wet >= 5 and seen_dry >= 5   # the rows did alternate
    assert_same_state(g, o, FIELDS + ["I", "T"])
    assert_same_clock(g, o)
    assert g.download_native("dmax").max() > 0
