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
