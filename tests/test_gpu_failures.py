"""Failure handling of the fused path (the try/catch of HydroPol2D_Main_While.m:926-993 and the
`unstable` flag of refreshing_timestep.m:357-359), made to happen from the host: a test hook
rejects chosen step attempts, a NaN depth is written into the state, min_time_step is set above
the CFL step, and the row-copy wait limit is set to zero polls.  Nothing faults or hangs the GPU:
every wait stays bounded and a timed-out block waits for its copies before it leaves.

The retries are checked bit for bit against the kernel-form oracle, which restates the same
rollback and the reference's new-step rule.
"""
import numpy as np
import pytest

from tests.cases import random_terrain, small_dambreak, small_urban
from tests.conftest import same_bits
from tests.test_gpu_parity import FIELDS, assert_same_clock, assert_same_state, make_pair

pytestmark = pytest.mark.gpu


def test_injected_rejections_are_retried_as_the_oracle(hp2d_lib, oracle_lib):
    case = small_dambreak(64, 256)
    g, o = make_pair(case, "fp32")
    for m in (g, o):
        m.inject_step_fault(6, 2)   # step 6 fails twice, then passes with a smaller step
    g.fused_steps(30)
    assert o.fused_steps(30) == 0
    assert_same_state(g, o, FIELDS)
    assert_same_clock(g, o)
    dg, do = g.diag(), o.diag()
    assert dg["retries"] == do["retries"] == 2
    assert dg["catch_index"] == do["catch_index"] == 3
    assert dg["max_time_step"] == do["max_time_step"] < case.params["max_time_step"]
    assert dg["status_bits"] & 1
    # the retries changed the step sequence: a run without them ends elsewhere
    f, _ = make_pair(case, "fp32")
    f.fused_steps(30)
    assert f.diag()["t"] != dg["t"]


def test_rejection_inside_a_graph_replay(hp2d_lib, oracle_lib):
    """A rejected step in the middle of a 32-launch CUDA graph halts the remaining launches of
    the replay; the call launches the missing steps after the retry."""
    case = small_urban(96, seed=3)
    g, o = make_pair(case, "fp32")
    for m in (g, o):
        m.inject_step_fault(45, 1)
    g.fused_steps(64)
    assert o.fused_steps(64) == 0
    assert g.diag()["k"] == o.diag()["k"] == 65
    assert_same_state(g, o, FIELDS + ["I", "T"])
    assert_same_clock(g, o)


def test_retries_exhausted_leave_the_last_accepted_state(hp2d_lib, oracle_lib):
    from hydropol2d_b200 import HP2DError
    case = small_dambreak(48, 160, seed=2)
    g, o = make_pair(case, "fp32")
    ref, _ = make_pair(case, "fp32")
    for m in (g, o):
        m.set_retry_policy(max_retries=2)
        m.inject_step_fault(5, 3)
    with pytest.raises(HP2DError) as e:
        g.fused_steps(20)
    assert e.value.status_name == "HP2D_NUMERICAL"
    assert o.fused_steps(20) == 4   # HP2D_NUMERICAL
    ref.fused_steps(4)
    assert g.diag()["k"] == 5
    for f in FIELDS:   # the state is the one after step 4, as if the attempts never ran
        assert same_bits(g.download_native(f), ref.download_native(f)), f
    assert_same_state(g, o, FIELDS)
    assert_same_clock(g, o)


def test_nan_depth_in_the_domain_is_rejected_before_stepping(hp2d_lib):
    from hydropol2d_b200 import HP2DError, SurfaceFlow
    case = random_terrain(40, 52, seed=3, walls=True)
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    g.fused_steps(3)   # NaN depths at NaN elevations (idx_nan walls) are fine
    d = g.download("depth")
    i, j = np.argwhere(np.isfinite(case.z))[100]
    d[i, j] = np.nan
    g.set_state(d)
    k0 = g.diag()["k"]
    with pytest.raises(HP2DError) as e:
        g.fused_steps(5)
    assert e.value.status_name == "HP2D_NUMERICAL"
    assert g.diag()["k"] == k0
    assert np.isnan(g.download("depth")[i, j])


def test_dt_floor_stops_when_asked(hp2d_lib, oracle_lib):
    from hydropol2d_b200 import HP2DError
    base = small_dambreak(48, 160, seed=4)
    base.params = dict(base.params, min_time_step=0.2)   # above the CFL step of the 30 m reservoir
    g, o = make_pair(base, "fp32")
    for m in (g, o):
        m.set_retry_policy(dt_floor_is_error=True)
    with pytest.raises(HP2DError) as e:
        g.fused_steps(10)
    assert e.value.status_name == "HP2D_DT_FLOOR"
    assert o.fused_steps(10) == 5   # HP2D_DT_FLOOR
    assert g.diag()["k"] == o.diag()["k"] == 2   # the step that hit the floor was kept
    assert g.diag()["unstable_steps"] == 1
    assert_same_state(g, o, FIELDS)
    # without the stop the run goes on and counts the floor hits
    for m in (g, o):
        m.set_retry_policy(dt_floor_is_error=False)
    g.fused_steps(10)
    assert o.fused_steps(10) == 0
    assert_same_state(g, o, FIELDS)
    assert_same_clock(g, o)
    assert g.diag()["unstable_steps"] > 1


@pytest.mark.parametrize("steps", [3, 40])
def test_row_copy_timeout_is_reported_and_the_context_stays_usable(steps, hp2d_lib, oracle_lib):
    """Zero polls make every ring wait give up at once: the step is rejected (the state stays
    the last accepted one) and the call returns HP2D_TIMEOUT; with the limit back the context
    steps on and matches the oracle."""
    from hydropol2d_b200 import HP2DError
    case = small_dambreak(64, 256, seed=7)
    g, o = make_pair(case, "fp32")
    g.fused_steps(10)
    o.fused_steps(10)
    before = {f: g.download_native(f) for f in FIELDS}
    k0 = g.diag()["k"]
    g.set_wait_limit(0)
    with pytest.raises(HP2DError) as e:
        g.fused_steps(steps)   # a single launch, or graph replays
    assert e.value.status_name == "HP2D_TIMEOUT"
    assert g.diag()["k"] == k0
    for f in FIELDS:
        assert same_bits(g.download_native(f), before[f]), f
    g.set_wait_limit(1 << 22)
    g.fused_steps(25)
    o.fused_steps(25)
    assert_same_state(g, o, FIELDS)
    assert_same_clock(g, o)


def test_ensemble_member_retry_equals_solo(hp2d_lib):
    """A member's rejected step is retried between launches as on its own."""
    from hydropol2d_b200 import SurfaceFlow
    from hydropol2d_b200.ensemble import Ensemble
    cases = [small_dambreak(48 + 16 * i, 160, seed=30 + i) for i in range(3)]
    ens = Ensemble()
    members, solos = [], []
    for i, c in enumerate(cases):
        m = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        s = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(m)
        c.apply(s)
        if i == 1:
            m.inject_step_fault(12, 1)
            s.inject_step_fault(12, 1)
        ens.add(m)
        members.append(m)
        solos.append(s)
    ens.steps(60)   # member 1's rejected step 12 halts it for the rest of these launches
    ens.steps(60)
    for i, (m, s) in enumerate(zip(members, solos)):
        k = m.diag()["k"]
        s.fused_steps(k - 1)
        assert s.diag()["k"] == k
        assert s.diag()["t"] == m.diag()["t"]
        for f in FIELDS:
            assert same_bits(m.download_native(f), s.download_native(f)), (i, f)
    assert members[1].diag()["retries"] == 1
    assert members[1].diag()["k"] < members[0].diag()["k"]
    ens.close()
