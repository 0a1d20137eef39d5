"""Velocity and hazard maxima on the GPU (hp2d_set_hazard_tracking): the fused step against the
kernel-form oracle bit for bit in FP32 and FP64, an ensemble member against its solo run, and
the C ABI's checks."""
import numpy as np
import pytest

from hydropol2d_b200 import synthetic as S
from tests.conftest import same_bits
from tests.test_gpu_parity import FIELDS, assert_same_clock, assert_same_state, make_pair

pytestmark = pytest.mark.gpu


def _maxima(m):
    return m.download("vmax"), m.download("hazard_max")


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_maxima_bit_exact(precision, hp2d_lib, oracle_lib):
    case = S.dambreak_case(32, 640, 5.0, seed=3, hours=0.05)   # long enough to keep dry blocks
    g, o = make_pair(case, precision)
    g.set_hazard_tracking(True)
    o.set_hazard_tracking(True)
    for chunk in (1, 7, 64, 300):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS, f"after chunk {chunk}")
        assert_same_clock(g, o)
        vg, hg = _maxima(g)
        assert same_bits(vg, o.download_native("vmax").astype(np.float64)), chunk
        assert same_bits(hg, o.download_native("hazard_max").astype(np.float64)), chunk
    assert np.nanmax(vg) > 1.0 and np.nanmax(hg) > 1.0
    assert g.diag()["skipped_read_cells"] > 0     # dry blocks skipped with the maxima on


def test_structures_and_hazard_together(hp2d_lib, oracle_lib):
    case = S.structures_case(40, 48, minutes=3.0, soil=True)
    g, o = make_pair(case, "fp32")
    g.set_hazard_tracking(True)
    o.set_hazard_tracking(True)
    g.fused_steps(200)
    o.fused_steps(200)
    assert_same_state(g, o, FIELDS, "structures + hazard")
    vg, hg = _maxima(g)
    assert same_bits(vg, o.download_native("vmax").astype(np.float64))
    assert same_bits(hg, o.download_native("hazard_max").astype(np.float64))


def test_ensemble_member_with_hazard(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    from hydropol2d_b200.ensemble import Ensemble
    cases = [S.dambreak_case(32, 96, 5.0, seed=5, hours=0.03), S.dambreak_case(64, 64, 5.0, seed=6, hours=0.03)]
    ens = Ensemble()
    solo = []
    for i, c in enumerate(cases):
        m = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(m)
        m.set_hazard_tracking(True)
        ens.add(m)
        s = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(s)
        s.set_hazard_tracking(True)
        solo.append(s)
    ens.run()
    for m, s in zip(ens.members, solo):
        s.run()
        for a, b in zip(_maxima(m), _maxima(s)):
            assert same_bits(a, b)
        assert same_bits(m.download_native("h"), s.download_native("h"))
    ens.close()


def test_hazard_checks(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    from hydropol2d_b200._abi import HP2DError
    case = S.dambreak_case(32, 64, 5.0, seed=3, hours=0.01)
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    with pytest.raises(HP2DError):
        g.download("vmax")                      # not tracked
    g.set_hazard_tracking(True)
    g.fused_steps(20)
    assert np.nanmax(g.download("vmax")) > 0
    g.set_hazard_tracking(True)                 # restarts at zero
    assert np.nanmax(g.download("vmax")) == 0
    g.close()
    slow = dict(case.params, time_step_change=1.0)   # velocities refreshed once a second only
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **slow)
    case.apply(g)
    with pytest.raises(HP2DError, match="refresh"):
        g.set_hazard_tracking(True)
    g.close()
