"""Row slabs of one grid on the GPU: every slab a context of its own rows plus two halo rows per
side, the driver combining the step maxima and exchanging the edge rows after each step.  The
slabs' own rows must equal one whole-grid context's, bit for bit, and so must the clock."""
import numpy as np
import pytest

from tests.cases import random_terrain, small_dambreak
from tests.conftest import same_bits

pytestmark = pytest.mark.gpu

STATE = ("h", "qx", "qy", "dmax")


def whole(case, precision):
    from hydropol2d_b200 import SurfaceFlow
    g = SurfaceFlow(*case.shape, case.resolution, precision, **case.params)
    case.apply(g)
    g.set_retry_policy(max_retries=0)
    return g


def check(grid, g, where):
    for f in STATE:
        assert same_bits(grid.gather(f), g.download_native(f)), f"{f} {where}"
    dg, ds = g.diag(), grid.diag()
    for k in ("t", "time_step", "k", "max_velocity", "unstable_steps"):
        assert ds[k] == dg[k], f"{k} {where}: slabs {ds[k]} whole {dg[k]}"


@pytest.mark.parametrize("precision,n", [("fp32", 2), ("fp32", 3), ("fp64", 3), ("fp32", 5)])
def test_dambreak_slabs_bit_exact(precision, n, hp2d_lib):
    from hydropol2d_b200.slabs import SlabGrid
    case = small_dambreak(96, 256, seed=11)
    g = whole(case, precision)
    grid = SlabGrid(case, n, precision)
    for chunk in (1, 5, 30):
        g.fused_steps(chunk)
        grid.step(chunk)
        check(grid, g, f"after {chunk}")
    grid.close()


@pytest.mark.parametrize("shape", [(45, 70), (64, 33)])
def test_rain_walls_slabs_bit_exact(shape, hp2d_lib):
    from hydropol2d_b200.slabs import SlabGrid
    case = random_terrain(*shape, seed=3 * shape[0], walls=True)
    case.d0 = np.where(np.isnan(case.d0), np.nan, np.abs(case.d0))
    g = whole(case, "fp32")
    grid = SlabGrid(case, 4, "fp32")
    for chunk in (3, 40):
        g.fused_steps(chunk)
        grid.step(chunk)
        check(grid, g, f"after {chunk}")
    # the ledgers add up over the slabs (sums in another order)
    dg = g.diag()
    rain = sum(s.ctx.diag()["rain_volume"] for s in grid.slabs)
    assert rain == pytest.approx(dg["rain_volume"], rel=1e-5)
    grid.close()


def test_refused_configurations(hp2d_lib):
    from hydropol2d_b200.slabs import SlabGrid
    case = small_dambreak(32, 64, seed=1)
    case.params = dict(case.params, flag_numerical_scheme=2)
    with pytest.raises(ValueError):
        SlabGrid(case, 2)
    case = small_dambreak(32, 64, seed=1)
    case.d0 = case.d0 - 1.0
    with pytest.raises(ValueError):
        SlabGrid(case, 2)
