"""Rain from gauges on the GPU: the device's inverse-distance maps equal the literal
restatement of Rainfall_Interpolator / idw_function bit for bit, shown by a run against the
kernel-form oracle fed the restated maps (FP32 and FP64)."""
import numpy as np
import pytest

from oracle import literal as L
from tests.cases import random_terrain
from tests.test_gpu_parity import FIELDS, assert_same_clock, assert_same_state, make_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_gauge_rain_bit_exact(precision, hp2d_lib, oracle_lib):
    case = random_terrain(40, 56, seed=6, rain=0.0)
    ny, nx = case.shape
    res = case.resolution
    rng = np.random.default_rng(3)
    xg = np.concatenate([[res * 5], rng.uniform(-50, res * nx + 50, 5)])   # one gauge on a cell centre
    yg = np.concatenate([[-res * 8], rng.uniform(-res * ny - 50, 50, 5)])
    rates = rng.uniform(0, 120, (6, 6))
    rates[2, 1] = np.nan
    rates[4, :] = np.nan
    g, o = make_pair(case, precision)
    g.set_rain_gauges(xg, yg, rates, 0.25)
    o.set_rain_maps(L.idw_rain_maps(xg, yg, rates, ny, nx, res), 0.25)
    for chunk in (3, 64, 128, 200):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS, f"after chunk {chunk}")
        assert_same_clock(g, o)
    assert g.diag()["rain_volume"] > 0
