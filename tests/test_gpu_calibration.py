"""Calibration through the batched ensemble: a Manning roughness recovered from an outlet
hydrograph the solver produced with a known roughness (Automatic_Calibrator_HydroPol2D.m's
loop, with every candidate of a generation one ensemble member)."""
from dataclasses import replace

import numpy as np
import pytest

from hydropol2d_b200 import synthetic
from hydropol2d_b200.calibration import calibrate, ensemble_hydrographs, objective

pytestmark = pytest.mark.gpu

TRUE_N = 0.03
TIMES = np.arange(2.0, 41.0, 2.0)        # observation clocks [min]


def _cases(ns):
    base = synthetic.vtilt_case(64, 64, 10.0)
    params = {**base.params, "routing_time": 40.0}
    return [replace(base, roughness=np.full(base.shape, float(n)), params=params) for n in ns]


def test_roughness_recovered_from_outlet_hydrograph():
    obs = ensemble_hydrographs(_cases([TRUE_N]), TIMES, chunk=8)[0]
    assert obs.max() > 0.1 and np.all(np.isfinite(obs))

    # the same member inside a larger batch reproduces the observation
    q = ensemble_hydrographs(_cases([0.02, TRUE_N, 0.05]), TIMES, chunk=8)
    assert np.allclose(q[1], obs, rtol=1e-5, atol=1e-7)
    assert objective(obs, q[0]) > objective(obs, q[1])
    assert objective(obs, q[2]) > objective(obs, q[1])

    calls = []

    def evaluate(pop):
        calls.append(len(pop))
        hyd = ensemble_hydrographs(_cases(pop[:, 0]), TIMES, chunk=8)
        return np.array([objective(obs, h, 5) for h in hyd])

    r = calibrate(evaluate, [0.01], [0.08], population=12, generations=3, seed=1)
    assert calls == [12, 12, 12]
    assert abs(r["x"][0] - TRUE_N) < 0.1 * TRUE_N
    assert r["objective"] < -0.98


def test_one_at_a_time_sensitivity():
    """Rougher planes delay and flatten the outlet peak; more rain raises peak, volume and the
    flooded area -- the baseline and the 6 variations run as one ensemble."""
    from hydropol2d_b200.calibration import sensitivity_oat

    def make(p):
        base = synthetic.vtilt_case(48, 48, 10.0)
        rain = (np.array([0.0, 20.0]), np.array([p["rain"], 0.0]))
        return replace(base, roughness=np.full(base.shape, p["n"]), rain_uniform=rain,
                       params={**base.params, "routing_time": 30.0})

    r = sensitivity_oat(make, {"n": 0.03, "rain": 100.0}, ["n", "rain"], [0.5, 1.0, 1.5], TIMES[:15])
    assert r["peak"].shape == (2, 3)
    assert abs(r["peak"][0, 1]) < 1e-6 and abs(r["volume"][1, 1]) < 1e-6      # factor 1 = baseline
    assert r["peak"][0, 0] > 0 > r["peak"][0, 2]                              # smoother -> higher peak
    assert r["peak"][1, 2] > 0 and r["volume"][1, 2] > 30.0                    # more rain
    assert r["flooded_area"][1, 2] >= 0 and r["baseline"]["flooded_area"] >= 0
