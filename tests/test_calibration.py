"""Objectives of Objective_Function_HydroPol2D.m:114-160 on hand-computed cases, the volume ->
discharge sampling and the evolutionary search on an analytic function (CPU only)."""
import numpy as np
import pytest

from hydropol2d_b200.calibration import calibrate, discharge_at, objective


def test_objective_kinds_by_hand():
    obs = np.array([1.0, 3.0, 2.0, 4.0])
    mod = np.array([1.5, 2.5, 2.0, 3.0])
    err2 = 0.25 + 0.25 + 0.0 + 1.0
    mbar = mod.mean()                                   # 2.25: the reference centres on the model
    den = np.sum((obs - mbar) ** 2)
    assert objective(obs, mod, 1) == pytest.approx(-(1.0 - err2 / den), rel=1e-15)
    ve = abs(np.sum(obs - mod)) / (obs.sum() + 1e-6)
    nse5 = 1.0 - err2 / (den + 1e-6)
    assert objective(obs, mod, 5) == pytest.approx(-(nse5 - 0.5 * ve), rel=1e-15)
    assert objective(obs, mod, 2) == pytest.approx(np.sqrt(err2 / 4), rel=1e-15)
    assert objective(obs, mod, 3) == pytest.approx(-np.corrcoef(obs, mod)[0, 1], rel=1e-15)
    assert objective(obs, mod, 4) == pytest.approx(1.0, rel=1e-15)
    with pytest.raises(ValueError):
        objective(obs, mod, 6)


def test_objective_perfect_and_gauge_weights():
    obs = np.array([[1.0, 10.0], [2.0, 30.0], [5.0, 20.0]])
    assert objective(obs, obs, 1) == pytest.approx(-1.0)
    assert objective(obs, obs, 5) == pytest.approx(-1.0)
    assert objective(obs, obs, 2) == 0.0
    mod = obs.copy()
    mod[:, 1] *= 1.1
    one = objective(obs[:, 1], mod[:, 1], 1)
    assert objective(obs, mod, 1) == pytest.approx(0.5 * (-1.0) + 0.5 * one)
    # a shorter model series is scored on the observations it covers
    assert objective(obs, obs[:2], 2) == 0.0


def test_discharge_from_cumulative_volume():
    q = 2.5                                              # m^3/s constant
    ts = np.array([0.7, 1.9, 3.1, 6.4, 9.0])             # minutes
    vs = q * ts * 60.0
    out = discharge_at(np.array([1.0, 2.0, 5.0, 8.0]), ts, vs)
    assert np.allclose(out, q, rtol=1e-12)
    # a volume step inside one interval lands in that interval only
    ts = np.array([1.0, 2.0, 3.0, 4.0])
    vs = np.array([0.0, 0.0, 120.0, 120.0])
    out = discharge_at(np.array([1.0, 2.0, 3.0, 4.0]), ts, vs)
    assert np.allclose(out, [0.0, 0.0, 2.0, 0.0])


def test_calibrate_finds_box_minimum_and_is_seeded():
    target = np.array([0.3, -1.2])

    def f(pop):
        return np.sum((pop - target) ** 2, axis=1)

    r = calibrate(f, [-2.0, -2.0], [2.0, 2.0], population=24, generations=8, seed=3)
    assert np.allclose(r["x"], target, atol=0.05)
    assert r["objective"] == pytest.approx(f(r["x"][None])[0])
    assert len(r["history"]) == 8
    for pop, _ in r["history"]:
        assert pop.shape == (24, 2) and np.all(pop >= -2.0) and np.all(pop <= 2.0)
    r2 = calibrate(f, [-2.0, -2.0], [2.0, 2.0], population=24, generations=8, seed=3)
    assert np.array_equal(r["x"], r2["x"])
    # generation 0 is a Latin hypercube: one point per stratum in each dimension
    pop0 = r["history"][0][0]
    for d in range(2):
        assert sorted(np.floor((pop0[:, d] + 2.0) / 4.0 * 24).astype(int)) == list(range(24))
    # the best objective never gets worse from one generation to the next (elitism)
    bests = [h[1].min() for h in r["history"]]
    assert all(b1 <= b0 for b0, b1 in zip(bests, bests[1:]))


def test_hydrograph_metrics_by_hand():
    from hydropol2d_b200.calibration import hydrograph_metrics
    q = np.array([[0.0, 2.0, 5.0, 5.0, 1.0], [1.0, 1.0, 1.0, 1.0, 1.0]])
    m = hydrograph_metrics(q, 2.0)
    assert list(m["peak"]) == [5.0, 1.0]
    assert list(m["volume"]) == [13.0 * 120.0, 5.0 * 120.0]
    assert list(m["time_to_peak"]) == [4.0, 0.0]      # first maximum, samples counted from 0
