"""Dam-breach inflow hydrograph (breach_hydrograph_CAV.m:6-46) for a rectangular reservoir,
checked against the model's closed forms, and its conversion into an inflow table (no GPU)."""
import math

import numpy as np
import pytest

from hydropol2d_b200.breach import breach_hydrograph_cav, inflow_table

G = 9.81


def test_peak_plateau_then_decay_rectangular_reservoir():
    h, W, B, A = 12.0, 300.0, 80.0, 2.0e5           # depth, dam length, breach, reservoir area
    t_min, q, d = breach_hydrograph_cav(h, W, B, 1.0, 1800.0, lambda x: A, lambda x: A * x)
    tp = 15 / 8 * W / math.sqrt(G * h)
    Qp = 8 / 27 * B * math.sqrt(G) * h ** 1.5
    assert t_min.size == 1801 and t_min[-1] == pytest.approx(30.0)
    plateau = t_min * 60 <= tp
    assert np.all(q[plateau] == Qp)
    # the decay of the model, and continuity at tp (the formula gives Qp there)
    Sf = A * h - Qp * tp
    t = t_min[~plateau] * 60
    expect = (-0.5 * (B * math.sqrt(G)) ** (2 / 3) * h * (tp - t) / Sf + Qp ** (-1 / 3)) ** -3
    assert np.allclose(q[~plateau], expect, rtol=1e-13)
    assert (-0.5 * (B * math.sqrt(G)) ** (2 / 3) * h * 0.0 / Sf + Qp ** (-1 / 3)) ** -3 == pytest.approx(Qp)
    assert np.all(np.diff(q[~plateau]) < 0)
    # drawdown: Qp dt / A per plateau second; after tp the reference's (Q_i + Q_{i-1}) dt / A
    n_p = int(plateau.sum())
    assert d[n_p - 1] == pytest.approx(h - n_p * Qp / A, rel=1e-12)
    i = n_p + 5
    assert d[i] == pytest.approx(d[i - 1] - (q[i] + q[i - 1]) / A, rel=1e-12)


def test_inflow_table_spreads_the_discharge():
    t_min, q, _ = breach_hydrograph_cav(8.0, 150.0, 40.0, 60.0, 3600.0, lambda x: 5e4, lambda x: 5e4 * x)
    rows, cols = np.array([3, 4, 5]), np.array([0, 0, 0])
    tab = inflow_table(t_min, q, rows, cols, 5.0)
    assert tab["t_start"].size == t_min.size + 1 and tab["rates"].shape == (t_min.size + 1, 1)
    # volume of the table (rate x duration over the cells) = the hydrograph's (piecewise constant)
    vol = np.sum(tab["rates"][:-1, 0] / 3.6e6 * 3 * 25.0 * np.diff(tab["t_start"]) * 60)
    assert vol == pytest.approx(np.sum(q) * 60.0, rel=1e-12)
    assert tab["rates"][-1, 0] == 0.0 and np.all(tab["gauge"] == 0)
