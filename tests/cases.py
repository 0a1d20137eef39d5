"""Small seeded cases shared by the parity tests (shapes chosen to cross tile edges)."""
from __future__ import annotations

import numpy as np

from hydropol2d_b200 import synthetic as S


def small_vtilt(ny=40, nx=40, dx=10.0):
    return S.vtilt_case(ny, nx, dx)


def small_urban(n=96, seed=3, hours=0.5):
    return S.urban_case(n, 2.0, seed=seed, hours=hours)


def small_dambreak(ny=64, nx=256, seed=5):
    return S.dambreak_case(ny, nx, 5.0, seed=seed, hours=0.5)


def random_terrain(ny, nx, seed=0, dx=5.0, walls=False, rain=40.0):
    """Rough random DEM with a wet random start, outlets on the last column; optional
    NaN (idx_nan) walls."""
    rng = np.random.default_rng(seed)
    z = S.gaussian_random_field(ny, nx, -3.0, seed) * 2.0 + np.linspace(5, 0, nx)[None, :]
    if walls:
        z[rng.random((ny, nx)) < 0.03] = np.nan
    d0 = np.where(rng.random((ny, nx)) < 0.5, rng.uniform(0, 300, (ny, nx)), 0.0)
    d0[np.isnan(z)] = np.nan
    rough = rng.choice([0.013, 0.03, 0.05, 0.1], size=(ny, nx))
    rows = np.arange(ny, dtype=np.int32)
    cols = np.full(ny, nx - 1, dtype=np.int32)
    params = dict(routing_time=30.0, alfa_min=0.5, alfa_max=0.7, outlet_type=1, slope_outlet=0.01,
                  min_time_step=0.01, max_time_step=10.0)
    return S.Case(f"random_{ny}x{nx}", z, rough, dx, rows, cols, params, d0,
                  rain_uniform=(np.array([0.0, 5.0]), np.array([rain, 0.0])))
