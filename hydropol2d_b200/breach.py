"""Dam-breach inflow hydrographs for dam-break ensembles.

``breach_hydrograph_cav`` restates breach_hydrograph_CAV.m:6-46, the instantaneous-breach
model the ensemble driver uses to feed each breach member through an inflow hydrograph
(HydroPol2D_Main_While_Ensemble.m:141-160): a constant peak outflow
Qp = 8/27 B sqrt(g) h^(3/2) until tp = 15/8 W / sqrt(g h), then the decay
Q(t) = (-1/2 (B sqrt(g))^(2/3) h (tp - t) / Sf + Qp^(-1/3))^(-3) with Sf = S0 - Qp tp, and the
reservoir depth drawn down by the outflow over the depth-area curve.  ``inflow_table`` turns a
hydrograph into the start-stamped table and cells of ``SurfaceFlow.set_inflow``.
"""
from __future__ import annotations

import math
from typing import Callable

import numpy as np

G = 9.81


def breach_hydrograph_cav(h: float, W: float, breach: float, dt: float, tf: float,
                          depth_area: Callable[[float], float], depth_volume: Callable[[float], float]):
    """Returns (time [min], flow [m^3/s], reservoir depth [m]) at t = 0, dt, ..., tf [s] for a
    reservoir of depth ``h`` [m] and dam length ``W`` [m] breached over ``breach`` [m].

    As the reference: the volume S0 = depth_volume(h); during the peak the depth falls by
    Qp dt / depth_area(previous depth); after tp it falls by (Q_i + Q_{i-1}) dt / depth_area
    (the reference takes MATLAB's mean of that single sum, which is the sum itself)."""
    tp = 15.0 / 8.0 * W / math.sqrt(G * h)
    S0 = depth_volume(h)
    Qp = 8.0 / 27.0 * breach * math.sqrt(G) * h ** 1.5
    Sf = S0 - Qp * tp
    n = int(math.floor(tf / dt + 1e-10)) + 1          # MATLAB's 0:dt:tf
    time = dt * np.arange(n, dtype=np.float64)
    flow = np.empty(n)
    depth = np.empty(n)
    h0 = h
    k = (breach * math.sqrt(G)) ** (2.0 / 3.0)
    for i in range(n):
        t = i * dt
        if t <= tp:
            flow[i] = Qp
            depth[i] = h0 - Qp * dt / depth_area(h0 if i == 0 else depth[i - 1])
        else:
            flow[i] = (-0.5 * k * h * (tp - t) / Sf + Qp ** (-1.0 / 3.0)) ** -3.0
            depth[i] = h0 - (flow[i] + flow[i - 1]) * dt / depth_area(depth[i - 1])
        h0 = depth[i]
    return time / 60.0, flow, depth


def inflow_table(time_min: np.ndarray, flow_m3s: np.ndarray, rows, cols, dx: float) -> dict:
    """``SurfaceFlow.set_inflow`` arguments for one gauge spreading ``flow_m3s`` over the cells
    (rows, cols): the discharge becomes a depth rate over the cells' area
    (Q / (n_cells dx^2) x 1000 x 3600 mm/h, HydroPol2D_Main_While_Ensemble.m:160) and sample i of
    the hydrograph holds from time_min[i] to time_min[i+1]; nothing flows after the last."""
    rows = np.asarray(rows, dtype=np.int32).ravel()
    cols = np.asarray(cols, dtype=np.int32).ravel()
    rate = np.asarray(flow_m3s, dtype=np.float64) / (rows.size * dx * dx) * 1000.0 * 3600.0
    t = np.asarray(time_min, dtype=np.float64)
    t_start = np.concatenate([t, [t[-1] + (t[1] - t[0] if t.size > 1 else 1.0)]])
    rates = np.concatenate([rate, [0.0]])[:, None]
    return dict(t_start=t_start, rates=rates, rows=rows, cols=cols, gauge=np.zeros(rows.size, np.int32))
