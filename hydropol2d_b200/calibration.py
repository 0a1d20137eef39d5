"""Calibration and sensitivity analysis on the batched ensemble: every candidate parameter set
of a generation (or every one-at-a-time variation) is one member of one ``Ensemble`` run.

Automatic_Calibrator_HydroPol2D.m minimises Objective_Function_HydroPol2D.m over the
parameters with MATLAB's genetic algorithm, one model run per candidate.  Here a generation's
candidates run together on the GPU and their outlet hydrographs are scored with the
reference's objectives (``objective``, Objective_Function_HydroPol2D.m:114-160); the search is
a small real-coded evolutionary loop of its own (elitism, blend crossover, Gaussian mutation
within the bounds), not a restatement of MATLAB's ``ga``.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np

SMALL = 1e-6   # Objective_Function_HydroPol2D.m:112


def objective(obs: np.ndarray, mod: np.ndarray, kind: int = 5) -> float:
    """Objective_Function_HydroPol2D.m:114-160 for one event: ``obs`` and ``mod`` are
    (n_times, n_gauges) discharges [m^3/s], gauges weighted equally; smaller is better.
    1: -NSE; 2: RMSE; 3: -r; 4: |peak difference|; 5: -(NSE - 0.5 VE).  As the reference, the
    NSE's denominator is taken about the MODELLED mean (kinds 1 and 5) and kind 5 adds 1e-6 to
    it and to the volume error's denominator."""
    obs = np.asarray(obs, dtype=np.float64).reshape(len(obs), -1)
    mod = np.asarray(mod, dtype=np.float64).reshape(len(mod), -1)
    n = mod.shape[0]
    o = obs[:n]
    w = np.full(mod.shape[1], 1.0 / mod.shape[1])
    if kind in (1, 5):
        den = np.sum((o - mod.mean(axis=0)) ** 2, axis=0) + (SMALL if kind == 5 else 0.0)
        nse = 1.0 - np.sum((o - mod) ** 2, axis=0) / den
        if np.any(np.isnan(nse)):
            raise ValueError("NSE is NaN")
        if kind == 1:
            return float(-np.sum(w * nse))
        ve = np.abs(np.sum(o - mod, axis=0) / (np.sum(o, axis=0) + SMALL))
        return float(-np.sum(w * (nse - 0.5 * ve)))
    if kind == 2:
        rmse = np.sqrt(np.sum((o - mod) ** 2, axis=0) / len(obs))
        return float(np.sum(w * rmse))
    if kind == 3:
        return float(-np.corrcoef(o.ravel(), mod.ravel())[0, 1])
    if kind == 4:
        return float(np.sum(np.abs(o.max(axis=0) - mod.max(axis=0))))
    raise ValueError("objective kind must be 1..5")


def discharge_at(times_min: np.ndarray, t_samples: Sequence[float], v_samples: Sequence[float]) -> np.ndarray:
    """Mean outlet discharge [m^3/s] over each observation interval (times_min[k-1],
    times_min[k]] from a run's cumulative outlet volume [m^3] sampled at clocks t_samples [min]
    (linear between samples; the first interval starts at 0)."""
    t = np.concatenate([[0.0], np.asarray(t_samples, dtype=np.float64)])
    v = np.concatenate([[0.0], np.asarray(v_samples, dtype=np.float64)])
    times = np.asarray(times_min, dtype=np.float64)
    vol = np.interp(times, t, v)
    prev = np.concatenate([[0.0], times[:-1]])
    vprev = np.concatenate([[0.0], vol[:-1]])
    return (vol - vprev) / ((times - prev) * 60.0)


def ensemble_runs(cases: Sequence, times_min: np.ndarray, device: int = 0, chunk: int = 32,
                  flood_depth_m: float | None = None) -> dict:
    """Runs ``cases`` (FP32 ``synthetic.Case``s on grids of any size) as one batched ensemble.
    Returns the outlet discharges at the observation times ("q", (members, n_times)) from each
    member's cumulative outlet volume sampled after every ``chunk`` launches and, with
    ``flood_depth_m``, the largest flooded area seen at those samples ("flooded_area" [m^2]:
    cells deeper than it x cell area, the Flooded_Area of save_output_maps.m:451 with 150 mm)."""
    from .ensemble import Ensemble
    from .surface import SurfaceFlow
    ens = Ensemble(device)
    try:
        for c in cases:
            m = SurfaceFlow(*c.shape, c.resolution, "fp32", device=device, **c.params)
            c.apply(m)
            ens.add(m)
        samples = [([], []) for _ in cases]
        area = np.zeros(len(cases))
        active = len(cases)
        while active:
            active = ens.steps(chunk)
            for i, (s, m) in enumerate(zip(samples, ens.members)):
                d = m.diag()
                s[0].append(d["t"])
                s[1].append(d["outlet_volume"])
                if flood_depth_m is not None:
                    wet = np.count_nonzero(m.download_native("h") > flood_depth_m)
                    area[i] = max(area[i], wet * m.resolution ** 2)
        out = {"q": np.stack([discharge_at(times_min, ts, vs) for ts, vs in samples])}
        if flood_depth_m is not None:
            out["flooded_area"] = area
        return out
    finally:
        ens.close()


def ensemble_hydrographs(cases: Sequence, times_min: np.ndarray, device: int = 0, chunk: int = 32) -> np.ndarray:
    """Outlet discharges of ``cases`` at the observation times, (members, n_times)."""
    return ensemble_runs(cases, times_min, device, chunk)["q"]


def hydrograph_metrics(q: np.ndarray, dt_min: float) -> dict:
    """Sensitivity_Analysis_HydroPol2D.m:152-157 for hydrographs sampled every ``dt_min``:
    peak flow [m^3/s], volume sum(q dt 60) [m^3] and time to peak (first maximum, samples
    from 0) [min]; ``q`` is (..., n_times)."""
    q = np.asarray(q, dtype=np.float64)
    return {"peak": q.max(axis=-1), "volume": (q * dt_min * 60.0).sum(axis=-1),
            "time_to_peak": np.argmax(q, axis=-1) * dt_min}


def sensitivity_oat(make_case: Callable[[dict], object], base: dict, names: Sequence[str],
                    factors: Sequence[float], times_min: np.ndarray, device: int = 0, chunk: int = 16,
                    flood_depth_m: float = 0.15) -> dict:
    """One-at-a-time sensitivity (Sensitivity_Analysis_HydroPol2D.m:82-171): every parameter in
    ``names`` is scaled by every factor while the others keep their ``base`` values; the
    baseline and all variations run as ONE batched ensemble.  Returns, per output, the
    percentage change against the baseline as (len(names), len(factors)) arrays ("peak",
    "volume", "time_to_peak", "flooded_area"), plus the baseline outputs."""
    times_min = np.asarray(times_min, dtype=np.float64)
    dt = float(times_min[1] - times_min[0])
    variants = [dict(base)]
    for n in names:
        for f in factors:
            variants.append(dict(base, **{n: base[n] * f}))
    runs = ensemble_runs([make_case(v) for v in variants], times_min, device, chunk, flood_depth_m)
    m = hydrograph_metrics(runs["q"], dt)
    m["flooded_area"] = runs["flooded_area"]
    out = {"baseline": {k: float(v[0]) for k, v in m.items()}}
    for k, v in m.items():
        b = v[0]
        out[k] = ((v[1:] - b) / b * 100.0).reshape(len(names), len(factors))
    return out


def calibrate(evaluate: Callable[[np.ndarray], np.ndarray], lower: Sequence[float], upper: Sequence[float],
              population: int = 24, generations: int = 4, elite: float = 0.25, seed: int = 0) -> dict:
    """Minimises ``evaluate`` over the box [lower, upper].  ``evaluate`` maps a
    (population, n_params) array to the objective of each row (one batched ensemble run per
    call).  Generation 0 is a Latin hypercube; later ones keep the elite fraction and fill up
    with blend crossovers of two elites plus Gaussian mutation (its scale shrinking by half per
    generation), clipped to the box.  Returns the best parameters, its objective and the
    history of (population, objectives) per generation."""
    lo = np.asarray(lower, dtype=np.float64)
    hi = np.asarray(upper, dtype=np.float64)
    rng = np.random.default_rng(seed)
    npar = lo.size
    u = (rng.permuted(np.tile(np.arange(population), (npar, 1)), axis=1).T + rng.random((population, npar))) / population
    pop = lo + u * (hi - lo)
    history = []
    best_x, best_f = None, np.inf
    n_elite = max(2, int(round(elite * population)))
    for gen in range(generations):
        f = np.asarray(evaluate(pop), dtype=np.float64)
        history.append((pop.copy(), f.copy()))
        order = np.argsort(f, kind="stable")
        if f[order[0]] < best_f:
            best_f, best_x = float(f[order[0]]), pop[order[0]].copy()
        if gen + 1 == generations:
            break
        elites = pop[order[:n_elite]]
        kids = []
        sigma = 0.2 * (hi - lo) * 0.5 ** gen
        while len(kids) < population - n_elite:
            a, b = elites[rng.integers(n_elite)], elites[rng.integers(n_elite)]
            alpha = rng.uniform(-0.25, 1.25, npar)
            kids.append(np.clip(a + alpha * (b - a) + rng.normal(0.0, sigma), lo, hi))
        pop = np.vstack([elites, np.asarray(kids)])
    return {"x": best_x, "objective": best_f, "history": history}
