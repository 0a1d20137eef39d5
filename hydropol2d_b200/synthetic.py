"""Seeded synthetic inputs of the benchmark configurations (no public dataset is involved).

* ``vtilt_case``    200 x 200, dx 10 m V-tilted catchment (two planes sloping 0.005 to a
                    channel sloping 0.002), n = 0.02, 100 mm/h for 30 min, 60 min, alpha 0.7.
                    Geometry follows Validation/Phase1_VTilted_Catchment/
                    generate_phase1_vtilted_domain.py:87-91.
* ``urban_case``    2048 x 2048, dx 2 m Gaussian random field (power spectrum k^-3, 40 m
                    relief) + rectangular buildings (+10 m, 30 % of cells); Voronoi LULC
                    (n in {0.013, 0.03, 0.05, 0.1}) and soil (Green-Ampt classes); 64 x 64
                    rain field U(0, 120) mm/h redrawn every 5 min; 2 h.
* ``dambreak_case`` 4096 x 8192 (ny x nx), dx 5 m fractal valley: parabolic cross-section
                    60 m deep + GRF of 5 m std; reservoir 30 m deep behind a wall over the
                    upstream 5 % (removed at t = 0); n = 0.035; 3 h.

All fields are float64 numpy arrays in the reference's units (m, mm, mm/h); the same
arrays feed the GPU library and the CPU restatements.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Case:
    name: str
    z: np.ndarray
    roughness: np.ndarray
    resolution: float
    outlet_rows: np.ndarray
    outlet_cols: np.ndarray
    params: dict
    d0: np.ndarray
    rain_uniform: tuple | None = None       # (t_start [min], rate [mm/h])
    rain_maps: np.ndarray | None = None     # (n, my, mx) float32 [mm/h]
    rain_map_dt: float = 5.0
    soil: dict | None = None                # set_soil kwargs
    I0: np.ndarray | None = None            # mm
    meta: dict = field(default_factory=dict)
    inflow: dict | None = None              # set_inflow kwargs (t_start, rates, rows, cols, gauge)
    stage: dict | None = None               # set_stage kwargs (t_start, depth_m, rows, cols, gauge)
    reservoirs: dict | None = None          # set_reservoirs kwargs (flag_reservoir = 1)

    @property
    def shape(self):
        return self.z.shape

    def apply(self, sf):
        """Upload the case into a SurfaceFlow (or an oracle with the same surface)."""
        sf.upload_static(self.z, self.roughness, self.outlet_rows, self.outlet_cols)
        if self.soil is not None:
            sf.set_soil(**self.soil)
        sf.set_state(self.d0, None, self.I0)
        if self.rain_uniform is not None:
            sf.set_rain_uniform(*self.rain_uniform)
        if self.rain_maps is not None:
            sf.set_rain_maps(self.rain_maps, self.rain_map_dt)
        if self.inflow is not None:
            sf.set_inflow(**self.inflow)
        if self.stage is not None:
            sf.set_stage(**self.stage)
        if self.reservoirs is not None:
            sf.set_reservoirs(**self.reservoirs)
        return sf


def gaussian_random_field(ny: int, nx: int, slope: float = -3.0, seed: int = 0) -> np.ndarray:
    """Zero-mean, unit-std field with isotropic power spectrum P(k) ~ k^slope (FFT method)."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((ny, nx))
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = np.inf
    amp = k ** (slope / 2.0)
    f = np.fft.irfft2(np.fft.rfft2(noise) * amp, s=(ny, nx))
    f -= f.mean()
    f /= f.std()
    return f


def voronoi_classes(ny: int, nx: int, n_seeds: int, n_classes: int, seed: int) -> np.ndarray:
    """Class map from a Voronoi partition of seeded random sites (nearest site wins)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    sites = rng.uniform([0, 0], [ny, nx], size=(n_seeds, 2))
    site_class = rng.integers(0, n_classes, size=n_seeds)
    tree = cKDTree(sites)
    out = np.empty((ny, nx), dtype=np.uint8)
    cols = np.arange(nx) + 0.5
    for r0 in range(0, ny, 256):
        rr = np.arange(r0, min(ny, r0 + 256)) + 0.5
        pts = np.stack(np.meshgrid(rr, cols, indexing="ij"), axis=-1).reshape(-1, 2)
        _, idx = tree.query(pts)
        out[r0:r0 + len(rr)] = site_class[idx].reshape(len(rr), nx)
    return out


def green_ampt_soil_tables(ksat_mmh, psi_mm, dtheta, theta_sat=0.45, theta_r=0.05, kr=0.0):
    """Per-class Green-Ampt tables with the reference's derived parameters
    (HydroPol2D_preprocessing.m:2250-2253: Tr = 4.5/sqrt(ksat/25.4) h,
    Lu = 4 sqrt(ksat/25.4) in, k_out = (theta_sat - theta_r) kr Lu 1000 mm/h;
    min_soil_moisture = eps mm, :2387-2388)."""
    ksat = np.asarray(ksat_mmh, dtype=np.float64)
    Tr = 4.5 / np.sqrt(ksat / 25.4)
    Lu = 4.0 * np.sqrt(ksat / 25.4) * 2.54 / 100.0
    k_out = (theta_sat - theta_r) * kr * Lu * 1000.0
    return dict(ksat=ksat, psi=np.asarray(psi_mm, dtype=np.float64),
                dtheta=np.asarray(dtheta, dtype=np.float64), Lu=Lu, k_out=k_out, Tr=Tr,
                min_soil_moisture=np.full(ksat.shape, np.finfo(np.float64).eps))


def vtilt_domain(ny: int, nx: int, dx: float, side_slope: float, long_slope: float,
                 z_outlet: float = 100.0, channel_cols: int = 2):
    """V-tilted DEM: rows run downstream toward row 0; the channel is the central
    ``channel_cols`` columns; planes slope toward it (generate_phase1_vtilted_domain.py:87-91)."""
    left = (nx - channel_cols) // 2
    x = np.arange(nx, dtype=np.float64) * dx
    y = np.arange(ny, dtype=np.float64) * dx
    x_left_end = left * dx
    x_channel_end = (left + channel_cols - 1) * dx
    base = z_outlet + long_slope * y[:, None] + 0.0 * x[None, :]
    z = base.copy()
    lm = x[None, :] < x_left_end
    rm = x[None, :] > x_channel_end
    z = np.where(lm, base + side_slope * (x_left_end - x[None, :]), z)
    z = np.where(rm, base + side_slope * (x[None, :] - x_channel_end), z)
    ch = np.arange(left, left + channel_cols)
    return z, ch


def vtilt_case(ny: int = 200, nx: int = 200, dx: float = 10.0) -> Case:
    z, ch = vtilt_domain(ny, nx, dx, 0.005, 0.002)
    rows = np.zeros(ch.size, dtype=np.int32)
    params = dict(routing_time=60.0, alfa_min=0.7, alfa_max=0.7, outlet_type=1, slope_outlet=0.002,
                  min_time_step=0.01, max_time_step=10.0)
    return Case("vtilt_200x200_dx10", z, np.full((ny, nx), 0.02), dx, rows, ch.astype(np.int32), params,
                np.zeros((ny, nx)), rain_uniform=(np.array([0.0, 30.0]), np.array([100.0, 0.0])))


def inflow_hydrograph_rates(q_m3s: np.ndarray, n_cells: int, dx: float) -> np.ndarray:
    """Discharge [m^3/s] spread over a gauge's cells as a depth rate [mm/h], the reference's
    conversion (Analytical_Catchments.m:118)."""
    return np.asarray(q_m3s, dtype=np.float64) / (n_cells * dx * dx) * 1000.0 * 3600.0


def inflow_case(ny: int = 96, nx: int = 96, dx: float = 10.0, minutes: float = 40.0, peak_m3s: float = 4.0) -> Case:
    """The V-tilted catchment, dry and without rain, fed by two inflow hydrographs: gauge 0
    on the channel's upstream cells (a triangular flood, 0 -> peak at 10 min -> 0 at 30 min,
    1-min steps) and gauge 1 on a block of cells of the left plane (a constant 0.2 m^3/s from
    minute 5).  Outlets on the channel's downstream end (row 0)."""
    z, ch = vtilt_domain(ny, nx, dx, 0.005, 0.002)
    rows = np.zeros(ch.size, dtype=np.int32)
    params = dict(routing_time=minutes, alfa_min=0.7, alfa_max=0.7, outlet_type=1, slope_outlet=0.002,
                  min_time_step=0.01, max_time_step=10.0)
    t = np.arange(0.0, 31.0)                      # start of each 1-min interval [min]
    q0 = np.interp(t + 0.5, [0.0, 10.0, 30.0], [0.0, peak_m3s, 0.0])
    q0[-1] = 0.0
    g0_r = np.full(ch.size, ny - 1, dtype=np.int32)
    g0_c = ch.astype(np.int32)
    br, bc = np.meshgrid(np.arange(ny // 2, ny // 2 + 3), np.arange(nx // 6, nx // 6 + 3), indexing="ij")
    g1_r, g1_c = br.ravel().astype(np.int32), bc.ravel().astype(np.int32)
    q1 = np.where(t >= 5.0, 0.2, 0.0)
    rates = np.stack([inflow_hydrograph_rates(q0, g0_r.size, dx), inflow_hydrograph_rates(q1, g1_r.size, dx)], axis=1)
    inflow = dict(t_start=t, rates=rates, rows=np.concatenate([g0_r, g1_r]), cols=np.concatenate([g0_c, g1_c]),
                  gauge=np.concatenate([np.zeros(g0_r.size, np.int32), np.ones(g1_r.size, np.int32)]))
    return Case(f"inflow_vtilt_{ny}x{nx}", z, np.full((ny, nx), 0.03), dx, rows, ch.astype(np.int32), params,
                np.zeros((ny, nx)), inflow=inflow)


def structures_case(ny: int = 48, nx: int = 48, dx: float = 10.0, minutes: float = 20.0, soil: bool = False,
                    maps: bool = False) -> Case:
    """The V-tilted catchment with a 0.6 m pond on the left plane drained by control structures
    (flag_reservoir = 1, Local_Inertial_Model_D4.m:318-344), rain at 50 mm/h for 10 min:
    structure 0 drains the pond's centre through two rating curves (crest 0.2 m into a cell
    down the plane, crest 0.4 m into a cell along it); structure 1 drains structure 0's first
    downstream cell into the channel (so it sees structure 0's transfer the same step);
    structure 2 drains a right-plane cell that only rain fills.  ``soil`` adds Green-Ampt
    classes, ``maps`` replaces the uniform rain by 8 x 8 rate maps."""
    z, ch = vtilt_domain(ny, nx, dx, 0.005, 0.002)
    rows = np.zeros(ch.size, dtype=np.int32)
    params = dict(routing_time=minutes, alfa_min=0.7, alfa_max=0.7, outlet_type=1, slope_outlet=0.002,
                  min_time_step=0.01, max_time_step=10.0, flag_reservoir=1)
    pr, pc = ny // 2, nx // 6
    d0 = np.zeros((ny, nx))
    d0[pr - 1:pr + 2, pc - 1:pc + 2] = 600.0
    res = dict(res_row=[pr, pr, ny - 3], res_col=[pc, pc + 6, nx - 5],
               k1=[3.0, 0.5, 1.0], h1=[0.2, 0.0, 0.001], k2=[1.5, 5.0 / 3.0, 1.0],
               ds1_row=[pr, ny // 3, ny - 3], ds1_col=[pc + 6, int(ch[0]), nx - 10],
               k3=[1.0, 0.0, 0.0], h2=[0.4, 0.0, 0.0], k4=[2.5, 0.0, 0.0],
               ds2_row=[pr + 5, -1, -1], ds2_col=[pc, -1, -1])
    c = Case(f"structures_vtilt_{ny}x{nx}", z, np.full((ny, nx), 0.03), dx, rows, ch.astype(np.int32), params,
             d0, rain_uniform=(np.array([0.0, 10.0]), np.array([50.0, 0.0])), reservoirs=res)
    if soil:
        cls = voronoi_classes(ny, nx, 12, 3, 5).astype(np.uint8)
        cls[:, ch] = 255
        c.soil = dict(soil_class=cls, **green_ampt_soil_tables([1.0, 10.0, 30.0], [50.0, 110.0, 200.0],
                                                                  [0.2, 0.3, 0.4]))
        c.I0 = np.full((ny, nx), 5.0)
        c.params["flag_infiltration"] = 1
    if maps:
        rng = np.random.default_rng(4)
        c.rain_uniform = None
        c.rain_maps = rng.uniform(0.0, 100.0, size=(3, 8, 8)).astype(np.float32)
        c.rain_map_dt = 5.0
    return c


def breach_inflow_case(ny: int = 128, nx: int = 512, dx: float = 5.0, seed: int = 11, minutes: float = 30.0,
                       breach_factor: float = 0.5, reservoir_depth: float = 20.0) -> Case:
    """The dam-break valley, dry, fed at its upstream edge by the breach outflow of a
    rectangular reservoir (``breach.breach_hydrograph_cav``: depth ``reservoir_depth``, dam length
    the valley width, breach ``breach_factor`` of it, 2 km^2 of surface, 1-min samples), as
    HydroPol2D_Main_While_Ensemble.m:141-160 feeds its breach members.  The inflow cells are the
    first column's cells within 2 m of the thalweg's elevation."""
    from .breach import breach_hydrograph_cav, inflow_table
    c = dambreak_case(ny, nx, dx, seed=seed, hours=minutes / 60.0)
    W = ny * dx
    area = 2.0e6
    t_min, q, _ = breach_hydrograph_cav(reservoir_depth, W, breach_factor * W, 60.0, minutes * 60.0,
                                        lambda h: area, lambda h: area * h)
    z0 = c.z[:, 0]
    rows = np.nonzero(z0 <= z0.min() + 2.0)[0]
    c.d0 = np.zeros_like(c.d0)
    c.inflow = inflow_table(t_min, q, rows, np.zeros(rows.size, np.int32), dx)
    c.name = f"breach_inflow_{ny}x{nx}"
    c.meta = dict(peak_m3s=float(q.max()), inflow_cells=int(rows.size))
    return c


def urban_case(n: int = 2048, dx: float = 2.0, seed: int = 7, hours: float = 2.0) -> Case:
    rng = np.random.default_rng(seed)
    grf = gaussian_random_field(n, n, -3.0, seed)
    z = (grf - grf.min()) / (grf.max() - grf.min()) * 40.0
    bld = np.zeros((n, n), dtype=bool)
    target = 0.30 * n * n
    while bld.sum() < target:
        h, w = rng.integers(4, 24, size=2)
        r, c = rng.integers(0, n - h), rng.integers(0, n - w)
        bld[r:r + h, c:c + w] = True
    z = z + 10.0 * bld
    lulc = voronoi_classes(n, n, 400, 4, seed + 1)
    nvals = np.array([0.013, 0.03, 0.05, 0.1])
    rough = nvals[lulc]
    soil = voronoi_classes(n, n, 300, 3, seed + 2)
    tabs = green_ampt_soil_tables([1.0, 10.0, 30.0], [50.0, 110.0, 200.0], [0.2, 0.3, 0.4])
    n_maps = int(np.ceil(hours * 60 / 5.0)) + 1
    maps = rng.uniform(0.0, 120.0, size=(n_maps, 64, 64)).astype(np.float32)
    edge_r = np.concatenate([np.zeros(n), np.full(n, n - 1), np.arange(1, n - 1), np.arange(1, n - 1)])
    edge_c = np.concatenate([np.arange(n), np.arange(n), np.zeros(n - 2), np.full(n - 2, n - 1)])
    params = dict(routing_time=hours * 60.0, alfa_min=0.5, alfa_max=0.7, outlet_type=2,
                  flag_infiltration=1, min_time_step=0.01, max_time_step=10.0)
    return Case(f"urban_{n}x{n}_dx{dx:g}", z, rough, dx, edge_r.astype(np.int32), edge_c.astype(np.int32),
                params, np.zeros((n, n)), rain_maps=maps, rain_map_dt=5.0,
                soil=dict(soil_class=soil, **tabs), I0=np.full((n, n), 5.0),
                meta=dict(buildings=float(bld.mean())))


def dambreak_case(ny: int = 4096, nx: int = 8192, dx: float = 5.0, seed: int = 11, hours: float = 3.0,
                  long_slope: float = 0.001) -> Case:
    """Valley along x (columns); reservoir over the first 5 % of columns."""
    grf = gaussian_random_field(ny, nx, -3.0, seed) * 5.0
    y = (np.arange(ny) + 0.5) / ny * 2.0 - 1.0
    x = np.arange(nx) * dx
    z = 60.0 * (y[:, None] ** 2) + long_slope * (x[-1] - x)[None, :] + grf + 20.0
    x_dam = int(round(0.05 * nx))
    thalweg = float(np.min(z[:, x_dam]))
    wse = thalweg + 30.0
    d0 = np.zeros((ny, nx))
    d0[:, :x_dam] = np.maximum(wse - z[:, :x_dam], 0.0) * 1000.0
    rows = np.arange(ny, dtype=np.int32)
    cols = np.full(ny, nx - 1, dtype=np.int32)
    params = dict(routing_time=hours * 60.0, alfa_min=0.5, alfa_max=0.7, outlet_type=1,
                  slope_outlet=long_slope, min_time_step=0.01, max_time_step=10.0)
    return Case(f"dambreak_{ny}x{nx}_dx{dx:g}", z, np.full((ny, nx), 0.035), dx, rows, cols, params, d0,
                meta=dict(x_dam=x_dam, wse=wse))


def _side(rng, lo: int = 256, hi: int = 1024, mult: int = 32) -> int:
    s = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
    return int(min(hi, max(lo, mult * round(s / mult))))


def ensemble_member_spec(i: int, seed: int = 2024, lo: int = 256, hi: int = 1024,
                         breach_share: float = 0.25) -> dict:
    """The seeded draws of ensemble member ``i`` (grid sides, roughness factor, forcing kind
    and its parameters) without building its arrays; ``ensemble_member`` builds from these."""
    rng = np.random.default_rng([seed, i])
    ny, nx = _side(rng, lo, hi), _side(rng, lo, hi)
    nfac = float(rng.uniform(0.7, 1.3))
    if rng.uniform() >= breach_share:
        rate = float(rng.uniform(20.0, 150.0))
        dur = float(rng.uniform(30.0, 90.0))
        return dict(kind="rain", ny=ny, nx=nx, n_factor=nfac, rate=rate, duration=dur)
    return dict(kind="breach", ny=ny, nx=nx, n_factor=nfac, breach_factor=float(rng.uniform(0.2, 1.0)))


def ensemble_member_cost(i: int, seed: int = 2024, lo: int = 256, hi: int = 1024, breach_share: float = 0.25,
                         rain_tail_min: float = 30.0, breach_minutes: float = 30.0) -> float:
    """A priori cell-updates of member ``i``: cells x (simulated seconds / a CFL timestep
    alpha dx / sqrt(g h)), with h the event's rain depth (rain members, at least 1 cm) or the
    reservoir depth (breach members).  Used to balance members across GPUs; the members'
    real step counts come from their own CFL sequence."""
    sp = ensemble_member_spec(i, seed, lo, hi, breach_share)
    cells = sp["ny"] * sp["nx"]
    if sp["kind"] == "rain":
        h = max(sp["rate"] * sp["duration"] / 60.0 / 1000.0, 0.01)
        dt = min(0.7 * 10.0 / np.sqrt(9.81 * h), 10.0)
        return float(cells * (sp["duration"] + rain_tail_min) * 60.0 / dt)
    h = 30.0 * max(sp["ny"] / 4096.0, 0.25)
    dt = min(0.5 * 5.0 / np.sqrt(9.81 * h), 10.0)
    return float(cells * breach_minutes * 60.0 / dt)


def ensemble_member(i: int, seed: int = 2024, lo: int = 256, hi: int = 1024, breach_share: float = 0.25,
                    rain_tail_min: float = 30.0, breach_minutes: float = 30.0) -> Case:
    """Member ``i`` of the batched-ensemble configuration (HydroPol2D_Main_While_Ensemble.m
    perturbs roughness and forcing per member; Probabilistic_dam_break_analysis.m varies the
    breach).  Seeded per member:

    * grid sides log-uniform in [lo, hi], multiples of 32 (ny and nx drawn separately);
    * rain members (share 1 - breach_share): the V-tilted catchment of the 200 x 200 case
      (dx 10 m, planes 0.005, channel 0.002) on the member's grid plus a member-seeded
      random field (k^-3, 0.5 m std), Manning n = 0.02 x U(0.7, 1.3), uniform rain
      U(20, 150) mm/h for U(30, 90) min, simulated to the end of rain + ``rain_tail_min``;
    * breach members: the dam-break valley on the member's grid (dx 5 m, valley depth and
      random field scaled with the grid's width), a wall across the valley at 5 % of the
      length with a breach of U(0.2, 1.0) x the valley width around the thalweg, n = 0.035
      x U(0.7, 1.3), ``breach_minutes`` simulated.
    """
    sp = ensemble_member_spec(i, seed, lo, hi, breach_share)
    ny, nx, nfac = sp["ny"], sp["nx"], sp["n_factor"]
    if sp["kind"] == "rain":
        dx = 10.0
        z, ch = vtilt_domain(ny, nx, dx, 0.005, 0.002)
        z = z + 0.5 * gaussian_random_field(ny, nx, -3.0, seed * 7919 + i)
        rate, dur = sp["rate"], sp["duration"]
        rows = np.zeros(ch.size, dtype=np.int32)
        params = dict(routing_time=dur + rain_tail_min, alfa_min=0.7, alfa_max=0.7, outlet_type=1,
                      slope_outlet=0.002, min_time_step=0.01, max_time_step=10.0)
        return Case(f"member{i}_rain_{ny}x{nx}", z, np.full((ny, nx), 0.02 * nfac), dx, rows,
                    ch.astype(np.int32), params, np.zeros((ny, nx)),
                    rain_uniform=(np.array([0.0, dur]), np.array([rate, 0.0])),
                    meta=dict(kind="rain", rate=rate, duration=dur, n_factor=nfac))
    dx = 5.0
    f = sp["breach_factor"]
    scale = ny / 4096.0
    grf = gaussian_random_field(ny, nx, -3.0, seed * 7919 + i) * 5.0 * scale
    y = (np.arange(ny) + 0.5) / ny * 2.0 - 1.0
    x = np.arange(nx) * dx
    z = 60.0 * scale * (y[:, None] ** 2) + 0.001 * (x[-1] - x)[None, :] + grf + 20.0
    x_dam = max(2, int(round(0.05 * nx)))
    half = max(1, int(round(0.5 * f * ny)))
    thalweg_row = int(np.argmin(z[:, x_dam]))
    lo_r, hi_r = max(0, thalweg_row - half), min(ny, thalweg_row + half)
    wse = float(z[thalweg_row, x_dam]) + 30.0 * max(scale, 0.25)
    wall = np.ones(ny, dtype=bool)
    wall[lo_r:hi_r] = False
    z[wall, x_dam] = wse + 5.0
    d0 = np.zeros((ny, nx))
    d0[:, :x_dam] = np.maximum(wse - z[:, :x_dam], 0.0) * 1000.0
    rows = np.arange(ny, dtype=np.int32)
    cols = np.full(ny, nx - 1, dtype=np.int32)
    params = dict(routing_time=breach_minutes, alfa_min=0.5, alfa_max=0.7, outlet_type=1,
                  slope_outlet=0.001, min_time_step=0.01, max_time_step=10.0)
    return Case(f"member{i}_breach_{ny}x{nx}", z, np.full((ny, nx), 0.035 * nfac), dx, rows, cols,
                params, d0, rain_uniform=(np.array([0.0]), np.array([0.0])),
                meta=dict(kind="breach", breach_factor=f, n_factor=nfac, x_dam=x_dam))


# van Genuchten parameters of three textures (Carsel & Parrish, 1988, Water Resour. Res. 24):
# sand, loam, clay; alpha [1/m], ksat [mm/h]
VG_TEXTURES = dict(theta_r=[0.045, 0.078, 0.068], theta_sat=[0.43, 0.43, 0.38], n_vg=[2.68, 1.56, 1.09],
                   alpha_vg=[14.5, 3.6, 0.8], ksat=[297.0, 10.4, 2.0])


def vg_soil(ny: int, nx: int, z: np.ndarray, seed: int = 3, soil_depth: float = 1.5, wt_below_m: float = 1.0,
            impervious_share: float = 0.1) -> dict:
    """set_soil_vg arguments for a seeded Voronoi texture map: soil 1.5 m deep, water table
    1 m below the surface (a groundwater head of z - 1 m), 10 % impervious cells."""
    rng = np.random.default_rng(seed)
    cls = voronoi_classes(ny, nx, 60, 3, seed)
    cls = np.where(rng.random((ny, nx)) < impervious_share, 255, cls).astype(np.uint8)
    return dict(soil_class=cls, **{k: np.asarray(v, dtype=np.float64) for k, v in VG_TEXTURES.items()},
                soil_depth=np.full((ny, nx), soil_depth), gw_head=np.asarray(z, dtype=np.float64) - wt_below_m)
