"""Oracle, literal form -- TEST INFRASTRUCTURE ONLY.

FP64 numpy restatement of HydroPol2D's surface-flow time step in the reference's own
whole-array operation order, units and quirks (depth in mm, face flux state in mm/h,
time step in minutes).  This is what the tests call "the reference's FP64 path": MATLAB
and GNU Octave are absent here, and the path's arithmetic lives entirely in the
reference's own .m files, so this restatement stands in for running them.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / reference legs of
``bench.py`` may import this module, and only as a checker or a timed CPU baseline.  The
product path (``hydropol2d_b200``) never calls it.

MATLAB semantics that matter for bit-level agreement and are reproduced on purpose:

* ``max(a, b)`` / ``min(a, b)`` ignore NaN -> ``np.fmax`` / ``np.fmin`` (never np.maximum).
* element-wise expressions evaluate left to right, so ``a*b*c/d`` is ``((a*b)*c)/d``.
* ``x.^(7/3)`` is ``pow(x, 2.3333333333333335)`` (numpy power calls C pow).

Every function cites the reference file:line it follows (paths relative to the project).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

G = 9.81
EPS64 = float(np.finfo(np.float64).eps)


# --------------------------------------------------------------------------------------
# Inertial_Solver.m
# --------------------------------------------------------------------------------------
def inertial_solver(scheme: int, q_p: np.ndarray, dt: float, Hf: np.ndarray, S: np.ndarray,
                    n_sq: np.ndarray, dx: float) -> np.ndarray:
    """``q = Inertial_Solver(flag_numerical_scheme, q_p, dt, Hf, S, n_sq, dx, idx_nan)``.

    Pages are the leading axis: ``q_p``, ``Hf``, ``S`` are (3, ny, nx); ``n_sq`` (ny, nx)
    broadcasts over pages as MATLAB's implicit expansion does.
    Scheme 1 (Bates): Inertial_Solver.m:23-26.  Scheme 2 (s-upwind): :29-78.
    Scheme 3 (s-centred): :81-121.
    """
    with np.errstate(all="ignore"):
        den = 1 + G * dt * n_sq * np.abs(q_p) / (Hf ** (7 / 3))
        if scheme == 1:
            return (q_p - G * Hf * dt * S) / den
        ny, nx = n_sq.shape
        if scheme == 2:
            q_up = np.zeros_like(q_p)
            q_up_neg = np.zeros_like(q_p)
            neg = np.zeros(q_p.shape, dtype=bool)
            neg[0] = q_p[0] < 0
            neg[1] = q_p[1] < 0
            if nx > 2:
                q_up[0][:, 1:nx - 1] = q_p[0][:, 0:nx - 2]
                q_up_neg[0][:, 1:nx - 1] = q_p[0][:, 2:nx]
            if ny > 2:
                q_up[1][1:ny - 1, :] = q_p[1][0:ny - 2, :]
                q_up_neg[1][1:ny - 1, :] = q_p[1][2:ny, :]
            q_up[neg] = q_up_neg[neg]
            theta = 1 - dt / dx * np.fmin(np.abs(q_p) / Hf, np.sqrt(G * Hf))
            return (theta * q_p + (1 - theta) * q_up - G * Hf * dt * S) / den
        if scheme == 3:
            theta = 1 - dt / dx * np.fmin(np.abs(q_p) / Hf, np.sqrt(G * Hf))
            theta[np.isnan(theta)] = 1
            q_avg = np.zeros_like(q_p)
            if nx > 2:
                q_avg[0][:, 1:nx - 1] = 1 / 2 * (q_p[0][:, 0:nx - 2] + q_p[0][:, 2:nx])
            if ny > 2:
                q_avg[1][1:ny - 1, :] = 1 / 2 * (q_p[1][0:ny - 2, :] + q_p[1][2:ny, :])
            return (theta * q_p + (1 - theta) * q_avg - G * Hf * dt * S) / den
    raise ValueError(f"flag_numerical_scheme={scheme} is not 1, 2 or 3")


# --------------------------------------------------------------------------------------
# Local_Inertial_Model_D4.m (non-subgrid, non-reservoir branch)
# --------------------------------------------------------------------------------------
def coarse_draining_limiter(Q: np.ndarray, d_tot_mm: np.ndarray, dt: float,
                            cell_area: float) -> np.ndarray:
    """``apply_coarse_draining_limiter`` -- Local_Inertial_Model_D4.m:799-858."""
    Q = Q.copy()
    ny, nx = d_tot_mm.shape
    area = cell_area * np.ones((ny, nx))
    with np.errstate(all="ignore"):
        available = np.fmax(d_tot_mm / 1000, 0) * area / max(dt, EPS64)
        Qx = Q[0].copy()
        Qy = Q[1].copy()
        out_rate = np.zeros((ny, nx)) + np.fmax(Qx, 0)
        out_rate[:, 1:] = out_rate[:, 1:] + np.fmax(-Qx[:, :-1], 0)
        out_rate = out_rate + np.fmax(Qy, 0)
        out_rate[:-1, :] = out_rate[:-1, :] + np.fmax(-Qy[1:, :], 0)
        scale = np.ones((ny, nx))
        need = (out_rate > available) & (out_rate > 0)
        scale[need] = available[need] / out_rate[need]
        scale[~np.isfinite(scale)] = 0
        scale = np.fmax(np.fmin(scale, 1), 0)
    if nx > 1:
        sub = Qx[:, :nx - 1].copy()
        pos = sub > 0
        neg = sub < 0
        sub[pos] = sub[pos] * scale[:, :nx - 1][pos]
        sub[neg] = sub[neg] * scale[:, 1:nx][neg]
        Qx[:, :nx - 1] = sub
        Qx[:, nx - 1] = 0
    if ny > 1:
        sub = Qy[1:ny, :].copy()
        pos = sub > 0
        neg = sub < 0
        sub[pos] = sub[pos] * scale[1:ny, :][pos]
        sub[neg] = sub[neg] * scale[:ny - 1, :][neg]
        Qy[1:ny, :] = sub
        Qy[0, :] = 0
    Q[0] = Qx
    Q[1] = Qy
    Q[~np.isfinite(Q)] = 0
    return Q


@dataclass
class LIOutputs:
    qout_left: np.ndarray
    qout_right: np.ndarray
    qout_up: np.ndarray
    qout_down: np.ndarray
    outlet_flow: np.ndarray
    d_t: np.ndarray
    I_tot_end_cell: np.ndarray
    outflow: np.ndarray          # (3, ny, nx) mm/h
    Hf: np.ndarray               # (3, ny, nx) m


def reservoir_transfers(d_tot, vol_flux, rs: dict, time_step: float, cell_area: float):
    """Local_Inertial_Model_D4.m:318-344 line by line (after the volume flux :313, before
    d_t :390): structure ii drains (res_row, res_col) through k1 max(dtsup-h1,0)^k2 into
    ds1 and, when ds2 exists, through (k3, h2, k4) into ds2.  Cells are 0-based; a ds1/ds2
    row that is negative or NaN is the reference's NaN.  Kept as the reference has it: the
    reservoir cell's Vol_Flux GAINS each transfer, and the first transfer is added to ds1 a
    second time in the second structure's branch.  Returns the new (d_tot, vol_flux)."""
    d_tot = np.array(d_tot, dtype=np.float64)
    vol_flux = np.array(vol_flux, dtype=np.float64)
    dt_h = time_step / 60

    def none(v):
        return not (v >= 0)

    dtsup = None
    for ii in range(len(rs["res_row"])):
        r = (int(rs["res_row"][ii]), int(rs["res_col"][ii]))
        if not none(rs["ds1_row"][ii]):
            ds1 = (int(rs["ds1_row"][ii]), int(rs["ds1_col"][ii]))
            dtsup = d_tot[r] / 1000
            available_volume = 1000 * (np.fmax(dtsup - rs["h1"][ii], 0)) / dt_h
            dh = np.fmin(rs["k1"][ii] * (np.fmax(dtsup - rs["h1"][ii], 0)) ** rs["k2"][ii] / cell_area * 1000 * 3600,
                         available_volume) * dt_h
            vol_flux[r] = vol_flux[r] + dh / 1000 * cell_area
            dtsup = dtsup - dh / 1000
            d_tot[ds1] = d_tot[ds1] + dh
        else:
            dh = 0
        if not none(rs["ds2_row"][ii]):
            if none(rs["ds1_row"][ii]):
                raise IndexError("yds1 is NaN where yds2 is not (the reference's indexing fails)")
            ds1 = (int(rs["ds1_row"][ii]), int(rs["ds1_col"][ii]))
            ds2 = (int(rs["ds2_row"][ii]), int(rs["ds2_col"][ii]))
            d_tot[ds1] = d_tot[ds1] + dh
            available_volume = 1000 * (np.fmax(dtsup - rs["h2"][ii], 0)) / dt_h
            dh = np.fmin(rs["k3"][ii] * (np.fmax(dtsup - rs["h2"][ii], 0)) ** rs["k4"][ii] / cell_area * 1000 * 3600,
                         available_volume) * dt_h
            vol_flux[r] = vol_flux[r] + dh / 1000 * cell_area
            d_tot[ds2] = d_tot[ds2] + dh
    return d_tot, vol_flux


def local_inertial_model_d4(z, d_tot, roughness_cell, roughness_squared, cell_area, time_step,
                            resolution, outlet_rows, outlet_cols, outlet_type, slope_outlet,
                            outflow, flag_numerical_scheme=1, flag_critical=0,
                            h_min=0.0, reservoirs: dict | None = None) -> LIOutputs:
    """``Local_Inertial_Model_D4`` with ``flag_subgrid=0``; ``reservoirs`` (``flag_reservoir=1``)
    is the structure table of ``reservoir_transfers``.

    Follows Local_Inertial_Model_D4.m:31-44 (depth, WSE), :89-142 (slopes, face depths,
    closed N/E boundary faces), :184 (Hf>=0), :198-201 (q_prev, dt), :263-264 (solver,
    NaN->0), :272-275 (critical clip), :292-307 (10 m/s clip, draining limiter), :309,
    :313-315 (volume flux), :347-350 (per-direction outputs), :389-393 and :415
    (continuity, d_t>=0), :417-498 (outlet sink) and :512-514 (I_tot_end_cell).
    Arrays are (ny, nx); ``outflow`` is (3, ny, nx) in mm/h; ``time_step`` in minutes.
    """
    z = np.asarray(z, dtype=np.float64)
    ny, nx = z.shape
    res = float(resolution)
    with np.errstate(all="ignore"):
        depth_cell = np.fmax(d_tot / 1000, 0)
        y = z + depth_cell
        Sx = np.zeros((ny, nx))
        Sy = np.zeros((ny, nx))
        Hf_x = np.zeros((ny, nx))
        Hf_y = np.zeros((ny, nx))
        zf_x = np.fmax(z[:, :-1], z[:, 1:])
        zf_y = np.fmax(z[:-1, :], z[1:, :])
        Sx[:, :-1] = (y[:, 1:] - y[:, :-1]) / res
        Sx[:, -1] = 0
        Sy[1:, :] = (y[:-1, :] - y[1:, :]) / res
        Sy[0, :] = 0
        Hf_x[:, :-1] = np.fmax(np.fmax(y[:, :-1], y[:, 1:]) - zf_x, 0)
        Hf_y[1:, :] = np.fmax(np.fmax(y[:-1, :], y[1:, :]) - zf_y, 0)
        Hf_x[:, -1] = 0
        Hf_y[0, :] = 0
        S = np.zeros((3, ny, nx))
        S[0] = Sx
        S[1] = Sy
        Hf = np.zeros((3, ny, nx))
        Hf[0] = Hf_x
        Hf[1] = Hf_y
        Hf[Hf < 0] = 0
        q_prev = outflow / 1000 / 3600 * (res * res) / res
        dt = time_step * 60
        q = inertial_solver(flag_numerical_scheme, q_prev, dt, Hf, S, roughness_squared, res)
        q[~np.isfinite(q)] = 0
        if flag_critical == 1:
            crit = Hf * np.sqrt(9.81 * Hf)
            q = np.fmin(np.fmax(q, -crit), crit)
        thr = Hf * 10
        q = np.fmin(np.fmax(q, -thr), thr)
        rate = q * res
        rate = coarse_draining_limiter(rate, d_tot, dt, cell_area)
        out = rate / cell_area * 1000 * 3600
        zc = np.zeros((ny, 1))
        zr = np.zeros((1, nx))
        vol_flux = dt * (np.concatenate([zc, rate[0][:, :nx - 1]], axis=1) - rate[0]
                         - rate[1] + np.concatenate([rate[1][1:, :], zr], axis=0))
        qout_left = -np.concatenate([zc, out[0][:, :nx - 1]], axis=1)
        qout_right = out[0].copy()
        qout_up = out[1].copy()
        qout_down = -np.concatenate([out[1][1:, :], zr], axis=0)
        d_src = d_tot
        if reservoirs is not None:
            d_src, vol_flux = reservoir_transfers(d_tot, vol_flux, reservoirs, time_step, cell_area)
        d_t = d_src + 1000 * vol_flux / (res * res)
        d_t[d_t < 0] = 0
        outlet_flow = np.zeros((ny, nx))
        out[2] = 0
        Hf[2] = 0
        rows = np.asarray(outlet_rows, dtype=np.int64).ravel()
        cols = np.asarray(outlet_cols, dtype=np.int64).ravel()
        if rows.size:
            idx = (rows, cols)
            h_out = np.fmax(d_t[idx], 0) / 1000
            if outlet_type == 1:
                s = np.asarray(slope_outlet, dtype=np.float64)
                if s.ndim == 0:
                    sqrt_s = math.sqrt(abs(float(s))) * np.ones(h_out.shape)
                else:
                    sqrt_s = np.sqrt(np.abs(s[idx]))
            else:
                h_safe = np.fmax(h_out, 1e-12)
                sqrt_s = np.sqrt(9.81 * roughness_squared[idx] * h_safe ** (-1 / 3))
                sqrt_s[~np.isfinite(sqrt_s)] = 0
            Hf3 = Hf[2]
            Hf3[idx] = h_out
            q_out = (1 / roughness_cell[idx]) * res * h_out ** (5 / 3) * sqrt_s / cell_area * 1000 * 3600
            qmax = np.fmax(d_t[idx] - 1000 * h_min, 0) / (time_step / 60)
            q_out = np.fmin(q_out, qmax)
            q_out[~np.isfinite(q_out)] = 0
            outlet_flow[idx] = q_out
            out[2] = outlet_flow
            d_t[idx] = d_t[idx] - q_out * (time_step / 60)
        I_tot_end_cell = np.abs(out.sum(axis=0)) * dt / 1000 * 1 / 3600 * (res * res)
    return LIOutputs(qout_left, qout_right, qout_up, qout_down, outlet_flow, d_t,
                     I_tot_end_cell, out, Hf)


# --------------------------------------------------------------------------------------
# Green-Ampt at the Infiltration_Module boundary
# --------------------------------------------------------------------------------------
@dataclass
class GAParams:
    """Per-cell Green-Ampt maps (mm, mm/h, h), built from per-class tables."""
    ksat: np.ndarray         # mm/h
    psi: np.ndarray          # mm
    dtheta: np.ndarray       # -
    Lu: np.ndarray           # m (upper soil layer; HydroPol2D_preprocessing.m:2251-2252)
    k_out: np.ndarray        # mm/h (HydroPol2D_preprocessing.m:2253)
    Tr: np.ndarray           # h   (HydroPol2D_preprocessing.m:2250)
    min_sm: np.ndarray       # mm  (HydroPol2D_preprocessing.m:2387-2388)
    active: np.ndarray       # bool, False = no soil (impervious), no infiltration


def green_ampt_infiltration(d_t, I_t, T, time_step, p: GAParams, resolution):
    """Explicit Green-Ampt infiltration in the current driver's order (rain first).

    Capacity, recovery timer and soil-storage update follow
    HydroPol2D_Main_While_Ensemble.m:274-298 with the post-rain depth in place of d_p
    (the current Infiltration_Module sees the rain added by Snow_Module.m:99);
    supply rate and the surface-depth update follow Infiltration_Module.m:179 and
    :444-445.  Returns (d_t, I_t, T, f[mm/h]).
    """
    dt_h = time_step / 60
    A = resolution * resolution
    C_a = resolution * resolution
    with np.errstate(all="ignore"):
        i_a = d_t / max(dt_h, 1e-12)
        I_p = I_t
        C = p.ksat * (1 + ((d_t + p.psi) * p.dtheta) / I_p)
        non_c = I_p > p.Lu * 1000
        C = np.where(non_c, p.ksat, C)
        idx_C = i_a <= C
        T_new = T - time_step / 60
        T_new = np.where(i_a > C, p.Tr, T_new)
        idx_T = T_new < 0
        f = np.fmin(C, i_a)
        I_new = np.fmax(I_p + f * time_step / 60 - p.k_out * idx_C.astype(np.float64) * time_step / 60,
                        p.min_sm)
        I_new = np.where(idx_T, p.min_sm, I_new)
        f = np.where(p.active, f, 0.0)
        I_new = np.where(p.active, I_new, I_t)
        T_new = np.where(p.active, T_new, T)
        d_new = d_t - f * dt_h * A / C_a
        d_new[d_new < 0] = 0
    return d_new, I_new, T_new, f


# --------------------------------------------------------------------------------------
# Infiltration_Module.m, van Genuchten-Mualem single-layer branch
# --------------------------------------------------------------------------------------
@dataclass
class VGParams:
    """Per-cell van Genuchten maps (built from per-class tables) and the module's scalars."""
    theta_r: np.ndarray
    theta_sat: np.ndarray
    n_vg: np.ndarray
    alpha_vg: np.ndarray      # 1/m
    ksat: np.ndarray          # mm/h
    soil_depth: np.ndarray    # m
    active: np.ndarray        # False = impervious (LULC_Properties.idx_imp): no infiltration
    l_vg: float = 0.5
    Ltop: float = 0.05
    dh_max: float = 1.0
    Ksurf_weight: float = 0.5


def vg_water_table_depth(z, soil_depth, h_t):
    """Infiltration_Module.m:192-199: saturated thickness and depth to the water table."""
    GW_Depth = h_t - (z - soil_depth)
    return np.fmax(soil_depth - GW_Depth, 0)


def vg_infiltration(d_t, I_t, time_step, p: VGParams, zwt, resolution):
    """Infiltration_Module.m:143-473 (flag_infiltration = 1 of the current module, no layered
    soil, no subgrid): supply :179-182, unsaturated capacity :205-217, bucket head :262-276,
    top-layer wetting :281-302, Mualem conductivity :307-318, surface interface :321-333,
    Darcy capacity :336-342, limits :345-352, storage and depth updates :356-372.
    Depths and storage in mm, time_step in minutes.  Returns (d_t, I_t, f [mm/h])."""
    dt_h = time_step / 60
    C_a = resolution * resolution
    with np.errstate(all="ignore"):
        eff_depth = d_t
        i_a = eff_depth / max(dt_h, 1e-12)
        h0 = np.fmax(eff_depth, 0) / 1000
        UZ_max_storage = zwt * (p.theta_sat - p.theta_r)
        S = np.fmax(I_t, 0) / 1000
        S_rem = np.fmax(UZ_max_storage - S, 0)
        idx_noUZ = (zwt <= 0) | (UZ_max_storage <= 0)
        theta_r, theta_s, n, a = p.theta_r, p.theta_sat, p.n_vg, p.alpha_vg
        Ks = p.ksat / 1000 / 3600
        m = 1 - 1 / n
        ell = p.l_vg
        Ltop = max(p.Ltop, 1e-6)
        dh_max = p.dh_max
        Lmix = Ltop
        zwt_safe = np.fmax(zwt, 1e-6)
        theta_bucket = theta_r + (S / zwt_safe)
        theta_bucket = np.fmax(theta_bucket, theta_r)
        theta_bucket = np.fmin(theta_bucket, theta_s)
        Se_bucket = (theta_bucket - theta_r) / np.fmax(theta_s - theta_r, 1e-12)
        Se_bucket = np.fmin(np.fmax(Se_bucket, 1e-6), 1)
        h_bucket = -(1 / a) * ((Se_bucket ** (-1 / m) - 1) ** (1 / n))
        h_bucket = np.where(Se_bucket >= 0.999999, 0.0, h_bucket)
        w_avail = np.fmax(eff_depth, 0) / 1000
        w_top_deficit = Lmix * np.fmax(theta_s - theta_bucket, 0)
        w_wet = np.fmin(w_avail, S_rem)
        w_wet = np.fmin(w_wet, w_top_deficit)
        w_wet = np.fmax(w_wet, 0)
        theta_top = theta_bucket + w_wet / Lmix
        theta_top = np.fmax(theta_top, theta_r)
        theta_top = np.fmin(theta_top, theta_s)
        Se_top = (theta_top - theta_r) / np.fmax(theta_s - theta_r, 1e-12)
        Se_top = np.fmin(np.fmax(Se_top, 1e-6), 1)
        term_top = 1 - Se_top ** (1 / m)
        term_top = np.fmin(np.fmax(term_top, 0), 1)
        Kr_top = Se_top ** ell * (1 - term_top ** m) ** 2
        Kr_top = np.fmin(np.fmax(Kr_top, 0), 1)
        Ktop = Ks * Kr_top
        Ksurf = Ks + np.zeros_like(Ktop)
        wK = min(max(p.Ksurf_weight, 0), 1)
        idx_wet_boundary = (i_a > 0) | (h0 > 0)
        Ksoil = np.where(idx_wet_boundary, wK * Ksurf + (1 - wK) * Ktop, Ktop)
        Ksoil = np.fmin(np.fmax(Ksoil, 0), Ksurf)
        dh = h0 - h_bucket
        dh = np.fmax(dh, 0)
        dh = np.fmin(dh, dh_max)
        grad = (dh / Ltop) + 1
        C = Ksoil * grad
        C = C * 1000 * 3600
        f_store_lim = (S_rem * 1000) / max(dt_h, 1e-12)
        f = np.fmin(i_a, C)
        f = np.fmin(f, f_store_lim)
        f = np.where(p.active, f, 0.0)
        f = np.where(idx_noUZ, 0.0, f)
        f = np.where(np.isnan(f), 0.0, f)
        f = np.fmax(f, 0)
        inf_volume_cell = f * dt_h
        I_new = I_t + inf_volume_cell
        I_new = np.fmin(I_new, UZ_max_storage * 1000)
        I_new = np.fmax(I_new, 0)
        I_new = np.where(p.active, I_new, I_t)
        d_new = d_t - inf_volume_cell * (resolution * resolution) / C_a
        d_new[d_new < 0] = 0
    return d_new, I_new, f


# --------------------------------------------------------------------------------------
# refreshing_timestep.m (inertial D4 branch)
# --------------------------------------------------------------------------------------
@dataclass
class CFLResult:
    time_calculation_routing: float   # s
    time_step: float                  # min
    max_velocity: float
    dt_adv: float
    dt_wave: float
    unstable: bool
    velocity_raster: np.ndarray | None = None   # max |face velocity| per cell [m/s] (:109-111)


def refreshing_timestep(Hf, qout_right, qout_up, resolution, depth_tolerance, alfa_min,
                        alfa_max, max_time_step, min_time_step, time_step_increments,
                        flag_timestep=1, flag_adaptive_timestepping=1) -> CFLResult:
    """refreshing_timestep.m:61-89, :94-134, :139-150, :181-242, :315-359 (D4, not CA)."""
    res = float(resolution)
    ny, nx = qout_right.shape
    with np.errstate(all="ignore"):
        flow_depth = Hf * 1000
        depth_ts = np.fmax.reduce(flow_depth / 1000, axis=0)
        safe = flow_depth.copy()
        safe[safe < depth_tolerance] = 1e12
        vel_right = (qout_right / 1000 / 3600) * res / (safe[0] / 1000)
        vel_left = -np.concatenate([np.zeros((ny, 1)), vel_right[:, 1:]], axis=1)
        vel_up = (qout_up / 1000 / 3600) * res / (safe[1] / 1000)
        vel_down = -np.concatenate([vel_up[1:, :], np.zeros((1, nx))], axis=0)
        raster = np.fmax(np.abs(vel_left), np.abs(vel_right))
        raster = np.fmax(raster, np.abs(vel_up))
        raster = np.fmax(raster, np.abs(vel_down))
        rc = 0.5 * (vel_right - vel_left)
        uc = 0.5 * (vel_up - vel_down)
        total = np.hypot(rc, uc)
        stagnant = total < 0.01
        max_velocity = float(np.fmax.reduce(total, axis=None))
        if max_velocity > 0:
            dt_adv = 1 * res / max(max_velocity, 1e-10)
            tsf = max(alfa_max - 2 * max(max_velocity - 5, 0), alfa_min)
            dt_adv = dt_adv * tsf
            dt_adv = float(min(dt_adv, max_time_step))
        else:
            dt_adv = max_time_step
        wc = np.sqrt(9.81 * np.fmax(depth_ts, 0))
        wc = np.fmax(wc, 1e-10)
        wc[np.isinf(wc)] = np.nan
        wc[stagnant] = np.nan
        if flag_adaptive_timestepping == 1:
            cand = alfa_min * res / wc
        else:
            cand = alfa_min * res / (raster + wc)
        dt_wave = float(np.nanmin(cand)) if np.any(~np.isnan(cand)) else math.nan
    if math.isnan(dt_wave):
        dt_wave = max_time_step
    new = min(dt_adv, dt_wave) if flag_timestep == 1 else dt_wave
    if math.isnan(new) or math.isinf(new):
        new = max_time_step
    tcr = max(time_step_increments * math.floor(new / time_step_increments), min_time_step)
    tcr = min(tcr, max_time_step)
    return CFLResult(tcr, tcr / 60, max_velocity, dt_adv, dt_wave, tcr == min_time_step, raster)


# --------------------------------------------------------------------------------------
# Hydrological_Model.m + HydroPol2D_Main_While.m loop (the full step)
# --------------------------------------------------------------------------------------
@dataclass
class RunConfig:
    """Inputs of one surface-flow run (units as the reference: m, mm, mm/h, s, min)."""
    z: np.ndarray
    roughness: np.ndarray
    resolution: float
    outlet_rows: np.ndarray
    outlet_cols: np.ndarray
    outlet_type: int = 1
    slope_outlet: float = 0.0
    d0: np.ndarray | None = None            # mm
    routing_time: float = 60.0              # min
    min_time_step: float = 0.01             # s
    max_time_step: float = 10.0             # s
    time_step_increments: float = 0.001     # s
    time_step_change: float = 0.0001        # s
    alfa_min: float = 0.5
    alfa_max: float = 0.5
    depth_tolerance: float = 1.0            # mm (CA_States.depth_tolerance)
    flag_timestep: int = 1
    flag_adaptive_timestepping: int = 1
    flag_critical: int = 0
    flag_numerical_scheme: int = 1
    arrival_threshold_mm: float = 10.0
    # rain: either uniform piecewise-constant series or 2-D rate maps (mm/h)
    rain_times_min: np.ndarray | None = None    # start time of each interval
    rain_rates_mmh: np.ndarray | None = None    # uniform rate per interval
    rain_maps_mmh: np.ndarray | None = None     # (n_maps, my, mx) coarse fields
    rain_map_dt_min: float = 5.0
    ga: GAParams | None = None
    I0: np.ndarray | None = None                # mm
    # inflow hydrographs: start-stamped times [min], rates (n_times, n_gauges) [mm/h] and
    # Wshed_Properties.inflow_cells as (n_gauges, ny, nx) 0/1 masks
    inflow_times_min: np.ndarray | None = None
    inflow_rates_mmh: np.ndarray | None = None
    inflow_cells: np.ndarray | None = None
    # stage hydrographs: start-stamped times [min], water depths (n_times, n_gauges) [m] and
    # Wshed_Properties.stage_mask as (n_gauges, ny, nx) 0/1 masks
    stage_times_min: np.ndarray | None = None
    stage_depth_m: np.ndarray | None = None
    stage_cells: np.ndarray | None = None
    # reservoir / control structures (flag_reservoir = 1): the table of reservoir_transfers
    reservoirs: dict | None = None
    # velocities.vmax_final / hazardmax_final of save_output_maps.m:588-604
    hazard_maps: bool = False
    fixed_time_step_s: float | None = None      # bypass refreshing_timestep


def bilinear_rain(field: np.ndarray, ny: int, nx: int, dtype=np.float64) -> np.ndarray:
    """Cell-centred bilinear interpolation of a coarse (my, mx) rate field to (ny, nx).

    Grid cell (i, j) samples the field at fy = (i+0.5)*my/ny - 0.5, fx likewise, clamped
    to the field's extent.  Shared definition with the CUDA rain sampler.
    """
    my, mx = field.shape
    f = field.astype(dtype)
    one = dtype(1)
    half = dtype(0.5)
    fy = (np.arange(ny, dtype=dtype) + half) * dtype(my / ny) - half
    fx = (np.arange(nx, dtype=dtype) + half) * dtype(mx / nx) - half
    fy = np.fmin(np.fmax(fy, dtype(0)), dtype(my - 1))
    fx = np.fmin(np.fmax(fx, dtype(0)), dtype(mx - 1))
    iy0 = np.floor(fy).astype(np.int64)
    ix0 = np.floor(fx).astype(np.int64)
    iy1 = np.minimum(iy0 + 1, my - 1)
    ix1 = np.minimum(ix0 + 1, mx - 1)
    wy = (fy - iy0.astype(dtype))[:, None]
    wx = (fx - ix0.astype(dtype))[None, :]
    f00 = f[iy0][:, ix0]
    f01 = f[iy0][:, ix1]
    f10 = f[iy1][:, ix0]
    f11 = f[iy1][:, ix1]
    top = (one - wx) * f00 + wx * f01
    bot = (one - wx) * f10 + wx * f11
    return ((one - wy) * top + wy * bot).astype(dtype)


def average_rate_over_step(times_end, values, t0: float, t1: float) -> float:
    """``localAverageRateOverStep`` (update_spatial_BC.m:1131-1184): the exact time average
    over [t0, t1] of an END-stamped piecewise-constant series -- value i holds from
    times_end[i-1] (times_end[0] minus the series' spacing for i = 0) up to times_end[i] and
    nothing after the last end; non-finite values contribute nothing.  0 when t1 <= t0."""
    times = np.asarray(times_end, dtype=np.float64)
    vals = np.asarray(values, dtype=np.float64)
    n = min(len(times), len(vals))
    if n == 0 or not (np.isfinite(t0) and np.isfinite(t1)) or t1 <= t0:
        return 0.0
    dt_force = times[1] - times[0] if n >= 2 else 0.0   # localEstimateConstantDt, :1240-1253
    if not np.isfinite(dt_force) or dt_force <= 0:
        dt_force = 0.0
    acc = 0.0
    for i in range(n):
        ts = times[0] - dt_force if i == 0 else times[i - 1]
        ov = max(0.0, min(t1, times[i]) - max(t0, ts))
        if ov > 0 and np.isfinite(vals[i]):
            acc += vals[i] * ov
        if times[i] >= t1:
            break
    return acc / (t1 - t0)


def advance_end_stamped_cursor(times, t_now: float, cursor: int) -> int:
    """localAdvanceEndStampedCursor (update_spatial_BC.m:1095-1129), 1-based as in MATLAB."""
    n = len(times)
    cursor = min(max(1, cursor), n)
    while cursor < n and t_now > times[cursor - 1]:
        cursor += 1
    return cursor


def average_input_rain_map_over_step(times_end, maps, t0: float, t1: float, cursor: int = 1,
                                     dt_force: float | None = None):
    """localAverageInputRainMapOverStep (update_spatial_BC.m:1287-1359) on maps already read and
    aligned ((n, ny, nx) [mm/h]): the time-averaged rate map over [t0, t1] and the new cursor.
    Map i holds from times_end[i-1] (times_end[0] - dt_force for the first) to times_end[i];
    dt_force defaults to localEstimateConstantDt (:1240-1253)."""
    times = np.asarray(times_end, dtype=np.float64)
    maps = np.asarray(maps, dtype=np.float64)
    zero = np.zeros(maps.shape[1:])
    if times.size == 0 or t1 <= t0:
        return zero, cursor
    dt_total = t1 - t0
    cursor = advance_end_stamped_cursor(times, t0, cursor)
    if dt_force is None:
        dt_force = times[1] - times[0] if times.size >= 2 else 0.0
        if not np.isfinite(dt_force) or dt_force <= 0:
            dt_force = 0.0
    ts = times[0] - dt_force if cursor == 1 else times[cursor - 2]
    te = times[cursor - 1]
    if t0 >= ts and t1 <= te:   # fast path: the step inside one forcing interval
        return maps[cursor - 1].copy(), cursor
    acc = zero.copy()
    for i in range(cursor, times.size + 1):
        ts = times[0] - dt_force if i == 1 else times[i - 2]
        te = times[i - 1]
        ov = max(0.0, min(t1, te) - max(t0, ts))
        if ov > 0:
            acc = acc + ov * maps[i - 1]
        if te >= t1:
            cursor = i
            break
    return acc / dt_total, cursor


def idw_rain_maps(x_gauge, y_gauge, rates, ny: int, nx: int, res: float, x_ul: float = 0.0,
                  y_ul: float = 0.0) -> np.ndarray:
    """Rainfall_Interpolator.m + idw_function.m (p = 2, Euclidean norm, no radius) for every
    record interval: (n_times, ny, nx) float32 maps [mm/h].  Cell (i, j) at
    (x_ul + res (j+1), y_ul - res (i+1)) (HydroPol2D_preprocessing.m:2420-2421); gauges with a
    NaN record are left out of that interval (update_spatial_BC.m:875-885), an interval without
    gauges is dry; the distance's square root and the gauge sums in order, in FP64."""
    xg = np.asarray(x_gauge, dtype=np.float64)
    yg = np.asarray(y_gauge, dtype=np.float64)
    r = np.asarray(rates, dtype=np.float64).reshape(-1, xg.size)
    X = x_ul + res * (np.arange(nx, dtype=np.float64) + 1.0)[None, :]
    Y = y_ul - res * (np.arange(ny, dtype=np.float64) + 1.0)[:, None]
    out = np.zeros((r.shape[0], ny, nx), dtype=np.float32)
    w = []
    for g in range(xg.size):
        dx = np.abs(X - xg[g])
        dy = np.abs(Y - yg[g])
        d = np.sqrt(dx * dx + dy * dy)
        d[d == 0] = np.finfo(np.float64).eps
        w.append(1.0 / (d * d))
    for m in range(r.shape[0]):
        num = np.zeros((ny, nx))
        den = np.zeros((ny, nx))
        for g in range(xg.size):
            if np.isnan(r[m, g]):
                continue
            num = num + w[g] * r[m, g]
            den = den + w[g]
        out[m] = np.where(den > 0, num / np.where(den > 0, den, 1.0), 0.0).astype(np.float32)
    return out


def rain_depth_mm(cfg: RunConfig, t0: float, t1: float, ny: int, nx: int):
    """Rain depth [mm] a step receives from the clock interval [t0, t1] [min]: the exact
    integral of the piecewise-constant rate over the interval / 60, which is what
    update_spatial_BC.m:435-470 (uniform series: average rate x interval / 60) and :536-558
    with :1287-1359 (rate maps: time-weighted map average x interval / 60) give.  The uniform
    series here is START-stamped -- rate q holds from times[q] up to times[q+1], the last one
    for ever -- and map m holds over [m, m+1) x map_dt and nothing after the last map
    (an end-stamped series converts by prepending its first start and appending a zero).
    Scalar for a uniform series, (ny, nx) for maps."""
    if t1 <= t0:
        return 0.0 if cfg.rain_maps_mmh is None else np.zeros((ny, nx))
    if cfg.rain_maps_mmh is not None:
        acc = np.zeros((ny, nx))
        dtm = cfg.rain_map_dt_min
        for m in range(cfg.rain_maps_mmh.shape[0]):
            ov = max(0.0, min(t1, (m + 1) * dtm) - max(t0, m * dtm))
            if ov > 0:
                acc = acc + ov * bilinear_rain(cfg.rain_maps_mmh[m], ny, nx)
        return acc / 60.0
    if cfg.rain_rates_mmh is None:
        return 0.0
    times = np.asarray(cfg.rain_times_min, dtype=np.float64)
    rates = np.asarray(cfg.rain_rates_mmh, dtype=np.float64)
    acc = 0.0
    for q in range(len(rates)):
        hi = times[q + 1] if q + 1 < len(times) else np.inf
        ov = max(0.0, min(t1, hi) - max(t0, times[q]))
        if ov > 0 and np.isfinite(rates[q]):
            acc += rates[q] * ov
    return acc / 60.0


def inflow_depth_mm(cfg: RunConfig, t0: float, t1: float) -> np.ndarray:
    """BC_States.inflow [mm] of update_spatial_BC.m:359-395: per gauge z the exact integral of
    its rate over [t0, t1] / 60 (delta_inflow_agg), spread over inflow_cells(:,:,z) and summed
    over gauges; NaN on idx_nan cells."""
    masks = np.asarray(cfg.inflow_cells, dtype=np.float64)
    times = np.asarray(cfg.inflow_times_min, dtype=np.float64)
    rates = np.asarray(cfg.inflow_rates_mmh, dtype=np.float64).reshape(times.size, -1)
    out = np.zeros(masks.shape[1:])
    if t1 > t0:
        for z in range(masks.shape[0]):
            acc = 0.0
            for q in range(times.size):
                hi = times[q + 1] if q + 1 < times.size else np.inf
                ov = max(0.0, min(t1, hi) - max(t0, times[q]))
                if ov > 0 and np.isfinite(rates[q, z]):
                    acc += rates[q, z] * ov
            out = out + acc / 60.0 * masks[z]
    out[np.isnan(cfg.z)] = np.nan
    return out


def next_rain_interval(a: float, b: float, t_previous: float, t: float, k: int, tcr_s: float):
    """The loop's bookkeeping of the rain interval.  At the end of iteration k (clock t, the
    end of step k) update_spatial_BC computes the depth the NEXT step applies over
    [t_previous, t] (HydroPol2D_Main_While.m:721); then t_previous becomes the clock
    increment on the first iteration and t after that (:734-738) and the clock advances by
    the new step (:779).  Returns the next step's (a, b) and the new t_previous."""
    return t_previous, t, (tcr_s / 60.0 if k == 1 else t)


@dataclass
class RunState:
    d: np.ndarray
    outflow: np.ndarray
    I: np.ndarray | None
    T: np.ndarray | None
    dmax: np.ndarray
    arrival: np.ndarray
    t: float
    k: int
    time_step: float
    time_save_previous: float = 0.0
    neg_warnings: int = 0
    unstable_steps: int = 0
    rain_volume: float = 0.0
    infiltration_volume: float = 0.0
    outlet_volume: float = 0.0
    inflow_volume: float = 0.0
    stage_volume: float = 0.0
    structure_volume: float = 0.0
    velocity_raster: np.ndarray | None = None    # of the last velocity refresh
    vmax_final: np.ndarray | None = None
    hazardmax_final: np.ndarray | None = None
    # rain interval [rain_a, rain_b] of the current step and the loop's t_previous [min]; the
    # first step's comes from the call before the loop (HydroPol2D_Main_While.m:115) with
    # t_previous = 0 (:120)
    rain_a: float = 0.0
    rain_b: float = 0.0
    t_previous: float = 0.0
    history: list = field(default_factory=list)


def velocity_hazard_snapshot(velocity_raster, depth_mm, idx_nan) -> np.ndarray:
    """snisb_velocity_hazard_snapshot (save_output_maps.m:832-848), the hazard output: depth [m]
    x velocity [m/s], 0 below 0.01 m and where non-finite, NaN on idx_nan cells."""
    depth_m = np.fmax(np.asarray(depth_mm, dtype=np.float64) / 1000, 0)
    v = np.array(velocity_raster, dtype=np.float64) + np.zeros(depth_m.shape)
    v[~np.isfinite(v)] = 0
    hazard = depth_m * v
    hazard[depth_m < 0.01] = 0
    hazard[~np.isfinite(hazard)] = 0
    hazard[idx_nan] = np.nan
    return hazard


def init_state(cfg: RunConfig) -> RunState:
    ny, nx = cfg.z.shape
    d = np.zeros((ny, nx)) if cfg.d0 is None else np.array(cfg.d0, dtype=np.float64)
    I = None if cfg.ga is None else np.array(cfg.I0, dtype=np.float64)
    # recovery timer starts at Tr (HydroPol2D_Main_While_Ensemble.m:266)
    T = None if cfg.ga is None else np.where(cfg.ga.active, cfg.ga.Tr, 0.0).astype(np.float64)
    ts = (cfg.fixed_time_step_s if cfg.fixed_time_step_s else cfg.min_time_step) / 60
    return RunState(d=d, outflow=np.zeros((3, ny, nx)), I=I, T=T,
                    dmax=np.full((ny, nx), -np.inf), arrival=np.full((ny, nx), np.inf),
                    t=cfg.min_time_step / 60, k=1, time_step=ts,
                    rain_a=0.0, rain_b=cfg.min_time_step / 60, t_previous=0.0)


def step(cfg: RunConfig, st: RunState) -> None:
    """One accepted step of HydroPol2D_Main_While.m:403-782 with the path's modules."""
    ny, nx = cfg.z.shape
    res = cfg.resolution
    A = res * res
    time_step = st.time_step
    # Hydrological_Model.m:14-55; rain via interception_module.m:68 + Snow_Module.m:99
    # the depth update_spatial_BC computed for this step at the end of the previous one
    delta_p = rain_depth_mm(cfg, st.rain_a, st.rain_b, ny, nx)
    d_t = st.d + delta_p
    st.rain_volume += float(np.nansum(np.broadcast_to(delta_p, (ny, nx)))) * A / 1000
    if cfg.ga is not None:
        d_t, st.I, st.T, f = green_ampt_infiltration(d_t, st.I, st.T, time_step, cfg.ga, res)
        st.infiltration_volume += float(np.nansum(f * (time_step / 60))) * A / 1000
    if cfg.inflow_cells is not None:   # Hydrological_Model.m:27-28, after the infiltration
        inflow = inflow_depth_mm(cfg, st.rain_a, st.rain_b)
        d_t = d_t + inflow
        st.inflow_volume += float(np.nansum(inflow)) * A / 1000
    if np.nanmin(d_t) < -1e-8:
        st.neg_warnings += 1
    else:
        d_t[d_t < 1e-6] = 0
    d_t[d_t < 0] = 0
    d_tot = d_t
    n = cfg.roughness
    out = local_inertial_model_d4(cfg.z, d_tot, n, n * n, A, time_step, res, cfg.outlet_rows,
                                  cfg.outlet_cols, cfg.outlet_type, cfg.slope_outlet, st.outflow,
                                  cfg.flag_numerical_scheme, cfg.flag_critical, reservoirs=cfg.reservoirs)
    if cfg.reservoirs is not None:   # what the transfers added: d_t + outlet water - (d_tot + fluxes)
        d_plain, vf = reservoir_transfers(d_tot, np.zeros_like(d_tot), cfg.reservoirs, time_step, A)
        st.structure_volume += (float(np.sum(d_plain - d_tot)) + float(np.sum(vf)) * 1000 / A) * A / 1000
    st.outlet_volume += float(np.nansum(out.outlet_flow)) * (time_step / 60) / 1000 * A
    # HydroPol2D_Main_While.m:691-705 (time_save gate) + refreshing_timestep.m
    if cfg.fixed_time_step_s:
        tcr = cfg.fixed_time_step_s
        cfl = None
    else:
        pos_save = math.ceil((st.t * 60) / cfg.time_step_change)
        time_save = (pos_save - 1) * cfg.time_step_change / 60
        delta = time_save - st.time_save_previous
        st.time_save_previous = time_save
        if delta > 0 or st.k == 1:
            cfl = refreshing_timestep(out.Hf, out.qout_right, out.qout_up, res,
                                      cfg.depth_tolerance, cfg.alfa_min, cfg.alfa_max,
                                      cfg.max_time_step, cfg.min_time_step,
                                      cfg.time_step_increments, cfg.flag_timestep,
                                      cfg.flag_adaptive_timestepping)
            tcr = cfl.time_calculation_routing
            st.unstable_steps += int(cfl.unstable)
        else:
            tcr = time_step * 60
            cfl = None
    # update_spatial_BC.m:316-357: stage cells take the gauge's depth at the clock t
    if cfg.stage_cells is not None:
        times = np.asarray(cfg.stage_times_min, dtype=np.float64)
        depth = np.asarray(cfg.stage_depth_m, dtype=np.float64).reshape(times.size, -1)
        hit = np.nonzero(times <= st.t)[0]
        z2 = int(hit[-1]) if hit.size else 0
        before = out.d_t.copy()
        for i in range(depth.shape[1]):
            out.d_t[np.asarray(cfg.stage_cells[i], dtype=bool)] = 1000.0 * depth[z2, i]
        st.stage_volume += float(np.nansum(out.d_t - before)) * A / 1000
    if cfg.hazard_maps:   # save_output_maps.m:588-604 with snisb_velocity_hazard_snapshot (:832-848)
        if cfl is not None:
            st.velocity_raster = cfl.velocity_raster
        hazard = velocity_hazard_snapshot(st.velocity_raster, out.d_t, np.isnan(cfg.z))
        if st.k == 1:
            st.vmax_final = np.array(st.velocity_raster, dtype=np.float64)
            st.hazardmax_final = hazard
        else:
            st.vmax_final = np.fmax(st.velocity_raster, st.vmax_final)
            st.hazardmax_final = np.fmax(hazard, st.hazardmax_final)
            st.hazardmax_final[np.isnan(hazard) & np.isnan(st.hazardmax_final)] = np.nan
    # save_output_maps.m:588-600 (running maximum depth) + arrival-time definition
    t_end_s = st.t * 60 + time_step * 60
    newly = (st.dmax < cfg.arrival_threshold_mm) & (out.d_t >= cfg.arrival_threshold_mm)
    st.arrival[newly] = t_end_s
    st.dmax = out.d_t.copy() if st.k == 1 else np.fmax(out.d_t, st.dmax)
    st.history.append((st.t, time_step, None if cfl is None else cfl.max_velocity))
    # HydroPol2D_Main_While.m:766-782 (state carry, clock by the new dt)
    st.d = out.d_t
    st.outflow = out.outflow
    st.rain_a, st.rain_b, st.t_previous = next_rain_interval(st.rain_a, st.rain_b, st.t_previous, st.t,
                                                             st.k, tcr)
    st.time_step = tcr / 60
    st.t = tcr / 60 + st.t
    st.k += 1
    st.last = out


def run(cfg: RunConfig, max_steps: int | None = None) -> RunState:
    st = init_state(cfg)
    while st.t <= cfg.routing_time + cfg.min_time_step / 60:
        if max_steps is not None and st.k > max_steps:
            break
        step(cfg, st)
    return st
