"""The reference's MATLAB entry points of the surface-flow step, by name and argument order,
over the C ABI.

MATLAB's layout is kept at this edge: grids are (ny, nx) arrays, page arrays such as
``outflow`` and ``Hf`` are (ny, nx, 3), outlet rows and columns are 1-based, and units are
the reference's (depth mm, flux mm/h, time step min, elevation m).  Every call runs on the
GPU through ``libhp2d.so``; there is no CPU path, so a missing library or device raises.

* ``Local_Inertial_Model_D4`` -- Local_Inertial_Model_D4.m:1-5, non-subgrid branch, schemes 1-3
  (Inertial_Solver.m:19-121).  Stateless: each call uploads z, roughness and the outlets to a
  cached context of the grid's shape, sets d_tot and outflow, runs ``hp2d_li_step`` and reads
  the outputs back.
* ``refreshing_timestep`` -- the refresh branch of the refreshing_timestep.m script
  (:61-89, :94-187, :205-242, :315-359), as a function of the workspace values the script
  reads, through ``hp2d_cfl_dt_noalloc`` (FP32 face arrays on the device).
* The Infiltration_Module script keeps its state (I_t and the recovery timer) in the
  caller's workspace between steps; here that workspace is a resident ``SurfaceFlow``
  context, whose ``hydrology_step`` is the script's drop-in.

Flags the build does not implement (``flag_subgrid = 1``, ``flag_reservoir`` other than 0/1,
``flag_numerical_scheme`` outside 1-3) raise ``HP2DError`` with ``HP2D_UNSUPPORTED_FLAG``, as the
C ABI does.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .surface import SurfaceFlow

_sessions: dict = {}


def _session(ny, nx, resolution, precision, params_key, params) -> SurfaceFlow:
    key = (ny, nx, float(resolution), precision, params_key)
    s = _sessions.get(key)
    if s is None:
        if len(_sessions) >= 4:
            for old in list(_sessions.values()):
                old.close()
            _sessions.clear()
        s = SurfaceFlow(ny, nx, resolution, precision, params=params)
        _sessions[key] = s
    return s


def close_sessions() -> None:
    """Frees the cached contexts (device memory) the stateless calls keep."""
    for s in _sessions.values():
        s.close()
    _sessions.clear()


def _outlets(row_outlet, col_outlet, ny, nx):
    rows = np.asarray(row_outlet if row_outlet is not None else [], dtype=np.int64).ravel()
    cols = np.asarray(col_outlet if col_outlet is not None else [], dtype=np.int64).ravel()
    if rows.size != cols.size:
        raise ValueError("row_outlet and col_outlet must have the same length")
    if rows.size and (rows.min() < 1 or rows.max() > ny or cols.min() < 1 or cols.max() > nx):
        raise ValueError("outlet rows/columns are 1-based and must lie inside the grid")
    return rows - 1, cols - 1


def Local_Inertial_Model_D4(flag_numerical_scheme, reservoir_x, reservoir_y, k1, h1, k2, k3, h2,
                            k4, yds1, xds1, yds2, xds2, flag_reservoir, z, d_tot, d_p,
                            roughness_cell, roughness_squared, cell_area, time_step, Resolution,
                            outlet_index, outlet_type, slope_outlet, row_outlet, col_outlet,
                            d_tolerance, outflow, idx_nan, flag_critical, flag_subgrid, nc, nf,
                            River_Width, River_Depth, Qc_prev, Qf_prev, Qci_prev, Qfi_prev,
                            C_a_prev, Subgrid_Properties, flag_overbanks, flag_inflow,
                            SubgridTables, *, precision: str = "fp64"):
    """``[qout_left, qout_right, qout_up, qout_down, outlet_flow, d_t, I_tot_end_cell, outflow,
    Hf, Qc, Qf, Qci, Qfi, C_a] = Local_Inertial_Model_D4(...)`` (Local_Inertial_Model_D4.m:1-5).

    With ``flag_reservoir = 1`` the reservoir tables (1-based cells, NaN for no downstream
    cell) drive the control-structure transfers (Local_Inertial_Model_D4.m:318-344).
    Arguments the non-subgrid branch never reads (d_p,
    outlet_index, d_tolerance, idx_nan, the subgrid inputs) are accepted and ignored, as in
    the reference (idx_nan is an unused argument of Inertial_Solver, in every scheme).  ``roughness_squared``
    must equal ``roughness_cell.^2`` and ``cell_area`` must be ``Resolution^2``: the library
    derives both from ``roughness_cell`` and ``Resolution``.  ``slope_outlet`` is a scalar or
    an (ny, nx) map sampled at the outlets (outlet_type 1).  ``precision`` selects the FP64
    (default, the reference's) or FP32 build.
    """
    if int(flag_subgrid) != 0 or int(flag_reservoir) not in (0, 1) or int(flag_numerical_scheme) not in (1, 2, 3):
        # the C ABI rejects these; raise the same error before touching the device
        raise _abi.HP2DError(2, "flag_subgrid = 1, flag_reservoir outside 0/1 and schemes other than 1-3 "
                                "are not implemented by this build")
    z = np.asarray(z, dtype=np.float64)
    if z.ndim != 2:
        raise ValueError("z must be an (ny, nx) array")
    ny, nx = z.shape
    res = float(Resolution)
    if not np.isclose(float(np.asarray(cell_area).ravel()[0]), res * res, rtol=1e-12, atol=0) or \
            np.asarray(cell_area).size != 1:
        raise ValueError("cell_area must be the scalar Resolution^2 outside the subgrid branch")
    n = np.broadcast_to(np.asarray(roughness_cell, dtype=np.float64), (ny, nx))
    n2 = np.broadcast_to(np.asarray(roughness_squared, dtype=np.float64), (ny, nx))
    fin = np.isfinite(n2) & np.isfinite(n)
    if not np.allclose(n2[fin], n[fin] * n[fin], rtol=1e-12, atol=0):
        raise ValueError("roughness_squared must equal roughness_cell.^2")
    rows, cols = _outlets(row_outlet, col_outlet, ny, nx)
    s = np.asarray(slope_outlet, dtype=np.float64)
    per_outlet = None
    scalar_slope = 0.0
    if s.ndim == 0 or s.size == 1:
        scalar_slope = float(s.ravel()[0])
    else:
        per_outlet = np.broadcast_to(s, (ny, nx))[rows, cols]
    params = _abi.default_params(outlet_type=int(outlet_type), slope_outlet=scalar_slope,
                                 flag_critical=int(flag_critical), flag_reservoir=int(flag_reservoir),
                                 flag_numerical_scheme=int(flag_numerical_scheme))
    pkey = (int(outlet_type), scalar_slope, int(flag_critical), int(flag_reservoir), int(flag_numerical_scheme))
    g = _session(ny, nx, res, precision, pkey, params)
    g.upload_static(z, n, rows, cols, per_outlet)
    if int(flag_reservoir) == 1:   # 1-based (x = column, y = row); NaN: no downstream cell
        def idx(v):
            a = np.asarray(v, dtype=np.float64).ravel()
            return np.where(np.isfinite(a), a - 1, -1).astype(np.int32)
        g.set_reservoirs(idx(reservoir_y), idx(reservoir_x), k1, h1, k2, idx(yds1), idx(xds1), k3, h2, k4,
                         idx(yds2), idx(xds2))
    of = np.asarray(outflow, dtype=np.float64)
    if of.shape != (ny, nx, 3) and of.shape != (ny, nx, 2):
        raise ValueError("outflow must be (ny, nx, 3) pages [mm/h]")
    pages = np.ascontiguousarray(np.moveaxis(of[:, :, :2], 2, 0))
    g.set_state(np.asarray(d_tot, dtype=np.float64), pages)
    g.li_step(float(time_step))
    d_t = g.download("depth")
    q_r = g.download("qout_right")
    q_u = g.download("qout_up")
    q_l = g.download("qout_left")
    q_d = g.download("qout_down")
    o_f = g.download("outlet_flow")
    i_tot = g.download("i_tot_end_cell")
    out = np.stack([q_r, q_u, o_f], axis=2)
    Hf = np.stack([g.download("hf_x"), g.download("hf_y"), g.download("hf_outlet")], axis=2)
    return q_l, q_r, q_u, q_d, o_f, d_t, i_tot, out, Hf, 0, 0, 0, 0, res * res


def refreshing_timestep(Hf, qout_right, qout_up, Resolution, depth_tolerance, alfa_min,
                        alfa_max, max_time_step, min_time_step, time_step_increments,
                        flag_timestep: int = 1, flag_adaptive_timestepping: int = 1,
                        device: int = 0):
    """Refresh branch of the refreshing_timestep.m script for the inertial D4 model.

    Reads what the script reads from its workspace -- ``Hf`` (ny, nx, 3) [m],
    ``flow_rate.qout_right_t``/``qout_up_t`` [mm/h], ``Resolution``,
    ``CA_States.depth_tolerance`` [mm], ``Courant_Parameters.alfa_min/alfa_max``,
    ``running_control.max/min_time_step`` and ``time_step_increments`` [s], the two flags --
    and returns ``(time_calculation_routing [s], time_step [min], max_velocity [m/s])``.
    The face arrays are rounded to FP32 on the way to the device (the FP32 build's state).
    """
    import torch
    if not torch.cuda.is_available():
        raise _abi.HP2DError(7, "no CUDA device: refreshing_timestep runs only on the GPU")
    qr = np.asarray(qout_right, dtype=np.float64)
    ny, nx = qr.shape
    res = float(Resolution)
    Hf = np.asarray(Hf, dtype=np.float64)
    if Hf.shape != (ny, nx, 3):
        raise ValueError("Hf must be (ny, nx, 3) pages [m]")
    # outflow [mm/h] -> discharge per unit width [m^2/s] (Local_Inertial_Model_D4.m:198)
    to_q = lambda a: (np.asarray(a, dtype=np.float64) / 1000 / 3600 * (res * res) / res)
    dev = torch.device("cuda", device)
    q_x = torch.from_numpy(np.ascontiguousarray(to_q(qr), dtype=np.float32)).to(dev)
    q_y = torch.from_numpy(np.ascontiguousarray(to_q(qout_up), dtype=np.float32)).to(dev)
    hf = torch.from_numpy(np.ascontiguousarray(np.moveaxis(Hf, 2, 0), dtype=np.float32)).to(dev)
    params = _abi.default_params(depth_tolerance=float(depth_tolerance), alfa_min=float(alfa_min),
                                 alfa_max=float(alfa_max), max_time_step=float(max_time_step),
                                 min_time_step=float(min_time_step),
                                 time_step_increments=float(time_step_increments),
                                 flag_timestep=int(flag_timestep),
                                 flag_adaptive_timestepping=int(flag_adaptive_timestepping))
    L = _abi.lib()
    ts = C.c_double()
    vm = C.c_double()
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev)
        st = L.hp2d_cfl_dt_noalloc(ny, nx, res, C.byref(params), C.c_void_p(q_x.data_ptr()),
                                   C.c_void_p(q_y.data_ptr()), C.c_void_p(hf.data_ptr()),
                                   C.c_void_p(stream.cuda_stream), C.byref(ts), C.byref(vm))
    if st != 0:
        raise _abi.HP2DError(st, L.hp2d_noalloc_error().decode())
    return ts.value * 60, ts.value, vm.value
