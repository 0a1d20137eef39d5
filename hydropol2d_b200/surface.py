"""Host-side handle of one resident grid: a thin Python layer over the C ABI.

Arrays cross as numpy (host) buffers; units are the reference's (mm, mm/h, min, m).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a, shape=None) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and out.shape != shape:
        out = np.ascontiguousarray(np.broadcast_to(out, shape), dtype=np.float64)
    return out


class SurfaceFlow:
    """One hp2d_ctx.  ``precision`` is "fp32" or "fp64"."""

    def __init__(self, ny: int, nx: int, resolution: float, precision: str = "fp32",
                 params: _abi.Params | None = None, device: int = 0, **param_kw):
        self._L = _abi.lib()
        self.ny, self.nx = int(ny), int(nx)
        self.resolution = float(resolution)
        self.precision = precision
        self.dtype = np.float32 if precision == "fp32" else np.float64
        prec = _abi.HP2D_FP32 if precision == "fp32" else _abi.HP2D_FP64
        self.params = params if params is not None else _abi.default_params(**param_kw)
        g = _abi.Grid(self.ny, self.nx, self.resolution, prec)
        h = C.c_void_p()
        st = self._L.hp2d_create(C.byref(g), C.byref(self.params), int(device), C.byref(h))
        if st != 0:
            raise _abi.HP2DError(st, self._L.hp2d_create_error().decode())
        self._h = h
        self.n_outlets = 0

    # ---------------------------------------------------------------- plumbing
    def _check(self, st: int):
        if st != 0:
            raise _abi.HP2DError(st, self._L.hp2d_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.hp2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---------------------------------------------------------------- inputs
    def upload_static(self, z, roughness, outlet_rows, outlet_cols, slope_per_outlet=None):
        shp = (self.ny, self.nx)
        z = _f64(z, shp)
        n = _f64(roughness, shp)
        rows = np.ascontiguousarray(outlet_rows, dtype=np.int32).ravel()
        cols = np.ascontiguousarray(outlet_cols, dtype=np.int32).ravel()
        sl = None if slope_per_outlet is None else _f64(slope_per_outlet).ravel()
        self._check(self._L.hp2d_upload_static(
            self._h, _dp(z), _dp(n), rows.ctypes.data_as(C.POINTER(C.c_int32)),
            cols.ctypes.data_as(C.POINTER(C.c_int32)), int(rows.size),
            None if sl is None else _dp(sl)))
        self.n_outlets = len(set(zip(rows.tolist(), cols.tolist())))

    def set_soil(self, soil_class, ksat, psi, dtheta, Lu, k_out, Tr, min_soil_moisture):
        cls = np.ascontiguousarray(soil_class, dtype=np.uint8).reshape(self.ny, self.nx)
        tabs = [_f64(v).ravel() for v in (ksat, psi, dtheta, Lu, k_out, Tr, min_soil_moisture)]
        ncls = tabs[0].size
        if any(t.size != ncls for t in tabs):
            raise ValueError("soil tables must have one entry per class")
        self._check(self._L.hp2d_set_soil(self._h, cls.ctypes.data_as(C.POINTER(C.c_uint8)), ncls,
                                          *[_dp(t) for t in tabs]))

    def set_soil_vg(self, soil_class, theta_r, theta_sat, n_vg, alpha_vg, ksat, soil_depth, gw_head=None,
                    l_vg=0.5, Ltop=0.05, dh_max=1.0, Ksurf_weight=0.5):
        """van Genuchten-Mualem soil (flag_infiltration=2): per-class tables, per-cell soil
        depth [m] and groundwater head [m] (None: water table at the soil bottom)."""
        shp = (self.ny, self.nx)
        cls = np.ascontiguousarray(soil_class, dtype=np.uint8).reshape(shp)
        tabs = [_f64(v).ravel() for v in (theta_r, theta_sat, n_vg, alpha_vg, ksat)]
        ncls = tabs[0].size
        if any(t.size != ncls for t in tabs):
            raise ValueError("soil tables must have one entry per class")
        sd = _f64(soil_depth, shp)
        gw = None if gw_head is None else _f64(gw_head, shp)
        self._check(self._L.hp2d_set_soil_vg(self._h, cls.ctypes.data_as(C.POINTER(C.c_uint8)), ncls,
                                             *[_dp(t) for t in tabs], _dp(sd), None if gw is None else _dp(gw),
                                             float(l_vg), float(Ltop), float(dh_max), float(Ksurf_weight)))

    def set_state(self, d, outflow=None, soil_storage=None):
        shp = (self.ny, self.nx)
        d = _f64(d, shp)
        of = None
        if outflow is not None:
            of = np.asarray(outflow, dtype=np.float64)
            of = np.ascontiguousarray(of[:2] if of.shape[0] >= 2 else of)
            if of.shape != (2, self.ny, self.nx):
                raise ValueError("outflow must be (2 or 3, ny, nx) pages [mm/h]")
        I = None if soil_storage is None else _f64(soil_storage, shp)
        self._check(self._L.hp2d_set_state(self._h, _dp(d), None if of is None else _dp(of),
                                           None if I is None else _dp(I)))

    def set_clock(self, t: float, time_step: float, k: int = 1):
        self._check(self._L.hp2d_set_clock(self._h, float(t), float(time_step), int(k)))

    def set_rain_clock(self, rain_t0: float, rain_t1: float, t_previous: float):
        """The clock interval whose rain the next step applies and the loop's t_previous
        [min] (``diag`` reports them), for an exact restart."""
        self._check(self._L.hp2d_set_rain_clock(self._h, float(rain_t0), float(rain_t1), float(t_previous)))

    def set_inflow(self, t_start, rates, rows, cols, gauge):
        """Inflow hydrographs: ``rates`` (n_times, n_gauges) [mm/h] on the start-stamped
        ``t_start`` [min]; cells ``rows``/``cols`` of gauge ``gauge`` (Wshed_Properties.inflow_cells).
        After ``upload_static``; ``rates`` with no gauges removes the inflow."""
        t = _f64(t_start).ravel()
        r = np.ascontiguousarray(np.asarray(rates, dtype=np.float64).reshape(t.size, -1))
        ng = r.shape[1]
        rr = np.ascontiguousarray(rows, dtype=np.int32).ravel()
        cc = np.ascontiguousarray(cols, dtype=np.int32).ravel()
        gg = np.ascontiguousarray(gauge, dtype=np.int32).ravel()
        ip = C.POINTER(C.c_int32)
        self._check(self._L.hp2d_set_inflow(self._h, int(ng), int(t.size), _dp(t), _dp(r), int(rr.size),
                                            rr.ctypes.data_as(ip), cc.ctypes.data_as(ip), gg.ctypes.data_as(ip)))

    def set_stage(self, t_start, depth_m, rows, cols, gauge):
        """Stage hydrographs: water depths ``depth_m`` (n_times, n_gauges) [m] on the start-stamped
        ``t_start`` [min]; cells ``rows``/``cols`` of gauge ``gauge`` (Wshed_Properties.stage_mask)."""
        t = _f64(t_start).ravel()
        d = np.ascontiguousarray(np.asarray(depth_m, dtype=np.float64).reshape(t.size, -1))
        rr = np.ascontiguousarray(rows, dtype=np.int32).ravel()
        cc = np.ascontiguousarray(cols, dtype=np.int32).ravel()
        gg = np.ascontiguousarray(gauge, dtype=np.int32).ravel()
        ip = C.POINTER(C.c_int32)
        self._check(self._L.hp2d_set_stage(self._h, int(d.shape[1]), int(t.size), _dp(t), _dp(d), int(rr.size),
                                           rr.ctypes.data_as(ip), cc.ctypes.data_as(ip), gg.ctypes.data_as(ip)))

    def set_dry_skip(self, on: bool = True):
        """Skipping of provably unchanged dry rows and blocks in the fused step (default on;
        results are identical either way)."""
        self._check(self._L.hp2d_set_dry_skip(self._h, 1 if on else 0))

    def set_hazard_tracking(self, on: bool = True):
        """Per-cell maxima of the velocity raster and of depth x velocity over the fused steps
        (velocities.vmax_final / hazardmax_final); read with download("vmax"/"hazard_max")."""
        self._check(self._L.hp2d_set_hazard_tracking(self._h, 1 if on else 0))

    def set_reservoirs(self, res_row, res_col, k1, h1, k2, ds1_row, ds1_col, k3, h2, k4, ds2_row, ds2_col):
        """Reservoir / control structures (``flag_reservoir = 1``): the reservoir_x/y, k1, h1, k2,
        k3, h2, k4, yds1/xds1, yds2/xds2 arguments of Local_Inertial_Model_D4 as arrays over the
        structures, 0-based cells, -1 rows for the reference's NaN (no downstream cell)."""
        i32 = [np.ascontiguousarray(a, dtype=np.int32).ravel() for a in (res_row, res_col, ds1_row, ds1_col,
                                                                          ds2_row, ds2_col)]
        f64 = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (k1, h1, k2, k3, h2, k4)]
        n = i32[0].size
        if any(a.size != n for a in i32 + f64):
            raise ValueError("every structure argument needs one entry per structure")
        ip = C.POINTER(C.c_int32)
        rr, rc, d1r, d1c, d2r, d2c = (a.ctypes.data_as(ip) for a in i32)
        self._check(self._L.hp2d_set_reservoirs(self._h, int(n), rr, rc, _dp(f64[0]), _dp(f64[1]), _dp(f64[2]), d1r, d1c,
                                                _dp(f64[3]), _dp(f64[4]), _dp(f64[5]), d2r, d2c))

    def set_rain_gauges(self, x_gauge, y_gauge, rates, record_dt: float, x_ul: float = 0.0, y_ul: float = 0.0):
        """Rain from gauges: ``rates`` (n_times, n_gauges) [mm/h] (NaN: no record) over intervals
        of ``record_dt`` minutes, interpolated by inverse-distance weighting to every cell."""
        x = _f64(x_gauge).ravel()
        y = _f64(y_gauge).ravel()
        r = np.ascontiguousarray(np.asarray(rates, dtype=np.float64).reshape(-1, x.size))
        self._check(self._L.hp2d_set_rain_gauges(self._h, int(x.size), _dp(x), _dp(y), int(r.shape[0]),
                                                 float(record_dt), _dp(r), float(x_ul), float(y_ul)))

    def set_map_records(self, time_records, n_slots: int, host: bool = False):
        """Keep the depth map after each step that passes a record time [min]
        (save_output_maps); ``n_slots`` maps are held on the device, or with ``host`` in
        page-locked host memory that the steps write across the host link themselves."""
        t = _f64(time_records).ravel()
        fn = self._L.hp2d_set_map_records_host if host else self._L.hp2d_set_map_records
        self._check(fn(self._h, int(t.size), _dp(t), int(n_slots)))

    def map_records(self) -> int:
        c = C.c_int64()
        self._check(self._L.hp2d_map_records(self._h, C.byref(c)))
        return c.value

    def download_map_record(self, index: int):
        """(depth [mm] as (ny, nx), clock [min]) of record ``index``."""
        out = np.empty((self.ny, self.nx), dtype=np.float64)
        t = C.c_double()
        self._check(self._L.hp2d_download_map_record(self._h, int(index), _dp(out), C.byref(t)))
        return out, t.value

    def set_rain_uniform(self, t_start, rate):
        t = _f64(t_start).ravel()
        r = _f64(rate).ravel()
        self._check(self._L.hp2d_set_rain_uniform(self._h, int(t.size), _dp(t), _dp(r)))

    def set_rain_maps_end_stamped(self, maps, t_end, dt_force: float | None = None):
        """Input rain maps [mm/h] (n, my, mx), map m over [t_end[m-1], t_end[m]) [min], the first
        from t_end[0] - dt_force (default t_end[1] - t_end[0], or 0 for one map)."""
        m = np.ascontiguousarray(maps, dtype=np.float32)
        if m.ndim == 2:
            m = m[None]
        te = np.ascontiguousarray(t_end, dtype=np.float64).reshape(-1)
        if te.size != m.shape[0]:
            raise ValueError("one end time per map")
        if dt_force is None:
            dt_force = float(te[1] - te[0]) if te.size >= 2 and te[1] > te[0] else 0.0
        self._check(self._L.hp2d_set_rain_maps_end_stamped(self._h, m.shape[0], m.shape[1], m.shape[2],
                                                           m.ctypes.data_as(C.POINTER(C.c_float)), _dp(te),
                                                           float(dt_force)))

    def set_rain_maps(self, maps, map_dt: float):
        m = np.ascontiguousarray(maps, dtype=np.float32)
        nm, my, mx = m.shape
        self._check(self._L.hp2d_set_rain_maps(self._h, nm, my, mx,
                                               m.ctypes.data_as(C.POINTER(C.c_float)), float(map_dt)))

    # ---------------------------------------------------------------- stages
    def hydrology_step(self, time_step: float):
        self._check(self._L.hp2d_hydrology_step(self._h, float(time_step)))

    def li_step(self, time_step: float):
        self._check(self._L.hp2d_li_step(self._h, float(time_step)))

    def cfl_dt(self):
        ts = C.c_double()
        vm = C.c_double()
        self._check(self._L.hp2d_cfl_dt(self._h, C.byref(ts), C.byref(vm)))
        return ts.value, vm.value

    def track_maxima(self, t_end: float):
        self._check(self._L.hp2d_track_maxima(self._h, float(t_end)))

    def fused_steps(self, n: int):
        self._check(self._L.hp2d_fused_steps(self._h, int(n)))

    def fused_steps_timed(self, n: int) -> float:
        """Runs n fused steps; returns their device time [ms] (CUDA events on the
        library's stream)."""
        ms = C.c_float()
        self._check(self._L.hp2d_fused_steps_timed(self._h, int(n), C.byref(ms)))
        return ms.value

    def set_layout(self, cells_per_lane: int):
        """1 or 2 cells per lane in the fused kernel (32- or 64-column strips)."""
        self._check(self._L.hp2d_set_layout(self._h, int(cells_per_lane)))

    def set_tuning(self, rows_per_warp: int):
        self._check(self._L.hp2d_set_tuning(self._h, int(rows_per_warp)))

    def autotune(self, trial_steps: int = 4) -> int:
        """Times ``trial_steps`` steps per launch shape from the current state, undoes them
        and keeps the fastest; returns the chosen rows per warp."""
        rpw = C.c_int32()
        self._check(self._L.hp2d_autotune(self._h, int(trial_steps), C.byref(rpw)))
        return rpw.value

    def run(self, max_steps: int = 0) -> int:
        done = C.c_int64()
        self._check(self._L.hp2d_run(self._h, int(max_steps), C.byref(done)))
        return done.value

    def set_retry_policy(self, max_retries: int = 8, factor_reduction: float = 2.0,
                         dt_floor_is_error: bool = False):
        """Retries of a rejected step (HydroPol2D_Main_While.m:926-993) and whether a step whose
        refreshed dt hits min_time_step ends the call with HP2D_DT_FLOOR."""
        self._check(self._L.hp2d_set_retry_policy(self._h, int(max_retries), float(factor_reduction),
                                                  int(bool(dt_floor_is_error))))

    def set_wait_limit(self, polls: int):
        """Polls of a row-copy wait before the step gives up with HP2D_TIMEOUT (default 4194304)."""
        self._check(self._L.hp2d_set_wait_limit(self._h, int(polls)))

    def set_temporal_blocking(self, steps_per_block: int):
        """K steps per launch at the frozen time step of the last refresh (2..4), 1 off, 0 chosen
        by ``autotune`` (see hp2d_set_temporal_blocking)."""
        self._check(self._L.hp2d_set_temporal_blocking(self._h, int(steps_per_block)))

    def inject_step_fault(self, k: int, attempts: int = 1):
        """Test hook: the next ``attempts`` attempts of step ``k`` are rejected."""
        self._check(self._L.hp2d_inject_step_fault(self._h, int(k), int(attempts)))

    # ---------------------------------------------------------------- row slabs
    def set_owned_rows(self, row0: int, row1: int):
        """This context holds one slab of a larger grid: rows [row0, row1) are its own, the rest
        halo rows (hydropol2d_b200.slabs drives it)."""
        self._check(self._L.hp2d_set_owned_rows(self._h, int(row0), int(row1)))

    def step_maxima(self) -> tuple[int, int, int]:
        """The last step's ordered speed^2 and celerity bits and the next step's clamp skip."""
        v, c, s = C.c_uint64(), C.c_uint64(), C.c_int32()
        self._check(self._L.hp2d_step_maxima(self._h, C.byref(v), C.byref(c), C.byref(s)))
        return v.value, c.value, s.value

    def apply_refresh(self, speed2_bits: int, celerity_bits: int, clamp_skip: int):
        self._check(self._L.hp2d_apply_refresh(self._h, int(speed2_bits), int(celerity_bits), int(clamp_skip)))

    def get_rows(self, row0: int, nrows: int) -> np.ndarray:
        """State records {h, q_x, q_y, dmax} of rows [row0, row0 + nrows), (nrows, nx, 4)."""
        out = np.empty((int(nrows), self.nx, 4), dtype=self.dtype)
        self._check(self._L.hp2d_copy_rows(self._h, int(row0), int(nrows), out.ctypes.data_as(C.c_void_p), 0))
        return out

    def set_rows(self, row0: int, block: np.ndarray):
        block = np.ascontiguousarray(block, dtype=self.dtype)
        if block.ndim != 3 or block.shape[1:] != (self.nx, 4):
            raise ValueError("rows must be an (nrows, nx, 4) array of state records")
        self._check(self._L.hp2d_copy_rows(self._h, int(row0), block.shape[0],
                                           block.ctypes.data_as(C.c_void_p), 1))

    # ---------------------------------------------------------------- outputs
    def download(self, field: str) -> np.ndarray:
        out = np.empty((self.ny, self.nx), dtype=np.float64)
        self._check(self._L.hp2d_download(self._h, _abi.FIELD[field], _dp(out), out.size))
        return out

    def download_into(self, field: str, out: np.ndarray) -> np.ndarray:
        """``download`` into a caller-owned C-contiguous float64 (ny, nx) array (for instance one
        in page-locked memory)."""
        if out.dtype != np.float64 or out.shape != (self.ny, self.nx) or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 (ny, nx) array")
        self._check(self._L.hp2d_download(self._h, _abi.FIELD[field], _dp(out), out.size))
        return out

    def download_native(self, field: str) -> np.ndarray:
        per_outlet = field in ("hf3", "qo")
        shape = (self.n_outlets,) if per_outlet else (self.ny, self.nx)
        out = np.empty(shape, dtype=self.dtype)
        self._check(self._L.hp2d_download_native(self._h, _abi.NATIVE[field],
                                                 out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def diag(self) -> dict:
        d = _abi.Diag()
        self._check(self._L.hp2d_get_diag(self._h, C.byref(d)))
        return {k: getattr(d, k) for k, _ in _abi.Diag._fields_}

    def stored_volume(self) -> float:
        v = C.c_double()
        self._check(self._L.hp2d_stored_volume(self._h, C.byref(v)))
        return v.value
