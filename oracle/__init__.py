"""Oracle package -- TEST INFRASTRUCTURE ONLY.

Two CPU restatements of HydroPol2D's surface-flow step:

* ``oracle.literal``: FP64 numpy, the reference's own whole-array operation order and
  units ("the reference's FP64 path").
* ``oracle.KernelFormOracle``: C++ (kernel_form.hpp via liboracle_hp2d.so), the
  algebraically identical form the CUDA kernels compute, in float or double.  The CUDA
  library must reproduce it bit for bit.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may use this
package; the product (hydropol2d_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
LIB_PATH = HERE / "liboracle_hp2d.so"

CXXFLAGS = ["-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
            f"-I{ROOT / 'include'}"]


def build(force: bool = False) -> Path:
    srcs = [HERE / "oracle_capi.cpp", HERE / "kernel_form.hpp", ROOT / "include" / "hp2d.h"]
    if not force and LIB_PATH.exists() and all(s.stat().st_mtime <= LIB_PATH.stat().st_mtime for s in srcs):
        return LIB_PATH
    # the system g++ ships the OpenMP runtime (libgomp); prefer it over $CXX
    cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else os.environ.get("CXX", "g++")
    tmp = LIB_PATH.with_suffix(".so.tmp")
    subprocess.run([cxx, *CXXFLAGS, str(HERE / "oracle_capi.cpp"), "-o", str(tmp)], check=True)
    tmp.replace(LIB_PATH)
    return LIB_PATH


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        from hydropol2d_b200 import _abi  # plain C structs of include/hp2d.h
        L = C.CDLL(str(LIB_PATH))
        P = C.POINTER
        vp = C.c_void_p
        dp = P(C.c_double)
        i32p = P(C.c_int32)
        sig = {
            "oracle_create": ([P(_abi.Grid), P(_abi.Params)], vp),
            "oracle_destroy": ([vp], None),
            "oracle_upload_static": ([vp, dp, dp, i32p, i32p, C.c_int32, dp], C.c_int),
            "oracle_set_soil": ([vp, P(C.c_uint8), C.c_int32, dp, dp, dp, dp, dp, dp, dp], C.c_int),
            "oracle_set_state": ([vp, dp, dp, dp], C.c_int),
            "oracle_set_depth": ([vp, dp], C.c_int),
            "oracle_set_clock": ([vp, C.c_double, C.c_double, C.c_int64], C.c_int),
            "oracle_set_rain_clock": ([vp, C.c_double, C.c_double, C.c_double], C.c_int),
            "oracle_set_map_records": ([vp, C.c_int32, dp], C.c_int),
            "oracle_set_stage": ([vp, C.c_int32, C.c_int32, dp, dp, C.c_int32, P(C.c_int32), P(C.c_int32),
                                  P(C.c_int32)], C.c_int),
            "oracle_set_reservoirs": ([vp, C.c_int32, i32p, i32p, dp, dp, dp, i32p, i32p, dp, dp, dp, i32p, i32p],
                                      C.c_int),
            "oracle_set_hazard_tracking": ([vp, C.c_int32], C.c_int),
            "oracle_map_records": ([vp], C.c_int64),
            "oracle_download_map_record": ([vp, C.c_int64, dp, dp], C.c_int),
            "oracle_set_inflow": ([vp, C.c_int32, C.c_int32, dp, dp, C.c_int32, P(C.c_int32), P(C.c_int32),
                                   P(C.c_int32), dp], C.c_int),
            "oracle_set_rain_uniform": ([vp, C.c_int32, dp, dp], C.c_int),
            "oracle_set_rain_maps": ([vp, C.c_int32, C.c_int32, C.c_int32, P(C.c_float), C.c_double], C.c_int),
            "oracle_set_rain_maps_end_stamped": ([vp, C.c_int32, C.c_int32, C.c_int32, P(C.c_float), P(C.c_double),
                                                  C.c_double], C.c_int),
            "oracle_hydrology_step": ([vp, C.c_double], C.c_int),
            "oracle_li_step": ([vp, C.c_double], C.c_int),
            "oracle_cfl_dt": ([vp, C.c_double, dp, dp], C.c_int),
            "oracle_track_maxima": ([vp, C.c_double], C.c_int),
            "oracle_steps": ([vp, C.c_int32], C.c_int),
            "oracle_run": ([vp, C.c_int64, P(C.c_int64)], C.c_int),
            "oracle_download_native": ([vp, C.c_int32, vp, C.c_size_t], C.c_int),
            "oracle_get_diag": ([vp, P(_abi.Diag)], C.c_int),
            "oracle_set_retry_policy": ([vp, C.c_int32, C.c_double, C.c_int32], C.c_int),
            "oracle_inject_step_fault": ([vp, C.c_int64, C.c_int32], C.c_int),
            "oracle_set_refresh_every": ([vp, C.c_int32], C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class KernelFormOracle:
    """Same call surface as hydropol2d_b200.SurfaceFlow, computed on the CPU."""

    NATIVE = {"h": 0, "qx": 1, "qy": 2, "I": 3, "T": 4, "dmax": 5, "arrival": 6, "hfx": 7,
              "hfy": 8, "hf3": 9, "qo": 10, "vmax": 11, "hazard_max": 12}

    def __init__(self, ny, nx, resolution, precision="fp32", params=None, **param_kw):
        from hydropol2d_b200 import _abi
        self._L = _load()
        self.ny, self.nx, self.resolution = int(ny), int(nx), float(resolution)
        self.precision = precision
        self.dtype = np.float32 if precision == "fp32" else np.float64
        self.params = params if params is not None else _abi.default_params(**param_kw)
        g = _abi.Grid(self.ny, self.nx, self.resolution, 0 if precision == "fp32" else 1)
        self._h = self._L.oracle_create(C.byref(g), C.byref(self.params))
        self.n_outlets = 0

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.oracle_destroy(self._h)
            self._h = None

    def upload_static(self, z, roughness, outlet_rows, outlet_cols, slope_per_outlet=None):
        z = np.ascontiguousarray(np.broadcast_to(z, (self.ny, self.nx)), dtype=np.float64)
        n = np.ascontiguousarray(np.broadcast_to(roughness, (self.ny, self.nx)), dtype=np.float64)
        rows = np.ascontiguousarray(outlet_rows, dtype=np.int32).ravel()
        cols = np.ascontiguousarray(outlet_cols, dtype=np.int32).ravel()
        sl = None if slope_per_outlet is None else np.ascontiguousarray(slope_per_outlet, dtype=np.float64).ravel()
        self._L.oracle_upload_static(self._h, _dp(z), _dp(n), rows.ctypes.data_as(C.POINTER(C.c_int32)),
                                     cols.ctypes.data_as(C.POINTER(C.c_int32)), int(rows.size),
                                     None if sl is None else _dp(sl))
        self.n_outlets = len(set(zip(rows.tolist(), cols.tolist())))
        self._z = z   # the inflow volume ledger counts gauge cells with a finite elevation

    def set_soil(self, soil_class, ksat, psi, dtheta, Lu, k_out, Tr, min_soil_moisture):
        cls = np.ascontiguousarray(soil_class, dtype=np.uint8).reshape(self.ny, self.nx)
        tabs = [np.ascontiguousarray(v, dtype=np.float64).ravel() for v in
                (ksat, psi, dtheta, Lu, k_out, Tr, min_soil_moisture)]
        self._L.oracle_set_soil(self._h, cls.ctypes.data_as(C.POINTER(C.c_uint8)), tabs[0].size,
                                *[_dp(t) for t in tabs])

    def set_state(self, d, outflow=None, soil_storage=None):
        d = np.ascontiguousarray(np.broadcast_to(d, (self.ny, self.nx)), dtype=np.float64)
        of = None if outflow is None else np.ascontiguousarray(np.asarray(outflow, dtype=np.float64)[:2])
        I = None if soil_storage is None else np.ascontiguousarray(
            np.broadcast_to(soil_storage, (self.ny, self.nx)), dtype=np.float64)
        self._L.oracle_set_state(self._h, _dp(d), None if of is None else _dp(of), None if I is None else _dp(I))

    def set_depth(self, d):
        d = np.ascontiguousarray(np.broadcast_to(d, (self.ny, self.nx)), dtype=np.float64)
        self._L.oracle_set_depth(self._h, _dp(d))

    def set_clock(self, t, time_step, k=1):
        self._L.oracle_set_clock(self._h, float(t), float(time_step), int(k))

    def set_inflow(self, t_start, rates, rows, cols, gauge):
        t = np.ascontiguousarray(t_start, dtype=np.float64).ravel()
        r = np.ascontiguousarray(np.asarray(rates, dtype=np.float64).reshape(t.size, -1))
        rr = np.ascontiguousarray(rows, dtype=np.int32).ravel()
        cc = np.ascontiguousarray(cols, dtype=np.int32).ravel()
        gg = np.ascontiguousarray(gauge, dtype=np.int32).ravel()
        ip = C.POINTER(C.c_int32)
        self._L.oracle_set_inflow(self._h, int(r.shape[1]), int(t.size), _dp(t), _dp(r), int(rr.size),
                                  rr.ctypes.data_as(ip), cc.ctypes.data_as(ip), gg.ctypes.data_as(ip),
                                  _dp(self._z))

    def set_stage(self, t_start, depth_m, rows, cols, gauge):
        t = np.ascontiguousarray(t_start, dtype=np.float64).ravel()
        d = np.ascontiguousarray(np.asarray(depth_m, dtype=np.float64).reshape(t.size, -1))
        rr = np.ascontiguousarray(rows, dtype=np.int32).ravel()
        cc = np.ascontiguousarray(cols, dtype=np.int32).ravel()
        gg = np.ascontiguousarray(gauge, dtype=np.int32).ravel()
        ip = C.POINTER(C.c_int32)
        self._L.oracle_set_stage(self._h, int(d.shape[1]), int(t.size), _dp(t), _dp(d), int(rr.size),
                                 rr.ctypes.data_as(ip), cc.ctypes.data_as(ip), gg.ctypes.data_as(ip))

    def set_hazard_tracking(self, on=True):
        self._L.oracle_set_hazard_tracking(self._h, 1 if on else 0)

    def set_reservoirs(self, res_row, res_col, k1, h1, k2, ds1_row, ds1_col, k3, h2, k4, ds2_row, ds2_col):
        i32 = [np.ascontiguousarray(a, dtype=np.int32).ravel() for a in (res_row, res_col, ds1_row, ds1_col,
                                                                          ds2_row, ds2_col)]
        f64 = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (k1, h1, k2, k3, h2, k4)]
        ip = C.POINTER(C.c_int32)
        rr, rc, d1r, d1c, d2r, d2c = (a.ctypes.data_as(ip) for a in i32)
        self._L.oracle_set_reservoirs(self._h, int(i32[0].size), rr, rc, _dp(f64[0]), _dp(f64[1]), _dp(f64[2]),
                                      d1r, d1c, _dp(f64[3]), _dp(f64[4]), _dp(f64[5]), d2r, d2c)

    def set_map_records(self, time_records, n_slots=None):
        t = np.ascontiguousarray(time_records, dtype=np.float64).ravel()
        self._L.oracle_set_map_records(self._h, int(t.size), _dp(t))

    def map_records(self):
        return int(self._L.oracle_map_records(self._h))

    def download_map_record(self, index):
        out = np.empty((self.ny, self.nx), dtype=np.float64)
        t = C.c_double()
        if self._L.oracle_download_map_record(self._h, int(index), _dp(out), C.byref(t)) != 0:
            raise IndexError(index)
        return out, t.value

    def set_rain_clock(self, rain_t0, rain_t1, t_previous):
        self._L.oracle_set_rain_clock(self._h, float(rain_t0), float(rain_t1), float(t_previous))

    def set_rain_uniform(self, t_start, rate):
        t = np.ascontiguousarray(t_start, dtype=np.float64).ravel()
        r = np.ascontiguousarray(rate, dtype=np.float64).ravel()
        self._L.oracle_set_rain_uniform(self._h, int(t.size), _dp(t), _dp(r))

    def set_rain_maps(self, maps, map_dt):
        m = np.ascontiguousarray(maps, dtype=np.float32)
        nm, my, mx = m.shape
        self._L.oracle_set_rain_maps(self._h, nm, my, mx, m.ctypes.data_as(C.POINTER(C.c_float)), float(map_dt))

    def set_rain_maps_end_stamped(self, maps, t_end, dt_force=None):
        m = np.ascontiguousarray(maps, dtype=np.float32)
        if m.ndim == 2:
            m = m[None]
        te = np.ascontiguousarray(t_end, dtype=np.float64).reshape(-1)
        if dt_force is None:
            dt_force = float(te[1] - te[0]) if te.size >= 2 and te[1] > te[0] else 0.0
        nm, my, mx = m.shape
        self._L.oracle_set_rain_maps_end_stamped(self._h, nm, my, mx, m.ctypes.data_as(C.POINTER(C.c_float)),
                                                 _dp(te), float(dt_force))

    def hydrology_step(self, time_step):
        self._L.oracle_hydrology_step(self._h, float(time_step))

    def li_step(self, time_step):
        self._L.oracle_li_step(self._h, float(time_step))
        self._last_ts = float(time_step)

    def cfl_dt(self):
        ts = C.c_double()
        vm = C.c_double()
        self._L.oracle_cfl_dt(self._h, getattr(self, "_last_ts", 1.0), C.byref(ts), C.byref(vm))
        return ts.value, vm.value

    def track_maxima(self, t_end):
        self._L.oracle_track_maxima(self._h, float(t_end))

    def fused_steps(self, n):
        """n accepted steps; returns the hp2d_status code (0, or HP2D_NUMERICAL / HP2D_DT_FLOOR)."""
        return self._L.oracle_steps(self._h, int(n))

    def run(self, max_steps=0):
        done = C.c_int64()
        self._L.oracle_run(self._h, int(max_steps), C.byref(done))
        return done.value

    def set_retry_policy(self, max_retries=8, factor_reduction=2.0, dt_floor_is_error=False):
        self._L.oracle_set_retry_policy(self._h, int(max_retries), float(factor_reduction),
                                        int(bool(dt_floor_is_error)))

    def set_temporal_blocking(self, steps_per_block):
        """The refresh schedule of temporal blocking: the time step is refreshed on step 1 and on
        the steps k with (k - 1) % K == 0 (K <= 1: every step)."""
        self._L.oracle_set_refresh_every(self._h, int(steps_per_block))

    def inject_step_fault(self, k, attempts=1):
        self._L.oracle_inject_step_fault(self._h, int(k), int(attempts))

    def download_native(self, field):
        per_outlet = field in ("hf3", "qo")
        shape = (self.n_outlets,) if per_outlet else (self.ny, self.nx)
        out = np.empty(shape, dtype=self.dtype)
        st = self._L.oracle_download_native(self._h, self.NATIVE[field], out.ctypes.data_as(C.c_void_p), out.nbytes)
        if st != 0:
            raise RuntimeError(f"oracle_download_native({field}) failed: {st}")
        return out

    def diag(self):
        from hydropol2d_b200 import _abi
        d = _abi.Diag()
        self._L.oracle_get_diag(self._h, C.byref(d))
        return {k: getattr(d, k) for k, _ in _abi.Diag._fields_}
