"""ctypes view of include/hp2d.h and the loader of the in-tree libhp2d.so.

There is no fallback: if the library is missing or no CUDA device is present, the calls
raise.  Plain C structs only -- no torch types cross this boundary.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import os

# the in-tree build; HP2D_LIBRARY names another build of the same library (A/B timing)
LIB_PATH = Path(os.environ.get("HP2D_LIBRARY") or Path(__file__).resolve().parent / "libhp2d.so")

HP2D_FP32 = 0
HP2D_FP64 = 1

STATUS = {
    0: "HP2D_OK", 1: "HP2D_INVALID_ARG", 2: "HP2D_UNSUPPORTED_FLAG", 3: "HP2D_CUDA_ERROR",
    4: "HP2D_NUMERICAL", 5: "HP2D_DT_FLOOR", 6: "HP2D_TIMEOUT", 7: "HP2D_NO_DEVICE",
    8: "HP2D_NOT_READY",
}

FIELD = {
    "depth": 0, "qout_right": 1, "qout_up": 2, "qout_left": 3, "qout_down": 4,
    "outlet_flow": 5, "hf_x": 6, "hf_y": 7, "hf_outlet": 8, "dmax": 9, "arrival": 10,
    "soil_storage": 11, "i_tot_end_cell": 12, "vmax": 13, "hazard_max": 14,
}

NATIVE = {
    "h": 0, "qx": 1, "qy": 2, "I": 3, "T": 4, "dmax": 5, "arrival": 6, "hfx": 7, "hfy": 8,
    "hf3": 9, "qo": 10,
}

# every symbol include/hp2d.h declares
EXPORTS = [
    "hp2d_create", "hp2d_destroy", "hp2d_last_error", "hp2d_create_error",
    "hp2d_upload_static", "hp2d_set_soil", "hp2d_set_soil_vg", "hp2d_set_state", "hp2d_set_clock", "hp2d_set_rain_clock",
    "hp2d_set_rain_uniform", "hp2d_set_rain_maps", "hp2d_set_rain_maps_end_stamped", "hp2d_set_rain_gauges", "hp2d_set_inflow", "hp2d_set_stage",
    "hp2d_set_reservoirs", "hp2d_set_hazard_tracking", "hp2d_set_dry_skip",
    "hp2d_set_map_records", "hp2d_set_map_records_host", "hp2d_map_records", "hp2d_download_map_record", "hp2d_hydrology_step", "hp2d_li_step",
    "hp2d_cfl_dt", "hp2d_track_maxima", "hp2d_fused_steps", "hp2d_fused_steps_timed",
    "hp2d_set_tuning", "hp2d_set_layout", "hp2d_run",
    "hp2d_set_retry_policy", "hp2d_set_wait_limit", "hp2d_inject_step_fault", "hp2d_set_temporal_blocking",
    "hp2d_set_owned_rows", "hp2d_step_maxima", "hp2d_apply_refresh", "hp2d_copy_rows",
    "hp2d_download",
    "hp2d_download_native", "hp2d_get_diag", "hp2d_stored_volume",
    "hp2d_cfl_dt_noalloc", "hp2d_noalloc_error",
    "hp2d_autotune",
    "hp2d_ensemble_create", "hp2d_ensemble_destroy", "hp2d_ensemble_last_error",
    "hp2d_ensemble_add", "hp2d_ensemble_set_tuning", "hp2d_ensemble_set_layout", "hp2d_ensemble_autotune",
    "hp2d_ensemble_steps", "hp2d_ensemble_steps_timed", "hp2d_ensemble_run",
]


# every symbol include/hp2d_nn.h declares (the learned screening network's kernels)
NN_EXPORTS = [
    "hp2d_nn_gemm", "hp2d_nn_conv3x3", "hp2d_nn_check", "hp2d_nn_error", "hp2d_nn_im2col3x3", "hp2d_nn_transpose",
    "hp2d_nn_maxpool2", "hp2d_nn_maxpool2_bwd", "hp2d_nn_upsample2", "hp2d_nn_upsample2_bwd",
    "hp2d_nn_copy_channels", "hp2d_nn_relu_bwd", "hp2d_nn_colsum", "hp2d_nn_mse", "hp2d_nn_adam",
    "hp2d_nn_flip3x3", "hp2d_nn_f32_to_bf16",
]

NN_EPI = {"f32": 0, "f32_atomic": 1, "bf16_bias_relu": 2, "bf16_bias": 3, "f32_bias": 4}


class Grid(C.Structure):
    _fields_ = [("ny", C.c_int32), ("nx", C.c_int32), ("resolution", C.c_double),
                ("precision", C.c_int32)]


class Params(C.Structure):
    _fields_ = [
        ("flag_numerical_scheme", C.c_int32), ("flag_critical", C.c_int32),
        ("flag_subgrid", C.c_int32), ("flag_D8", C.c_int32), ("flag_reservoir", C.c_int32),
        ("flag_infiltration", C.c_int32), ("flag_timestep", C.c_int32),
        ("flag_adaptive_timestepping", C.c_int32), ("outlet_type", C.c_int32),
        ("slope_outlet", C.c_double), ("min_time_step", C.c_double),
        ("max_time_step", C.c_double), ("time_step_increments", C.c_double),
        ("time_step_change", C.c_double), ("routing_time", C.c_double),
        ("alfa_min", C.c_double), ("alfa_max", C.c_double), ("depth_tolerance", C.c_double),
        ("arrival_threshold", C.c_double),
    ]


class Diag(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("time_step", C.c_double), ("k", C.c_int64),
        ("max_velocity", C.c_double), ("rain_volume", C.c_double),
        ("infiltration_volume", C.c_double), ("outlet_volume", C.c_double),
        ("neg_depth_warnings", C.c_int64), ("unstable_steps", C.c_int64),
        ("status_bits", C.c_int64),
        ("rain_t0", C.c_double), ("rain_t1", C.c_double), ("t_previous", C.c_double),
        ("inflow_volume", C.c_double), ("stage_volume", C.c_double),
        ("structure_volume", C.c_double), ("skipped_cells", C.c_int64), ("skipped_read_cells", C.c_int64),
        ("retries", C.c_int64), ("catch_index", C.c_int32), ("steps_per_block", C.c_int32), ("max_time_step", C.c_double),
    ]


def default_params(**kw) -> Params:
    """Reference defaults (Config/input_data_bypass_script.m:160-170, :330-380)."""
    d = dict(flag_numerical_scheme=1, flag_critical=0, flag_subgrid=0, flag_D8=0,
             flag_reservoir=0, flag_infiltration=0, flag_timestep=1,
             flag_adaptive_timestepping=1, outlet_type=1, slope_outlet=0.0,
             min_time_step=0.01, max_time_step=10.0, time_step_increments=0.001,
             time_step_change=0.0001, routing_time=60.0, alfa_min=0.5, alfa_max=0.5,
             depth_tolerance=1.0, arrival_threshold=10.0)
    unknown = set(kw) - set(d)
    if unknown:
        raise TypeError(f"unknown hp2d_params fields: {sorted(unknown)}")
    d.update(kw)
    return Params(**d)


_lib = None


def lib() -> C.CDLL:
    """The loaded libhp2d.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m hydropol2d_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    P = C.POINTER
    vp = C.c_void_p
    dp = P(C.c_double)
    i32p = P(C.c_int32)
    sig = {
        "hp2d_create": ([P(Grid), P(Params), C.c_int32, P(vp)], C.c_int),
        "hp2d_destroy": ([vp], C.c_int),
        "hp2d_last_error": ([vp], C.c_char_p),
        "hp2d_create_error": ([], C.c_char_p),
        "hp2d_upload_static": ([vp, dp, dp, i32p, i32p, C.c_int32, dp], C.c_int),
        "hp2d_set_soil": ([vp, P(C.c_uint8), C.c_int32, dp, dp, dp, dp, dp, dp, dp], C.c_int),
        "hp2d_set_soil_vg": ([vp, P(C.c_uint8), C.c_int32, dp, dp, dp, dp, dp, dp, dp, C.c_double, C.c_double,
                              C.c_double, C.c_double], C.c_int),
        "hp2d_set_state": ([vp, dp, dp, dp], C.c_int),
        "hp2d_set_clock": ([vp, C.c_double, C.c_double, C.c_int64], C.c_int),
        "hp2d_set_rain_clock": ([vp, C.c_double, C.c_double, C.c_double], C.c_int),
        "hp2d_set_map_records": ([vp, C.c_int32, P(C.c_double), C.c_int32], C.c_int),
        "hp2d_set_map_records_host": ([vp, C.c_int32, P(C.c_double), C.c_int32], C.c_int),
        "hp2d_set_stage": ([vp, C.c_int32, C.c_int32, P(C.c_double), P(C.c_double), C.c_int32,
                            P(C.c_int32), P(C.c_int32), P(C.c_int32)], C.c_int),
        "hp2d_set_hazard_tracking": ([vp, C.c_int32], C.c_int),
        "hp2d_set_dry_skip": ([vp, C.c_int32], C.c_int),
        "hp2d_set_reservoirs": ([vp, C.c_int32, P(C.c_int32), P(C.c_int32), P(C.c_double), P(C.c_double),
                                 P(C.c_double), P(C.c_int32), P(C.c_int32), P(C.c_double), P(C.c_double),
                                 P(C.c_double), P(C.c_int32), P(C.c_int32)], C.c_int),
        "hp2d_set_rain_gauges": ([vp, C.c_int32, P(C.c_double), P(C.c_double), C.c_int32, C.c_double,
                                  P(C.c_double), C.c_double, C.c_double], C.c_int),
        "hp2d_map_records": ([vp, P(C.c_int64)], C.c_int),
        "hp2d_download_map_record": ([vp, C.c_int64, P(C.c_double), P(C.c_double)], C.c_int),
        "hp2d_set_inflow": ([vp, C.c_int32, C.c_int32, P(C.c_double), P(C.c_double), C.c_int32,
                             P(C.c_int32), P(C.c_int32), P(C.c_int32)], C.c_int),
        "hp2d_set_rain_uniform": ([vp, C.c_int32, dp, dp], C.c_int),
        "hp2d_set_rain_maps": ([vp, C.c_int32, C.c_int32, C.c_int32, P(C.c_float), C.c_double], C.c_int),
        "hp2d_set_rain_maps_end_stamped": ([vp, C.c_int32, C.c_int32, C.c_int32, P(C.c_float), P(C.c_double),
                                            C.c_double], C.c_int),
        "hp2d_hydrology_step": ([vp, C.c_double], C.c_int),
        "hp2d_li_step": ([vp, C.c_double], C.c_int),
        "hp2d_cfl_dt": ([vp, dp, dp], C.c_int),
        "hp2d_track_maxima": ([vp, C.c_double], C.c_int),
        "hp2d_fused_steps": ([vp, C.c_int32], C.c_int),
        "hp2d_fused_steps_timed": ([vp, C.c_int32, P(C.c_float)], C.c_int),
        "hp2d_set_tuning": ([vp, C.c_int32], C.c_int),
        "hp2d_set_layout": ([vp, C.c_int32], C.c_int),
        "hp2d_run": ([vp, C.c_int64, P(C.c_int64)], C.c_int),
        "hp2d_set_retry_policy": ([vp, C.c_int32, C.c_double, C.c_int32], C.c_int),
        "hp2d_set_wait_limit": ([vp, C.c_int64], C.c_int),
        "hp2d_inject_step_fault": ([vp, C.c_int64, C.c_int32], C.c_int),
        "hp2d_set_temporal_blocking": ([vp, C.c_int32], C.c_int),
        "hp2d_set_owned_rows": ([vp, C.c_int32, C.c_int32], C.c_int),
        "hp2d_step_maxima": ([vp, P(C.c_uint64), P(C.c_uint64), P(C.c_int32)], C.c_int),
        "hp2d_apply_refresh": ([vp, C.c_uint64, C.c_uint64, C.c_int32], C.c_int),
        "hp2d_copy_rows": ([vp, C.c_int32, C.c_int32, vp, C.c_int32], C.c_int),
        "hp2d_download": ([vp, C.c_int32, dp, C.c_size_t], C.c_int),
        "hp2d_download_native": ([vp, C.c_int32, vp, C.c_size_t], C.c_int),
        "hp2d_get_diag": ([vp, P(Diag)], C.c_int),
        "hp2d_stored_volume": ([vp, dp], C.c_int),
        "hp2d_cfl_dt_noalloc": ([C.c_int32, C.c_int32, C.c_double, P(Params), vp, vp, vp, vp, dp, dp], C.c_int),
        "hp2d_noalloc_error": ([], C.c_char_p),
        "hp2d_autotune": ([vp, C.c_int32, P(C.c_int32)], C.c_int),
        "hp2d_ensemble_create": ([C.c_int32, P(vp)], C.c_int),
        "hp2d_ensemble_destroy": ([vp], C.c_int),
        "hp2d_ensemble_last_error": ([vp], C.c_char_p),
        "hp2d_ensemble_add": ([vp, vp], C.c_int),
        "hp2d_ensemble_set_tuning": ([vp, C.c_int32], C.c_int),
        "hp2d_ensemble_set_layout": ([vp, C.c_int32], C.c_int),
        "hp2d_ensemble_autotune": ([vp, C.c_int32, P(C.c_int32)], C.c_int),
        "hp2d_ensemble_steps": ([vp, C.c_int32, P(C.c_int32)], C.c_int),
        "hp2d_ensemble_steps_timed": ([vp, C.c_int32, P(C.c_int32), P(C.c_float)], C.c_int),
        "hp2d_ensemble_run": ([vp, C.c_int64, P(C.c_int64)], C.c_int),
    }
    i32, i64, f32 = C.c_int32, C.c_int64, C.c_float
    sig.update({
        "hp2d_nn_gemm": ([i32, i32, i32, vp, i32, vp, i32, vp, i32, vp, i32, i32, vp], C.c_int),
        "hp2d_nn_conv3x3": ([vp, i32, i32, i32, i32, vp, i32, i32, vp, vp, i32, i32, vp], C.c_int),
        "hp2d_nn_check": ([], C.c_int),
        "hp2d_nn_error": ([], C.c_char_p),
        "hp2d_nn_im2col3x3": ([vp, i32, i32, i32, i32, vp, i32, i32, vp], C.c_int),
        "hp2d_nn_transpose": ([vp, i32, i32, i32, vp, i32, vp], C.c_int),
        "hp2d_nn_maxpool2": ([vp, i32, i32, i32, i32, vp, vp], C.c_int),
        "hp2d_nn_maxpool2_bwd": ([vp, vp, vp, i32, i32, i32, i32, vp, i32, vp], C.c_int),
        "hp2d_nn_upsample2": ([vp, i32, i32, i32, i32, vp, vp], C.c_int),
        "hp2d_nn_upsample2_bwd": ([vp, i32, i32, i32, i32, vp, vp], C.c_int),
        "hp2d_nn_copy_channels": ([vp, i32, i32, i32, i64, vp, i32, i32, vp], C.c_int),
        "hp2d_nn_relu_bwd": ([vp, vp, i64, vp], C.c_int),
        "hp2d_nn_colsum": ([vp, i64, i32, i32, vp, vp], C.c_int),
        "hp2d_nn_mse": ([vp, i32, vp, vp, i64, i32, f32, vp, vp, i32, vp], C.c_int),
        "hp2d_nn_adam": ([vp, vp, vp, vp, vp, i64, f32, f32, f32, f32, f32, i32, vp], C.c_int),
        "hp2d_nn_flip3x3": ([vp, i32, i32, i32, vp, i32, vp], C.c_int),
        "hp2d_nn_f32_to_bf16": ([vp, vp, i64, vp], C.c_int),
    })
    for name, (args, res) in sig.items():
        try:
            f = getattr(L, name)
        except AttributeError:
            if os.environ.get("HP2D_LIBRARY"):   # another build for A/B timing: bind what it has
                continue
            raise
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


class HP2DError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        self.status_name = STATUS.get(status, str(status))
        super().__init__(f"{self.status_name}: {message}")
