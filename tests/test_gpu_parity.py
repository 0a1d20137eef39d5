"""CUDA library vs the kernel-form oracle, bit for bit (FP32 and FP64), through the C ABI.

The oracle (oracle/kernel_form.hpp) restates Local_Inertial_Model_D4.m,
Inertial_Solver.m, the Green-Ampt capacity of HydroPol2D_Main_While_Ensemble.m:274-298
at the Infiltration_Module boundary and refreshing_timestep.m; these tests require the
GPU to produce the same bits for every state field, the same timestep sequence and the
same clock.
"""
import numpy as np
import pytest

from tests.cases import random_terrain, small_dambreak, small_urban, small_vtilt
from tests.conftest import first_mismatch, same_bits

pytestmark = pytest.mark.gpu

FIELDS = ["h", "qx", "qy", "dmax", "arrival"]


def make_pair(case, precision):
    import oracle
    from hydropol2d_b200 import SurfaceFlow
    g = SurfaceFlow(*case.shape, case.resolution, precision, **case.params)
    o = oracle.KernelFormOracle(*case.shape, case.resolution, precision, **case.params)
    case.apply(g)
    case.apply(o)
    return g, o


def assert_same_state(g, o, fields, where=""):
    for f in fields:
        a = g.download_native(f)
        b = o.download_native(f)
        assert same_bits(a, b), f"{where} field {f}: first mismatch {first_mismatch(a, b)}"


def assert_same_clock(g, o):
    dg, do = g.diag(), o.diag()
    for k in ("t", "time_step", "k", "max_velocity", "neg_depth_warnings", "unstable_steps"):
        assert dg[k] == do[k], f"{k}: gpu {dg[k]} oracle {do[k]}"
    # the volume ledger is a diagnostic: per-lane partial sums are kept in the state
    # precision and summed in a different order than the oracle's sequential FP64 sum
    rel = 1e-5 if g.precision == "fp32" else 1e-9
    for k in ("rain_volume", "infiltration_volume", "outlet_volume"):
        assert dg[k] == pytest.approx(do[k], rel=rel, abs=1e-9), k


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_fused_vtilt_bit_exact(precision, hp2d_lib, oracle_lib):
    case = small_vtilt(40, 40)
    g, o = make_pair(case, precision)
    for chunk in (1, 7, 40, 33, 64):  # single launches and CUDA-graph replays
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS, f"after chunk {chunk}")
        assert_same_clock(g, o)


@pytest.mark.parametrize("shape", [(37, 41), (16, 64), (17, 65), (33, 130), (5, 300)])
def test_fused_ragged_shapes_bit_exact(shape, hp2d_lib, oracle_lib):
    case = random_terrain(*shape, seed=sum(shape), walls=True)
    g, o = make_pair(case, "fp32")
    for chunk in (1, 3, 40):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS, f"{shape} chunk {chunk}")
        assert_same_clock(g, o)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_fused_urban_green_ampt_bit_exact(precision, hp2d_lib, oracle_lib):
    case = small_urban(96, seed=3)
    g, o = make_pair(case, precision)
    for chunk in (1, 50, 100):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS + ["I", "T"], f"chunk {chunk}")
        assert_same_clock(g, o)


def test_fused_dambreak_bit_exact(hp2d_lib, oracle_lib):
    case = small_dambreak(64, 256)
    g, o = make_pair(case, "fp32")
    g.fused_steps(120)
    o.fused_steps(120)
    assert_same_state(g, o, FIELDS)
    assert_same_clock(g, o)
    assert same_bits(g.download_native("qo"), o.download_native("qo"))
    assert same_bits(g.download_native("hf3"), o.download_native("hf3"))


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_unfused_stages_bit_exact(precision, hp2d_lib, oracle_lib):
    """hp2d_hydrology_step / hp2d_li_step / hp2d_cfl_dt / hp2d_track_maxima, as a MATLAB
    caller would sequence them (HydroPol2D_Main_While.m:424, :596-615, :705, :749)."""
    case = small_urban(64, seed=9)
    g, o = make_pair(case, precision)
    ts = case.params["min_time_step"] / 60
    t = case.params["min_time_step"] / 60
    for k in range(60):
        g.set_clock(t, ts, k + 1)
        o.set_clock(t, ts, k + 1)
        g.hydrology_step(ts)
        o.hydrology_step(ts)
        assert_same_state(g, o, ["h", "I", "T"], f"hydrology {k}")
        g.li_step(ts)
        o.li_step(ts)
        assert_same_state(g, o, ["h", "qx", "qy", "hfx", "hfy", "qo", "hf3"], f"li {k}")
        tg, vg = g.cfl_dt()
        to, vo = o.cfl_dt()
        assert (tg, vg) == (to, vo), k
        g.track_maxima(t + ts)
        o.track_maxima(t + ts)
        assert_same_state(g, o, ["dmax", "arrival"], f"track {k}")
        t = tg + t
        ts = tg


def test_fused_equals_unfused_sequence(hp2d_lib):
    """The fused kernel and the unfused stage kernels agree bit for bit on the GPU."""
    from hydropol2d_b200 import SurfaceFlow
    case = random_terrain(48, 80, seed=4)
    a = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    b = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(a)
    case.apply(b)
    for _ in range(25):
        d = b.diag()
        t, ts, k = d["t"], d["time_step"], d["k"]
        b.hydrology_step(ts)
        b.li_step(ts)
        new_ts, _ = b.cfl_dt()
        b.track_maxima(t + ts)
        b.set_clock(new_ts + t, new_ts, k + 1)
        a.fused_steps(1)
        for f in FIELDS:
            assert same_bits(a.download_native(f), b.download_native(f)), f
        assert a.diag()["t"] == b.diag()["t"]


def test_vtilt_mirror_symmetry_exact(hp2d_lib):
    """V-tilted symmetry gate of run_local_inertial_ca_hydrodynamics_validation.m:197
    (RMSE < 1e-8 m); the FP32 kernels keep it exactly."""
    from hydropol2d_b200 import SurfaceFlow
    case = small_vtilt(60, 50)
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    g.fused_steps(300)
    h = g.download_native("h")
    assert np.array_equal(h, h[:, ::-1])
    assert h.max() > 0


def test_capi_errors(hp2d_lib):
    from hydropol2d_b200 import HP2DError, SurfaceFlow
    g = SurfaceFlow(8, 8, 1.0, "fp32")
    with pytest.raises(HP2DError) as e:
        g.cfl_dt()
    assert e.value.status_name == "HP2D_NOT_READY"
    with pytest.raises(HP2DError):
        g.fused_steps(1)  # static data missing
    with pytest.raises(HP2DError) as e:
        g.upload_static(np.zeros((8, 8)), np.full((8, 8), 0.03), [9], [0])
    assert e.value.status_name == "HP2D_INVALID_ARG"
