"""The MATLAB-signature mirror (hydropol2d_b200.reference_api) against the literal FP64
restatement of the same functions, called the way HydroPol2D_Main_While calls them
(Local_Inertial_Model_D4 at HydroPol2D_Main_While.m:596-615, refreshing_timestep at :705).
"""
import math

import numpy as np
import pytest

from tests.cases import random_terrain


def _lim_args(case, d_tot, outflow, time_step, outlet_type=1):
    """The 45 positional arguments of Local_Inertial_Model_D4.m:1-5 (MATLAB layout)."""
    ny, nx = case.z.shape
    res = case.resolution
    n = case.roughness
    empty = np.zeros(0)
    return (1, empty, empty, empty, empty, empty, empty, empty, empty, empty, empty, empty, empty,
            0, case.z, d_tot, d_tot, n, n ** 2, res * res, time_step, res,
            np.zeros((ny, nx), bool), outlet_type, case.params["slope_outlet"],
            case.outlet_rows + 1, case.outlet_cols + 1, 1.0, outflow, np.isnan(case.z), 0, 0,
            0, 0, 0, 0, 0, 0, 0, 0, res * res, None, 0, 0, None)


def test_unsupported_flags_raise_before_device():
    from hydropol2d_b200 import HP2DError, reference_api
    case = random_terrain(8, 8, seed=1)
    args = list(_lim_args(case, case.d0, np.zeros((8, 8, 3)), 0.01))
    for pos, v in ((0, 4), (13, 2), (31, 1)):   # flag_numerical_scheme=4, flag_reservoir=2, flag_subgrid=1
        bad = list(args)
        bad[pos] = v
        with pytest.raises(HP2DError) as e:
            reference_api.Local_Inertial_Model_D4(*bad)
        assert e.value.status_name == "HP2D_UNSUPPORTED_FLAG"


def test_roughness_squared_must_match():
    from hydropol2d_b200 import reference_api
    case = random_terrain(8, 8, seed=1)
    args = list(_lim_args(case, case.d0, np.zeros((8, 8, 3)), 0.01))
    args[18] = args[18] * 1.01
    with pytest.raises(ValueError):
        reference_api.Local_Inertial_Model_D4(*args)


@pytest.mark.gpu
@pytest.mark.parametrize("outlet_type", [1, 2])
def test_local_inertial_model_d4_matches_literal(outlet_type):
    """Two chained calls (the second with the fluxes of the first as outflow_prev), FP64,
    against oracle/literal.local_inertial_model_d4.  The library evaluates the algebraically
    identical kernel form, so agreement is to round-off."""
    from hydropol2d_b200 import reference_api
    from oracle import literal
    case = random_terrain(37, 45, seed=4, walls=True)
    ny, nx = case.z.shape
    d = case.d0.copy()
    outflow = np.zeros((ny, nx, 3))
    d_lit = d.copy()
    of_lit = np.zeros((3, ny, nx))
    for time_step in (0.02, 0.015):
        got = reference_api.Local_Inertial_Model_D4(*_lim_args(case, d, outflow, time_step, outlet_type))
        ref = literal.local_inertial_model_d4(
            case.z, d_lit, case.roughness, case.roughness ** 2, case.resolution ** 2, time_step,
            case.resolution, case.outlet_rows, case.outlet_cols, outlet_type,
            case.params["slope_outlet"], of_lit)
        q_l, q_r, q_u, q_d, o_f, d_t, i_tot, out, Hf = got[:9]
        pairs = [(d_t, ref.d_t, 1e-9), (q_r, ref.qout_right, 1e-6), (q_u, ref.qout_up, 1e-6),
                 (q_l, ref.qout_left, 1e-6), (q_d, ref.qout_down, 1e-6),
                 (o_f, ref.outlet_flow, 1e-6), (i_tot, ref.I_tot_end_cell, 1e-9),
                 (np.moveaxis(out, 2, 0), ref.outflow, 1e-6), (np.moveaxis(Hf, 2, 0), ref.Hf, 1e-12)]
        for a, b, atol in pairs:
            fin = np.isfinite(b)
            assert np.array_equal(np.isfinite(a), fin)
            np.testing.assert_allclose(a[fin], b[fin], rtol=1e-9, atol=atol)
        assert got[9:13] == (0, 0, 0, 0) and got[13] == case.resolution ** 2
        d, outflow = d_t, out
        d_lit, of_lit = ref.d_t, ref.outflow


@pytest.mark.gpu
def test_refreshing_timestep_matches_literal():
    """The FP32 device reduction against the FP64 literal script: the new step agrees to
    one time_step_increments (the floor snap can fall either side of a boundary the FP32
    rounding moves), the maximum velocity to FP32 round-off."""
    from hydropol2d_b200 import reference_api
    from oracle import literal
    case = random_terrain(64, 96, seed=7)
    ny, nx = case.z.shape
    ref_li = literal.local_inertial_model_d4(
        case.z, case.d0, case.roughness, case.roughness ** 2, case.resolution ** 2, 0.02,
        case.resolution, case.outlet_rows, case.outlet_cols, 1, case.params["slope_outlet"],
        np.zeros((3, ny, nx)))
    kw = dict(depth_tolerance=1.0, alfa_min=0.5, alfa_max=0.7, max_time_step=10.0,
              min_time_step=0.01, time_step_increments=0.001)
    Hf = np.moveaxis(ref_li.Hf, 0, 2)
    tcr, ts, vmax = reference_api.refreshing_timestep(Hf, ref_li.qout_right, ref_li.qout_up,
                                                      case.resolution, **kw)
    lit = literal.refreshing_timestep(ref_li.Hf, ref_li.qout_right, ref_li.qout_up,
                                      case.resolution, **kw)
    assert vmax > 0
    assert math.isclose(vmax, lit.max_velocity, rel_tol=2e-6)
    assert abs(tcr - lit.time_calculation_routing) <= 0.001 + 1e-12
    assert math.isclose(ts, tcr / 60, rel_tol=1e-15)


@pytest.mark.gpu
def test_local_inertial_model_d4_with_reservoirs_matches_literal():
    """flag_reservoir = 1 through the MATLAB signature: 1-based reservoir tables with NaN for
    a missing downstream cell, two chained calls, FP64, against the literal restatement."""
    from hydropol2d_b200 import reference_api
    from oracle import literal
    case = random_terrain(30, 36, seed=7)
    ny, nx = case.z.shape
    d = case.d0.copy()
    d[10, 10] = 900.0
    d[20, 5] = 400.0
    tab = dict(res_row=np.array([10, 20]), res_col=np.array([10, 5]), k1=np.array([2.0, 0.7]),
               h1=np.array([0.3, 0.1]), k2=np.array([1.5, 2.0]), ds1_row=np.array([12, 10]),
               ds1_col=np.array([14, 14]), k3=np.array([1.0, 0.0]), h2=np.array([0.5, 0.0]),
               k4=np.array([2.5, 0.0]), ds2_row=np.array([8.0, np.nan]), ds2_col=np.array([3.0, np.nan]))
    outflow = np.zeros((ny, nx, 3))
    d_lit, of_lit = d.copy(), np.zeros((3, ny, nx))
    for time_step in (0.02, 0.015):
        args = list(_lim_args(case, d, outflow, time_step))
        args[1], args[2] = tab["res_col"] + 1, tab["res_row"] + 1          # reservoir_x, reservoir_y
        args[3], args[4], args[5] = tab["k1"], tab["h1"], tab["k2"]
        args[6], args[7], args[8] = tab["k3"], tab["h2"], tab["k4"]
        args[9], args[10] = tab["ds1_row"] + 1, tab["ds1_col"] + 1         # yds1, xds1
        args[11], args[12] = tab["ds2_row"] + 1, tab["ds2_col"] + 1        # yds2, xds2 (NaN stays)
        args[13] = 1
        got = reference_api.Local_Inertial_Model_D4(*args)
        ref = literal.local_inertial_model_d4(
            case.z, d_lit, case.roughness, case.roughness ** 2, case.resolution ** 2, time_step,
            case.resolution, case.outlet_rows, case.outlet_cols, 1, case.params["slope_outlet"], of_lit,
            reservoirs=tab)
        fin = np.isfinite(ref.d_t)
        np.testing.assert_allclose(got[5][fin], ref.d_t[fin], rtol=1e-9, atol=1e-9)
        plain = literal.local_inertial_model_d4(
            case.z, d_lit, case.roughness, case.roughness ** 2, case.resolution ** 2, time_step,
            case.resolution, case.outlet_rows, case.outlet_cols, 1, case.params["slope_outlet"], of_lit)
        if time_step == 0.02:   # the first call moves water (the steep cells drain below the crests)
            assert np.nanmax(np.abs(ref.d_t - plain.d_t)) > 1.0
        d, outflow = got[5], got[7]
        d_lit, of_lit = ref.d_t, ref.outflow
