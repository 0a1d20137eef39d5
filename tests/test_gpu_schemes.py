"""Inertial_Solver's schemes 2 (s-upwind) and 3 (s-centred) (Inertial_Solver.m:29-121) and the
critical-velocity clip of Local_Inertial_Model_D4.m:272-275 (flag_critical = 1) on the GPU:
bit for bit against the kernel-form oracle in FP32 and FP64, on the fused step (single launches
and CUDA-graph replays, both strip layouts), the unfused hp2d_li_step, and ensemble members;
and through the MATLAB-signature mirror against the literal FP64 restatement.
"""
import numpy as np
import pytest

from tests.cases import random_terrain, small_dambreak, small_urban
from tests.conftest import same_bits
from tests.test_gpu_parity import FIELDS, assert_same_clock, assert_same_state, make_pair

pytestmark = pytest.mark.gpu


def with_params(case, **kw):
    case.params = dict(case.params, **kw)
    return case


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("scheme", [2, 3])
def test_fused_dambreak_schemes_bit_exact(precision, scheme, hp2d_lib, oracle_lib):
    case = with_params(small_dambreak(64, 256), flag_numerical_scheme=scheme)
    g, o = make_pair(case, precision)
    for chunk in (1, 7, 40, 64):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS, f"scheme {scheme} chunk {chunk}")
        assert_same_clock(g, o)
    assert same_bits(g.download_native("qo"), o.download_native("qo"))


@pytest.mark.parametrize("layout", [1, 2])
@pytest.mark.parametrize("scheme", [2, 3])
def test_fused_schemes_ragged_walls_layouts(layout, scheme, hp2d_lib, oracle_lib):
    """Ragged shapes with NaN walls, strips of 32 and 64 columns (the strip's first lane reads
    its left neighbour's previous flux from memory) and short row blocks."""
    for shape in ((37, 41), (17, 130), (70, 61)):
        case = with_params(random_terrain(*shape, seed=sum(shape) + scheme, walls=True), flag_numerical_scheme=scheme)
        g, o = make_pair(case, "fp32")
        g.set_layout(layout)
        g.set_tuning(8)
        for chunk in (1, 3, 36):
            g.fused_steps(chunk)
            o.fused_steps(chunk)
            assert_same_state(g, o, FIELDS, f"{shape} layout {layout} chunk {chunk}")
            assert_same_clock(g, o)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_fused_urban_scheme3_green_ampt(precision, hp2d_lib, oracle_lib):
    case = with_params(small_urban(96, seed=4), flag_numerical_scheme=3)
    g, o = make_pair(case, precision)
    g.fused_steps(80)
    o.fused_steps(80)
    assert_same_state(g, o, FIELDS + ["I", "T"])
    assert_same_clock(g, o)


@pytest.mark.parametrize("scheme", [1, 2, 3])
def test_critical_clip_bit_exact(scheme, hp2d_lib, oracle_lib):
    """flag_critical = 1 on a steep dam-break: the clip binds (the run differs from the one
    without it) and the GPU reproduces the oracle."""
    base = small_dambreak(48, 192, seed=6)
    base.z = base.z * 4.0
    case = with_params(base, flag_critical=1, flag_numerical_scheme=scheme)
    g, o = make_pair(case, "fp32")
    g.fused_steps(90)
    o.fused_steps(90)
    assert_same_state(g, o, FIELDS)
    assert_same_clock(g, o)
    free = with_params(small_dambreak(48, 192, seed=6), flag_critical=0, flag_numerical_scheme=scheme)
    free.z = free.z * 4.0
    f, _ = make_pair(free, "fp32")
    f.fused_steps(90)
    assert not same_bits(f.download_native("h"), g.download_native("h"))


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("scheme,critical", [(2, 0), (3, 1)])
def test_unfused_li_step_schemes(precision, scheme, critical, hp2d_lib, oracle_lib):
    case = with_params(random_terrain(40, 52, seed=12, walls=True), flag_numerical_scheme=scheme,
                       flag_critical=critical)
    g, o = make_pair(case, precision)
    g.fused_steps(20)
    o.fused_steps(20)
    for k in range(15):
        ts = g.diag()["time_step"]
        g.hydrology_step(ts)
        o.hydrology_step(ts)
        g.li_step(ts)
        o.li_step(ts)
        assert_same_state(g, o, ["h", "qx", "qy", "hfx", "hfy"], f"li {k}")
        assert g.cfl_dt() == o.cfl_dt()


def test_ensemble_members_scheme2_equal_solo(hp2d_lib):
    """Members running scheme 2 in the batched persistent kernel give the bits of solo runs."""
    from hydropol2d_b200 import SurfaceFlow
    from hydropol2d_b200.ensemble import Ensemble
    cases = [with_params(small_dambreak(48 + 16 * i, 160 + 32 * i, seed=20 + i), flag_numerical_scheme=2)
             for i in range(3)]
    ens = Ensemble()
    members, solos = [], []
    for c in cases:
        m = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        s = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(m)
        c.apply(s)
        ens.add(m)
        members.append(m)
        solos.append(s)
    ens.steps(70)
    for m, s in zip(members, solos):
        s.fused_steps(70)
        for f in FIELDS:
            assert same_bits(m.download_native(f), s.download_native(f)), f
    ens.close()


def test_ensemble_rejects_mixed_schemes(hp2d_lib):
    from hydropol2d_b200 import HP2DError, SurfaceFlow
    from hydropol2d_b200.ensemble import Ensemble
    a = with_params(small_dambreak(32, 96, seed=1), flag_numerical_scheme=1)
    b = with_params(small_dambreak(32, 96, seed=2), flag_numerical_scheme=3)
    ens = Ensemble()
    for c in (a, b):
        m = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(m)
        ens.add(m)
    with pytest.raises(HP2DError) as e:
        ens.steps(1)
    assert e.value.status_name == "HP2D_INVALID_ARG"
    ens.close()


@pytest.mark.parametrize("scheme,critical", [(2, 0), (3, 0), (2, 1)])
def test_reference_api_schemes_against_literal(scheme, critical, hp2d_lib):
    """The MATLAB-signature mirror with flag_numerical_scheme / flag_critical (FP64 build)
    against the literal restatement of Local_Inertial_Model_D4 + Inertial_Solver."""
    from hydropol2d_b200 import reference_api
    from oracle import literal as L
    from tests.test_reference_api import _lim_args
    case = random_terrain(30, 44, seed=31, walls=True)
    rng = np.random.default_rng(5)
    ny, nx = case.shape
    outflow = np.zeros((ny, nx, 3))
    outflow[..., 0] = rng.normal(0, 3e4, (ny, nx))
    outflow[..., 1] = rng.normal(0, 3e4, (ny, nx))
    outflow[:, -1, 0] = 0
    outflow[0, :, 1] = 0
    d = np.where(np.isnan(case.z), np.nan, rng.uniform(0, 400, (ny, nx)))
    ts = 1.0 / 60
    args = list(_lim_args(case, d, outflow, ts))
    args[0] = scheme
    args[30] = critical
    out = reference_api.Local_Inertial_Model_D4(*args)
    lit = L.local_inertial_model_d4(case.z, d, case.roughness, case.roughness ** 2, case.resolution ** 2, ts,
                                    case.resolution, case.outlet_rows, case.outlet_cols, 1,
                                    case.params["slope_outlet"], np.moveaxis(outflow, -1, 0),
                                    flag_numerical_scheme=scheme, flag_critical=critical)
    assert np.allclose(out[5], lit.d_t, rtol=1e-10, atol=1e-9, equal_nan=True)
    assert np.allclose(out[1], lit.qout_right, rtol=1e-9, atol=1e-7)
    assert np.allclose(out[2], lit.qout_up, rtol=1e-9, atol=1e-7)
    reference_api.close_sessions()
