"""The kernel-form restatement (oracle/kernel_form.hpp, FP64) against the literal one
(oracle/literal.py): the rewrites listed in kernel_form.hpp are algebraically exact, so the two
agree to round-off; the full loop agrees until a timestep-snapping tie (floor(dt/inc)) flips.
"""
import numpy as np
import pytest

from oracle import literal as L
from tests.cases import random_terrain, small_urban, small_vtilt


def literal_cfg(case):
    p = case.params
    kw = dict(z=case.z, roughness=case.roughness, resolution=case.resolution, outlet_rows=case.outlet_rows,
              outlet_cols=case.outlet_cols, outlet_type=p.get("outlet_type", 1),
              slope_outlet=p.get("slope_outlet", 0.0), d0=case.d0, routing_time=p["routing_time"],
              alfa_min=p["alfa_min"], alfa_max=p["alfa_max"])
    if case.rain_uniform is not None:
        kw["rain_times_min"], kw["rain_rates_mmh"] = case.rain_uniform
    if case.rain_maps is not None:
        kw["rain_maps_mmh"] = case.rain_maps.astype(np.float64)
        kw["rain_map_dt_min"] = case.rain_map_dt
    if case.soil is not None:
        s = case.soil
        cls = s["soil_class"]
        act = cls != 255
        c = np.where(act, cls, 0)
        kw["ga"] = L.GAParams(ksat=s["ksat"][c], psi=s["psi"][c], dtheta=s["dtheta"][c], Lu=s["Lu"][c],
                              k_out=s["k_out"][c], Tr=s["Tr"][c], min_sm=s["min_soil_moisture"][c], active=act)
        kw["I0"] = case.I0
    if case.inflow is not None:
        f = case.inflow
        masks = np.zeros((np.asarray(f["rates"]).reshape(len(f["t_start"]), -1).shape[1],) + case.shape)
        for r, c, g in zip(f["rows"], f["cols"], f["gauge"]):
            masks[g, r, c] += 1.0
        kw["inflow_times_min"], kw["inflow_rates_mmh"], kw["inflow_cells"] = f["t_start"], f["rates"], masks
    stage = getattr(case, "stage", None)
    if stage is not None:
        d = np.asarray(stage["depth_m"]).reshape(len(stage["t_start"]), -1)
        masks = np.zeros((d.shape[1],) + case.shape)
        for r, c, g in zip(stage["rows"], stage["cols"], stage["gauge"]):
            masks[g, r, c] = 1.0
        kw["stage_times_min"], kw["stage_depth_m"], kw["stage_cells"] = stage["t_start"], d, masks
    if getattr(case, "reservoirs", None) is not None:
        kw["reservoirs"] = {k: np.asarray(v, dtype=np.float64) for k, v in case.reservoirs.items()}
    return L.RunConfig(**kw)


def kernel_form(case):
    import oracle
    o = oracle.KernelFormOracle(*case.shape, case.resolution, "fp64", **case.params)
    case.apply(o)
    return o


def test_full_loop_vtilt_agrees(oracle_lib):
    case = small_vtilt(40, 40)
    cfg = literal_cfg(case)
    st = L.init_state(cfg)
    o = kernel_form(case)
    for k in range(200):
        L.step(cfg, st)
        o.fused_steps(1)
        d = o.diag()
        assert d["time_step"] == pytest.approx(st.time_step, rel=1e-12)
        assert d["t"] == pytest.approx(st.t, rel=1e-12)
        h = o.download_native("h") * 1000
        assert np.allclose(h, st.d, rtol=1e-9, atol=1e-9), k
    dm = o.download_native("dmax") * 1000
    assert np.allclose(dm, st.dmax, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("seed,walls", [(1, False), (2, False), (3, False), (4, True), (5, True)])
def test_li_step_agrees_on_random_states(oracle_lib, seed, walls):
    """One Local_Inertial_Model_D4 call on a random wet state with random prior fluxes; with
    walls, cells of NaN elevation (idx_nan) whose faces keep the inside cell's depth as Hf
    (MATLAB's max skips NaN) while passing no flow."""
    case = random_terrain(23, 37, seed=seed, walls=walls)
    rng = np.random.default_rng(seed)
    ny, nx = case.shape
    outflow = np.zeros((3, ny, nx))
    outflow[0] = rng.normal(0, 50, (ny, nx))
    outflow[1] = rng.normal(0, 50, (ny, nx))
    outflow[0][:, -1] = 0
    outflow[1][0, :] = 0
    d = np.where(rng.random((ny, nx)) < 0.7, rng.uniform(0, 500, (ny, nx)), 0.0)
    d[np.isnan(case.z)] = np.nan
    ts = 0.5 / 60
    lit = L.local_inertial_model_d4(case.z, d, case.roughness, case.roughness ** 2, case.resolution ** 2, ts,
                                    case.resolution, case.outlet_rows, case.outlet_cols, 1,
                                    case.params["slope_outlet"], outflow)
    o = kernel_form(case)
    o.set_state(d, outflow)
    o.li_step(ts)
    h = o.download_native("h") * 1000
    assert np.allclose(h, lit.d_t, rtol=1e-12, atol=1e-12, equal_nan=True)
    qr = o.download_native("qx") * 3.6e6 / case.resolution
    qu = o.download_native("qy") * 3.6e6 / case.resolution
    assert np.allclose(qr, lit.qout_right, rtol=1e-11, atol=1e-9)
    assert np.allclose(qu, lit.qout_up, rtol=1e-11, atol=1e-9)
    assert np.allclose(o.download_native("hfx"), lit.Hf[0], rtol=1e-12, atol=1e-14)
    assert np.allclose(o.download_native("hfy"), lit.Hf[1], rtol=1e-12, atol=1e-14)
    if walls:
        nan_face = np.isnan(case.z[:, 1:]) ^ np.isnan(case.z[:, :-1])
        assert (lit.Hf[0][:, :-1][nan_face] > 0).any()   # the rule is exercised
    # refreshing_timestep on that state
    cfl = L.refreshing_timestep(lit.Hf, lit.qout_right, lit.qout_up, case.resolution, 1.0, 0.5, 0.7, 10.0,
                                0.01, 0.001)
    ts_k, vm_k = o.cfl_dt()
    assert vm_k == pytest.approx(cfl.max_velocity, rel=1e-12)
    assert ts_k == pytest.approx(cfl.time_step, rel=1e-12)


def test_green_ampt_step_agrees(oracle_lib):
    case = small_urban(48, seed=5)
    cfg = literal_cfg(case)
    st = L.init_state(cfg)
    o = kernel_form(case)
    ts = 2.0 / 60
    d = np.random.default_rng(0).uniform(0, 30, case.shape)
    o.set_state(d, None, case.I0)
    o.hydrology_step(ts)
    dl, Il, Tl, f = L.green_ampt_infiltration(d + L.rain_depth_mm(cfg, st.rain_a, st.rain_b, *case.shape), st.I, st.T,
                                              ts, cfg.ga, case.resolution)
    dl[dl < 1e-6] = 0
    assert np.allclose(o.download_native("h") * 1000, dl, rtol=1e-10, atol=1e-9)
    assert np.allclose(o.download_native("I") * 1000, Il, rtol=1e-10, atol=1e-9)
    assert np.allclose(o.download_native("T") / 3600, Tl, rtol=1e-12)


def test_rcbrt_accuracy(oracle_lib):
    """x^(7/3) and x^(5/3) of the Newton iteration against libm in double: within 3e-6 in
    float (~50 ulp: the iteration's residual 1 - x r^3 is formed from rounded products) and
    1e-13 in double.  Both are far below the FP32-vs-FP64 differences the accuracy tests bound."""
    import ctypes as C
    import oracle
    L_ = oracle._load()
    f = L_.oracle_pow_check
    f.argtypes = [C.c_int32, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    xs = np.concatenate([np.logspace(-30, 5, 4000), [1e-38, 3e-39, 1.0, 2.0, 1e-320]])
    for prec, tol in ((0, 3e-6), (1, 1e-13)):
        a = np.empty_like(xs)
        b = np.empty_like(xs)
        f(prec, xs.size, xs.ctypes.data_as(C.POINTER(C.c_double)), a.ctypes.data_as(C.POINTER(C.c_double)),
          b.ctypes.data_as(C.POINTER(C.c_double)))
        xr = xs.astype(np.float32).astype(np.float64) if prec == 0 else xs
        ok = xr > (1e-15 if prec == 0 else 1e-130)   # results above the smallest normal
        assert np.all(np.abs(a[ok] / xr[ok] ** (7 / 3) - 1) < tol)
        assert np.all(np.abs(b[ok] / xr[ok] ** (5 / 3) - 1) < tol)


def test_qdiv_within_one_ulp(oracle_lib):
    """The kernels' FP32 quotient (seeded reciprocal, three Newton steps, one residual
    correction) against the exact quotient: at most one ulp off, over quotients spanning
    the ranges the step produces (fluxes over face depths and Bates denominators)."""
    import ctypes as C
    import oracle
    L_ = oracle._load()
    f = L_.oracle_qdiv_check
    fp = C.POINTER(C.c_float)
    f.argtypes = [C.c_int32, fp, fp, fp]
    rng = np.random.default_rng(0)
    n = 200000
    a = (rng.uniform(-1, 1, n) * 10.0 ** rng.uniform(-20, 5, n)).astype(np.float32)
    b = (10.0 ** rng.uniform(-30, 9, n)).astype(np.float32)
    a[:5] = [0.0, -0.0, 1.0, 3.0, -7.0]
    b[:5] = [3.0, 3.0, 3.0, 1e-3, 1e9]
    q = np.empty(n, dtype=np.float32)
    f(n, a.ctypes.data_as(fp), b.ctypes.data_as(fp), q.ctypes.data_as(fp))
    exact = a.astype(np.float64) / b.astype(np.float64)
    fin = np.isfinite(exact) & (np.abs(exact) < 3e38) & (np.abs(exact) > 1e-37)
    ulp = np.spacing(np.abs(exact[fin]).astype(np.float32)).astype(np.float64)
    err = np.abs(q[fin].astype(np.float64) - exact[fin]) / ulp
    assert err.max() <= 1.0, err.max()
    assert q[0] == 0.0 and q[1] == 0.0   # a zero numerator gives a zero (its sign is not kept)


def _prior_state(case, seed, scale_mmh):
    rng = np.random.default_rng(seed)
    ny, nx = case.shape
    outflow = np.zeros((3, ny, nx))
    outflow[0] = rng.normal(0, scale_mmh, (ny, nx))
    outflow[1] = rng.normal(0, scale_mmh, (ny, nx))
    outflow[0][:, -1] = 0
    outflow[1][0, :] = 0
    d = np.where(rng.random((ny, nx)) < 0.7, rng.uniform(0, 500, (ny, nx)), 0.0)
    d[np.isnan(case.z)] = np.nan
    return d, outflow


@pytest.mark.parametrize("scheme", [2, 3])
@pytest.mark.parametrize("seed,walls", [(6, False), (7, True)])
def test_li_step_schemes_2_3_agree(oracle_lib, scheme, seed, walls):
    """Inertial_Solver's s-upwind (2) and s-centred (3) schemes (Inertial_Solver.m:29-121) in the
    kernel form against the literal restatement: one Local_Inertial_Model_D4 call on a random
    wet state with random prior fluxes, which the schemes mix with their neighbours'."""
    case = random_terrain(23, 37, seed=seed, walls=walls)
    d, outflow = _prior_state(case, seed, 2e4)
    ts = 0.5 / 60
    lit = L.local_inertial_model_d4(case.z, d, case.roughness, case.roughness ** 2, case.resolution ** 2, ts,
                                    case.resolution, case.outlet_rows, case.outlet_cols, 1,
                                    case.params["slope_outlet"], outflow, flag_numerical_scheme=scheme)
    bates = L.local_inertial_model_d4(case.z, d, case.roughness, case.roughness ** 2, case.resolution ** 2, ts,
                                      case.resolution, case.outlet_rows, case.outlet_cols, 1,
                                      case.params["slope_outlet"], outflow, flag_numerical_scheme=1)
    assert np.abs(lit.qout_right - bates.qout_right).max() > 1.0   # the scheme changes the fluxes
    import oracle
    o = oracle.KernelFormOracle(*case.shape, case.resolution, "fp64",
                                **dict(case.params, flag_numerical_scheme=scheme))
    case.apply(o)
    o.set_state(d, outflow)
    o.li_step(ts)
    assert np.allclose(o.download_native("h") * 1000, lit.d_t, rtol=1e-11, atol=1e-10, equal_nan=True)
    qr = o.download_native("qx") * 3.6e6 / case.resolution
    qu = o.download_native("qy") * 3.6e6 / case.resolution
    assert np.allclose(qr, lit.qout_right, rtol=1e-10, atol=1e-8)
    assert np.allclose(qu, lit.qout_up, rtol=1e-10, atol=1e-8)


@pytest.mark.parametrize("scheme", [1, 2])
def test_li_step_critical_clip_agrees(oracle_lib, scheme):
    """flag_critical = 1 (Local_Inertial_Model_D4.m:272-275): |q| <= Hf sqrt(g Hf) after the
    solver; a steep random state with large prior fluxes makes the clip bind on many faces."""
    case = random_terrain(31, 29, seed=8)
    case.z = case.z * 6.0   # steep: supercritical faces within one step
    d, outflow = _prior_state(case, 8, 2e6)
    ts = 2.0 / 60
    kw = dict(flag_numerical_scheme=scheme)
    args = (case.z, d, case.roughness, case.roughness ** 2, case.resolution ** 2, ts, case.resolution,
            case.outlet_rows, case.outlet_cols, 1, case.params["slope_outlet"], outflow)
    lit = L.local_inertial_model_d4(*args, flag_critical=1, **kw)
    free = L.local_inertial_model_d4(*args, flag_critical=0, **kw)
    clipped = np.abs(lit.qout_right - free.qout_right) > 1e-6
    assert clipped.sum() > 20   # the clip binds
    import oracle
    o = oracle.KernelFormOracle(*case.shape, case.resolution, "fp64",
                                **dict(case.params, flag_critical=1, **kw))
    case.apply(o)
    o.set_state(d, outflow)
    o.li_step(ts)
    assert np.allclose(o.download_native("h") * 1000, lit.d_t, rtol=1e-11, atol=1e-10)
    qr = o.download_native("qx") * 3.6e6 / case.resolution
    qu = o.download_native("qy") * 3.6e6 / case.resolution
    assert np.allclose(qr, lit.qout_right, rtol=1e-10, atol=1e-8)
    assert np.allclose(qu, lit.qout_up, rtol=1e-10, atol=1e-8)


@pytest.mark.parametrize("scheme,critical", [(2, 0), (3, 0), (1, 1), (3, 1)])
def test_full_loop_dambreak_schemes_agree(oracle_lib, scheme, critical):
    """The whole loop (rain-free dam-break, adaptive dt) with the diffusive schemes and the
    critical clip: kernel form against literal for 120 steps, to round-off relative to the
    reservoir depth (the dam-break amplifies the two forms' different roundings to ~1e-11 of
    the depth scale over these steps)."""
    from tests.cases import small_dambreak
    case = small_dambreak(24, 96, seed=9)
    case.params = dict(case.params, flag_numerical_scheme=scheme, flag_critical=critical)
    cfg = literal_cfg(case)
    cfg.flag_numerical_scheme = scheme
    cfg.flag_critical = critical
    st = L.init_state(cfg)
    o = kernel_form(case)
    for k in range(120):
        L.step(cfg, st)
        o.fused_steps(1)
        d = o.diag()
        assert d["time_step"] == pytest.approx(st.time_step, rel=1e-12), k
        h = o.download_native("h") * 1000
        assert np.abs(h - st.d).max() <= 1e-9 * np.abs(st.d).max(), k


def test_block_refresh_schedule(oracle_lib):
    """The temporal-blocking schedule of the kernel-form oracle: with K = 3 the time step is
    refreshed on step 1 and on the steps k with (k - 1) % 3 == 0 only, and K = 1 is the per-step
    path."""
    from tests.cases import small_dambreak
    case = small_dambreak(24, 96, seed=9)
    o = kernel_form(case)
    o.set_temporal_blocking(3)
    per = kernel_form(case)
    prev = o.diag()["time_step"]
    changed = []
    for _ in range(30):
        k = o.diag()["k"]
        o.fused_steps(1)
        per.fused_steps(1)
        ts = o.diag()["time_step"]
        if ts != prev:
            changed.append(k)
        prev = ts
    assert changed and all(k == 1 or (k - 1) % 3 == 0 for k in changed), changed
    assert o.diag()["t"] != per.diag()["t"]
    one = kernel_form(case)
    one.set_temporal_blocking(1)
    one.fused_steps(30)
    assert one.diag()["t"] == per.diag()["t"]
