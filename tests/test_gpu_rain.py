"""Rain timing on the GPU against the kernel-form oracle, bit for bit: the rain interval each
step applies (update_spatial_BC over [t_previous, t] at the end of the step before,
HydroPol2D_Main_While.m:721, :734-738), rate maps blended over a step that straddles two of
them, an explicit hp2d_set_rain_clock, and the map-interval check."""
import numpy as np
import pytest

from tests.cases import random_terrain, small_vtilt
from tests.test_gpu_parity import FIELDS, assert_same_clock, assert_same_state, make_pair

pytestmark = pytest.mark.gpu


def _interval(d):
    return d["rain_t0"], d["rain_t1"], d["t_previous"]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_uniform_rain_interval_sequence(precision, hp2d_lib, oracle_lib):
    case = small_vtilt(32, 32)
    g, o = make_pair(case, precision)
    for chunk in (1, 1, 1, 2, 40):
        assert _interval(g.diag()) == _interval(o.diag())
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS, f"after chunk {chunk}")
        assert_same_clock(g, o)
    assert _interval(g.diag()) == _interval(o.diag())


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_maps_straddling_steps(precision, hp2d_lib, oracle_lib):
    """Maps every 0.2 min (12 s >= max_time_step 10 s): many steps take rain from two maps,
    and after the last map no rain falls."""
    case = random_terrain(40, 72, seed=3)
    rng = np.random.default_rng(1)
    maps = rng.uniform(0, 200, (6, 9, 13)).astype(np.float32)
    g, o = make_pair(case, precision)
    g.set_rain_maps(maps, 0.2)
    o.set_rain_maps(maps, 0.2)
    for chunk in (5, 64, 64, 128):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert_same_state(g, o, FIELDS, f"after chunk {chunk}")
        assert_same_clock(g, o)
    assert g.diag()["t"] > 6 * 0.2   # the run went past the last map


def test_unfused_sequence_with_maps_matches_fused(hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    from tests.conftest import same_bits
    case = random_terrain(24, 40, seed=7)
    maps = np.random.default_rng(2).uniform(0, 150, (4, 5, 7)).astype(np.float32)
    a = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    b = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    for s in (a, b):
        case.apply(s)
        s.set_rain_maps(maps, 0.2)
    for _ in range(30):
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
        assert _interval(a.diag()) == _interval(b.diag())


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_set_rain_clock(precision, hp2d_lib, oracle_lib):
    case = small_vtilt(24, 24)
    g, o = make_pair(case, precision)
    g.fused_steps(10)
    o.fused_steps(10)
    for m in (g, o):
        m.set_rain_clock(0.25, 3.5, 2.0)
    assert _interval(g.diag()) == (0.25, 3.5, 2.0)
    g.fused_steps(12)
    o.fused_steps(12)
    assert_same_state(g, o, FIELDS)
    assert_same_clock(g, o)


def test_maps_shorter_than_the_largest_step_are_rejected(hp2d_lib):
    from hydropol2d_b200 import HP2DError, SurfaceFlow
    case = small_vtilt(16, 16)
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    with pytest.raises(HP2DError):
        g.set_rain_maps(np.zeros((2, 4, 4), np.float32), 0.1)   # 6 s < max_time_step 10 s
    g.close()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_end_stamped_input_maps(precision, hp2d_lib, oracle_lib):
    """Input rain maps (flag_input_rainfall_map): uneven end-stamped intervals, the first from
    t_end[0] - dt_force > 0, full-resolution maps (each cell its own value) and coarse ones; the
    run goes past the last map."""
    case = random_terrain(40, 72, seed=4, walls=True)
    case.rain_uniform = None
    rng = np.random.default_rng(6)
    t_end = np.array([0.5, 0.8, 1.3, 1.6])   # [0.3, 0.5), [0.5, 0.8), ...: all >= 10 s
    for maps in (rng.uniform(0, 200, (4, 40, 72)).astype(np.float32),
                 rng.uniform(0, 200, (4, 7, 9)).astype(np.float32)):
        g, o = make_pair(case, precision)
        g.set_rain_maps_end_stamped(maps, t_end, 0.2)
        o.set_rain_maps_end_stamped(maps, t_end, 0.2)
        for chunk in (3, 40, 100, 200):
            g.fused_steps(chunk)
            o.fused_steps(chunk)
            assert_same_state(g, o, FIELDS, f"{maps.shape} after chunk {chunk}")
            assert_same_clock(g, o)
        assert g.diag()["t"] > 1.6
        g.close()


def test_input_rain_rasters_from_files(tmp_path, hp2d_lib, oracle_lib):
    """GeoTIFF rate rasters at four times the grid's cell size, read and aligned as
    raster_cutter.m does, on the GPU and in the oracle: the same bits."""
    from hydropol2d_b200 import raster_rain as RR
    from hydropol2d_b200.outputs import GeoRef, write_geotiff
    case = random_terrain(48, 64, seed=8, walls=True)
    case.rain_uniform = None
    dem = GeoRef(x_ul=500000.0, y_ul=7000000.0, res=case.resolution)
    rng = np.random.default_rng(8)
    paths = []
    for m in range(3):
        p = str(tmp_path / f"rain_{m}.tif")
        write_geotiff(p, rng.uniform(0, 150, (14, 18)), GeoRef(dem.x_ul - 7.0, dem.y_ul + 3.0, 4 * dem.res))
        paths.append(p)
    g, o = make_pair(case, "fp32")
    mg = RR.set_input_rain(g, paths, [0.4, 0.8, 1.2], dem, case.z)
    mo = RR.set_input_rain(o, paths, [0.4, 0.8, 1.2], dem, case.z)
    assert np.array_equal(mg, mo) and mg.shape == (3, 48, 64) and np.all(mg >= 0)
    g.fused_steps(300)
    o.fused_steps(300)
    assert_same_state(g, o, FIELDS)
    assert_same_clock(g, o)
    assert g.diag()["rain_volume"] > 0
    g.close()


def test_end_stamped_intervals_shorter_than_the_largest_step_are_rejected(hp2d_lib):
    from hydropol2d_b200 import HP2DError, SurfaceFlow
    case = small_vtilt(16, 16)
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    with pytest.raises(HP2DError):
        g.set_rain_maps_end_stamped(np.zeros((2, 4, 4), np.float32), [0.5, 0.6], 0.5)   # 6 s
    with pytest.raises(HP2DError):
        g.set_rain_maps_end_stamped(np.zeros((2, 4, 4), np.float32), [0.5, 0.4], 0.5)   # decreasing
    g.set_rain_maps_end_stamped(np.zeros((2, 4, 4), np.float32), [0.5, 0.5], 0.5)        # empty interval: fine
    g.close()
