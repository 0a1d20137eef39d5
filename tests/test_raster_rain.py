"""Input rain rasters (flags.flag_input_rainfall_map = 1) on the CPU.

* reading: the GeoTIFFs outputs.write_geotiff writes, and LZW-compressed float TIFFs with the
  GeoTIFF pixel-scale / tie-point tags (Pillow);
* alignment as localReadAlignRain + raster_cutter.m: identity on the grid's own cells (MATLAB's
  NaN-ignoring max(Z, 0)), bilinear sampling of a coarser raster at the grid's points against a
  hand computation, zero outside the source, on walls, and for NaN / negative / > 300 mm/h;
* quality control of localGetInputRainMapCached: a map above 300 mm/h is replaced by the previous
  file's;
* timing: literal.average_input_rain_map_over_step (localAverageInputRainMapOverStep, with its
  cursor and fast path) against a direct overlap sum, and the kernel-form oracle's end-stamped
  maps against the literal over a run (rain volume).
"""
import numpy as np
import pytest

from hydropol2d_b200.outputs import GeoRef, write_geotiff
from hydropol2d_b200 import raster_rain as RR
from oracle import literal as L


def test_read_own_and_pillow_geotiffs(tmp_path):
    from PIL import Image, TiffImagePlugin
    z = np.arange(12, dtype=np.float64).reshape(3, 4)
    write_geotiff(str(tmp_path / "a.tif"), z, GeoRef(100.0, 900.0, 30.0))
    got, g = RR.read_raster(str(tmp_path / "a.tif"))
    assert np.array_equal(got, z) and (g.x_ul, g.y_ul, g.res) == (100.0, 900.0, 30.0)
    info = TiffImagePlugin.ImageFileDirectory_v2()
    info[33550] = (30.0, 30.0, 0.0)
    info.tagtype[33550] = 12
    info[33922] = (1.0, 2.0, 0.0, 130.0, 840.0, 0.0)   # raster point (1, 2) at world (130, 840)
    info.tagtype[33922] = 12
    Image.fromarray(z.astype(np.float32)).save(str(tmp_path / "b.tif"), tiffinfo=info, compression="tiff_lzw")
    got, g = RR.read_raster(str(tmp_path / "b.tif"))
    assert np.array_equal(got, z) and (g.x_ul, g.y_ul, g.res) == (100.0, 900.0, 30.0)


def test_align_on_the_grids_own_cells():
    z = np.array([[1.0, -2.0, np.nan], [400.0, 5.0, 6.0]])
    valid = np.ones((2, 3), dtype=bool)
    got = RR.align(z, GeoRef(0.0, 20.0, 10.0), GeoRef(0.0, 20.0, 10.0), 2, 3, valid)
    # no resampling: only max(Z, 0), NaN-ignoring (the > 300 check is the caller's)
    assert np.array_equal(got, np.array([[1.0, 0.0, 0.0], [400.0, 5.0, 6.0]]))


def test_align_samples_a_coarser_raster_bilinearly():
    rng = np.random.default_rng(2)
    src = rng.uniform(0, 100, (4, 5))
    src[3, 4] = 350.0          # > 300 after sampling near it: zeroed
    sg = GeoRef(x_ul=0.0, y_ul=400.0, res=100.0)
    dem = GeoRef(x_ul=30.0, y_ul=370.0, res=25.0)
    ny, nx = 14, 18
    valid = np.ones((ny, nx), dtype=bool)
    valid[5, 7] = False
    got = RR.align(src, sg, dem, ny, nx, valid)
    xs = sg.x_ul + np.arange(5) * sg.res
    ys = sg.y_ul - np.arange(4) * sg.res
    for i in range(ny):
        for j in range(nx):
            x, y = dem.x_ul + j * dem.res, dem.y_ul - i * dem.res
            if not valid[i, j] or x > xs[-1] or y < ys[-1]:
                assert got[i, j] == 0.0, (i, j)
                continue
            c = min(int((x - xs[0]) // sg.res), 3)
            r = min(int((ys[0] - y) // sg.res), 2)
            tx = (x - xs[c]) / sg.res
            ty = (ys[r] - y) / sg.res
            v = ((1 - tx) * (1 - ty) * src[r, c] + tx * (1 - ty) * src[r, c + 1]
                 + (1 - tx) * ty * src[r + 1, c] + tx * ty * src[r + 1, c + 1])
            want = 0.0 if v > 300.0 else v
            assert got[i, j] == pytest.approx(want, rel=1e-12, abs=1e-12), (i, j)
    assert np.all(got >= 0.0) and np.all(got <= 300.0)


def test_align_refuses_another_coordinate_system():
    with pytest.raises(ValueError):
        RR.align(np.zeros((2, 2)), GeoRef(0, 0, 10, epsg=4326), GeoRef(0, 0, 5, epsg=31983), 4, 4,
                 np.ones((4, 4), dtype=bool))


def test_quality_control_takes_the_previous_map():
    valid = np.ones((2, 2), dtype=bool)
    valid[0, 1] = False
    a = np.full((2, 2), 10.0)
    b = np.full((2, 2), 20.0)
    b[1, 1] = 301.0
    c = np.full((2, 2), 30.0)
    maps = RR.quality_controlled([b, a, b, c], valid)
    assert maps.dtype == np.float32
    assert maps[0][1, 1] == 301.0   # the first file's previous is itself (localClampIndex to 1)
    assert np.all(maps[2][valid] == 10.0)                   # replaced by the previous file's map
    assert np.all(maps[3][valid] == 30.0)
    assert np.all(maps[:, 0, 1] == 0.0)                      # walls


def _direct_average(times, maps, dt_force, t0, t1):
    acc = np.zeros(maps.shape[1:])
    for i in range(len(times)):
        ts = times[0] - dt_force if i == 0 else times[i - 1]
        ov = max(0.0, min(t1, times[i]) - max(t0, ts))
        acc += ov * maps[i]
    return acc / (t1 - t0)


def test_literal_average_with_cursor_and_fast_path():
    rng = np.random.default_rng(5)
    times = np.array([7.5, 15.0, 20.0, 35.0])   # uneven, first interval [2.5, 7.5] (dt_force 7.5)
    maps = rng.uniform(0, 50, (4, 3, 3))
    cursor = 1
    t = 0.0
    while t < 40.0:
        t1 = t + rng.uniform(0.3, 4.0)
        got, cursor = L.average_input_rain_map_over_step(times, maps, t, t1, cursor)
        assert np.allclose(got, _direct_average(times, maps, 7.5, t, t1), rtol=1e-12, atol=1e-12), (t, t1)
        t = t1
    got, _ = L.average_input_rain_map_over_step(times, maps, 16.0, 18.0, 1)   # fast path: map 3 itself
    assert np.array_equal(got, maps[2])


def test_kernel_form_oracle_end_stamped_maps_against_literal(oracle_lib):
    """Rain volume over a run: the oracle's end-stamped maps against the literal average over
    each step's rain interval, summed over the finite cells."""
    import oracle
    from tests.cases import random_terrain
    case = random_terrain(24, 30, seed=9, walls=True)
    case.rain_uniform = None
    rng = np.random.default_rng(9)
    times = np.array([1.0, 1.4, 2.2, 3.0])   # first map from 0.6 min
    maps = rng.uniform(0, 120, (4, 24, 30)).astype(np.float32)
    o = oracle.KernelFormOracle(*case.shape, case.resolution, "fp64", **case.params)
    case.apply(o)
    o.set_rain_maps_end_stamped(maps, times, 0.4)
    finite = np.isfinite(case.d0)
    area = case.resolution ** 2
    want = 0.0
    cursor = 1
    for _ in range(3000):
        if o.diag()["t"] > 3.3:
            break
        d = o.diag()
        a, b = d["rain_t0"], d["rain_t1"]
        avg, cursor = L.average_input_rain_map_over_step(times, maps, a, b, cursor, dt_force=0.4)
        want += float(np.sum((avg * (b - a) / 60.0)[finite])) / 1000.0 * area
        o.fused_steps(1)
    assert o.diag()["t"] > 3.2
    assert o.diag()["rain_volume"] == pytest.approx(want, rel=1e-9)
