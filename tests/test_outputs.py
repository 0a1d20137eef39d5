"""Output files (no GPU): GeoTIFF round trip through the module's reader and through Pillow,
the GeoTIFF keys, MATLAB's num2str for the record file names, the maxima masks of
post_processing.m and the save_map_hydro chunks read back with scipy."""
import os

import numpy as np
import pytest

from hydropol2d_b200 import outputs as O


def test_num2str_matches_matlab_rules():
    assert O.num2str(2.0) == "2"
    assert O.num2str(0.25) == "0.25"
    assert O.num2str(3.14159265) == "3.1416"
    assert O.num2str(0.123456) == "0.12346"
    assert O.num2str(123.456789) == "123.4568"
    assert O.num2str(1.0 / 3.0) == "0.33333"


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_geotiff_round_trip(tmp_path, dtype):
    rng = np.random.default_rng(0)
    z = rng.normal(size=(7, 13)).astype(dtype)
    z[2, 3] = np.nan
    geo = O.GeoRef(x_ul=500000.0, y_ul=7400000.0, res=5.0, epsg=31983)
    p = str(tmp_path / "a.tif")
    O.write_geotiff(p, z, geo, dtype=dtype)
    back, g2 = O.read_geotiff(p)
    assert back.dtype == np.dtype(dtype) and back.shape == z.shape
    assert np.array_equal(back, z, equal_nan=True)
    assert (g2.x_ul, g2.y_ul, g2.res, g2.epsg) == (500000.0, 7400000.0, 5.0, 31983)
    if dtype == np.float32:   # an independent reader
        from PIL import Image
        im = np.array(Image.open(p))
        assert np.array_equal(im, z, equal_nan=True)


def test_geotiff_without_epsg(tmp_path):
    p = str(tmp_path / "b.tif")
    O.write_geotiff(p, np.arange(6.0).reshape(2, 3), O.GeoRef(1.0, 2.0, 0.5))
    z, g = O.read_geotiff(p)
    assert g.epsg is None and g.res == 0.5 and z[1, 2] == 5.0


def test_export_maxima_masks(tmp_path):
    dmax = np.array([[5.0, 20.0], [np.inf, 300.0]])       # mm
    vmax = np.array([[1.0, 2.0], [3.0, np.nan]])
    hz = np.array([[0.1, 0.04], [9.0, 0.5]])
    files = O.export_maxima(str(tmp_path), O.GeoRef(), dmax, vmax, hz, depth_wse=0.01)
    names = [os.path.basename(f) for f in files]
    assert names == ["Maximum_Depths.tif", "Maximum_Velocity.tif", "Maximum_Hazard.tif"]
    d, _ = O.read_geotiff(files[0])
    v, _ = O.read_geotiff(files[1])
    h, _ = O.read_geotiff(files[2])
    assert np.isnan(d[0, 0]) and d[0, 1] == 0.02 and np.isnan(d[1, 0]) and d[1, 1] == 0.3
    assert np.isnan(v[0, 0]) and v[0, 1] == 2.0 and v[1, 0] == 3.0 and np.isnan(v[1, 1])
    assert np.isnan(h[0, 0]) and h[0, 1] == 0.04 and h[1, 1] == 0.5


def test_depth_records_and_chunks(tmp_path):
    from scipy.io import loadmat
    maps = [np.full((3, 4), float(i)) for i in range(26)]
    times = [15.0 * (i + 1) for i in range(26)]
    files = O.export_depth_records(str(tmp_path), O.GeoRef(), maps[:3], times[:3],
                                   idx_nan=np.eye(3, 4, dtype=bool))
    assert [os.path.basename(f) for f in files] == ["Flood_Depths_t_0.25_h.tif", "Flood_Depths_t_0.5_h.tif",
                                                    "Flood_Depths_t_0.75_h.tif"]
    z, _ = O.read_geotiff(files[2])
    assert np.isnan(z[1, 1]) and z[0, 1] == 0.002
    chunks = O.write_map_chunks(str(tmp_path), maps)
    assert [os.path.basename(c) for c in chunks] == ["save_map_hydro_1.mat", "save_map_hydro_2.mat",
                                                     "save_map_hydro_3.mat"]
    m = loadmat(chunks[1], simplify_cells=True)["Maps"]["Hydro"]["d"]
    assert m.shape == (3, 4, 12) and m[0, 0, 0] == 12.0 and m[0, 0, 11] == 23.0
    last = loadmat(chunks[2], simplify_cells=True)["Maps"]["Hydro"]["d"]
    assert last.shape == (3, 4, 2)


def test_timeseries_netcdf_layout(tmp_path):
    """Dimensions, coordinates (cell centres, y ascending), flipped rows, single precision, the
    fill value and the CF attributes of initializeTimeSeriesNetCDF (post_processing.m:2811-3154)."""
    from scipy.io import netcdf_file
    from hydropol2d_b200.outputs import GeoRef, write_timeseries_netcdf
    rng = np.random.default_rng(4)
    maps = rng.uniform(0, 2, (3, 5, 7))
    maps[1, 0, 0] = np.nan
    geo = GeoRef(x_ul=1000.0, y_ul=5000.0, res=10.0, epsg=31983)
    p = write_timeseries_netcdf(str(tmp_path / "Flood_Depths_timeseries.nc"), maps, [0.5, 1.0, 1.5], geo)
    with netcdf_file(p, "r", mmap=False) as f:
        assert f.dimensions == {"x": 7, "y": 5, "time": 3}
        assert np.allclose(f.variables["x"][:], 1005.0 + 10.0 * np.arange(7))
        assert np.allclose(f.variables["y"][:], 4955.0 + 10.0 * np.arange(5))   # ascending
        assert list(f.variables["time"][:]) == [0.5, 1.0, 1.5]
        v = f.variables["flood_depth"]
        assert v.dimensions == ("time", "y", "x") and v.data.dtype.newbyteorder("=") == np.float32
        got = np.array(v[:])
        assert np.array_equal(got[:, ::-1, :], maps.astype(np.float32), equal_nan=True)   # north row first again
        assert np.isnan(got[1, -1, 0])
        assert v.units == b"m" and v.grid_mapping == b"crs" and v.coordinates == b"x y time"
        assert np.isnan(v._FillValue)
        assert f.variables["time"].units == b"hours since simulation start"
        assert f.variables["crs"].epsg_code == b"EPSG:31983"
        assert f.variables["x"].standard_name == b"projection_x_coordinate"
        assert f.title == b"Flood depth time series" and f.source == b"HydroPol2D export"
