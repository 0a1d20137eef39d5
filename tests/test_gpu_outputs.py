"""A run's output files from the device results: map records as Flood_Depths_t_<h>_h.tif and
save_map_hydro chunks, the maximum depth, velocity and hazard rasters."""
import os

import numpy as np
import pytest

from hydropol2d_b200 import outputs as O
from hydropol2d_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def test_export_run(tmp_path, hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    case = S.dambreak_case(48, 128, 5.0, seed=3, hours=0.1)
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    g.set_hazard_tracking(True)
    records = np.array([1.0, 2.0, 3.0, 4.5])
    g.set_map_records(records, 8)
    g.run()
    assert g.map_records() == 4
    geo = O.GeoRef(x_ul=300000.0, y_ul=7500000.0, res=case.resolution, epsg=31983)
    files = O.export_run(g, str(tmp_path), geo, time_records=records)
    names = sorted(os.path.basename(f) for f in files)
    assert names == sorted(["Flood_Depths_t_0.016667_h.tif", "Flood_Depths_t_0.033333_h.tif",
                            "Flood_Depths_t_0.05_h.tif", "Flood_Depths_t_0.075_h.tif",
                            "save_map_hydro_1.mat", "Maximum_Depths.tif", "Maximum_Velocity.tif",
                            "Maximum_Hazard.tif"]), names
    d, gr = O.read_geotiff(os.path.join(str(tmp_path), "Maximum_Depths.tif"))
    dmax = g.download("dmax") / 1000.0
    wet = dmax >= 0.01
    assert np.array_equal(d[wet], dmax[wet]) and np.all(np.isnan(d[~wet]))
    assert gr.epsg == 31983 and gr.x_ul == 300000.0
    h, _ = O.read_geotiff(os.path.join(str(tmp_path), "Maximum_Hazard.tif"))
    v, _ = O.read_geotiff(os.path.join(str(tmp_path), "Maximum_Velocity.tif"))
    assert np.nanmax(v) > 1.0 and np.nanmax(h) > 1.0
    assert np.all(h[wet] <= v[wet] * d[wet] * (1 + 1e-6) + 1e-9)
    rec, t = g.download_map_record(1)
    r, _ = O.read_geotiff(os.path.join(str(tmp_path), "Flood_Depths_t_0.033333_h.tif"))
    assert np.array_equal(r, rec / 1000.0)
    g.close()


def test_export_run_netcdf_time_series(tmp_path, hp2d_lib):
    from scipy.io import netcdf_file
    from hydropol2d_b200 import SurfaceFlow
    case = S.dambreak_case(48, 128, 5.0, seed=3, hours=0.1)
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    records = np.array([1.0, 2.0, 3.0, 4.5])
    g.set_map_records(records, 8)
    g.run()
    geo = O.GeoRef(x_ul=300000.0, y_ul=7500000.0, res=case.resolution, epsg=31983)
    files = O.export_run(g, str(tmp_path), geo, time_records=records, netcdf=True)
    nc = [f for f in files if f.endswith("Flood_Depths_timeseries.nc")]
    assert len(nc) == 1
    with netcdf_file(nc[0], "r", mmap=False) as f:
        assert list(f.variables["time"][:]) == list(records / 60.0)
        z = np.array(f.variables["flood_depth"][:])[:, ::-1, :]
        for i in range(4):
            rec, _ = g.download_map_record(i)
            assert np.array_equal(z[i], (rec / 1000.0).astype(np.float32))
    g.close()
