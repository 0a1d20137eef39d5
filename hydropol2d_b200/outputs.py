"""Output files of a run in the reference's formats: GeoTIFF rasters named as post_processing.m
names them, and the save_map_hydro_<store>.mat chunks of save_output_maps.m.

* ``write_geotiff`` / ``read_geotiff``: single-band, uncompressed, one strip per row, IEEE
  float samples, with the GeoTIFF model tags (pixel scale, tie point at the upper-left corner,
  PixelIsArea, optional EPSG code) that MATLAB's ``geotiffwrite`` puts on a projected raster.
* ``export_maxima``: Maximum_Depths.tif [m], Maximum_Velocity.tif [m/s], Maximum_Hazard.tif
  [m^2/s], NaN where the maximum depth stays below ``depth_wse`` or the value is not finite
  (post_processing.m:1796-1828, :1940-1970).
* ``export_depth_records``: Flood_Depths_t_<hours>_h.tif for each map record [m], NaN on the
  idx_nan cells (post_processing.m:1482-1524 with flag_elapsed_time = 1).
* ``write_map_chunks``: the depth records [mm] in files of ``saver_memory_maps`` maps, variable
  ``Maps.Hydro.d`` (ny, nx, k) (save_output_maps.m:565-580).  The reference saves MAT 7.3
  (HDF5); these are MAT 5 files, which MATLAB's ``load`` reads the same way.
* ``write_timeseries_netcdf``: one time series of maps in one NetCDF file with the variables,
  dimensions and CF attributes of initializeTimeSeriesNetCDF / appendTimeSliceToNetCDF
  (post_processing.m:2811-3154, :3236-3248): x, y (cell centres, y ascending, so the maps' rows
  are flipped), time, a scalar crs, and the data variable (time, y, x) in single precision.
  The reference writes the netcdf4 (HDF5) flavour with deflate; this writes the classic 64-bit
  offset flavour (no HDF5 library here), which every NetCDF reader takes.
"""
from __future__ import annotations

import math
import os
import struct
from dataclasses import dataclass

import numpy as np


@dataclass
class GeoRef:
    """Upper-left corner of the grid [m] (GIS_data.xulcorner / yulcorner), cell size [m] and
    the projected coordinate system's EPSG code (None: left out)."""
    x_ul: float = 0.0
    y_ul: float = 0.0
    res: float = 1.0
    epsg: int | None = None


def num2str(x: float) -> str:
    """MATLAB's num2str for a real scalar: integers as integers, otherwise
    max(floor(log10|x|), 0) + 5 significant digits."""
    x = float(x)
    if x == int(x) and abs(x) < 1e15:
        return str(int(x))
    digits = max(int(math.floor(math.log10(abs(x)))), 0) + 5
    return f"{x:.{digits}g}"


_TYPES = {2: ("s", 1), 3: ("H", 2), 4: ("I", 4), 12: ("d", 8)}


def write_geotiff(path: str, z: np.ndarray, geo: GeoRef, dtype=np.float64) -> None:
    z = np.ascontiguousarray(np.asarray(z, dtype=dtype))
    if z.ndim != 2:
        raise ValueError("a GeoTIFF raster is 2-D")
    ny, nx = z.shape
    bps = z.dtype.itemsize * 8
    row_bytes = nx * z.dtype.itemsize
    keys = [1, 1, 0, 0, 1024, 0, 1, 1, 1025, 0, 1, 1]          # model: projected; raster: area
    if geo.epsg is not None:
        keys += [3072, 0, 1, int(geo.epsg)]
    keys[3] = (len(keys) - 4) // 4
    nodata = b"nan\x00"
    tags = [  # (tag, type, values)
        (256, 4, [nx]), (257, 4, [ny]), (258, 3, [bps]), (259, 3, [1]), (262, 3, [1]),
        (273, 4, None), (277, 3, [1]), (278, 4, [1]), (279, 4, [row_bytes] * ny), (284, 3, [1]),
        (339, 3, [3]),
        (33550, 12, [geo.res, geo.res, 0.0]),
        (33922, 12, [0.0, 0.0, 0.0, geo.x_ul, geo.y_ul, 0.0]),
        (34735, 3, keys),
        (42113, 2, nodata),
    ]
    n_tags = len(tags)
    ifd_off = 8
    ifd_size = 2 + 12 * n_tags + 4
    extra_off = ifd_off + ifd_size
    extra = bytearray()
    data_off = None

    def payload(typ, vals):
        if typ == 2:
            return bytes(vals)
        fmt, _ = _TYPES[typ]
        return struct.pack("<" + fmt * len(vals), *vals)

    # the strip offsets come after the extra block, whose size does not depend on them
    sizes = []
    for tag, typ, vals in tags:
        count = ny if tag == 273 else len(vals)
        size = count * _TYPES[typ][1]
        sizes.append(size)
    extra_len = sum(s + (s & 1) for s in sizes if s > 4)
    data_off = extra_off + extra_len
    data_off += (-data_off) % 8
    offsets = [data_off + i * row_bytes for i in range(ny)]
    entries = []
    for (tag, typ, vals), size in zip(tags, sizes):
        if tag == 273:
            vals = offsets
        raw = payload(typ, vals)
        count = len(vals)
        if size <= 4:
            entries.append(struct.pack("<HHI", tag, typ, count) + raw.ljust(4, b"\x00"))
        else:
            entries.append(struct.pack("<HHII", tag, typ, count, extra_off + len(extra)))
            extra += raw
            if len(extra) & 1:
                extra += b"\x00"
    assert len(extra) == extra_len
    with open(path, "wb") as f:
        f.write(b"II" + struct.pack("<HI", 42, ifd_off))
        f.write(struct.pack("<H", n_tags) + b"".join(entries) + struct.pack("<I", 0))
        f.write(bytes(extra))
        f.write(b"\x00" * (data_off - extra_off - len(extra)))
        f.write(z.tobytes())


def read_geotiff(path: str) -> tuple[np.ndarray, GeoRef]:
    """Reads what ``write_geotiff`` writes (little-endian, uncompressed, one band)."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:4] != b"II*\x00":
        raise ValueError("not a little-endian TIFF")
    (ifd,) = struct.unpack_from("<I", buf, 4)
    (n,) = struct.unpack_from("<H", buf, ifd)
    tags = {}
    for i in range(n):
        tag, typ, count = struct.unpack_from("<HHI", buf, ifd + 2 + 12 * i)
        fmt, size = _TYPES[typ]
        at = ifd + 2 + 12 * i + 8
        if count * size > 4:
            (at,) = struct.unpack_from("<I", buf, at)
        if typ == 2:
            tags[tag] = buf[at:at + count]
        else:
            tags[tag] = list(struct.unpack_from("<" + fmt * count, buf, at))
    nx, ny, bps = tags[256][0], tags[257][0], tags[258][0]
    if tags[259][0] != 1 or tags[339][0] != 3:
        raise ValueError("only uncompressed IEEE float rasters")
    dt = np.dtype("<f8" if bps == 64 else "<f4")
    rows = [np.frombuffer(buf, dtype=dt, count=nx, offset=o) for o in tags[273]]
    z = np.stack(rows) if len(tags[273]) == ny else np.frombuffer(buf, dtype=dt, count=nx * ny,
                                                                   offset=tags[273][0]).reshape(ny, nx)
    keys = tags.get(34735, [])
    epsg = None
    for k in range(4, len(keys), 4):
        if keys[k] == 3072:
            epsg = keys[k + 3]
    tp = tags[33922]
    return np.array(z), GeoRef(x_ul=tp[3], y_ul=tp[4], res=tags[33550][0], epsg=epsg)


def export_maxima(directory: str, geo: GeoRef, dmax_mm: np.ndarray, vmax: np.ndarray | None = None,
                  hazard_max: np.ndarray | None = None, depth_wse: float = 0.01) -> list[str]:
    os.makedirs(directory, exist_ok=True)
    d = np.asarray(dmax_mm, dtype=np.float64) / 1000.0
    shallow = d < depth_wse
    out = []

    def put(name, z):
        z = np.array(z, dtype=np.float64)
        z[~np.isfinite(z)] = np.nan
        z[shallow] = np.nan
        p = os.path.join(directory, name)
        write_geotiff(p, z, geo)
        out.append(p)

    put("Maximum_Depths.tif", d)
    if vmax is not None:
        put("Maximum_Velocity.tif", vmax)
    if hazard_max is not None:
        put("Maximum_Hazard.tif", hazard_max)
    return out


def export_depth_records(directory: str, geo: GeoRef, depths_mm, times_min, idx_nan=None) -> list[str]:
    os.makedirs(directory, exist_ok=True)
    out = []
    for d, t in zip(depths_mm, times_min):
        z = np.asarray(d, dtype=np.float64) / 1000.0
        if idx_nan is not None:
            z[np.asarray(idx_nan, dtype=bool)] = np.nan
        p = os.path.join(directory, f"Flood_Depths_t_{num2str(t / 60.0)}_h.tif")
        write_geotiff(p, z, geo)
        out.append(p)
    return out


def write_map_chunks(directory: str, depths_mm, saver_memory_maps: int = 12, first_store: int = 1) -> list[str]:
    """Writes every ``saver_memory_maps`` depth maps as save_map_hydro_<store>.mat; a last
    partial chunk is written too (the reference keeps it in memory to the end of the run)."""
    from scipy.io import savemat
    os.makedirs(directory, exist_ok=True)
    maps = [np.asarray(d, dtype=np.float64) for d in depths_mm]
    out = []
    for s, i in enumerate(range(0, len(maps), saver_memory_maps)):
        stack = np.stack(maps[i:i + saver_memory_maps], axis=2)
        p = os.path.join(directory, f"save_map_hydro_{first_store + s}.mat")
        savemat(p, {"Maps": {"Hydro": {"d": stack}}})
        out.append(p)
    return out


def write_timeseries_netcdf(path: str, maps, times, geo: GeoRef, var_name: str = "flood_depth",
                            long_name: str = "Flood depth", units: str = "m",
                            time_units: str = "hours since simulation start", calendar: str = "none",
                            fill_value: float = float("nan")) -> str:
    """``maps``: (nt, ny, nx) in the variable's units, row 0 the northern row; ``times`` in
    ``time_units``.  Projected coordinates (metres) from ``geo``."""
    from scipy.io import netcdf_file
    maps = np.asarray(maps, dtype=np.float64)
    if maps.ndim != 3:
        raise ValueError("maps must be (nt, ny, nx)")
    nt, ny, nx = maps.shape
    times = np.asarray(times, dtype=np.float64).reshape(-1)
    if times.size != nt:
        raise ValueError("one time per map")
    # intrinsicToWorld of the cell centres of a map-cells reference whose columns start north
    x = geo.x_ul + (np.arange(1, nx + 1) - 0.5) * geo.res
    y = geo.y_ul - (np.arange(1, ny + 1) - 0.5) * geo.res
    flip = ny >= 2 and y[1] < y[0]
    if flip:
        y = y[::-1]
    if os.path.exists(path):
        os.remove(path)
    f = netcdf_file(path, "w", version=2)
    try:
        f.createDimension("x", nx)
        f.createDimension("y", ny)
        f.createDimension("time", nt)
        vx = f.createVariable("x", "d", ("x",))
        vy = f.createVariable("y", "d", ("y",))
        vt = f.createVariable("time", "d", ("time",))
        crs = f.createVariable("crs", "i", ())
        var = f.createVariable(var_name, "f", ("time", "y", "x"))
        vx[:] = x
        vy[:] = y
        vt[:] = times
        crs.data[()] = 0   # (assignValue indexes a 0-d array with [:] under numpy 2)
        for v, std, lng, ax in ((vx, "projection_x_coordinate", "x coordinate of projection", "X"),
                                (vy, "projection_y_coordinate", "y coordinate of projection", "Y")):
            v.standard_name, v.long_name, v.units, v.axis = std, lng, "m", ax
        vt.standard_name, vt.long_name, vt.units, vt.calendar, vt.axis = "time", "time", time_units, calendar, "T"
        crs.grid_mapping_name = "transverse_mercator"
        crs.long_name = "projected"
        if geo.epsg is not None:
            crs.epsg_code = f"EPSG:{int(geo.epsg)}"
        var._FillValue = np.float32(fill_value)
        var.long_name, var.units = long_name, units
        var.coordinates = "x y time"
        var.grid_mapping = "crs"
        for i in range(nt):   # appendTimeSliceToNetCDF: single precision, rows flipped
            z = maps[i].astype(np.float32)
            var[i] = z[::-1] if flip else z
        f.title = f"{long_name} time series"
        f.source = "HydroPol2D export"
    finally:
        f.close()
    return path


def export_run(sf, directory: str, geo: GeoRef, time_records=None, depth_wse: float = 0.01,
               netcdf: bool = False) -> list[str]:
    """All of the above for a ``SurfaceFlow`` after its run: the map records (when kept), named
    by ``time_records`` [min] as post_processing.m names record i (else by the clock of the
    step that took it), the maximum depth, and the velocity and hazard maxima (when tracked);
    with ``netcdf`` also the records' time series (Flood_Depths_timeseries.nc, hours)."""
    from ._abi import HP2DError
    out = []
    recs = [sf.download_map_record(i) for i in range(sf.map_records())]
    if recs:
        depths = [d for d, _ in recs]
        times = [t for _, t in recs] if time_records is None else list(time_records)[:len(recs)]
        out += export_depth_records(directory, geo, depths, times)
        out += write_map_chunks(directory, depths)
        if netcdf:   # post_processing.m:1397-1410, :1527-1547 (flag_wse = 0)
            out.append(write_timeseries_netcdf(os.path.join(directory, "Flood_Depths_timeseries.nc"),
                                               np.stack(depths) / 1000.0, np.asarray(times, dtype=float) / 60.0,
                                               geo))
    vmax = hz = None
    try:
        vmax, hz = sf.download("vmax"), sf.download("hazard_max")
    except HP2DError:   # not tracked
        pass
    out += export_maxima(directory, geo, sf.download("dmax"), vmax, hz, depth_wse)
    return out
