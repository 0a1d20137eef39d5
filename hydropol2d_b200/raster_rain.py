"""Input rain rasters (flags.flag_input_rainfall_map = 1): GeoTIFF rate maps [mm/h] read, aligned
to the grid and quality-controlled as update_spatial_BC.m does it, then handed to the device as
end-stamped full-resolution rain maps (hp2d_set_rain_maps_end_stamped).

* ``read_raster``: a single-band GeoTIFF (the files ``outputs.write_geotiff`` writes, or any
  TIFF Pillow opens with the GeoTIFF pixel-scale and tie-point tags).
* ``align``: localReadAlignRain (update_spatial_BC.m:1018-1063) with raster_cutter.m for a source
  in the grid's projected coordinate system: when the source's cell size or shape differs from
  the grid's, it is sampled bilinearly (griddedInterpolant 'linear', no extrapolation) at the
  grid's points, on the coordinates raster_cutter uses for both (XWorldLimits(1) + (0:n-1) dx,
  YWorldLimits(2) - (0:n-1) dy); points outside the source or outside the DEM's valid cells get
  0, and NaN, negative or > 300 mm/h values 0 (raster_cutter.m:56-81); finally max(Z, 0) with
  MATLAB's NaN-ignoring max (a NaN becomes 0).  Sources in another coordinate system would
  need projinv/projfwd and are refused.
* ``quality_controlled``: localGetInputRainMapCached (:903-963): a map whose largest value
  exceeds 300 mm/h is replaced by the previous file's map (the first file's own for the first);
  the walls (NaN elevation) get 0 here -- their depth is NaN on the device, so no rain is
  counted there either way.
* ``set_input_rain``: all of it for a list of files with their end times.
"""
from __future__ import annotations

import numpy as np

from .outputs import GeoRef, read_geotiff

QC_MAX_MMH = 300.0


def read_raster(path: str) -> tuple[np.ndarray, GeoRef]:
    try:
        return read_geotiff(path)
    except Exception:
        pass
    from PIL import Image
    with Image.open(path) as im:
        z = np.asarray(im, dtype=np.float64)
        tags = im.tag_v2
        scale = tags.get(33550)
        tie = tags.get(33922)
    if scale is None or tie is None:
        raise ValueError(f"{path}: no GeoTIFF pixel scale / tie point")
    # tie point (I, J, K, X, Y, Z): raster point (I, J) at world (X, Y), pixel-is-area corners
    res = float(scale[0])
    if abs(float(scale[1]) - res) > 1e-9 * max(res, 1.0):
        raise ValueError(f"{path}: cells are not square")
    return z, GeoRef(x_ul=float(tie[3]) - float(tie[0]) * res, y_ul=float(tie[4]) + float(tie[1]) * res, res=res)


def align(z_src: np.ndarray, src: GeoRef, dem: GeoRef, ny: int, nx: int, dem_valid: np.ndarray) -> np.ndarray:
    """(ny, nx) FP64 rate map [mm/h] on the grid; ``dem_valid`` = ~isnan(elevation)."""
    z_src = np.asarray(z_src, dtype=np.float64)
    if src.epsg is not None and dem.epsg is not None and src.epsg != dem.epsg:
        raise ValueError("the rain raster is in another coordinate system than the grid (no reprojection here)")
    need = abs(src.res - dem.res) > 1e-9 or z_src.shape != (ny, nx)
    if not need:
        z = z_src
    else:
        from scipy.interpolate import RegularGridInterpolator
        nrs, ncs = z_src.shape
        xs = src.x_ul + np.arange(ncs) * src.res
        ys = src.y_ul - np.arange(nrs) * src.res          # rows start from north
        xq = dem.x_ul + np.arange(nx) * dem.res
        yq = dem.y_ul - np.arange(ny) * dem.res
        f = RegularGridInterpolator((ys[::-1], xs), z_src[::-1], method="linear", bounds_error=False,
                                    fill_value=np.nan)
        Y, X = np.meshgrid(yq, xq, indexing="ij")
        z = f(np.stack([Y.ravel(), X.ravel()], axis=1)).reshape(ny, nx)
        z[~np.asarray(dem_valid, dtype=bool)] = 0.0
        z[np.isnan(z) | (z < 0) | (z > QC_MAX_MMH)] = 0.0
    return np.fmax(z, 0.0)


def quality_controlled(maps: list[np.ndarray], dem_valid: np.ndarray) -> np.ndarray:
    """(n, ny, nx) float32 maps ready for the device."""
    out = np.empty((len(maps),) + maps[0].shape, dtype=np.float32)
    walls = ~np.asarray(dem_valid, dtype=bool)
    for i, z in enumerate(maps):
        if np.nanmax(z) > QC_MAX_MMH:
            z = maps[max(i - 1, 0)]
        z = np.where(np.isnan(z), 0.0, z)
        z[walls] = 0.0
        out[i] = z
    return out


def set_input_rain(sf, paths, t_end_min, dem: GeoRef, elevation: np.ndarray, dt_force: float | None = None) -> np.ndarray:
    """Reads, aligns and quality-controls the rasters ``paths`` (end-stamped at ``t_end_min``)
    and sets them on ``sf`` (a SurfaceFlow, or the oracle); returns the device maps."""
    ny, nx = elevation.shape
    valid = ~np.isnan(np.asarray(elevation, dtype=np.float64))
    aligned = []
    for p in paths:
        z, g = read_raster(p)
        aligned.append(align(z, g, dem, ny, nx, valid))
    maps = quality_controlled(aligned, valid)
    sf.set_rain_maps_end_stamped(maps, t_end_min, dt_force)
    return maps
