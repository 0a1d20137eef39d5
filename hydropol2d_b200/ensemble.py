"""Batched ensemble over the C ABI: many ``SurfaceFlow`` members of uneven grid sizes
advanced together by one persistent kernel per step (``hp2d_ensemble_*``).

Replaces the member loop of HydroPol2D_Main_While_Ensemble.m:46-139 and the per-member runs
of Probabilistic_dam_break_analysis.m:8-60.  Each member keeps its own dt and clock; the
members' results are read from the members themselves.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .surface import SurfaceFlow


class Ensemble:
    """An hp2d_ensemble on ``device`` holding FP32 ``SurfaceFlow`` members."""

    def __init__(self, device: int = 0):
        self._L = _abi.lib()
        h = C.c_void_p()
        st = self._L.hp2d_ensemble_create(int(device), C.byref(h))
        if st != 0:
            raise _abi.HP2DError(st, self._L.hp2d_create_error().decode())
        self._h = h
        self.members: list[SurfaceFlow] = []

    def _check(self, st: int):
        if st != 0:
            raise _abi.HP2DError(st, self._L.hp2d_ensemble_last_error(self._h).decode())

    def add(self, member: SurfaceFlow) -> None:
        self._check(self._L.hp2d_ensemble_add(self._h, member._h))
        self.members.append(member)

    def set_tuning(self, rows_per_warp: int) -> None:
        self._check(self._L.hp2d_ensemble_set_tuning(self._h, int(rows_per_warp)))

    def set_layout(self, cells_per_lane: int) -> None:
        self._check(self._L.hp2d_ensemble_set_layout(self._h, int(cells_per_lane)))

    def autotune(self, trial_steps: int = 4) -> int:
        rpw = C.c_int32()
        self._check(self._L.hp2d_ensemble_autotune(self._h, int(trial_steps), C.byref(rpw)))
        return rpw.value

    def steps(self, n: int) -> int:
        """Runs n launches; returns how many members are still running."""
        act = C.c_int32()
        self._check(self._L.hp2d_ensemble_steps(self._h, int(n), C.byref(act)))
        return act.value

    def steps_timed(self, n: int) -> tuple[int, float]:
        act = C.c_int32()
        ms = C.c_float()
        self._check(self._L.hp2d_ensemble_steps_timed(self._h, int(n), C.byref(act), C.byref(ms)))
        return act.value, ms.value

    def run(self, max_steps: int = 0) -> int:
        """Until every member reaches its routing_time; returns the launches made."""
        done = C.c_int64()
        self._check(self._L.hp2d_ensemble_run(self._h, int(max_steps), C.byref(done)))
        return done.value

    def cells(self) -> int:
        return int(sum(m.ny * m.nx for m in self.members))

    def cell_updates(self) -> int:
        """Sum over members of cells x accepted steps so far."""
        return int(sum(m.ny * m.nx * (m.diag()["k"] - 1) for m in self.members))

    def close(self, members: bool = True) -> None:
        if getattr(self, "_h", None):
            self._L.hp2d_ensemble_destroy(self._h)
            self._h = None
        if members:
            for m in self.members:
                m.close()
            self.members = []

    def __del__(self):
        try:
            self.close(members=False)
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def peak_depth_stats(maximum_depths: np.ndarray, threshold: float = 0.3) -> dict:
    """Per-pixel statistics over members of one common grid, as
    Probabilistic_dam_break_analysis.m:8-60 computes them: ``maximum_depths`` is
    (ny, nx, members) in metres; the flood mask is depth > ``threshold`` (0.3 m there);
    returns the per-pixel mean and sample standard deviation (MATLAB ``std``, N-1) of the
    mask and of the depth, and the union mask over members."""
    d = np.asarray(maximum_depths, dtype=np.float64)
    mask = d > threshold
    ddof = 1 if d.shape[2] > 1 else 0
    return dict(total_mask=mask.any(axis=2),
                mean_cell_mask=mask.mean(axis=2), stdev_mask=mask.std(axis=2, ddof=ddof),
                mean_cell=d.mean(axis=2), stdev=d.std(axis=2, ddof=ddof))
