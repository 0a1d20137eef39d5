"""One grid split into row slabs, one context per slab (no counterpart in the reference, which
runs one grid on one GPU: HP2D_HPC_Config.sbatch asks for one).

Slab s owns rows [r0_s, r1_s) of the grid and holds up to two halo rows on each side, copies of
the neighbouring slabs' edge rows: the draining limiter makes a cell's new state depend on cells
two away, so a slab whose halo rows hold the right state at the start of a step computes its own
rows exactly.  Every step is then:

1. each slab runs one fused step (its CFL maxima, ledgers and depth checks over its own rows:
   hp2d_set_owned_rows);
2. the slabs' maxima are combined -- the largest speed^2, the largest wave-celerity term, the
   clamp skip of the next step if any slab asks for it -- and every slab redoes the step's
   time-step refresh with them (hp2d_step_maxima, hp2d_apply_refresh), so all slabs agree on the
   refreshed step and the clock (refreshing_timestep.m over the whole grid);
3. each slab's two edge rows go into its neighbours' halo rows (hp2d_copy_rows).

The slabs then step as the whole grid would, bit for bit.  ``SlabGrid`` keeps the slabs in one
process (on one device, or round-robin over several); ``SlabRank`` is one slab per rank of a
torch.distributed group: step 2 is an all-reduce (max) of three integers, step 3 point-to-point
transfers of 2 x nx records to each neighbour (NCCL on GPUs).  Unsupported here: infiltration,
rain maps, map records, inflow / stage / control structures, hazard maps and step retries.
"""
from __future__ import annotations

import numpy as np

from .surface import SurfaceFlow

HALO = 2


def slab_rows(ny: int, n: int) -> list[tuple[int, int]]:
    """Own rows of n slabs, as even as possible (every slab at least HALO rows)."""
    if n < 1 or ny < n * HALO:
        raise ValueError(f"{ny} rows cannot be split into {n} slabs of at least {HALO} rows")
    edges = [round(ny * s / n) for s in range(n + 1)]
    return [(edges[s], edges[s + 1]) for s in range(n)]


def _build(case, r0: int, r1: int, precision: str, device: int) -> tuple[SurfaceFlow, int]:
    ny, nx = case.shape
    if case.soil is not None or case.rain_maps is not None or case.inflow is not None or \
            case.stage is not None or case.reservoirs is not None:
        raise ValueError("row slabs support uniform rain only (no infiltration, rain maps, inflow, "
                         "stage or control structures)")
    if int(case.params.get("flag_numerical_scheme", 1)) != 1:
        raise ValueError("row slabs carry two halo rows: the local-inertial scheme (1) only")
    d0 = np.asarray(case.d0, dtype=np.float64)
    if np.any(d0[np.isfinite(d0)] < 0):
        # the first step's clamp skip is each slab's own verdict: with non-negative depths and
        # rain every slab says no
        raise ValueError("row slabs start from non-negative depths")
    lo, hi = max(r0 - HALO, 0), min(r1 + HALO, ny)
    g = SurfaceFlow(hi - lo, nx, case.resolution, precision, device=device, **case.params)
    rows = np.asarray(case.outlet_rows, dtype=np.int64)
    cols = np.asarray(case.outlet_cols, dtype=np.int64)
    sel = (rows >= lo) & (rows < hi)
    g.upload_static(case.z[lo:hi], case.roughness[lo:hi], rows[sel] - lo, cols[sel])
    g.set_state(d0[lo:hi])
    if case.rain_uniform is not None:
        g.set_rain_uniform(*case.rain_uniform)
    g.set_owned_rows(r0 - lo, r1 - lo)
    g.set_retry_policy(max_retries=0)
    return g, lo


class _Slab:
    def __init__(self, ctx: SurfaceFlow, lo: int, r0: int, r1: int):
        self.ctx, self.lo, self.r0, self.r1 = ctx, lo, r0, r1

    @property
    def top_halo(self) -> int:
        return self.r0 - self.lo

    @property
    def bottom_halo(self) -> int:
        return self.lo + self.ctx.ny - self.r1

    def rows(self, g0: int, n: int) -> np.ndarray:
        """n state-record rows from global row g0 (host copy)."""
        return self.ctx.get_rows(g0 - self.lo, n)

    def put_rows(self, g0: int, block: np.ndarray) -> None:
        self.ctx.set_rows(g0 - self.lo, block)


class SlabGrid:
    """The row slabs of one grid in one process (contexts on ``devices`` round-robin)."""

    def __init__(self, case, n_slabs: int, precision: str = "fp32", devices=(0,)):
        self.shape = case.shape
        self.slabs = []
        for s, (r0, r1) in enumerate(slab_rows(case.shape[0], n_slabs)):
            ctx, lo = _build(case, r0, r1, precision, devices[s % len(devices)])
            self.slabs.append(_Slab(ctx, lo, r0, r1))

    def step(self, n: int = 1) -> None:
        for _ in range(n):
            for s in self.slabs:
                s.ctx.fused_steps(1)
            m = [s.ctx.step_maxima() for s in self.slabs]
            v, c, skip = max(x[0] for x in m), max(x[1] for x in m), max(x[2] for x in m)
            for s in self.slabs:
                s.ctx.apply_refresh(v, c, skip)
            self._exchange()

    def _exchange(self) -> None:
        for a, b in zip(self.slabs[:-1], self.slabs[1:]):   # a above b
            if b.top_halo:
                b.put_rows(b.r0 - b.top_halo, a.rows(a.r1 - b.top_halo, b.top_halo))
            if a.bottom_halo:
                a.put_rows(a.r1, b.rows(b.r0, a.bottom_halo))

    def gather(self, field: str) -> np.ndarray:
        """The whole grid's field from the slabs' own rows (download_native fields)."""
        return np.concatenate([s.ctx.download_native(field)[s.r0 - s.lo:s.r1 - s.lo] for s in self.slabs])

    def diag(self) -> dict:
        return self.slabs[0].ctx.diag()

    def close(self) -> None:
        for s in self.slabs:
            s.ctx.close()


class SlabRank:
    """Slab ``rank`` of ``world`` for one rank of a torch.distributed group; ``engine`` is the
    slab's context (a SurfaceFlow built by ``build``, or any object with its fused_steps /
    step_maxima / apply_refresh / get_rows / set_rows methods)."""

    def __init__(self, engine, lo: int, r0: int, r1: int, rank: int, world: int, group=None, device=None):
        self.s = _Slab(engine, lo, r0, r1)
        self.rank, self.world, self.group, self.device = rank, world, group, device

    @classmethod
    def build(cls, case, rank: int, world: int, precision: str = "fp32", device: int = 0, group=None):
        r0, r1 = slab_rows(case.shape[0], world)[rank]
        ctx, lo = _build(case, r0, r1, precision, device)
        return cls(ctx, lo, r0, r1, rank, world, group, device)

    def _tensor(self, a):
        import torch
        t = torch.from_numpy(np.ascontiguousarray(a))
        return t.to(f"cuda:{self.device}") if self.device is not None and torch.cuda.is_available() else t

    def _empty(self, nrows: int) -> np.ndarray:
        probe = self.s.rows(self.s.r0, 0)
        return np.empty((nrows,) + probe.shape[1:], dtype=probe.dtype)

    def step(self, n: int = 1) -> None:
        import torch
        import torch.distributed as dist
        for _ in range(n):
            self.s.ctx.fused_steps(1)
            v, c, skip = self.s.ctx.step_maxima()
            # ordered bits of non-negative floats are below 2^63: they fit a signed int64
            t = self._tensor(np.array([v, c, skip], dtype=np.int64))
            dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
            v, c, skip = (int(x) for x in t.cpu().numpy())
            self.s.ctx.apply_refresh(v, c, skip)
            self._exchange(torch, dist)

    def _exchange(self, torch, dist) -> None:
        s = self.s
        ops = []
        bufs = []
        if self.rank > 0:        # edge rows up, halo rows from above
            up = self._tensor(s.rows(s.r0, HALO))
            down_in = self._tensor(self._empty(s.top_halo))
            ops += [dist.P2POp(dist.isend, up, self.rank - 1, self.group),
                    dist.P2POp(dist.irecv, down_in, self.rank - 1, self.group)]
            bufs.append((s.r0 - s.top_halo, down_in))
        if self.rank < self.world - 1:   # edge rows down, halo rows from below
            dn = self._tensor(s.rows(s.r1 - HALO, HALO))
            up_in = self._tensor(self._empty(s.bottom_halo))
            ops += [dist.P2POp(dist.isend, dn, self.rank + 1, self.group),
                    dist.P2POp(dist.irecv, up_in, self.rank + 1, self.group)]
            bufs.append((s.r1, up_in))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for g0, t in bufs:
            s.put_rows(g0, t.cpu().numpy())

    def own(self, field: str) -> np.ndarray:
        return self.s.ctx.download_native(field)[self.s.r0 - self.s.lo:self.s.r1 - self.s.lo]
