"""Row slabs of one grid (hydropol2d_b200.slabs) on the CPU: the row split, and the driver's
combine + halo exchange, in one process and over gloo ranks, with a stand-in engine whose step
is a radius-2 row stencil scaled by the last combined maxima -- so a wrong halo row or a wrong
combine changes the own rows, and the slabs match the whole grid bit for bit only when both are
right.  The GPU form (real contexts, against one whole-grid context) is tests/test_gpu_slabs.py."""
import json
import os
import socket

import numpy as np
import pytest

from hydropol2d_b200.slabs import HALO, SlabGrid, SlabRank, _Slab, slab_rows


def _bits(x: float) -> int:
    return int(np.float64(x).view(np.int64))   # ordered for non-negative doubles


class FakeSlab:
    """Rows [lo, hi) of a (ny, nx, 4) record grid, own rows [own0, own1) in local indices."""

    def __init__(self, full: np.ndarray, lo: int, hi: int, own0: int, own1: int):
        self.st = full[lo:hi].copy()
        self.ny, self.nx = self.st.shape[:2]
        self.own = slice(own0, own1)
        self.scale = 1.0
        self.skip = 0
        self.last = (0, 0, 0)

    def fused_steps(self, n: int):
        for _ in range(n):
            p = np.pad(self.st, ((2, 2), (0, 0), (0, 0)))   # rows past the context read 0
            w = (0.05, 0.2, 0.5, 0.2, 0.05)
            new = sum(wi * p[i:i + self.ny] for i, wi in enumerate(w))
            new = new * (1.0 - 1e-3 * self.scale) + (0.0 if self.skip else 1e-4)
            new = np.roll(new, 1, axis=1)   # lateral motion inside rows
            self.st = new
            o = new[self.own]
            self.last = (_bits(o[..., 0].max()), _bits(o[..., 1].max()), int(o[..., 2].max() > 0.9))

    def step_maxima(self):
        return self.last

    def apply_refresh(self, v, c, skip):
        self.scale = float(np.int64(v).view(np.float64)) + float(np.int64(c).view(np.float64))
        self.skip = skip

    def get_rows(self, row0, nrows):
        return self.st[row0:row0 + nrows].copy()

    def set_rows(self, row0, block):
        self.st[row0:row0 + block.shape[0]] = block


def _full_grid(ny, nx, seed):
    return np.random.default_rng(seed).uniform(0.0, 1.0, (ny, nx, 4))


def _whole(full, steps):
    e = FakeSlab(full, 0, full.shape[0], 0, full.shape[0])
    for _ in range(steps):
        e.fused_steps(1)
        e.apply_refresh(*e.step_maxima())
    return e.st


def _fake_slabs(full, n):
    ny = full.shape[0]
    out = []
    for r0, r1 in slab_rows(ny, n):
        lo, hi = max(r0 - HALO, 0), min(r1 + HALO, ny)
        out.append(_Slab(FakeSlab(full, lo, hi, r0 - lo, r1 - lo), lo, r0, r1))
    return out


@pytest.mark.parametrize("ny,n", [(10, 1), (10, 3), (37, 4), (8, 4), (100, 7)])
def test_slab_rows_partition(ny, n):
    rows = slab_rows(ny, n)
    assert rows[0][0] == 0 and rows[-1][1] == ny
    assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
    sizes = [r1 - r0 for r0, r1 in rows]
    assert min(sizes) >= HALO and max(sizes) - min(sizes) <= 1


def test_slab_rows_refuses_thin_slabs():
    with pytest.raises(ValueError):
        slab_rows(7, 4)
    with pytest.raises(ValueError):
        slab_rows(10, 0)


@pytest.mark.parametrize("ny,n", [(9, 2), (24, 3), (41, 5), (8, 4)])
def test_in_process_slabs_match_the_whole_grid(ny, n):
    full = _full_grid(ny, 13, seed=ny + n)
    ref = _whole(full, 25)
    grid = SlabGrid.__new__(SlabGrid)
    grid.shape = full.shape[:2]
    grid.slabs = _fake_slabs(full, n)
    grid.step(25)
    got = np.concatenate([s.ctx.st[s.r0 - s.lo:s.r1 - s.lo] for s in grid.slabs])
    assert np.array_equal(got, ref)


def test_a_missing_exchange_is_seen():
    """The check above has teeth: without the halo exchange the own rows drift."""
    full = _full_grid(24, 13, seed=3)
    ref = _whole(full, 10)
    grid = SlabGrid.__new__(SlabGrid)
    grid.shape = full.shape[:2]
    grid.slabs = _fake_slabs(full, 3)
    grid._exchange = lambda: None
    grid.step(10)
    got = np.concatenate([s.ctx.st[s.r0 - s.lo:s.r1 - s.lo] for s in grid.slabs])
    assert not np.array_equal(got, ref)


def _rank_main(rank, world, port, ny, steps, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        full = _full_grid(ny, 11, seed=ny)
        r0, r1 = slab_rows(ny, world)[rank]
        lo, hi = max(r0 - HALO, 0), min(r1 + HALO, ny)
        sr = SlabRank(FakeSlab(full, lo, hi, r0 - lo, r1 - lo), lo, r0, r1, rank, world)
        sr.step(steps)
        own = sr.s.ctx.st[r0 - lo:r1 - lo]
        np.save(f"{out}.{rank}.npy", own)
        with open(f"{out}.{rank}.json", "w") as f:
            json.dump({"scale": sr.s.ctx.scale, "skip": sr.s.ctx.skip}, f)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,ny", [(2, 17), (3, 30)])
def test_slab_ranks_over_gloo_match_the_whole_grid(tmp_path, world, ny):
    import torch.multiprocessing as mp
    out = str(tmp_path / "slab")
    steps = 12
    mp.spawn(_rank_main, args=(world, _free_port(), ny, steps, out), nprocs=world, join=True)
    full = _full_grid(ny, 11, seed=ny)
    e = FakeSlab(full, 0, ny, 0, ny)
    for _ in range(steps):
        e.fused_steps(1)
        e.apply_refresh(*e.step_maxima())
    got = np.concatenate([np.load(f"{out}.{r}.npy") for r in range(world)])
    assert np.array_equal(got, e.st)
    for r in range(world):   # every rank holds the combined scalars
        d = json.load(open(f"{out}.{r}.json"))
        assert d["scale"] == e.scale and d["skip"] == e.skip
