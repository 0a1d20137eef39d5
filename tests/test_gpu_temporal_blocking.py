"""Temporal blocking (hp2d_set_temporal_blocking): K steps per launch on 2-D tiles with halos staged
in shared memory by TMA, at the time step of the last refresh, which runs only on step 1 and on the
steps k with (k - 1) % K == 0.  The kernel-form oracle restates that schedule
(set_temporal_blocking), and the GPU must match it bit for bit: every state field, the outlet
arrays, the clock and the step sequence, through blocks, the single steps around them, replayed
blocks and the row-copy timeout.
"""
import numpy as np
import pytest

from tests.cases import random_terrain, small_dambreak
from tests.conftest import same_bits
from tests.test_gpu_parity import FIELDS, assert_same_clock, assert_same_state, make_pair

pytestmark = pytest.mark.gpu


def blocked_pair(case, k):
    g, o = make_pair(case, "fp32")
    g.set_temporal_blocking(k)
    o.set_temporal_blocking(k)
    return g, o


@pytest.mark.parametrize("k", [2, 3, 4])
def test_blocks_bit_exact_with_the_oracle(k, hp2d_lib, oracle_lib):
    case = small_dambreak(100, 300, seed=5)   # 5 x 4 tiles, the last ones ragged
    g, o = blocked_pair(case, k)
    for chunk in (1, 1, 7, 13, 40, 64):   # blocks and the single steps that align them
        g.fused_steps(chunk)
        assert o.fused_steps(chunk) == 0
        assert_same_state(g, o, FIELDS, f"K={k} chunk {chunk}")
        assert_same_clock(g, o)
    assert same_bits(g.download_native("qo"), o.download_native("qo"))
    assert same_bits(g.download_native("hf3"), o.download_native("hf3"))
    # the schedule is not the per-step one
    f, _ = make_pair(case, "fp32")
    f.fused_steps(g.diag()["k"] - 1)
    assert f.diag()["t"] != g.diag()["t"]


@pytest.mark.parametrize("shape", [(37, 41), (33, 130), (97, 70)])
def test_blocks_ragged_grids_with_walls(shape, hp2d_lib, oracle_lib):
    case = random_terrain(*shape, seed=sum(shape), walls=True)
    case.rain_uniform = None   # blocks run without rain
    g, o = blocked_pair(case, 3)
    for chunk in (2, 9, 30):
        g.fused_steps(chunk)
        assert o.fused_steps(chunk) == 0
        assert_same_state(g, o, FIELDS, f"{shape} chunk {chunk}")
        assert_same_clock(g, o)


def test_rejected_step_inside_a_block_is_replayed(hp2d_lib, oracle_lib):
    """A step that the test hook rejects inside a block: the block is not committed, its steps
    run one per launch, the rejected step is retried with the reference's smaller step."""
    case = small_dambreak(64, 256, seed=6)
    g, o = blocked_pair(case, 4)
    for m in (g, o):
        m.inject_step_fault(11, 1)
    g.fused_steps(30)
    assert o.fused_steps(30) == 0
    assert_same_state(g, o, FIELDS)
    assert_same_clock(g, o)
    assert g.diag()["retries"] == o.diag()["retries"] == 1


def test_block_timeout_leaves_the_state(hp2d_lib, oracle_lib):
    from hydropol2d_b200 import HP2DError
    case = small_dambreak(64, 256, seed=7)
    g, o = blocked_pair(case, 2)
    g.fused_steps(9)
    o.fused_steps(9)
    before = {f: g.download_native(f) for f in FIELDS}
    k0 = g.diag()["k"]
    g.set_wait_limit(0)
    with pytest.raises(HP2DError) as e:
        g.fused_steps(4)
    assert e.value.status_name == "HP2D_TIMEOUT"
    assert g.diag()["k"] == k0
    for f in FIELDS:
        assert same_bits(g.download_native(f), before[f]), f
    g.set_wait_limit(1 << 22)
    g.fused_steps(12)
    o.fused_steps(12)
    assert_same_state(g, o, FIELDS)
    assert_same_clock(g, o)


def test_autotune_chooses_the_block_depth(hp2d_lib, oracle_lib):
    """steps_per_block 0: hp2d_autotune times blocks of 2..4 steps against single steps and
    keeps the fastest; the run then follows that depth's schedule."""
    import oracle
    case = small_dambreak(128, 512, seed=8)
    g, _ = make_pair(case, "fp32")
    g.fused_steps(5)
    g.set_temporal_blocking(0)
    g.autotune(4)
    k = g.diag()["steps_per_block"]
    assert k in (1, 2, 3, 4)
    g.fused_steps(24)
    ref = oracle.KernelFormOracle(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(ref)
    ref.fused_steps(5)
    ref.set_temporal_blocking(k)
    ref.fused_steps(24)
    assert_same_state(g, ref, FIELDS)
    assert_same_clock(g, ref)


def test_unsupported_configurations_are_refused(hp2d_lib):
    from hydropol2d_b200 import HP2DError, SurfaceFlow
    case = random_terrain(40, 40, seed=1)   # uniform rain
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    g.set_temporal_blocking(2)
    with pytest.raises(HP2DError) as e:
        g.fused_steps(4)
    assert e.value.status_name == "HP2D_UNSUPPORTED_FLAG"
    g.set_temporal_blocking(1)
    g.fused_steps(4)
    h = SurfaceFlow(16, 16, 1.0, "fp64")
    with pytest.raises(HP2DError) as e:
        h.set_temporal_blocking(2)
    assert e.value.status_name == "HP2D_UNSUPPORTED_FLAG"
