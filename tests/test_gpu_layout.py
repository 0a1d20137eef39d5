"""Both layouts of the fused kernel (one cell per lane in 32-column strips, two cells per
lane in 64-column strips; hp2d_set_layout) against the kernel-form oracle, bit for bit: every
state field, the timestep sequence and the clock.  The layout changes only which lane computes
which cell, so the arithmetic per cell is the same."""
import pytest

from tests.cases import random_terrain, small_dambreak, small_urban, small_vtilt
from tests.test_gpu_parity import FIELDS, assert_same_clock, assert_same_state, make_pair

pytestmark = pytest.mark.gpu

CASES = {
    "vtilt": lambda: small_vtilt(40, 40),
    "urban_ga": lambda: small_urban(n=96, seed=3, hours=0.05),
    "dambreak": lambda: small_dambreak(64, 256),
    "ragged_walls": lambda: random_terrain(37, 131, seed=2, walls=True),
    "narrow": lambda: random_terrain(29, 61, seed=8),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("layout", [1, 2])
def test_layout_bit_exact(name, precision, layout):
    case = CASES[name]()
    g, o = make_pair(case, precision)
    g.set_layout(layout)
    g.set_tuning(16 if name != "dambreak" else 24)
    for chunk in (7, 40):
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        fields = FIELDS + (["I"] if case.soil is not None else [])
        assert_same_state(g, o, fields, f"{name} after {chunk}")
        assert_same_clock(g, o)
    g.close()


def test_layouts_agree_and_autotune_picks_one():
    from hydropol2d_b200 import SurfaceFlow
    case = random_terrain(64, 200, seed=5)
    a = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    b = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(a)
    case.apply(b)
    b.set_layout(2)
    a.fused_steps(50)
    b.fused_steps(50)
    from tests.conftest import same_bits
    for f in FIELDS:
        assert same_bits(a.download_native(f), b.download_native(f)), f
    assert b.autotune(3) >= 4
    b.fused_steps(10)
    a.fused_steps(10)
    for f in FIELDS:
        assert same_bits(a.download_native(f), b.download_native(f)), f
    a.close()
    b.close()
