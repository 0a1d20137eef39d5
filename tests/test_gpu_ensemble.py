"""Batched ensemble (hp2d_ensemble_*) and autotuner (hp2d_autotune) parity.

Members of uneven sizes advance in one persistent launch per step, each with its own dt
and clock; every member must end bit-identical to the FP32 kernel-form restatement run on
its own, whatever launch shape the ensemble or the autotuner picks.
"""
import numpy as np
import pytest

from tests.conftest import first_mismatch, same_bits

pytestmark = pytest.mark.gpu

FIELDS = ("h", "qx", "qy", "dmax", "arrival")


def small_members(n=6, minutes=2.0, seed=5):
    from hydropol2d_b200 import synthetic as S
    out = []
    for i in range(n):
        c = S.ensemble_member(i, seed=seed, lo=32, hi=160, breach_share=0.4)
        c.params = dict(c.params, routing_time=minutes)
        out.append(c)
    return out


def oracle_final(case):
    import oracle
    o = oracle.KernelFormOracle(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(o)
    o.run()
    return {f: o.download_native(f) for f in FIELDS}, o.diag()


def member(case, rpw=None):
    from hydropol2d_b200 import SurfaceFlow
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    if rpw:
        g.set_tuning(rpw)
    return g


def check_member(g, ref, diag_ref, name):
    for f in FIELDS:
        got = g.download_native(f)
        assert same_bits(got, ref[f]), (name, f, first_mismatch(got, ref[f]))
    d = g.diag()
    for k in ("t", "time_step", "k", "unstable_steps", "neg_depth_warnings"):
        assert d[k] == diag_ref[k], (name, k, d[k], diag_ref[k])
    for k in ("rain_volume", "outlet_volume"):
        assert np.isclose(d[k], diag_ref[k], rtol=1e-5, atol=1e-9), (name, k, d[k], diag_ref[k])


@pytest.mark.parametrize("rpw,layout", [(8, 1), (24, 1), (16, 2), (32, 2)])
def test_ensemble_members_match_oracle(rpw, layout):
    from hydropol2d_b200.ensemble import Ensemble
    cases = small_members()
    refs = [oracle_final(c) for c in cases]
    assert len({r[1]["k"] for r in refs}) > 1, "members should take different step counts"
    with Ensemble() as ens:
        for c in cases:
            ens.add(member(c))
        ens.set_tuning(rpw)
        ens.set_layout(layout)
        launches = ens.run()
        assert launches >= max(r[1]["k"] for r in refs) - 1
        assert ens.steps(3) == 0   # launches after the end leave every member alone
        for g, c, (ref, dref) in zip(ens.members, cases, refs):
            check_member(g, ref, dref, c.name)


def test_ensemble_in_chunks_and_autotuned():
    """Stepping in uneven chunks, with an autotune pass (trial steps undone) in between,
    reaches the same bits."""
    from hydropol2d_b200.ensemble import Ensemble
    cases = small_members(n=4, seed=9)
    refs = [oracle_final(c) for c in cases]
    with Ensemble() as ens:
        for c in cases:
            ens.add(member(c))
        assert ens.steps(7) == 4
        chosen = ens.autotune(3)
        assert chosen >= 4
        ens.steps(40)   # crosses the 32-launch graph chunk
        ens.run()
        for g, c, (ref, dref) in zip(ens.members, cases, refs):
            check_member(g, ref, dref, c.name)


def test_autotune_leaves_state_untouched():
    from tests.cases import small_urban
    case = small_urban(n=96, seed=3, hours=0.1)
    ref, dref = oracle_final(case)
    g = member(case)
    g.fused_steps(5)
    before = {f: g.download_native(f) for f in FIELDS}
    d0 = g.diag()
    rpw = g.autotune(3)
    assert rpw >= 4
    for f in FIELDS:
        assert same_bits(g.download_native(f), before[f]), f
    assert g.diag() == d0
    g.run()
    check_member(g, ref, dref, case.name)
    g.close()


def test_ensemble_rejects_bad_members():
    from hydropol2d_b200 import HP2DError, SurfaceFlow
    from hydropol2d_b200.ensemble import Ensemble
    from tests.cases import small_urban
    cases = small_members(n=1)
    with Ensemble() as ens:
        with pytest.raises(HP2DError) as e:
            ens.steps(1)
        assert e.value.status_name == "HP2D_NOT_READY"
        g64 = SurfaceFlow(16, 16, 1.0, "fp64")
        with pytest.raises(HP2DError) as e:
            ens.add(g64)
        assert e.value.status_name == "HP2D_INVALID_ARG"
        g64.close()
        ens.add(member(cases[0]))
        with pytest.raises(HP2DError):
            ens.add(ens.members[0])
        u = small_urban(n=64, seed=1, hours=0.05)   # Green-Ampt + rain maps
        ens.add(member(u))
        with pytest.raises(HP2DError) as e:
            ens.steps(1)
        assert e.value.status_name == "HP2D_INVALID_ARG"
