"""Map records on the GPU against the kernel-form oracle, bit for bit: the depth maps after the
steps that pass a record time and their clocks, a record whose step is the last of a call
(taken by the host), the slot ring, and records of ensemble members."""
import numpy as np
import pytest

from tests.cases import random_terrain, small_vtilt
from tests.conftest import same_bits
from tests.test_gpu_parity import make_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,host", [("fp32", False), ("fp64", False), ("fp32", True), ("fp64", True)])
def test_records_bit_exact(precision, host, hp2d_lib, oracle_lib):
    """host: the record ring in page-locked host memory, written by the steps themselves."""
    case = small_vtilt(32, 40)
    case.params = dict(case.params, routing_time=8.0)
    times = np.arange(0.0, 8.01, 0.25)
    g, o = make_pair(case, precision)
    g.set_map_records(times, 64, host=host)
    o.set_map_records(times)
    for chunk in (1, 7, 33, 64, 100000):     # calls end between and right after record events
        g.fused_steps(chunk)
        o.fused_steps(chunk)
        assert g.map_records() == o.map_records()
    n = g.map_records()
    assert n >= 25
    for i in range(n):
        dg, tg = g.download_map_record(i)
        do, to = o.download_map_record(i)
        assert tg == to, i
        assert same_bits(dg, do), i


def test_record_ring_keeps_the_last_slots(hp2d_lib):
    from hydropol2d_b200 import HP2DError, SurfaceFlow
    case = random_terrain(24, 32, seed=2)
    case.params = dict(case.params, routing_time=4.0)
    g = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(g)
    g.set_map_records(np.arange(0.0, 4.01, 0.1), 5)
    g.run()
    n = g.map_records()
    assert n > 5
    ts = [g.download_map_record(i)[1] for i in range(n - 5, n)]
    assert all(b > a for a, b in zip(ts, ts[1:]))
    with pytest.raises(HP2DError):
        g.download_map_record(n - 6)            # overwritten
    with pytest.raises(HP2DError):
        g.download_map_record(n)                # not taken


def test_ensemble_members_record(hp2d_lib, oracle_lib):
    import oracle
    from hydropol2d_b200 import SurfaceFlow
    from hydropol2d_b200.ensemble import Ensemble
    cases = [random_terrain(24, 40, seed=3), random_terrain(40, 24, seed=4)]
    times = np.arange(0.0, 3.01, 0.2)
    ens = Ensemble()
    ors = []
    for c in cases:
        c.params = dict(c.params, routing_time=3.0)
        m = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(m)
        m.set_map_records(times, 32)
        ens.add(m)
        o = oracle.KernelFormOracle(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(o)
        o.set_map_records(times)
        o.run()
        ors.append(o)
    ens.run()
    for m, o in zip(ens.members, ors):
        assert m.map_records() == o.map_records() > 5
        for i in range(m.map_records()):
            dg, tg = m.download_map_record(i)
            do, to = o.download_map_record(i)
            assert tg == to and same_bits(dg, do)
    ens.close()
