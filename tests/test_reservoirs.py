"""Reservoir / control structures (flag_reservoir = 1, Local_Inertial_Model_D4.m:318-344) in
the two oracles (no GPU): the literal restatement against hand arithmetic, including the
reference's bookkeeping (the reservoir's volume term gains each transfer, the first transfer
reaches ds1 twice with a second structure), then the kernel-form restatement against the
literal one through a run, and the water balance with the structures' volume."""
import math

import numpy as np
import pytest

from hydropol2d_b200 import synthetic as S
from oracle import literal as L
from tests.test_oracle_crosscheck import kernel_form, literal_cfg


def _dh(d_mm, k, h, p, A, ts):
    q = max(d_mm / 1000 - h, 0.0)
    return min(k * q ** p / A * 1000 * 3600, 1000 * q / (ts / 60)) * (ts / 60)


def test_transfers_by_hand():
    d = np.zeros((4, 4))
    d[1, 1] = 500.0
    d[2, 2] = 80.0
    vf = np.zeros((4, 4))
    A, ts = 100.0, 0.1
    rs = dict(res_row=[1, 2], res_col=[1, 2], k1=[3.0, 2.0], h1=[0.2, 0.05], k2=[1.5, 1.0],
              ds1_row=[2, 0], ds1_col=[2, 3], k3=[1.0, 0.0], h2=[0.4, 0.0], k4=[2.5, 0.0],
              ds2_row=[3, np.nan], ds2_col=[0, np.nan])
    d2, vf2 = L.reservoir_transfers(d, vf, rs, ts, A)
    dh1 = _dh(500.0, 3.0, 0.2, 1.5, A, ts)
    q2 = max(0.5 - dh1 / 1000 - 0.4, 0.0)
    dh2 = min(1.0 * q2 ** 2.5 / A * 3.6e6, 1000 * q2 / (ts / 60)) * (ts / 60)
    assert dh1 > 1.0 and dh2 > 0.0
    # structure 1 reads cell (2, 2) after structure 0 added 2 dh1 to it
    dh3 = _dh(80.0 + 2 * dh1, 2.0, 0.05, 1.0, A, ts)
    assert vf2[1, 1] == pytest.approx((dh1 + dh2) / 1000 * A, rel=1e-14)
    assert d2[2, 2] == pytest.approx(80.0 + 2 * dh1, rel=1e-14)
    assert d2[3, 0] == pytest.approx(dh2, rel=1e-14)
    assert vf2[2, 2] == pytest.approx(dh3 / 1000 * A, rel=1e-14)
    assert d2[0, 3] == pytest.approx(dh3, rel=1e-14)
    assert d2[1, 1] == 500.0                 # the reservoir's own d_tot is left alone
    # the available-volume cap: a huge coefficient moves exactly the water above the crest
    big = dict(rs, k1=[1e9, 2.0])
    d3, vf3 = L.reservoir_transfers(d, vf, big, ts, A)
    assert vf3[1, 1] / A * 1000 == pytest.approx(300.0 + 0.0, rel=1e-12)   # q2 = 0: dh2 = 0


def test_transfers_need_ds1_for_ds2():
    rs = dict(res_row=[0], res_col=[0], k1=[1.0], h1=[0.0], k2=[1.0], ds1_row=[np.nan], ds1_col=[np.nan],
              k3=[1.0], h2=[0.0], k4=[1.0], ds2_row=[1], ds2_col=[1])
    with pytest.raises(IndexError):
        L.reservoir_transfers(np.ones((2, 2)), np.zeros((2, 2)), rs, 0.1, 1.0)


@pytest.mark.parametrize("soil,maps", [(False, False), (True, False), (False, True)])
def test_kernel_form_follows_literal(oracle_lib, soil, maps):
    case = S.structures_case(32, 32, minutes=6.0, soil=soil, maps=maps)
    cfg = literal_cfg(case)
    st = L.init_state(cfg)
    o = kernel_form(case)
    for k in range(2000):
        if st.t > cfg.routing_time + cfg.min_time_step / 60:
            break
        L.step(cfg, st)
        o.fused_steps(1)
        if k % 50 == 0:
            h = o.download_native("h") * 1000
            assert np.allclose(h, st.d, rtol=1e-9, atol=1e-9), k
    d = o.diag()
    assert d["t"] == pytest.approx(st.t, rel=1e-12)
    assert st.structure_volume > 1.0
    assert d["structure_volume"] == pytest.approx(st.structure_volume, rel=1e-9)


def test_water_balance_with_structures(oracle_lib):
    case = S.structures_case(32, 32, minutes=6.0)
    o = kernel_form(case)
    v0 = float(np.sum(case.d0)) / 1000 * case.resolution ** 2
    o.run()
    d = o.diag()
    stored = float(np.nansum(o.download_native("h"))) * case.resolution ** 2
    lhs = stored + d["outlet_volume"] + d["infiltration_volume"]
    rhs = v0 + d["rain_volume"] + d["structure_volume"]
    assert d["structure_volume"] > 0
    assert lhs == pytest.approx(rhs, rel=1e-7)
    assert lhs <= rhs * (1 + 1e-12)
