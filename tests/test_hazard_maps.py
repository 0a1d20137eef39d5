"""Velocity and hazard maxima (velocities.vmax_final / hazardmax_final, save_output_maps.m:588-604,
snisb_velocity_hazard_snapshot :832-848) in the two oracles (no GPU): the snapshot rule by hand,
then the kernel-form restatement against the literal one through a dam-break run."""
import numpy as np
import pytest

from hydropol2d_b200 import synthetic as S
from oracle import literal as L
from tests.test_oracle_crosscheck import kernel_form, literal_cfg


def test_snapshot_by_hand():
    v = np.array([[1.0, 2.0, np.inf], [0.5, np.nan, 3.0]])
    d = np.array([[5.0, 100.0, 200.0], [2000.0, 300.0, np.nan]])     # mm
    nanmask = np.array([[False, False, False], [False, False, True]])
    hz = L.velocity_hazard_snapshot(v, d, nanmask)
    assert hz[0, 0] == 0.0                  # 5 mm is below 1 cm
    assert hz[0, 1] == pytest.approx(0.2)
    assert hz[0, 2] == 0.0                  # non-finite velocity counts as 0
    assert hz[1, 0] == pytest.approx(1.0)
    assert hz[1, 1] == 0.0
    assert np.isnan(hz[1, 2])


def test_kernel_form_follows_literal(oracle_lib):
    case = S.dambreak_case(32, 96, 5.0, seed=3, hours=0.05)
    cfg = literal_cfg(case)
    cfg.hazard_maps = True
    st = L.init_state(cfg)
    o = kernel_form(case)
    o.set_hazard_tracking(True)
    for k in range(4000):
        if st.t > cfg.routing_time + cfg.min_time_step / 60:
            break
        L.step(cfg, st)
        o.fused_steps(1)
    assert k > 50
    vm = o.download_native("vmax")
    hm = o.download_native("hazard_max")
    assert np.nanmax(st.vmax_final) > 1.0 and np.nanmax(st.hazardmax_final) > 1.0
    assert np.allclose(vm, st.vmax_final, rtol=1e-9, atol=1e-12)
    assert np.allclose(hm, st.hazardmax_final, rtol=1e-9, atol=1e-12)
    # the hazard maximum is bounded by the product of the two maxima
    assert np.all(hm <= vm * o.download_native("dmax") * (1 + 1e-12) + 1e-15)
