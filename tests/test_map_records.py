"""Map records (save_output_maps.m:25-27, :160-166) in the kernel-form oracle (no GPU): the
record events follow the reference's rule -- after step k, t_save = t + the new step; a map is
kept when the last record time below t_save has advanced -- restated here over the literal
restatement's clock sequence."""
import numpy as np
import pytest

from oracle import literal as L
from tests.cases import small_vtilt
from tests.test_oracle_crosscheck import kernel_form, literal_cfg


def record_events(clock_seq, times):
    """Steps (0-based) that record, from the (t_k, new dt_k [min]) sequence of a run."""
    last = int(np.searchsorted(times, clock_seq[0][0], side="left")) - 1   # initial: below t_1
    out = []
    for k, (t, dt_new) in enumerate(clock_seq):
        idx = int(np.searchsorted(times, t + dt_new, side="left")) - 1
        if idx > last:
            out.append(k)
            last = idx
    return out


def test_record_events_follow_the_reference_rule(oracle_lib):
    case = small_vtilt(24, 24)
    case.params = dict(case.params, routing_time=6.0)
    times = np.arange(0.0, 6.01, 0.5)                 # record every 30 s, from 0
    cfg = literal_cfg(case)
    st = L.init_state(cfg)
    seq = []
    while st.t <= cfg.routing_time + cfg.min_time_step / 60:
        t0 = st.t
        L.step(cfg, st)
        seq.append((t0, st.time_step))
    expect = record_events(seq, times)
    o = kernel_form(case)
    o.set_map_records(times)
    o.run()
    assert o.map_records() == len(expect) >= 10
    for i, k in enumerate(expect):
        _, t = o.download_map_record(i)
        assert t == pytest.approx(seq[k][0], rel=1e-12)
    # the last record holds a depth map of the run (finite where the DEM is)
    d, _ = o.download_map_record(len(expect) - 1)
    assert np.isfinite(d).all() and d.max() > 0
