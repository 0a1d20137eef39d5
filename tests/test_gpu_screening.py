"""The screening pipeline end to end at a small size (64 x 64 members, short runs): solver
data, three networks trained on it, screening of held-out members.  What the trained
networks gain over the same networks untrained is their held-out loss; the members/h and
accuracy figures of the full-size study are reported by bench.py --surrogate."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trained_screener_beats_untrained_on_heldout_members():
    from hydropol2d_b200 import screening
    res = screening.study(n_train=128, n_test=32, size=64, epochs=6, batch=16, n_fp64=4,
                          member_kw=dict(rain_tail_min=5.0, breach_minutes=5.0))
    assert np.isfinite(res["final_loss"]).all()
    assert res["heldout_loss"]["trained"] < 0.5 * res["heldout_loss"]["untrained"], res["heldout_loss"]
    assert 0 <= res["rerun_members"] <= res["n_test"]
    # members that were not rerun carry the surrogate's map, the rest the solver's
    assert res["accepted_in_subset"] <= res["fp64_subset"]
