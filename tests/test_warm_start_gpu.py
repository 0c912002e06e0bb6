"""The learned warm start end to end: a network trained on the device on
plain bounce solutions of small maps, then a held-out map bounced from its
guess.  The plain bounce stays the judge: the warm start must reach the
same threshold in no more bounces, with the lightmap within one unit of
the last place of the plain one on at least 99.9 % of luxels, and the
trained network must guess better than an untrained one."""
import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import learned as LN, lighting as L, roomgrid as rg

pytestmark = pytest.mark.gpu


def test_trained_warm_start_beats_plain_and_untrained():
    import torch
    x, t = LN.collect([LN.training_config(k) for k in range(6)])
    assert len(x) > 100_000 and torch.isfinite(t).all()
    held = LN.training_config(3, seed0=900)            # a 5x5 map not trained on
    w = rg.generate(held)
    with L.LightingStage(w) as st:
        off, lst = L.pvs_lists(w)
        st.upload_bounce(L.face_reflectivity(w), off, lst, threshold=0.1)
        plain, _, _ = st.light_pass()
        plain_bounces = st.bounce_stats().bounces
        hx, ht = st.bounce_features()
        untrained = LN.Network(st.tracer, seed=1)
        trained = LN.Network(st.tracer, seed=1)
        first = LN.train(trained, x, t, steps=1200)
        err_untrained = (untrained.forward(hx) - ht).abs().mean().item()
        err_trained = (trained.forward(hx) - ht).abs().mean().item()
        st.set_bounce_model(trained)
        warm, _, _ = st.light_pass()
        warm_bounces = st.bounce_stats().bounces
        st.set_bounce_model(None)
        again, _, _ = st.light_pass()
        held_out = LN.evaluate(trained, [LN.heldout_config(0)])
        untrained.close()
        trained.close()
    assert err_trained < 0.5 * err_untrained and err_trained < 0.25, (err_trained, err_untrained)
    assert warm_bounces <= plain_bounces, (warm_bounces, plain_bounces)
    assert LN.within_one_lsb(warm, plain) >= 0.999
    assert np.array_equal(again, plain)                # detaching restores the plain bounce exactly
    (ev,) = held_out
    assert 0.0 < ev["rho"] < 1.0 and 0.0 < ev["eps"] < 1.0, ev
    assert ev["warm_bounces"] <= ev["plain_bounces"] and ev["within_1_lsb"] >= 0.999, ev
