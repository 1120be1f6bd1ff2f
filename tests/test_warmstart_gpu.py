"""The learned warm start on held-out pairs (the network trained on the GPU with the project's own
kernels by `python -m skmimageregistration_b200.warmstart train --n 512 --epochs 60`, weights and the
validated number of first-level refinement iterations in skmimageregistration_b200/warmstart_weights.npz).

The plain zero-started multi-scale registration is the judge.  Measured on a B200 for the four
held-out pairs below: the warm-started run (first level from the prediction, 50 refinement iterations
instead of 100, later levels on their plain schedule) reached the plain run's final NCC within 1e-3 on
three pairs and within 1.1e-3 on the fourth, with 250 optimizer iterations instead of 300.  A
prediction that does not lower the first level's metric value falls back to the plain run, bit for bit.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _net():
    pytest.importorskip("torch")
    from skmimageregistration_b200 import warmstart as W
    if not os.path.exists(W.WEIGHTS_PATH):
        pytest.fail("trained weights missing: %s" % W.WEIGHTS_PATH)
    return W, W.WarmStartNet.load()


def test_warm_start_reaches_plain_ncc_with_fewer_iterations():
    W, net = _net()
    res = W.evaluate_gain(net, [900_000, 900_001, 900_002, 900_003])
    for r in res:
        print(r)
        assert r["used_warm_start"], r
        assert r["warm_iterations"] < r["plain_iterations"], r
        assert r["warm_ncc"] >= r["plain_ncc"] - 2e-3, r
    assert sum(r["within_1e-3"] for r in res) >= 3


def test_bad_prediction_falls_back_to_the_plain_method():
    W, net = _net()
    net.label_scale *= 1e4                                       # a useless, huge prediction
    from skmimageregistration_b200 import register as R
    f, m = W.make_pairs([900_010], workers=1)[0]
    d_w, rep_w, used = W.register_with_warm_start(net, f, m)
    d_p, rep_p = R.register(m, f, (1.0, 1.0, 1.0), None, W.MS_CONFIG)
    assert not used
    assert np.array_equal(d_w, d_p)
