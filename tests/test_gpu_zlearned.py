"""What the trained weights buy: a short training run of the unrolled
weighted min-sum on this package's own demapper output, then a held-out
comparison against plain normalised min-sum under the same flooding
schedule (BCH-arbitrated block errors, mean iterations)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_training_lowers_loss_and_iterations():
    import torch
    from atsc3_b200 import evaluate as EV
    from atsc3_b200 import learned as LR
    rate, mod, n = "8/15", "64QAM", 64800
    thr = 11.0                                    # near the waterfall
    al, be, hist, man = LR.train(rate, n, mod, steps=80, nblk=64, iters=12,
                                 esn0=(thr - 0.5, thr + 1.5), channel="mixed",
                                 seed=3, log_every=20)
    assert hist[-1][1] < hist[0][1]               # the loss went down
    code = LR.WmsCode(rate, n)
    w = LR.inference_weights(al, be, code.buckets)
    rows = EV.sweep(rate, mod, w, [thr + 0.6], 1200, chunk=600)
    p, l = rows[0]["plain"], rows[0]["learned"]
    # fewer iterations at no worse block error rate
    assert l["mean_iters"] < p["mean_iters"]
    assert l["block_errors"] <= p["block_errors"] + 2
