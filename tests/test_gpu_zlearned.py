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


def test_compare_decoders_same_blocks():
    """The four-decoder comparison at the 6/15 16-NUC operating point on a
    small held-out set: the learned and the exact sum-product flooding
    decoders need fewer iterations than plain min-sum, the layered schedule
    fewer still, and the learned and sum-product decoders leave no block
    without a zero syndrome."""
    from atsc3_b200 import evaluate as EV
    r = EV.compare_decoders("6/15", "16QAM", 8.25, 200, chunk=200)
    d = r["decoders"]
    assert set(d) == {"plain flooding min-sum", "learned flooding min-sum",
                      "float64 sum-product flooding", "plain layered min-sum"}
    plain = d["plain flooding min-sum"]["mean_iters"]
    assert d["learned flooding min-sum"]["mean_iters"] < plain
    assert d["float64 sum-product flooding"]["mean_iters"] < plain
    assert d["plain layered min-sum"]["mean_iters"] < d["learned flooding min-sum"]["mean_iters"]
    assert d["learned flooding min-sum"]["block_errors"] == 0
    assert d["float64 sum-product flooding"]["block_errors"] == 0
