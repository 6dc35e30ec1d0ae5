"""Negative controls, as the reference's lab/m6_bicm.py:484-516 gates carry:
the full chain decodes a clean-ish link, and the SAME cells fed wrongly --
rotated by 90 degrees, conjugated, shuffled, or de-interleaved with the
inverted group-wise interleaver -- must not decode (BCH not clean).  A parity
test that passed on a vacuous decoder would fail here."""
import numpy as np
import pytest

from atsc3_b200 import codes as C

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,mod,rate,esn0", [(16200, "64QAM", "11/15", 16.0),
                                             (64800, "16QAM", "6/15", 9.0)])
def test_controls_must_not_decode(n, mod, rate, esn0):
    import torch
    from atsc3_b200 import bch as BCH
    from atsc3_b200 import demap as DM
    from atsc3_b200 import ldpc as LDPC
    from atsc3_b200 import synth
    from atsc3_b200.pipeline import FecPipeline
    tx = synth.Transmitter(n, mod, rate, device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(17)
    pay = torch.randint(0, 2, (4, tx.kp), generator=g, device="cuda", dtype=torch.uint8)
    x, _ = tx.encode(pay)
    y, s2 = synth.channel(x, esn0, "awgn", g)
    p = FecPipeline(n, mod, rate, iters=50, alpha=0.75)
    ok = p.decode(y, float(s2))["ok"].cpu().numpy()
    assert ok.tolist() == [1, 1, 1, 1]                       # the positive leg
    perm = torch.from_numpy(np.random.default_rng(3).permutation(y.shape[1])).cuda()
    for name, bad in (("rotated", y * 1j), ("conjugated", y.conj()),
                      ("shuffled", y[:, perm])):
        r = p.decode(bad.contiguous(), float(s2))["ok"].cpu().numpy()
        assert r.sum() == 0, name
    # inverted group-wise interleaver
    lq = torch.from_numpy(np.array(C.bicm_map(n, mod, rate, gw_invert=True),
                                   np.int32)).cuda()
    q = DM.demap(y, mod, rate, sigma2=float(s2), n=n, deinterleave=False)
    lam = torch.empty((4, n), dtype=torch.float32, device="cuda")
    lam[:, lq.long()] = q
    o = LDPC.decode_flood(p.plan, lam, iters=50, want_bits=False, want_hard=True)
    chk = BCH.bch_check(o["hard"], C.kldpc(rate, n), n, want_payload=False)
    assert int(chk["ok"].sum()) == 0
