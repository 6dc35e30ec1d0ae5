"""The demapper and BICM de-interleaver for every MODCOD the thresholds
table lists (both code lengths, every rate, QPSK to 4096-point; the 1024-
and 4096-point alphabets are the uniform-QAM stand-ins): noisy random cells
with a supplied per-cell sigma2 (the bit-exact path), GPU LLRs in q order and
in codeword order identical to the oracle's (lab/m44_ldm.py:2431-2494
metric and minima, / sigma2 per cell as lab/m9_fast.py:1096-1115, then
lam[lam_of_q] = q)."""
import json
import os
import zlib

import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C

pytestmark = pytest.mark.gpu

TH = json.load(open(os.path.join(os.path.dirname(C.__file__), "data", "thresholds.json")))
MODCODS = sorted(tuple(k.split("|")) for k in TH)


@pytest.mark.parametrize("n,mod,rate", MODCODS)
def test_demap_deinterleave_every_modcod(n, mod, rate):
    import torch
    from atsc3_b200 import demap as DM
    n = int(n)
    nb = C.MOD_BITS[mod]
    ncell = n // nb
    pts = np.asarray(C.alphabet(mod, rate), np.complex128)
    rng = np.random.default_rng(zlib.crc32(f"{n}|{mod}|{rate}".encode()))
    lab = rng.integers(0, len(pts), (2, ncell))
    s2 = (0.02 + 0.2 * rng.random((2, ncell))).astype(np.float32)
    noise = (rng.standard_normal((2, ncell)) + 1j * rng.standard_normal((2, ncell)))
    cells = (pts[lab] + np.sqrt(s2 / 2) * noise).astype(np.complex64)
    q = oracle.demap(cells, pts, nb, s2)
    lam = oracle.deinterleave(q, C.bicm_map(n, mod, rate), n)
    tc = torch.from_numpy(cells).cuda()
    ts = torch.from_numpy(s2).cuda()
    got_q = DM.demap(tc, mod, rate, sigma2=ts, deinterleave=False).cpu().numpy()
    got = DM.demap(tc, mod, rate, sigma2=ts, n=n).cpu().numpy()
    assert np.array_equal(got_q.view(np.uint32), np.asarray(q, np.float32).view(np.uint32))
    assert np.array_equal(got.view(np.uint32), np.asarray(lam, np.float32).view(np.uint32))
