"""The whole chain for every MODCOD of the thresholds table: one real
codeword (two for 16200) at the MODCOD's measured threshold + 1 dB, AWGN,
supplied sigma2, through ``FecPipeline.decode`` (demap + de-interleave,
edge-buffer LDPC in kernel semantics, BCH + descramble) against the oracle
chain (lab/m44_ldm.py:2348-2390 order: demap, lam[lam_of_q] = q,
lab/ldpc_kernel.c, BCH remainder, descramble): LLRs, conv, its, bad, BCH
verdict and payload bytes identical."""
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
def test_pipeline_every_modcod(n, mod, rate):
    import torch
    from atsc3_b200.pipeline import FecPipeline
    n = int(n)
    nblk = 2 if n == 16200 else 1
    nb = C.MOD_BITS[mod]
    kp = C.kpayload(rate, n)
    k = C.ldpc_params(rate, n)[1]
    pts = np.asarray(C.alphabet(mod, rate), np.complex128)
    pay, cells, s2 = oracle.synth_case(
        lambda p: oracle.transmit(p, n, mod, rate, pts=pts)[0], nblk, kp, n // nb,
        TH[f"{n}|{mod}|{rate}"] + 1.0, "awgn", zlib.crc32(f"{n}|{mod}|{rate}".encode()))
    q = oracle.demap(cells, pts, nb, s2)
    lam = oracle.deinterleave(q, C.bicm_map(n, mod, rate), n)
    bits, conv, its, bad = oracle.flood(lam, C.csr(rate, n), n, iters=50, alpha=0.75)
    ok = [s == 0 for s in oracle.bch_syndrome(bits[:, :k], n)]
    want_pay = np.packbits(bits[:, :kp] ^ C.scrambler_sequence(kp)[None, :], axis=1)
    p = FecPipeline(n, mod, rate, iters=50, alpha=0.75, device=torch.device("cuda"))
    ws = p.decode(torch.from_numpy(np.ascontiguousarray(cells, np.complex64)).cuda(),
                  float(s2))
    torch.cuda.synchronize()
    assert np.array_equal(ws["lam"].cpu().numpy().view(np.uint32),
                          np.asarray(lam, np.float32).view(np.uint32))
    assert ws["conv"].cpu().numpy().astype(bool).tolist() == conv.tolist()
    assert ws["its"].cpu().numpy().tolist() == its.tolist()
    assert ws["bad"].cpu().numpy().tolist() == bad.tolist()
    assert ws["ok"].cpu().numpy().astype(bool).tolist() == ok
    assert np.array_equal(ws["payload"].cpu().numpy(), want_pay)
