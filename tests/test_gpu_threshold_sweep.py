"""Every A/322 code with real codewords at its measured 16-NUC threshold
(atsc3_b200/data/thresholds.json; converging and stuck blocks mixed), the
default GPU decoder against the C oracle in the three decode variants the
drop-ins offer: kernel semantics in float32 (lab/ldpc_kernel.c), torch
semantics in float32 and in float64 (lab/m9_gpu.py, lab/m3_ldpc.py:560-630).
bits, conv, its and bad identical."""
import json
import os

import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C

pytestmark = pytest.mark.gpu

TH = json.load(open(os.path.join(os.path.dirname(C.__file__), "data", "thresholds.json")))
MOD = "16QAM"


@pytest.mark.parametrize("n", [16200, 64800])
@pytest.mark.parametrize("rate", C.RATES)
def test_code_at_threshold_all_variants(rate, n):
    import torch
    from atsc3_b200 import ldpc as LDPC
    nblk = 10 if n == 16200 else 5
    pay, cells, s2 = oracle.synth_case(
        lambda p: oracle.transmit(p, n, MOD, rate)[0], nblk, C.kpayload(rate, n),
        C.cells_per_block(n, MOD), TH[f"{n}|{MOD}|{rate}"], "awgn",
        2000 + int(rate.split("/")[0]))
    q = oracle.demap(cells, C.points_for(MOD, rate), C.MOD_BITS[MOD], s2)
    lam = oracle.deinterleave(q, C.bicm_map(n, MOD, rate), n).astype(np.float32)
    tabs = C.csr(rate, n)
    for sem, dt in (("kernel", np.float32), ("torch", np.float32), ("torch", np.float64)):
        x = lam.astype(dt)
        want = oracle.flood(x, tabs, n, iters=50, alpha=0.75,
                            semantics=1 if sem == "torch" else 0, dtype=dt)
        plan = LDPC.plan_for(rate, n, dtype=np.dtype(dt).name)
        o = LDPC.decode_flood(plan, torch.from_numpy(x).cuda(), iters=50, alpha=0.75,
                              semantics=sem)
        tag = (sem, np.dtype(dt).name)
        assert np.array_equal(o["bits"].cpu().numpy(), want[0]), tag
        assert o["conv"].cpu().numpy().astype(bool).tolist() == want[1].tolist(), tag
        assert o["its"].cpu().numpy().tolist() == want[2].tolist(), tag
        assert o["bad"].cpu().numpy().tolist() == want[3].tolist(), tag
