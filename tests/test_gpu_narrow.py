"""GpuMinSum(dtype="bfloat16"/"float16") on the GPU against
``oracle.flood_torch_narrow`` (the reference's torch decoder in that dtype,
lab/m9_gpu.py:138-220, pinned against the reference itself by
tests/test_oracle_narrow.py): bits, conv, its and bad identical.  All three cases
mix converging and stuck blocks (16200 6/15 at 1.5 dB; the Type A 16200 3/15 at
-3.75 dB: two of six converge; 64800 8/15 at its
measured threshold, 7.75 dB: one block converges at 28 iterations, two stick
with 6 and 2 unsatisfied checks in bfloat16)."""
import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["bfloat16", "float16"])
@pytest.mark.parametrize("rate,n,mod,esn0,chan,nblk", [
    ("6/15", 16200, "QPSK", 1.5, "awgn", 6),
    ("3/15", 16200, "QPSK", -3.75, "awgn", 6),
    ("8/15", 64800, "16QAM", 7.75, "awgn", 3)])
def test_gpuminsum_narrow_vs_oracle(dtype, rate, n, mod, esn0, chan, nblk):
    import torch
    from atsc3_b200 import ldpc
    pay, cells, s2 = oracle.synth_case(
        lambda p: oracle.transmit(p, n, mod, rate)[0], nblk, C.kpayload(rate, n),
        C.cells_per_block(n, mod), esn0, chan, 21)
    q = oracle.demap(cells, C.points_for(mod, rate), C.MOD_BITS[mod], s2)
    lam = oracle.deinterleave(q, C.bicm_map(n, mod, rate), n)
    tdt = torch.bfloat16 if dtype == "bfloat16" else torch.float16
    lam_n = torch.from_numpy(np.ascontiguousarray(lam, np.float64)).to(tdt).float().numpy()
    want = oracle.flood_torch_narrow(lam_n, C.csr(rate, n), n, iters=30, alpha=0.75,
                                     dtype=dtype)
    cptr, cidx, vptr, vedge = C.csr(rate, n)
    checks = [cidx[cptr[c]:cptr[c + 1]].tolist() for c in range(len(cptr) - 1)]
    got = ldpc.GpuMinSum(checks, n, iters=30, dtype=dtype).decode(lam)
    for a, b, k in zip(got, want, ("bits", "conv", "its", "bad")):
        assert np.array_equal(np.asarray(a), np.asarray(b)), k
