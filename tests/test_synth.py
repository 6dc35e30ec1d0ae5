"""The package transmitter (torch, used by the bench) against the oracle and
the reference codeword digests -- CPU tensors, no GPU needed."""
import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C
from atsc3_b200 import synth
from golden_util import golden, sha

CASES = sorted(golden()[0]["cases"])


@pytest.mark.parametrize("name", CASES)
def test_transmitter_matches_reference_codewords(name):
    import torch
    c = golden()[0]["cases"][name]
    n, mod, rate = c["n"], c["mod"], c["rate"]
    rng = np.random.default_rng(c["seed"])
    pay = rng.integers(0, 2, (c["nblk"], C.kpayload(rate, n)), dtype=np.uint8)
    tx = synth.Transmitter(n, mod, rate, device="cpu")
    cells, cw = tx.encode(torch.from_numpy(pay))
    assert sha(cw.numpy()) == c["cw_sha"]
    ocells, _ = oracle.transmit(pay, n, mod, rate)
    assert np.array_equal(cells.numpy(), ocells.astype(np.complex64))


def test_standin_constellations_roundtrip():
    import torch
    for mod in ("1024QAM", "4096QAM"):
        tx = synth.Transmitter(64800, mod, "10/15", device="cpu")
        pay = torch.randint(0, 2, (1, tx.kp), dtype=torch.uint8)
        cells, cw = tx.encode(pay)
        assert cells.shape == (1, C.cells_per_block(64800, mod))
        cptr, cidx, _, _ = C.csr("10/15", 64800)
        syn = np.bitwise_xor.reduceat(cw.numpy()[:, cidx], cptr[:-1], axis=1)
        assert not syn.any()
