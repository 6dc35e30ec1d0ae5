"""BCH syndromes on the GPU for all 24 codes (both lengths, every rate):
random K_ldpc-bit messages and one valid BCH codeword per code through
``bch_syndrome_batch`` (the m9_accel drop-in), equal to the oracle's
big-integer remainder (lab/m6_bicm.py:269-280); the valid codeword's
syndrome is 0."""
import zlib

import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [16200, 64800])
@pytest.mark.parametrize("rate", C.RATES)
def test_bch_syndrome_every_code(rate, n):
    from atsc3_b200 import bch
    k = C.ldpc_params(rate, n)[1]
    rng = np.random.default_rng(zlib.crc32(f"{n}|{rate}".encode()))
    msgs = rng.integers(0, 2, (4, k), dtype=np.uint8)
    info = rng.integers(0, 2, (1, C.kpayload(rate, n)), dtype=np.uint8)
    msgs[3] = oracle.bch_encode(info, n)[0]
    want = oracle.bch_syndrome(msgs, n)
    got = bch.bch_syndrome_batch(msgs, n)
    assert got == list(want)
    assert got[3] == 0 and all(s != 0 for s in got[:3])
