"""The oracle's exact sum-product (oracle.sum_product) reproduces the
reference's own lab/m16_margin.py:325-390 outputs stored in
tests/golden/golden_sp.npz, on the same seeded inputs."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_sp.npz")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cases():
    return json.loads(str(np.load(GOLD)["meta_json"]))["cases"]


@pytest.mark.parametrize("name", sorted(cases()))
def test_oracle_sum_product_matches_reference(name):
    c = cases()[name]
    lam, cw = oracle.near_miss_llr(c["rate"], c["n"], c["nblk"], c["mu"], c["seed"])
    assert sha(lam) == c["llr"]
    bits, conv, its, bad = oracle.sum_product(lam, C.csr(c["rate"], c["n"]),
                                              c["n"], iters=c["iters"])
    assert conv.tolist() == c["conv"]
    assert its.tolist() == c["its"]
    assert bad.tolist() == c["bad"]
    assert sha(bits.astype(np.uint8)) == c["bits"]
