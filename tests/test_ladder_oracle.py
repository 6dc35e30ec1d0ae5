"""The oracle's alpha ladder (oracle.ladder over the oracle's flooding
decoder) reproduces the reference's own batched ladder,
lab/m44_ldm.py:2497-2526 over its compiled lab/ldpc_kernel.c, stored in
tests/golden/golden_ladder.npz."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_ladder.npz")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def golden():
    return json.loads(str(np.load(GOLD)["meta_json"]))


@pytest.mark.parametrize("name", sorted(golden()["cases"]))
def test_oracle_ladder_matches_reference(name):
    g = golden()
    c = g["cases"][name]
    lam, cw = oracle.near_miss_llr(c["rate"], c["n"], c["nblk"], c["mu"], c["seed"])
    assert sha(lam) == c["llr"]
    bits, conv, its, bad, kept = oracle.ladder(lam, C.csr(c["rate"], c["n"]), c["n"],
                                               alphas=tuple(g["ladder"]), iters=c["iters"])
    assert conv.tolist() == c["conv"] and bad.tolist() == c["bad"]
    assert sha(bits) == c["bits"]
