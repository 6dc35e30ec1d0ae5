"""The oracle's CPE restatement (oracle.cpe_correct) reproduces the
reference's own lab/m6_cells.py:176-209 outputs stored in
tests/golden/golden_cpe.npz, bit for bit, on the same seeded pools."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_cpe.npz")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cases():
    return json.loads(str(np.load(GOLD)["meta_json"]))["cases"]


def case_inputs(c):
    return oracle.cpe_pool(c["nsym"], c["per_sym"], [tuple(m) for m in c["mods"]],
                           c["seed"])


@pytest.mark.parametrize("name", sorted(cases()))
def test_oracle_cpe_matches_reference(name):
    c = cases()[name]
    pool, sym, alph, region, dummy = case_inputs(c)
    assert sha(pool) == c["pool"]
    out, gains = oracle.cpe_correct(pool, sym, alph, region, dummy, iters=c["iters"])
    assert sha(out) == c["out"]
    assert [[g.real, g.imag] for _, g in sorted(gains.items())] == c["gains"]
