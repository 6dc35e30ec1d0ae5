"""Time de-interleaver index maps (CPU): the oracle and the product's host
maps (atsc3_b200/timeint.py, which drive csrc/timeint.cu) against the
reference's own outputs stored in tests/golden/golden_ti.npz
(lab/m6_tbi.py, lab/m10_cti.py, lab/m9_fast.py:1087-1093), the A/327
Figure 6.5 worked example, and the structural properties the reference's
gates check (bijection, round trip)."""
import functools
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from atsc3_b200 import timeint as T

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_ti.npz")


@functools.lru_cache(maxsize=1)
def golden():
    z = np.load(GOLD)
    arrs = {k: z[k] for k in z.files}
    return json.loads(str(arrs.pop("meta_json"))), arrs


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_fig_6_5_worked_example():
    meta, _ = golden()
    g = meta["gold_fig_6_5"]
    nr, nc, nv = g["nrows"], g["ncols"], g["n_virtual"]
    mem = [""] * (nr * nv) + list("abcd") + list("efgh")
    for order in (oracle.tbi_read_order(nr, nc, nv), T.tbi_read_order(nr, nc, nv)):
        assert [mem[nv * nr + t] for t in order] == g["expect"]


def test_tbi_maps_match_reference():
    meta, arrs = golden()
    for c in meta["tbi"]:
        nr, nc, nv = c["nrows"], c["ncols"], c["n_virtual"]
        order = T.tbi_read_order(nr, nc, nv)
        assert sha(order.astype(np.int64)) == c["read_order"], (nr, nc, nv)
        if nr * nc <= 64:
            assert np.array_equal(oracle.tbi_read_order(nr, nc, nv),
                                  arrs[f"tbi_{nr}_{nc}_{nv}"])
        pos = T.tbi_positions(nr, nc, nv)
        for j, digest in enumerate(c["fec_block"]):
            assert sha(pos[j].astype(np.int64)) == digest, (nr, nc, nv, j)


def test_hybrid_index_is_the_reference_cached_gather():
    meta, _ = golden()
    for c in meta["hti"]:
        ti = T.HybridTI(c["nrows"], c["ncols"], nti=c["nti"])
        assert sha(ti.index().astype(np.int64)) == c["index"]
        assert ti.launch_args()[0] == 1          # closed form on the GPU


def test_cti_matches_reference():
    meta, _ = golden()
    for c in meta["cti"]:
        rng = np.random.default_rng(c["seed"])
        recv = rng.integers(0, 1 << 30, c["n"]).astype(np.int64)
        out, valid = oracle.cti_deinterleave(recv, c["nrows"], c["start_row"], c["n"])
        assert sha(out) == c["out"] and sha(valid.astype(np.uint8)) == c["valid"]
        ti = T.ConvolutionalTI(c["nrows"], c["start_row"], C=0, nblk=1, ncell=c["n"])
        idx = ti.index(c["n"])[0].astype(np.int64)
        got = np.where(idx >= 0, recv[np.maximum(idx, 0)], 0)
        assert sha(got) == c["out"]
        assert int((idx >= 0).sum()) == c["n_valid"]


@pytest.mark.parametrize("nr,nc,nv", [(2700, 37, 0), (2700, 37, 5), (8100, 1, 0),
                                      (2025, 16, 7)])
def test_tbi_bijection_and_round_trip(nr, nc, nv):
    order = T.tbi_read_order(nr, nc, nv)
    assert np.array_equal(np.sort(order), np.arange(nr * (nc - nv)))
    x = np.random.default_rng(nr + nc).permutation(nr * (nc - nv))
    tx = x[order]                                   # interleave
    assert np.array_equal(oracle.tbi_deinterleave(tx, nr, nc, nv), x)
    ti = T.HybridTI(nr, nc, nti=1, n_virtual=nv)
    assert np.array_equal(tx[ti.index()].ravel(), x)


def test_bad_geometry_rejected():
    with pytest.raises(ValueError):
        T.HybridTI(4, 3, n_virtual=3)
    with pytest.raises(ValueError):
        T.ConvolutionalTI(0, 0)
