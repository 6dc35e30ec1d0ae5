#!/usr/bin/env python3
"""Golden vectors of the reference's time de-interleavers.

Runs ONLY where a Felbs/atsc3 checkout exists (ATSC3_REFERENCE, default
/root/reference): imports the reference's lab/m6_tbi.py (twisted block
interleaver, A/322 7.1.5.4) and lab/m10_cti.py (convolutional interleaver,
A/322 7.1.4), evaluates their index maps and de-interleavers on seeded
inputs, and writes digests and small arrays to tests/golden/golden_ti.npz.
The tests never import the reference.

    python tests/golden/make_golden_ti.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("ATSC3_REFERENCE", "/root/reference")
sys.dont_write_bytecode = True
sys.path.insert(0, REF)
sys.path.insert(0, os.path.join(REF, "lab"))

import m6_tbi as T                             # noqa: E402
import m10_cti as CT                           # noqa: E402

OUT = os.path.join(HERE, "golden_ti.npz")
# (nrows, ncols, n_virtual)
TBI = [(4, 3, 1), (4, 3, 0), (12, 5, 2), (2700, 37, 0), (8100, 39, 3),
       (16200, 4, 0), (2025, 16, 7)]
# (nrows, start_row, n)
CTI = [(8, 5, 4096), (512, 191, 700000), (1024, 1002, 2200000)]
# the cached hybrid-TI gather of lab/m9_fast.py:1087-1093: (nrows, ncols, nti)
HTI = [(2700, 37, 2), (16200, 4, 3)]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    meta = {"tbi": [], "cti": [], "hti": []}
    arrs = {}
    for nr, nc, nv in TBI:
        order = T.read_order(nr, nc, nv)
        per_block = [sha(T.fec_block(np.arange(nr * (nc - nv), dtype=np.int64),
                                     j, nr, nc, nv).astype(np.int64))
                     for j in range(nc - nv)]
        meta["tbi"].append({"nrows": nr, "ncols": nc, "n_virtual": nv,
                            "read_order": sha(order.astype(np.int64)),
                            "fec_block": per_block})
        if nr * nc <= 64:
            arrs[f"tbi_{nr}_{nc}_{nv}"] = order.astype(np.int64)
    for nrows, start, n in CTI:
        rng = np.random.default_rng(nrows + start)
        recv = rng.integers(0, 1 << 30, n).astype(np.int64)
        out, valid = CT.deinterleave(recv, nrows, start)
        meta["cti"].append({"nrows": nrows, "start_row": start, "n": n,
                            "seed": nrows + start, "out": sha(out.astype(np.int64)),
                            "valid": sha(valid.astype(np.uint8)),
                            "n_valid": int(valid.sum())})
    for nrows, ncols, nti in HTI:
        per_ti = nrows * ncols
        hidx = np.array([ti * per_ti + T.fec_block(np.arange(per_ti), j, nrows,
                                                   ncols, 0)
                         for ti in range(nti) for j in range(ncols)], np.int64)
        meta["hti"].append({"nrows": nrows, "ncols": ncols, "nti": nti,
                            "index": sha(hidx)})
    meta["gold_fig_6_5"] = T.GOLD
    arrs["meta_json"] = np.array(json.dumps(meta))
    np.savez_compressed(OUT, **arrs)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
