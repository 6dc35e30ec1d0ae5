#!/usr/bin/env python3
"""Golden vectors of the reference's common phase error correction.

Runs ONLY where a Felbs/atsc3 checkout exists (ATSC3_REFERENCE, default
/root/reference): corrects seeded synthetic cell pools (the oracle's
`cpe_pool`, plain numpy) with the reference's own lab/m6_cells.py:176-209
cpe_correct and writes digests of its outputs to tests/golden/golden_cpe.npz.
The tests never import the reference.

    python tests/golden/make_golden_cpe.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("ATSC3_REFERENCE", "/root/reference")
sys.dont_write_bytecode = True
sys.path.insert(0, ROOT)
sys.path.insert(0, REF)
sys.path.insert(0, os.path.join(REF, "lab"))

import oracle                                  # noqa: E402
import m6_cells as CE                          # noqa: E402

OUT = os.path.join(HERE, "golden_cpe.npz")
# (name, nsym, cells per symbol, (mod, rate) of regions 0 and 1, seed, iters)
CASES = [("cpe_64_16", 6, 2000, (("64QAM", "8/15"), ("16QAM", "6/15")), 3, 3),
         ("cpe_256_qpsk", 4, 3001, (("256QAM", "10/15"), ("QPSK", "4/15")), 4, 3),
         ("cpe_16_16_it5", 3, 1500, (("16QAM", "9/15"), ("16QAM", "6/15")), 5, 5)]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    meta = {"cases": {}}
    for name, nsym, per, mods, seed, iters in CASES:
        pool, sym, alph, region, dummy = oracle.cpe_pool(nsym, per, mods, seed)
        out, gains = CE.cpe_correct(pool, sym, alph, region, dummy, iters=iters)
        meta["cases"][name] = {
            "nsym": nsym, "per_sym": per, "mods": [list(m) for m in mods],
            "seed": seed, "iters": iters, "pool": sha(pool), "out": sha(out),
            "gains": [[g.real, g.imag] for _, g in sorted(gains.items())]}
        print(name, sha(out)[:12])
    np.savez_compressed(OUT, meta_json=np.array(json.dumps(meta)))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
