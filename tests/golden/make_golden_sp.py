#!/usr/bin/env python3
"""Golden vectors of the reference's exact sum-product rescue.

Runs ONLY where a Felbs/atsc3 checkout exists (ATSC3_REFERENCE, default
/root/reference): decodes seeded consistent-Gaussian LLRs (the oracle's
`near_miss_llr`, plain numpy) with the reference's own
lab/m16_margin.py:325-390 sum_product_decode_batch over the reference's
parity checks (lab/m3_ldpc.py:166-212) and writes digests of its outputs to
tests/golden/golden_sp.npz.  The tests never import the reference.

    python tests/golden/make_golden_sp.py
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
import m3_ldpc as LD                           # noqa: E402
import m16_margin as M16                       # noqa: E402

OUT = os.path.join(HERE, "golden_sp.npz")
# (name, rate, n, nblk, mu, seed, iters)
CASES = [("sp_8_15_a", "8/15", 16200, 6, 2.5, 3, 60),
         ("sp_8_15_b", "8/15", 16200, 4, 2.6, 9, 45),
         ("sp_4_15", "4/15", 16200, 4, 1.3, 5, 50)]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    meta = {"cases": {}}
    for name, rate, n, nblk, mu, seed, iters in CASES:
        lam, cw = oracle.near_miss_llr(rate, n, nblk, mu, seed)
        checks = LD.parity_check(rate, n)
        bits, conv, its, bad = M16.sum_product_decode_batch(
            lam.astype(np.float64), checks, n, iters=iters)
        meta["cases"][name] = {
            "rate": rate, "n": n, "nblk": nblk, "mu": mu, "seed": seed,
            "iters": iters, "llr": sha(lam), "bits": sha(bits.astype(np.uint8)),
            "conv": [bool(x) for x in conv], "its": [int(x) for x in its],
            "bad": [int(x) for x in bad],
            "bits_equal_codeword": [bool((bits[b] == cw[b]).all())
                                    for b in range(nblk)]}
        print(name, meta["cases"][name]["conv"], meta["cases"][name]["its"],
              meta["cases"][name]["bad"])
    np.savez_compressed(OUT, meta_json=np.array(json.dumps(meta)))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
