#!/usr/bin/env python3
"""Golden vectors of the reference's alpha ladder.

Runs ONLY where a Felbs/atsc3 checkout exists (ATSC3_REFERENCE, default
/root/reference): decodes seeded consistent-Gaussian LLRs (the oracle's
`near_miss_llr`, plain numpy) with the reference's own batched ladder,
lab/m44_ldm.py:2497-2526 ldpc_batch (rungs 1.0, 0.85, 0.75 from
lab/m6_bicm.py:313, sum-product rescue off), whose min-sum is the
reference's compiled lab/ldpc_kernel.c (oracle/_ref, built by
oracle/build.py, handed to lab/m3_ldpc.py's loader), and writes digests to
tests/golden/golden_ladder.npz.  The tests never import the reference.

    python tests/golden/make_golden_ladder.py
"""
from __future__ import annotations

import ctypes
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
os.environ.pop("ATSC3_LDM_SP", None)

import oracle                                  # noqa: E402
from oracle import build as OB                 # noqa: E402
import m3_ldpc as LD                           # noqa: E402
import m6_bicm as B                            # noqa: E402
import m44_ldm as L                            # noqa: E402

OUT = os.path.join(HERE, "golden_ladder.npz")
# (name, n, mod, rate, nblk, mu, seed, iters)
CASES = [("ladder_6_15", 64800, "16QAM", "6/15", 6, 2.1, 11, 30),
         ("ladder_6_15_near", 64800, "16QAM", "6/15", 4, 1.9, 12, 30),
         ("ladder_11_15", 16200, "64QAM", "11/15", 8, 5.0, 3, 25)]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def ref_kernel():
    OB.build()
    lib = ctypes.CDLL(OB.REF_SO)
    lib.ldpc_kernel_abi.restype = ctypes.c_int32
    i32 = np.ctypeslib.ndpointer(np.int32, flags="C")
    f32 = np.ctypeslib.ndpointer(np.float32, flags="C")
    u8 = np.ctypeslib.ndpointer(np.uint8, flags="C")
    lib.ldpc_minsum_f32.restype = ctypes.c_int32
    lib.ldpc_minsum_f32.argtypes = [f32, ctypes.c_int32, ctypes.c_int32,
                                    ctypes.c_int32, ctypes.c_int32, i32, i32,
                                    i32, i32, ctypes.c_int32, ctypes.c_float,
                                    u8, u8, i32, i32, f32]
    return lib


def main():
    LD._KERNEL_STATE["lib"] = ref_kernel()
    meta = {"ladder": list(B.PlpChain.ALPHA_LADDER), "cases": {}}
    for name, n, mod, rate, nblk, mu, seed, iters in CASES:
        lam, cw = oracle.near_miss_llr(rate, n, nblk, mu, seed)
        ch = B.PlpChain(n, mod, rate, iters=iters)
        bits, conv, bad = L.ldpc_batch(lam, ch, gpu=None, iters=iters,
                                       threads=1, alpha=None)
        meta["cases"][name] = {"n": n, "rate": rate, "nblk": nblk, "mu": mu,
                               "seed": seed, "iters": iters, "llr": sha(lam),
                               "bits": sha(bits.astype(np.uint8)),
                               "conv": [bool(x) for x in conv],
                               "bad": [int(x) for x in bad]}
        print(name, meta["cases"][name]["conv"], meta["cases"][name]["bad"])
    np.savez_compressed(OUT, meta_json=np.array(json.dumps(meta)))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
