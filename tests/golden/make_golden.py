#!/usr/bin/env python3
"""Generate the golden vectors that pin the oracle to the reference.

Runs ONLY where a Felbs/atsc3 checkout exists (ATSC3_REFERENCE, default
/root/reference): it imports the reference's own Python (lab/m3_ldpc.py,
lab/m6_bicm.py, lab/m44_ldm.py, lab/m9_accel.py) and its compiled
lab/ldpc_kernel.c (through oracle/_ref, built by oracle/build.py), runs them
on seeded synthetic inputs and writes digests and small arrays to
tests/golden/golden.npz.  The tests never import the reference; they
recompute everything with the oracle and compare with this file.

    python tests/golden/make_golden.py
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
import m6_bicm as B                            # noqa: E402
import m9_accel                                # noqa: E402
import spec_bitint as BI                       # noqa: E402

OUT = os.path.join(HERE, "golden.npz")

# (name, n, mod, rate, nblk, esn0_db, channel, seed)
CASES = [
    ("c16_64qam_11_15", 16200, "64QAM", "11/15", 6, 15.5, "awgn", 5),
    ("c16_qpsk_2_15", 16200, "QPSK", "2/15", 4, 1.0, "awgn", 6),
    ("c16_256qam_13_15", 16200, "256QAM", "13/15", 3, 22.0, "awgn", 7),
    ("c64_256qam_10_15", 64800, "256QAM", "10/15", 3, 20.0, "awgn", 11),
    ("c64_16qam_6_15_ray", 64800, "16QAM", "6/15", 2, 8.0, "rayleigh", 12),
    ("c64_64qam_7_15", 64800, "64QAM", "7/15", 2, 13.0, "awgn", 13),
    ("c64_qpsk_5_15", 64800, "QPSK", "5/15", 2, 0.5, "awgn", 14),
]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def ref_demap(cells, ch, s2):
    """lab/m44_ldm.py:2454-2494 per-bit minima over the reference's own
    `_point_metric`, divided by the SUPPLIED sigma2 (scalar or per cell)."""
    import m44_ldm as L
    pts = B.points_for(ch.mod, ch.rate)
    nb = ch.mod_bits
    nblk, ncell = cells.shape
    pr = np.asarray(pts.real, np.float32)
    pi = np.asarray(pts.imag, np.float32)
    p2f = (pts.real ** 2 + pts.imag ** 2).astype(np.float32)
    z = np.asarray(cells, np.complex128)
    zr = np.asarray(z.real, np.float32)
    zi = np.asarray(z.imag, np.float32)
    q = L._point_metric(zr.ravel(), zi.ravel(), pr, pi, p2f).reshape(
        nblk, ncell, len(pts))
    s2 = s2 if np.ndim(s2) == 0 else np.asarray(s2, np.float32)
    qr = q.reshape(nblk, ncell, *([2] * nb))
    sub = tuple(range(2, 2 + nb - 1))
    out = np.empty((nblk, ncell, nb), np.float32)
    head = (slice(None), slice(None))
    for i in range(nb):
        a = qr[head + (slice(None),) * i + (1,)].min(axis=sub)
        b = qr[head + (slice(None),) * i + (0,)].min(axis=sub)
        out[:, :, i] = (a - b) / s2
    return out.reshape(nblk, ncell * nb)


def main():
    import m44_ldm as L
    meta = {"tables": {}, "bicm": {}, "cases": {}, "bch": {}}
    arrs = {}
    # --- code tables -------------------------------------------------------
    for n in (16200, 64800):
        for r in BI.RATES:
            checks = LD.parity_check(r, n)
            tabs = LD._kernel_tables(checks, n)
            meta["tables"][f"{n}:{r}"] = [sha(np.asarray(t, np.int32))
                                          for t in tabs[:4]]
    for (n, mod, r) in sorted(BI.GROUPWISE):
        if BI.DEMUX[(n, mod)][1] is None:
            continue
        meta["bicm"][f"{n}:{mod}:{r}"] = sha(B.bicm_map(n, mod, r).astype(np.int32))
    # --- BCH: random messages, both lengths, plus all-zero / all-one --------
    rng = np.random.default_rng(99)
    for n, k in ((16200, 11880), (16200, 2160), (64800, 43200), (64800, 25920)):
        m = rng.integers(0, 2, (6, k)).astype(np.uint8)
        m = np.concatenate([m, np.zeros((1, k), np.uint8),
                            np.ones((1, k), np.uint8)])
        syn = m9_accel.bch_syndrome_batch(m, n)
        syn1 = [B.bch_syndrome(row, n) for row in m[:2]]
        assert syn[:2] == syn1
        arrs[f"bch_msg/{n}:{k}"] = np.packbits(m, axis=1)
        meta["bch"][f"{n}:{k}"] = [hex(s) for s in syn]
    # --- decode cases -------------------------------------------------------
    for name, n, mod, rate, nblk, esn0, chan, seed in CASES:
        ch = B.PlpChain(n, mod, rate, iters=50)
        cw_ref = []

        def tx(pay):
            rows = []
            for p in pay:
                scr = np.asarray(p, np.uint8) ^ __import__("m4_scrambler").sequence(len(p))
                nouter = B.bch_encode(scr, n)
                cw = LD.encode(nouter, rate, n)
                cw_ref.append(cw)
                rows.append(B.map_cells(cw[ch.lam_of_q], mod, rate))
            return np.array(rows)

        pay, cells, s2 = oracle.synth_case(tx, nblk, ch.kpayload,
                                           ch.cells_per_fec, esn0, chan, seed)
        q = ref_demap(cells, ch, s2)
        lam = np.empty((nblk, n), np.float32)
        lam[:, ch.lam_of_q] = q
        tabs = LD._kernel_tables(ch.checks, n)
        bits, conv, its, bad = oracle.flood_ref(lam, tabs[:4], n, iters=50,
                                                alpha=0.75)
        # the reference's own Python dispatch reaches the same kernel
        LD._KERNEL_STATE["lib"] = None
        os.environ.pop("ATSC3_LDPC_KERNEL", None)
        syn = m9_accel.bch_syndrome_batch(bits[:, :ch.kldpc], n)
        seq = __import__("m4_scrambler").sequence(ch.kpayload)
        payload = np.packbits(bits[:, :ch.kpayload] ^ seq[None, :], axis=1)
        c = {"n": n, "mod": mod, "rate": rate, "nblk": nblk, "esn0": esn0,
             "channel": chan, "seed": seed,
             "payload_sha": sha(pay), "cw_sha": sha(np.array(cw_ref)),
             "cells_sha": sha(cells), "llr_q_sha": sha(q),
             "lam_sha": sha(lam),
             "bits_sha": sha(bits), "conv": conv.astype(int).tolist(),
             "its": its.tolist(), "bad": bad.tolist(),
             "bch": [hex(s) for s in syn],
             "payload_bytes_sha": sha(payload),
             "payload_ok": [bool(np.array_equal(
                 np.unpackbits(payload[i])[:ch.kpayload], pay[i]))
                 for i in range(nblk)]}
        # a few raw LLR values for human inspection
        arrs[f"llr_head/{name}"] = q[:, :64].copy()
        # float64 torch/numpy semantics on the 16200 cases (slow for 64800)
        if n == 16200:
            b64, c64, i64, d64 = LD.min_sum_decode_batch(
                lam.astype(np.float64), ch.checks, n, iters=50, alpha=0.75,
                dtype=np.float64)
            c["f64_bits_sha"] = sha(b64)
            c["f64_conv"] = c64.astype(int).tolist()
            c["f64_its"] = i64.tolist()
            c["f64_bad"] = d64.tolist()
        # row-estimated sigma2 demap (lab/m44_ldm.py:2454) on the same cells
        qe = L.demap_batch_qam(np.asarray(cells, np.complex128), ch, None, 1)
        c["llr_q_est_sha"] = sha(qe)
        arrs[f"llr_est_head/{name}"] = qe[:, :64].copy()
        meta["cases"][name] = c
        print(name, "conv", int(conv.sum()), "/", nblk, "its", its.tolist(),
              "bch0", sum(1 for s in syn if s == 0))
    arrs["meta_json"] = np.array(json.dumps(meta, sort_keys=True))
    np.savez_compressed(OUT, **arrs)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
