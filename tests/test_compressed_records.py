"""The GPU decoders keep one record per check (min1*alpha, min2*alpha, the
first-minimum position, one sign bit per edge) instead of one message per
edge.  This numpy model of exactly that state, driven by the same tables,
must reproduce the per-edge oracle bit for bit -- a CPU check of the
algorithm the flooding kernel implements."""
import numpy as np

import oracle
from atsc3_b200 import codes as C


def compressed_flood(llr, rate, n, iters, alpha):
    cptr, cidx, vptr, vedge = C.csr(rate, n)
    nc = len(cptr) - 1
    deg = np.diff(cptr)
    chk = np.repeat(np.arange(nc), deg)
    pos = np.arange(len(cidx)) - cptr[chk]
    al = np.float32(alpha)
    out = []
    for lam in np.atleast_2d(llr).astype(np.float32):
        tot = lam.copy()
        A = np.zeros(nc, np.float32)
        Bm = np.zeros(nc, np.float32)
        F = np.zeros(nc, np.int64)
        S = np.zeros(len(cidx), bool)          # sign bit per edge
        res = None
        for it in range(iters + 1):
            t = tot[cidx]
            syn = np.bitwise_xor.reduceat((t < 0).astype(np.uint8), cptr[:-1])
            bad = int(syn.sum())
            if bad == 0 or it == iters:
                res = ((tot < 0).astype(np.uint8), bad == 0, it,
                       0 if bad == 0 else bad)
                break
            mo = np.where(pos == F[chk], Bm[chk], A[chk])
            mo = np.where(S, -mo, mo).astype(np.float32)
            v = (t - mo).astype(np.float32)
            sg = v < 0
            mag = np.abs(v)
            # first minimum and second minimum with multiplicity, per check
            order = np.lexsort((pos, mag, chk))
            first_e = order[cptr[:-1]]
            second_e = order[cptr[:-1] + 1]
            min1, min2 = mag[first_e], mag[second_e]
            par = np.bitwise_xor.reduceat(sg.astype(np.uint8), cptr[:-1])
            A = (min1 * al).astype(np.float32)
            Bm = (min2 * al).astype(np.float32)
            F = pos[first_e]
            S = sg ^ par[chk].astype(bool)
            m = np.where(pos == F[chk], Bm[chk], A[chk])
            m = np.where(S, -m, m).astype(np.float32)
            s = np.zeros(n, np.float32)
            mv = m[vedge]
            for k in range(int(np.diff(vptr).max())):
                has = np.diff(vptr) > k
                idx = vptr[:-1][has] + k
                s[has] = (s[has] + mv[idx]).astype(np.float32)
            tot = (lam + s).astype(np.float32)
        out.append(res)
    return ([r[0] for r in out], [r[1] for r in out], [r[2] for r in out],
            [r[3] for r in out])


def test_compressed_state_equals_per_edge_messages():
    rng = np.random.default_rng(8)
    for rate, n in (("11/15", 16200), ("4/15", 16200)):
        tabs = C.csr(rate, n)
        llr = (rng.standard_normal((2, n)) * 2.0 + 1.2).astype(np.float32)
        a = compressed_flood(llr, rate, n, 8, 0.75)
        b = oracle.flood(llr, tabs, n, iters=8, alpha=0.75)
        assert np.array_equal(np.array(a[0]), b[0])
        assert list(a[1]) == b[1].tolist()
        assert list(a[2]) == b[2].tolist()
        assert list(a[3]) == b[3].tolist()
