"""The quasi-cyclic decoder's circulant descriptors, expanded on the CPU with
the kernel's own index formulas, must reproduce the CSR tables exactly: every
check's columns in position order, and every bit's (check, position) list in
the reference summation order (vedge)."""
import numpy as np
import pytest

from atsc3_b200 import codes as C
from atsc3_b200 import native as N

QZ = 360


def qc_tables(rate, n, cluster):
    typ, K, M1, M2, Q1, Q = C.ldpc_params(rate, n)
    rowptr, addr = [np.ascontiguousarray(a, np.int32) for a in C.address_rows(rate, n)]
    meta = np.zeros(48, np.int32)
    args = [n, K, Q, rowptr.ctypes.data, addr.ctypes.data, cluster]
    N.call("atsc3_ldpc_qc_tables_host", *args, meta.ctypes.data, None, None,
           None, None, None, None)
    nbi = K // QZ
    rdesc = np.zeros((meta[0], 2), np.int32)
    rptr = np.zeros(Q + 1, np.int32)
    cdesc = np.zeros((meta[1], 4), np.int32)
    cptr = np.zeros(nbi + 1, np.int32)
    s0 = np.zeros(nbi * QZ, np.uint8)
    rowinfo = np.zeros((Q, 2), np.int32)
    N.call("atsc3_ldpc_qc_tables_host", *args, meta.ctypes.data,
           rdesc.ctypes.data, rptr.ctypes.data, cdesc.ctypes.data,
           cptr.ctypes.data, s0.ctypes.data, rowinfo.ctypes.data)
    return K, Q, meta, rdesc, rptr, cdesc, cptr, s0, rowinfo


@pytest.mark.parametrize("rate", ["6/15", "8/15", "10/15", "13/15"])
@pytest.mark.parametrize("cluster", [4, 8])
def test_qc_descriptors_reproduce_csr(rate, cluster):
    n = 64800
    K, Q, meta, rdesc, rptr, cdesc, cptr, s0, rowinfo = qc_tables(rate, n, cluster)
    ccp, cidx, vptr, vedge = C.csr(rate, n)
    rb = meta[8:8 + cluster + 1]
    ncp = meta[3]
    chk = np.repeat(np.arange(len(ccp) - 1), np.diff(ccp))
    pos = np.arange(len(cidx)) - ccp[chk]
    # check side: columns in position order
    for r in range(Q):
        d = rptr[r + 1] - rptr[r]
        for k in range(0, QZ, 7):
            cols = []
            for i in range(d):
                base, u = rdesc[rptr[r] + i]
                cols.append(base + k + (QZ if k < u else 0))
            cols.append(K + QZ * (r - 1) + k if r >= 1 else K + k)
            if r >= 1 or k >= 1:
                cols.append(K + QZ * r + k if r >= 1 else K + QZ * (Q - 1) + k - 1)
            a = Q * k + r
            assert cols == cidx[ccp[a]:ccp[a + 1]].tolist(), (r, k)

    def rec_to_check(rank, off):
        r = rb[rank] + off // QZ
        return Q * (off % QZ) + r

    # variable side: (check, position) in summation order
    nbi = K // QZ
    for lam in list(range(0, K, 97)) + list(range(K, n, 89)) + [n - 1]:
        b, mm = divmod(lam, QZ)
        got = []
        if b < nbi:
            cs, d = cptr[b], cptr[b + 1] - cptr[b]
            for t in range(d):
                i = s0[b * QZ + mm] + t
                i = i - d if i >= d else i
                rk_pos, rowoff, u, _ = cdesc[cs + i]
                kk = (u + mm) % QZ
                got.append((rec_to_check(rk_pos & 0xFF, rowoff + kk), rk_pos >> 8))
        else:
            tt = b - nbi
            rk, roff = rowinfo[tt]
            dt = rk >> 8
            got.append((rec_to_check(rk & 0xFF, roff + mm), dt + 1 if tt >= 1 else dt))
            if tt + 1 < Q:
                rk2, roff2 = rowinfo[tt + 1]
                got.append((rec_to_check(rk2 & 0xFF, roff2 + mm), rk2 >> 8))
            elif mm + 1 < QZ:
                rk2, roff2 = rowinfo[0]
                got.append((rec_to_check(rk2 & 0xFF, roff2 + mm + 1), (rk2 >> 8) + 1))
        want = [(int(chk[e]), int(pos[e])) for e in vedge[vptr[lam]:vptr[lam + 1]]]
        assert got == want, lam
    # work split covers every (column, chunk) item exactly once
    wb = meta[25:25 + cluster + 1]
    assert wb[0] == 0 and wb[-1] == (nbi + Q) * 12 and (np.diff(wb) >= 0).all()
    assert ncp == meta[4] * QZ and rb[-1] == Q


def test_qc_rejects_shared_blocks():
    # 16200 6/15 has two circulants in one block: the CSR decoder serves it
    typ, K, M1, M2, Q1, Q = C.ldpc_params("6/15", 16200)
    rowptr, addr = [np.ascontiguousarray(a, np.int32) for a in C.address_rows("6/15", 16200)]
    meta = np.zeros(48, np.int32)
    rc = N.lib().atsc3_ldpc_qc_tables_host(16200, K, Q, rowptr.ctypes.data,
                                           addr.ctypes.data, 1, meta.ctypes.data,
                                           None, None, None, None, None, None)
    assert rc == -4
