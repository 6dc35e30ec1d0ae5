"""The quasi-cyclic decoder's edge-slot descriptors, expanded on the CPU with
the kernel's own index formulas, must reproduce the CSR tables exactly: every
check's columns in position order, and every bit's (check, position) list in
the reference summation order (vedge)."""
import numpy as np
import pytest

from atsc3_b200 import codes as C
from atsc3_b200 import native as N

QZ = 360
WRAP = 1 << 8


def qc_tables(rate, n, cluster):
    typ, K, M1, M2, Q1, Q = C.ldpc_params(rate, n)
    rowptr, addr = [np.ascontiguousarray(a, np.int32) for a in C.address_rows(rate, n)]
    meta = np.zeros(48, np.int32)
    args = [n, K, Q, rowptr.ctypes.data, addr.ctypes.data, cluster]
    N.call("atsc3_ldpc_qc_tables_host", *args, meta.ctypes.data, None, None,
           None, None, None)
    nb = n // QZ
    rdesc = np.zeros((meta[0], 4), np.int32)
    rptr = np.zeros(Q + 1, np.int32)
    cdesc = np.zeros((meta[1], 4), np.int32)
    cptr = np.zeros(nb + 1, np.int32)
    s0 = np.zeros(nb * QZ, np.uint8)
    N.call("atsc3_ldpc_qc_tables_host", *args, meta.ctypes.data,
           rdesc.ctypes.data, rptr.ctypes.data, cdesc.ctypes.data,
           cptr.ctypes.data, s0.ctypes.data)
    return K, Q, meta, rdesc, rptr, cdesc, cptr, s0


@pytest.mark.parametrize("rate", ["6/15", "8/15", "10/15", "13/15"])
@pytest.mark.parametrize("cluster", [4, 8])
def test_qc_descriptors_reproduce_csr(rate, cluster):
    n = 64800
    K, Q, meta, rdesc, rptr, cdesc, cptr, s0 = qc_tables(rate, n, cluster)
    ccp, cidx, vptr, vedge = C.csr(rate, n)
    cpc, ncp, per = meta[2], meta[3], meta[4]
    tot_bytes = cpc * QZ * 4
    chk = np.repeat(np.arange(len(ccp) - 1), np.diff(ccp))
    pos = np.arange(len(cidx)) - ccp[chk]
    # check side: columns in position order
    for r in range(Q):
        for k in list(range(0, QZ, 7)) + [0, 1, QZ - 1]:
            cols = []
            for j, (x, base, u, _) in enumerate(rdesc[rptr[r]:rptr[r + 1]]):
                assert (x >> 16) == j
                if (x & WRAP) and k == 0:
                    continue
                col = (x & 0xFF) * cpc + base // (QZ * 4)
                assert base % (QZ * 4) == 0
                cols.append(col * QZ + (k - u) % QZ)
            a = Q * k + r
            assert cols == cidx[ccp[a]:ccp[a + 1]].tolist(), (r, k)
    # variable side: (check, position) in summation order
    for lam in list(range(0, n, 61)) + [n - 1, n - 2, K, K - 1]:
        b, mm = divmod(lam, QZ)
        cs, d = cptr[b], cptr[b + 1] - cptr[b]
        got = []
        for t in range(d):
            i = s0[b * QZ + mm] + t
            i = i - d if i >= d else i
            x, rowbase, u, _ = cdesc[cs + i]
            if (x & WRAP) and mm == QZ - 1:
                continue
            rrow = (x & 0xFF) * per + (rowbase - tot_bytes) // (QZ * 16)
            assert (rowbase - tot_bytes) % (QZ * 16) == 0
            got.append((Q * ((u + mm) % QZ) + rrow, int(x >> 16)))
        want = [(int(chk[e]), int(pos[e])) for e in vedge[vptr[lam]:vptr[lam + 1]]]
        assert got == want, lam
    wb = meta[25:25 + cluster + 1]
    nb = n // QZ
    assert wb[0] == 0 and wb[-1] == nb * 12 and (np.diff(wb) >= 0).all()
    assert ncp == per * QZ and meta[8 + cluster] == Q
    assert meta[7] == tot_bytes + ncp * 16 + 256


def test_qc_rejects_shared_blocks():
    # 16200 6/15 has two circulants in one block: the CSR decoder serves it
    typ, K, M1, M2, Q1, Q = C.ldpc_params("6/15", 16200)
    rowptr, addr = [np.ascontiguousarray(a, np.int32) for a in C.address_rows("6/15", 16200)]
    meta = np.zeros(48, np.int32)
    rc = N.lib().atsc3_ldpc_qc_tables_host(16200, K, Q, rowptr.ctypes.data,
                                           addr.ctypes.data, 1, meta.ctypes.data,
                                           None, None, None, None, None)
    assert rc == -4
