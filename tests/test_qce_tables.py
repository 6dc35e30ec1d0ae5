"""The edge-buffer quasi-cyclic decoder's descriptors, expanded on the CPU with
the kernel's own index formulas (csrc/ldpc_qce.cu), must reproduce the CSR
tables: every check's columns (in position order, unless two circulants
share a block), every bit's checks in the reference summation order (vedge),
each edge owning exactly one slot entry, and every slot inside its owner's
shared memory."""
import numpy as np
import pytest

from atsc3_b200 import codes as C
from atsc3_b200 import native as N

QZ = 360
WRAP = 1 << 8
SLOT = QZ * 4


def qce_tables(rate, n, cluster):
    typ, K, M1, M2, Q1, Q = C.ldpc_params(rate, n)
    rowptr, addr = [np.ascontiguousarray(a, np.int32) for a in C.address_rows(rate, n)]
    meta = np.zeros(48, np.int32)
    args = [n, K, Q, rowptr.ctypes.data, addr.ctypes.data, cluster]
    N.call("atsc3_ldpc_qce_tables_host", *args, meta.ctypes.data, None, None,
           None, None, None)
    nb = n // QZ
    rdesc = np.zeros((meta[0], 4), np.int32)
    rptr = np.zeros(Q + 1, np.int32)
    cdesc = np.zeros((nb, 4), np.int32)
    ccols = np.zeros(nb, np.int32)
    s0 = np.zeros(nb * QZ, np.uint8)
    N.call("atsc3_ldpc_qce_tables_host", *args, meta.ctypes.data,
           rdesc.ctypes.data, rptr.ctypes.data, cdesc.ctypes.data,
           ccols.ctypes.data, s0.ctypes.data)
    return K, Q, meta, rdesc, rptr, cdesc, ccols, s0


@pytest.mark.parametrize("rate,n,cluster", [("6/15", 64800, 8), ("10/15", 64800, 8),
                                            ("6/15", 64800, 6), ("12/15", 64800, 7),
                                            ("13/15", 64800, 16), ("8/15", 64800, 4),
                                            ("11/15", 16200, 2), ("7/15", 16200, 1),
                                            ("6/15", 16200, 2), ("8/15", 16200, 3),
                                            ("10/15", 16200, 2), ("12/15", 16200, 2),
                                            ("13/15", 16200, 2)])
def test_qce_descriptors_reproduce_csr(rate, n, cluster):
    K, Q, meta, rdesc, rptr, cdesc, ccols, s0 = qce_tables(rate, n, cluster)
    ccp, cidx, vptr, vedge = C.csr(rate, n)
    nb = n // QZ
    smem, part_off, maxs = meta[2], meta[3], meta[6]
    cb = meta[25:25 + cluster + 1]
    rb = meta[8:8 + cluster + 1]
    assert cb[0] == 0 and cb[-1] == nb and (np.diff(cb) >= 0).all()
    assert rb[0] == 0 and rb[-1] == Q
    assert sorted(ccols.tolist()) == list(range(nb))
    buf_off = meta[7]
    assert part_off >= nb * 12 * 4 and buf_off >= part_off + 256
    assert smem == buf_off + maxs * SLOT
    # slot totals per CTA differ by at most one column's slots
    tot = [int(cdesc[ccols[cb[c]:cb[c + 1]], 0].sum()) for c in range(cluster)]
    assert max(tot) == maxs and max(tot) - min(tot) <= cdesc[:, 0].max()
    # column descriptors: slots contiguous from buf_off in every owner
    for c in range(cluster):
        off = buf_off
        for g in ccols[cb[c]:cb[c + 1]]:
            d, base, wrap, own = cdesc[g]
            assert own == c and base == off
            off += d * SLOT
        assert off <= smem
    # (owner, byte offset) -> (column, slot index), to decode row slots
    slot_of = {}
    for g in range(nb):
        d, base, wrap, own = cdesc[g]
        for i in range(d):
            slot_of[(own, base + i * SLOT)] = (g, i)
    chk = np.repeat(np.arange(len(ccp) - 1), np.diff(ccp))
    seen = {}
    # check side: the check's columns, one slot entry per edge
    for r in range(Q):
        for k in list(range(0, QZ, 7)) + [1, QZ - 1]:
            cols = []
            for j, (x, off, u, bmo) in enumerate(rdesc[rptr[r]:rptr[r + 1]]):
                assert (x >> 16) == j
                if (x & WRAP) and k == 0:
                    continue
                g, i = slot_of[(x & 0xFF, off)]
                assert bmo == g * 12 * 4
                mm = (k - u) % QZ
                cols.append(g * QZ + mm)
                key = (g, i, mm)
                assert key not in seen
                seen[key] = Q * k + r
            a = Q * k + r
            want = cidx[ccp[a]:ccp[a + 1]].tolist()
            # the same edges; in the same order unless two circulants share a
            # block (then the slot order is fixed while the bit order within
            # the block depends on k; the check update is order-free)
            assert sorted(cols) == want, (r, k)
            if len({c // QZ for c in cols}) == len(cols):
                assert cols == want, (r, k)
    # variable side: rotated slot order = vedge order, and the slot entry
    # read for each (check, position) is the one that check writes
    for lam in list(range(0, n, 53)) + [n - 1, n - 2, K, K - 1]:
        g, mm = divmod(lam, QZ)
        d, base, wrap, own = cdesc[g]
        got = []
        for t in range(d):
            i = s0[g * QZ + mm] + t
            i = i - d if i >= d else i
            if i == wrap and mm == QZ - 1:
                continue
            if (g, i, mm) in seen:
                got.append(seen[(g, i, mm)])
            else:
                got.append(("unvisited", g, i, mm))
        # the checks of the bit in summation order (the variable sum is the
        # only order-sensitive arithmetic)
        want = [int(chk[e]) for e in vedge[vptr[lam]:vptr[lam + 1]]]
        sampled = [w for w in want if (w // Q) in set(range(0, QZ, 7)) | {1, QZ - 1}]
        got_s = [x for x in got if not (isinstance(x, tuple) and x[0] == "unvisited")]
        assert got_s == sampled, lam
        assert len(got) == len(want), lam


def _tables_from(n, K, Q, rowptr, addr, cluster):
    meta = np.zeros(48, np.int32)
    nb = n // QZ
    f = N.lib().atsc3_ldpc_qce_tables_host
    rc = f(n, K, Q, rowptr.ctypes.data, addr.ctypes.data, cluster, meta.ctypes.data,
           None, None, None, None, None)
    if rc:
        return rc, None
    rdesc = np.zeros((meta[0], 4), np.int32)
    rptr = np.zeros(Q + 1, np.int32)
    cdesc = np.zeros((nb, 4), np.int32)
    ccols = np.zeros(nb, np.int32)
    s0 = np.zeros(nb * QZ, np.uint8)
    f(n, K, Q, rowptr.ctypes.data, addr.ctypes.data, cluster, meta.ctypes.data,
      rdesc.ctypes.data, rptr.ctypes.data, cdesc.ctypes.data, ccols.ctypes.data,
      s0.ctypes.data)
    return 0, (meta, rdesc, rptr, cdesc, ccols, s0)


def test_qce_repeated_address_cancels_and_bad_input_is_refused():
    """An address listed twice in a row of the table cancels in GF(2)
    (lab/m3_ldpc.py:199-211): the descriptors equal those of the table
    without it.  A cluster outside 1..16 and an address outside the parity
    range are invalid arguments."""
    typ, K, M1, M2, Q1, Q = C.ldpc_params("7/15", 16200)
    rowptr, addr = [np.asarray(a, np.int32) for a in C.address_rows("7/15", 16200)]
    g0 = addr[rowptr[0]:rowptr[1]].tolist()
    x = g0[2]
    twice = np.array(g0 + [x] + addr[rowptr[1]:].tolist(), np.int32)
    rp_twice = np.concatenate([[0], rowptr[1:] + 1]).astype(np.int32)
    drop = np.array(g0[:2] + g0[3:] + addr[rowptr[1]:].tolist(), np.int32)
    rp_drop = np.concatenate([[0], rowptr[1:] - 1]).astype(np.int32)
    # three copies: the cancelled pair leaves one, as in the original table
    thrice = np.array(g0 + [x, x] + addr[rowptr[1]:].tolist(), np.int32)
    rp_thrice = np.concatenate([[0], rowptr[1:] + 2]).astype(np.int32)
    rc_a, a = _tables_from(16200, K, Q, rp_twice, twice, 2)
    rc_b, b = _tables_from(16200, K, Q, rp_drop, drop, 2)
    rc_c, c = _tables_from(16200, K, Q, rp_thrice, thrice, 2)
    rc_d, d = _tables_from(16200, K, Q, np.asarray(rowptr, np.int32), addr, 2)
    assert rc_a == rc_b == rc_c == rc_d == 0
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    for u, v in zip(c, d):
        assert np.array_equal(u, v)
    rc, _ = _tables_from(16200, K, Q, np.asarray(rowptr, np.int32), addr, 17)
    assert rc == -3
    bad = addr.copy()
    bad[0] = 16200 - K + 3
    rc, _ = _tables_from(16200, K, Q, np.asarray(rowptr, np.int32), bad, 2)
    assert rc == -3


def test_qce_shared_memory_fits_b200_at_cluster_6():
    """Every 64800 Type B code fits a 6-CTA cluster within the 227 KB
    opt-in limit; every 16200 Type B code (6/15 .. 13/15) fits 2 CTAs."""
    for num in (6, 8, 9, 10, 11, 12, 13):
        meta = qce_tables(f"{num}/15", 64800, 6)[2]
        assert meta[2] <= 232448, (num, meta[2])
    for num in (6, 7, 8, 9, 10, 11, 12, 13):
        meta = qce_tables(f"{num}/15", 16200, 2)[2]
        assert meta[2] <= 232448, (num, meta[2])
