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


def zones(rate, n):
    """(K, accumulator block rows, identity block rows) of an A/322 code."""
    typ, K, M1, M2, Q1, Q2 = C.ldpc_params(rate, n)
    return (K, Q2, 0) if typ == "B" else (K, Q1, Q2)


def qce_tables(rate, n, cluster):
    K, QA, QB = zones(rate, n)
    Q = QA + QB
    rowptr, addr = [np.ascontiguousarray(a, np.int32) for a in C.address_rows(rate, n)]
    meta = np.zeros(96, np.int32)
    args = [n, K, QA, QB, rowptr.ctypes.data, addr.ctypes.data, cluster]
    N.call("atsc3_ldpc_qce_tables_host2", *args, meta.ctypes.data, None, None,
           None, None, None, None, None, None)
    nb = n // QZ
    rdesc = np.zeros((meta[0], 4), np.int32)
    rptr = np.zeros(Q + 1, np.int32)
    cdesc = np.zeros((nb, 4), np.int32)
    ccols = np.zeros(nb, np.int32)
    s0 = np.zeros(nb * QZ, np.uint8)
    s0b = np.zeros(nb * QZ, np.uint8)
    itab = np.zeros((meta[61], 4), np.int32)
    hitems = np.zeros(max(1, meta[62 + cluster]), np.int32)
    N.call("atsc3_ldpc_qce_tables_host2", *args, meta.ctypes.data,
           rdesc.ctypes.data, rptr.ctypes.data, cdesc.ctypes.data,
           ccols.ctypes.data, s0.ctypes.data, s0b.ctypes.data, itab.ctypes.data,
           hitems.ctypes.data)
    return K, QA, QB, meta, rdesc, rptr, cdesc, ccols, s0, s0b, itab, hitems[:meta[62 + cluster]]


def check_index(r, k, QA, QB):
    """Check index of block row r, lane k: r + QA*k in the accumulator rows,
    360*QA + (r - QA) + QB*k in the identity rows (lab/m3_ldpc.py:63-82)."""
    return r + QA * k if r < QA else QZ * QA + (r - QA) + QB * k


TYPE_A = [("2/15", 16200, 2), ("3/15", 16200, 3), ("5/15", 16200, 2),
          ("2/15", 64800, 6), ("4/15", 64800, 7), ("5/15", 64800, 8),
          ("7/15", 64800, 7), ("3/15", 64800, 6)]


@pytest.mark.parametrize("rate,n,cluster", [("6/15", 64800, 8), ("10/15", 64800, 8),
                                            ("6/15", 64800, 6), ("12/15", 64800, 7),
                                            ("13/15", 64800, 16), ("8/15", 64800, 4),
                                            ("11/15", 16200, 2), ("7/15", 16200, 1),
                                            ("6/15", 16200, 2), ("8/15", 16200, 3),
                                            ("10/15", 16200, 2), ("12/15", 16200, 2),
                                            ("13/15", 16200, 2)] + TYPE_A)
def test_qce_descriptors_reproduce_csr(rate, n, cluster):
    K, QA, QB, meta, rdesc, rptr, cdesc, ccols, s0, s0b, itab, hitems = qce_tables(rate, n, cluster)
    Q = QA + QB
    ccp, cidx, vptr, vedge = C.csr(rate, n)
    nb = n // QZ
    smem, part_off, maxs = meta[2], meta[3], meta[6]
    cb = meta[25:25 + cluster + 1]
    ci = meta[42:42 + cluster + 1]
    assert cb[0] == 0 and cb[-1] == nb and (np.diff(cb) >= 0).all()
    assert ci[-1] == Q * 12 and (np.diff(ci) >= 0).all()
    # light ranges + heavy lists: every check item exactly once; heavy items
    # (the accumulator rows of a Type A code) dealt round-robin
    hoff = meta[62:62 + cluster + 1]
    items = [i for c in range(cluster) for i in range(ci[c], ci[c + 1])]
    items += hitems.tolist()
    assert sorted(items) == list(range(Q * 12))
    if meta[79]:
        assert ci[0] == meta[79] * 12 and meta[79] == QA
        sizes = np.diff(hoff)
        assert sizes.max() - sizes.min() <= 1
    else:
        assert ci[0] == 0 and len(hitems) == 0
    assert sorted(ccols.tolist()) == list(range(nb))
    buf_off = meta[7]
    assert part_off >= nb * 12 * 4 and buf_off >= part_off + 256
    assert smem == buf_off + maxs * SLOT
    own_of = cdesc[:, 3] & 0xFF
    dA_of = cdesc[:, 3] >> 8
    # slot totals per CTA differ by at most one column's slots
    tot = [int(cdesc[ccols[cb[c]:cb[c + 1]], 0].sum()) for c in range(cluster)]
    assert max(tot) == maxs and max(tot) - min(tot) <= cdesc[:, 0].max()
    # column descriptors: slots contiguous from buf_off in every owner
    for c in range(cluster):
        off = buf_off
        for g in ccols[cb[c]:cb[c + 1]]:
            d, base, wrap, _ = cdesc[g]
            assert own_of[g] == c and base == off
            off += d * SLOT
        assert off <= smem
    # (owner, byte offset) -> (column, slot index), to decode row slots
    slot_of = {}
    for g in range(nb):
        d, base, wrap, _ = cdesc[g]
        for i in range(d):
            slot_of[(int(own_of[g]), base + i * SLOT)] = (g, i)
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
                # zone-A slots of a column come first
                assert (i < dA_of[g]) == (r < QA)
                mm = (k - u) % QZ
                cols.append(g * QZ + mm)
                key = (g, i, mm)
                assert key not in seen
                seen[key] = check_index(r, k, QA, QB)
            a = check_index(r, k, QA, QB)
            want = cidx[ccp[a]:ccp[a + 1]].tolist()
            # the same edges; in the same order unless two circulants share a
            # block (then the slot order is fixed while the bit order within
            # the block depends on k; the check update is order-free)
            assert sorted(cols) == want, (r, k)
            if len({c // QZ for c in cols}) == len(cols):
                assert cols == want, (r, k)
    visited = set(seen.values())
    # variable side: zone A rotated at s0, then zone B rotated at s0b (a
    # column of one zone: its zone rotated at s0) = vedge order
    for lam in list(range(0, n, 53)) + [n - 1, n - 2, K, K - 1]:
        g, mm = divmod(lam, QZ)
        d, base, wrap, _ = cdesc[g]
        dA = int(dA_of[g])
        segs = [(0, d, int(s0[lam]))] if dA in (0, d) else \
            [(0, dA, int(s0[lam])), (dA, d - dA, int(s0b[lam]))]
        order = []
        for lo, dz, rot in segs:
            order += [lo + (rot + t) % dz for t in range(dz)]
        got = []
        for i in order:
            if i == wrap and mm == QZ - 1:
                continue
            got.append(seen.get((g, i, mm), ("unvisited", g, i, mm)))
        # the checks of the bit in summation order (the variable sum is the
        # only order-sensitive arithmetic)
        want = [int(chk[e]) for e in vedge[vptr[lam]:vptr[lam + 1]]]
        sampled = [w for w in want if w in visited]
        got_s = [x for x in got if not (isinstance(x, tuple) and x[0] == "unvisited")]
        assert got_s == sampled, lam
        assert len(got) == len(want), lam
    # variable-phase items (64 bits each: two bits a lane): the pair path
    # sums slot 0 then slot 1 (no rotation), the register path takes 1..4
    # slots of one zone, the two-segment path only columns with slots in
    # both zones
    for x, y, z, w in itab:
        g, mm0 = divmod(int(y), QZ)
        d, dA, mode = z & 0xFF, (w >> 16) & 0xFF, (z >> 25) & 3
        assert d == cdesc[g][0] and dA == dA_of[g]
        bits = range(g * QZ + mm0, g * QZ + min(QZ, mm0 + 64))   # 64-bit items
        assert mm0 % 64 == 0
        if mode == 0:
            # (bit 359 of the wrap column has one real edge and the -0.0
            # entry, whose place in the sum does not matter)
            wrapcol = cdesc[g][2] >= 0
            assert d == 2 and all(s0[b] % 2 == 0 for b in bits
                                  if not (wrapcol and b % QZ == QZ - 1))
        elif mode == 1:
            assert d <= 4 and dA in (0, d) and (w >> 24) & 0xFF == 0xFF
        elif mode == 3:
            assert 0 < dA < d
        else:
            assert dA in (0, d)


def _tables_from(n, K, Q, rowptr, addr, cluster):
    meta = np.zeros(96, np.int32)
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
        meta = qce_tables(f"{num}/15", 64800, 6)[3]
        assert meta[2] <= 232448, (num, meta[2])
    for num in (6, 7, 8, 9, 10, 11, 12, 13):
        meta = qce_tables(f"{num}/15", 16200, 2)[3]
        assert meta[2] <= 232448, (num, meta[2])


@pytest.mark.parametrize("rate,n,cluster", [("6/15", 64800, 6), ("10/15", 64800, 6),
                                            ("7/15", 64800, 7), ("11/15", 16200, 2)])
def test_variable_items_dealt_evenly_to_warp_bins(rate, n, cluster):
    """The host deals each CTA's variable-phase items to 32 warp bins, the
    most expensive first, each to the least-loaded bin: the bins' estimated
    costs then differ by at most the largest item's (1330 + 140 x the column
    degree, two zones +200), the item list keeps every item once, and the
    exported bin offsets (atsc3_ldpc_qce_bins_host) cut each CTA's items
    into QBINS consecutive, non-overlapping runs."""
    K, QA, QB, meta, rdesc, rptr, cdesc, ccols, s0, s0b, itab, hitems = \
        qce_tables(rate, n, cluster)
    lo, hi = int(meta[80]), int(meta[81])
    dmax = int(cdesc[:, 0].max())
    assert 0 < lo <= hi and hi - lo <= 1530 + 140 * dmax
    starts = sorted((int(y), int(x)) for x, y, z, w in itab)
    assert len(starts) == len(set(starts)) == len(itab)
    qbins = int(meta[82])
    rowptr, addr = [np.ascontiguousarray(a, np.int32) for a in C.address_rows(rate, n)]
    wbin = np.zeros(cluster * (qbins + 1), np.int32)
    N.call("atsc3_ldpc_qce_bins_host", n, K, QA, QB, rowptr.ctypes.data,
           addr.ctypes.data, cluster, wbin.ctypes.data)
    wbin = wbin.reshape(cluster, qbins + 1)
    assert (wbin[:, 0] == 0).all() and (np.diff(wbin, axis=1) >= 0).all()
    assert int(wbin[:, qbins].sum()) == len(itab)
