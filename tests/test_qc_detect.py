"""atsc3_ldpc_qc_detect: the host-pointer drop-in (ldpc_minsum_f32) recognises
an A/322 Type B code in the CSR tables it is handed and decodes it with the
edge-buffer quasi-cyclic decoder.  The recognition must accept exactly the
reference's tables (lab/m3_ldpc.py:459-482) of every Type B code, recover the
address table the quasi-cyclic plan is built from, and refuse Type A codes and
any table whose edges are not in the reference order (those go to the CSR
decoder, whose summation order follows vedge as given)."""
import numpy as np
import pytest

from atsc3_b200 import codes as C
from atsc3_b200 import native as N

CODES = [(r, n) for n in (16200, 64800) for r in C.RATES]


def detect(cptr, cidx, vptr, vedge, n, fn="atsc3_ldpc_qc_detect"):
    nc = len(cptr) - 1
    ne = len(cidx)
    kq = np.zeros(3, np.int32)
    rowptr = np.zeros(n // 360 + 1, np.int32)
    addr = np.zeros(max(ne, 1), np.int32)
    arrs = [np.ascontiguousarray(a, np.int32) for a in (cptr, cidx, vptr, vedge)]
    rc = getattr(N.lib(), fn)(*[a.ctypes.data for a in arrs], n, nc, ne,
                              kq.ctypes.data, rowptr.ctypes.data, addr.ctypes.data)
    return rc, kq, rowptr, addr


def reference_addresses(rate, n):
    """Per 360-group, the checks of bit 360g: the Annex A addresses with pairs
    that cancel in GF(2) removed, ascending."""
    rowptr, addr = C.address_rows(rate, n)
    out = []
    for g in range(len(rowptr) - 1):
        xs, cnt = np.unique(np.asarray(addr[rowptr[g]:rowptr[g + 1]]), return_counts=True)
        out.append(xs[cnt % 2 == 1].tolist())
    return out


@pytest.mark.parametrize("rate,n", CODES)
def test_detects_type_b_and_recovers_addresses(rate, n):
    typ, K, M1, M2, Q1, Q2 = C.ldpc_params(rate, n)
    rc, kq, rowptr, addr = detect(*C.csr(rate, n), n)
    if typ == "A":
        assert rc == -4
        return
    assert rc == 0, N.lib().atsc3_last_error()
    assert kq[:2].tolist() == [K, Q2]
    want = reference_addresses(rate, n)
    assert rowptr[K // 360] == sum(len(w) for w in want)
    got = [addr[rowptr[g]:rowptr[g + 1]].tolist() for g in range(K // 360)]
    assert got == want


def test_refuses_tables_out_of_reference_order():
    n = 16200
    cptr, cidx, vptr, vedge = [np.array(a) for a in C.csr("8/15", n)]
    assert detect(cptr, cidx, vptr, vedge, n)[0] == 0
    # a bit's edges listed in another order (the CSR decoder would sum them in
    # that order, the quasi-cyclic one would not)
    v = int(np.argmax(np.diff(vptr)))
    ve = vedge.copy()
    ve[vptr[v]:vptr[v + 1]] = ve[vptr[v]:vptr[v + 1]][::-1]
    assert detect(cptr, cidx, vptr, ve, n)[0] == -4
    # columns of one check out of ascending order
    ci = cidx.copy()
    ci[cptr[5]], ci[cptr[5] + 1] = ci[cptr[5] + 1], ci[cptr[5]]
    assert detect(cptr, ci, vptr, np.argsort(ci, kind="stable"), n)[0] == -4


def test_refuses_a_code_that_is_not_quasi_cyclic():
    n = 16200
    cptr, cidx, vptr, vedge = C.csr("8/15", n)
    checks = [list(cidx[cptr[c]:cptr[c + 1]]) for c in range(len(cptr) - 1)]
    # move one info edge of check 0 to another info column: still a valid
    # code with the same degrees, no longer a circulant shift
    c0 = checks[0][0]
    checks[0][0] = c0 + 1 if c0 + 1 not in checks[0] else c0 + 2
    checks[0].sort()
    t = C.csr_from_checks(checks, n)
    assert detect(*t, n)[0] == -4
    # a parity part that is not the accumulator
    checks = [list(cidx[cptr[c]:cptr[c + 1]]) for c in range(len(cptr) - 1)]
    checks[7] = [x for x in checks[7] if x < C.kldpc("8/15", n)]
    t = C.csr_from_checks(checks, n)
    assert detect(*t, n)[0] == -4


def test_refuses_inconsistent_tables_without_reading_past_them():
    n = 16200
    cptr, cidx, vptr, vedge = [np.array(a) for a in C.csr("8/15", n)]
    bad = cidx.copy()
    bad[3] = n + 5
    assert detect(cptr, bad, vptr, vedge, n)[0] == -4
    vp = vptr.copy()
    vp[-1] += 1
    assert detect(cptr, cidx, vp, vedge, n)[0] == -4


@pytest.mark.parametrize("rate,n", CODES)
def test_detect2_both_types(rate, n):
    """atsc3_ldpc_qc_detect2 recognises every A/322 code: Type B with qb = 0
    as above, Type A with qa = Q1, qb = Q2 and the address table's rows for
    the information groups and the accumulator parity groups."""
    typ, K, M1, M2, Q1, Q2 = C.ldpc_params(rate, n)
    rc, kq, rowptr, addr = detect(*C.csr(rate, n), n, fn="atsc3_ldpc_qc_detect2")
    assert rc == 0, N.lib().atsc3_last_error()
    nrows = K // 360 + (Q1 if typ == "A" else 0)
    assert kq.tolist() == ([K, Q2, 0] if typ == "B" else [K, Q1, Q2])
    want = reference_addresses(rate, n)
    assert len(want) == nrows
    got = [addr[rowptr[g]:rowptr[g + 1]].tolist() for g in range(nrows)]
    assert got == want


def test_detect2_refuses_a_broken_type_a_code():
    n = 16200
    cptr, cidx, vptr, vedge = C.csr("3/15", n)
    K = C.kldpc("3/15", n)
    checks = [list(cidx[cptr[c]:cptr[c + 1]]) for c in range(len(cptr) - 1)]
    # an identity parity bit moved onto the neighbouring check
    last = len(checks) - 1
    bit = [x for x in checks[last] if x >= K][0]
    checks[last].remove(bit)
    checks[last - 1] = sorted(checks[last - 1] + [bit])
    assert detect(*C.csr_from_checks(checks, n), n, fn="atsc3_ldpc_qc_detect2")[0] == -4
    # one info edge of an accumulator row shifted to the next column
    checks = [list(cidx[cptr[c]:cptr[c + 1]]) for c in range(len(cptr) - 1)]
    c0 = checks[3][0]
    checks[3][0] = c0 + 1 if c0 + 1 not in checks[3] else c0 + 2
    checks[3].sort()
    assert detect(*C.csr_from_checks(checks, n), n, fn="atsc3_ldpc_qc_detect2")[0] == -4
