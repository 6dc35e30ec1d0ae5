"""Host-side fault handling (no GPU needed): every malformed call is refused
with the C ABI's invalid-argument code (-3) or unsupported code (-4), or a
Python exception, before anything is launched -- the reference's silent CPU
fallbacks (lab/m9_fast.py:196-204, lab/m3_ldpc.py:448-454) have no
counterpart here."""
import ctypes

import numpy as np
import pytest

from atsc3_b200 import codes as C
from atsc3_b200 import native as N

L = N.lib()


def test_null_plans_and_bad_sizes_are_invalid_arguments():
    vp = ctypes.c_void_p
    assert L.atsc3_ldpc_qce_decode(None, None, 64800, 1, 50, 0.75, 0, None, 0,
                                   None, 0, None, None, None, 0, None) == -3
    assert L.atsc3_ldpc_qc_decode(None, None, 64800, 1, 50, 0.75, 0, None, 0,
                                  None, 0, None, None, None, 0, None) == -3
    assert L.atsc3_ldpc_sp_decode(None, None, None, None, 0, 1, 1, None, 1, 1,
                                  10, None, 1, None, None, None, None, None) == -3
    assert L.atsc3_cpe_correct(None, 10, None, 1, None, None, 0, None, 0, None,
                               3, None, None, None, None) == -3
    assert L.atsc3_demap_gather(None, 10, 1, 10, None, 4, 7, None, 0, 0, 0, 0,
                                None, 1.0, None, None, 40, None) == -3
    assert L.atsc3_demap_gather(None, 10, 1, 10, None, 5, 0, None, 0, 0, 0, 0,
                                None, 1.0, None, None, 50, None) == -3
    msg = L.atsc3_last_error().decode()
    assert "nbits" in msg


def test_demap_gather_geometry_checks():
    dummy = ctypes.c_void_p(64)              # never dereferenced: refused first
    # hybrid TI: per_ti below Nr*Nc
    assert L.atsc3_demap_gather(dummy, 100, 2, 10, dummy, 4, 1, None, 0, 3, 20,
                                0, None, 1.0, None, dummy, 40, None) == -3
    # CTI: Nrows 0
    assert L.atsc3_demap_gather(dummy, 100, 2, 10, dummy, 4, 2, None, 0, 0, 0,
                                0, None, 1.0, None, dummy, 40, None) == -3
    # table mode without a table
    assert L.atsc3_demap_gather(dummy, 100, 2, 10, dummy, 4, 0, None, 0, 0, 0,
                                0, None, 1.0, None, dummy, 40, None) == -3
    # misaligned cells
    assert L.atsc3_demap_gather(ctypes.c_void_p(65), 100, 2, 10, dummy, 4, 1,
                                None, 0, 5, 50, 0, None, 1.0, None, dummy, 40,
                                None) == -3


def test_code_tables_refused():
    """A malformed code (addresses outside the parity range), a code that is
    not 360-circulant, a cluster size outside 1..16."""
    typ, K, M1, M2, Q1, Q = C.ldpc_params("10/15", 64800)
    rowptr, addr = [np.ascontiguousarray(a, np.int32) for a in C.address_rows("10/15", 64800)]
    meta = np.zeros(48, np.int32)
    bad = addr.copy()
    bad[3] = 64800 - K + 5
    f = L.atsc3_ldpc_qce_tables_host
    assert f(64800, K, Q, rowptr.ctypes.data, bad.ctypes.data, 6, meta.ctypes.data,
             None, None, None, None, None) == -3
    assert f(64801, K, Q, rowptr.ctypes.data, addr.ctypes.data, 6, meta.ctypes.data,
             None, None, None, None, None) == -3
    assert f(64800, K, Q, rowptr.ctypes.data, addr.ctypes.data, 0, meta.ctypes.data,
             None, None, None, None, None) == -3


def test_python_wrappers_refuse_bad_inputs():
    """Wrong dtype / device / shape / contiguity raise before any launch."""
    import torch
    from atsc3_b200 import ldpc as LDPC
    from atsc3_b200 import timeint as T

    class FakePlan:
        n, dtype, kind = 64800, "float32", "qce"

    with pytest.raises(TypeError):
        LDPC.decode_flood(FakePlan(), torch.zeros((2, 64800)))          # CPU tensor
    with pytest.raises(TypeError):
        LDPC.sp_decode({"n": 16200}, torch.zeros((1, 16200), dtype=torch.float64))
    with pytest.raises(TypeError):
        T.demap_deinterleave(torch.zeros(10, dtype=torch.complex64),
                             T.HybridTI(5, 2), "QPSK", "2/15", 16200, sigma2=1.0)
    with pytest.raises(ValueError):
        T.HybridTI(4, 3, n_virtual=3)
    with pytest.raises(ValueError):
        T.ConvolutionalTI(8, -1)


def test_type_a_tables_refused():
    """The two-zone builder refuses a zone split that does not add up to the
    parity length, a decreasing rowptr, a nonzero rowptr[0], and an identity
    address beyond the parity range; atsc3_ldpc_qc_detect2 refuses null
    outputs."""
    rate, n = "7/15", 64800
    typ, K, M1, M2, Q1, Q2 = C.ldpc_params(rate, n)
    rowptr, addr = [np.ascontiguousarray(a, np.int32) for a in C.address_rows(rate, n)]
    meta = np.zeros(96, np.int32)
    f = L.atsc3_ldpc_qce_tables_host2

    def call(qa, qb, rp, ad):
        return f(n, K, qa, qb, rp.ctypes.data, ad.ctypes.data, 7, meta.ctypes.data,
                 None, None, None, None, None, None, None, None)

    assert call(Q1, Q2, rowptr, addr) == 0
    assert call(Q1 + 1, Q2, rowptr, addr) == -3           # zones do not add up
    assert call(0, Q2 + Q1, rowptr, addr) == -3           # no accumulator rows
    rp = rowptr.copy()
    rp[5] = rp[4] - 1
    assert call(Q1, Q2, rp, addr) == -3                   # decreasing rowptr
    rp = rowptr.copy()
    rp[0] = 1
    assert call(Q1, Q2, rp, addr) == -3
    bad = addr.copy()
    bad[-1] = n - K
    assert call(Q1, Q2, rowptr, bad) == -3                # past the parity range
    cptr, cidx, vptr, vedge = [np.ascontiguousarray(t, np.int32) for t in C.csr(rate, n)]
    assert L.atsc3_ldpc_qc_detect2(cptr.ctypes.data, cidx.ctypes.data, vptr.ctypes.data,
                                   vedge.ctypes.data, n, len(cptr) - 1, len(cidx),
                                   None, None, None) == -3
