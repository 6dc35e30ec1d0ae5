"""libatsc3_fec.so on the CPU: it loads, exports every symbol the header
declares, and its host-side table build encodes the CSR tables exactly.
No CUDA call is made."""
import ctypes
import os
import re

import numpy as np
import pytest

from atsc3_b200 import codes as C
from atsc3_b200 import native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "atsc3_fec.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b([a-z_0-9]+)\s*\(", txt)) - {"if"})


def test_library_exports_every_declared_symbol():
    L = N.lib()
    syms = header_symbols()
    assert "ldpc_minsum_f32" in syms and "ldpc_kernel_abi" in syms
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) <= set(N.SIGNATURES)
    assert L.ldpc_kernel_abi() == 1


def host_tables(rate, n, cluster):
    tabs = [np.ascontiguousarray(t, np.int32) for t in C.csr(rate, n)]
    nc = len(tabs[0]) - 1
    ne = len(tabs[1])
    sizes = np.zeros(6, np.int64)
    args = [t.ctypes.data for t in tabs] + [n, nc, ne, cluster]
    N.call("atsc3_ldpc_tables_host", *args, sizes.ctypes.data, None, None,
           None, None)
    cent = np.zeros(sizes[0], np.uint16)
    cs = np.zeros(sizes[1], np.int32)
    vent = np.zeros(sizes[2], np.uint32)
    vs = np.zeros(sizes[3], np.int32)
    N.call("atsc3_ldpc_tables_host", *args, sizes.ctypes.data,
           cent.ctypes.data, cs.ctypes.data, vent.ctypes.data, vs.ctypes.data)
    return tabs, cent, cs, vent, vs, int(sizes[4]), int(sizes[5])


@pytest.mark.parametrize("rate,n,cluster", [("11/15", 16200, 1),
                                            ("6/15", 64800, 4),
                                            ("7/15", 64800, 8),
                                            ("2/15", 64800, 16)])
def test_host_tables_encode_csr(rate, n, cluster):
    (cptr, cidx, vptr, vedge), cent, cs, vent, vs, ncp, nvlog2 = \
        host_tables(rate, n, cluster)
    nc = len(cptr) - 1
    assert ncp % 32 == 0 and ncp * cluster >= nc
    assert (1 << nvlog2) * cluster >= n
    deg = np.diff(cptr)
    for s in range(len(cs) - 1):
        dm = cs[s + 1] - cs[s]
        blk = cent[cs[s] * 32:(cs[s] + dm) * 32].reshape(dm, 32)
        for l in range(32):
            c = 32 * s + l
            col = blk[:, l]
            if c >= nc:
                assert (col == 0xFFFF).all()
                continue
            assert np.array_equal(col[:deg[c]], cidx[cptr[c]:cptr[c + 1]])
            assert (col[deg[c]:] == 0xFFFF).all()
    vdeg = np.diff(vptr)
    for s in range(len(vs) - 1):
        dm = vs[s + 1] - vs[s]
        blk = vent[vs[s] * 32:(vs[s] + dm) * 32].reshape(dm, 32)
        for l in range(32):
            i = 32 * s + l
            col = blk[:, l]
            if i >= n:
                assert (col == 0xFFFFFFFF).all()
                continue
            e = col[:vdeg[i]]
            chk = (e >> 16 & 15).astype(np.int64) * ncp + (e & 0xFFFF)
            pos = (e >> 20).astype(np.int64)
            assert np.array_equal(cptr[chk] + pos, vedge[vptr[i]:vptr[i + 1]])
            assert (col[vdeg[i]:] == 0xFFFFFFFF).all()


def test_host_tables_reject_bad_input():
    tabs = [np.ascontiguousarray(t, np.int32).copy()
            for t in C.csr("11/15", 16200)]
    nc, ne = len(tabs[0]) - 1, len(tabs[1])
    sizes = np.zeros(6, np.int64)

    def rc(t, cluster=1):
        return N.lib().atsc3_ldpc_tables_host(
            *[a.ctypes.data for a in t], 16200, nc, ne, cluster,
            sizes.ctypes.data, None, None, None, None)

    assert rc(tabs) == 0
    assert rc(tabs, cluster=3) == -3
    bad = [a.copy() for a in tabs]
    bad[1][5] = 16200                       # cidx out of range
    assert rc(bad) == -3
    bad = [a.copy() for a in tabs]
    j = bad[2][1]                           # first edge of variable 1
    bad[3][[0, j]] = bad[3][[j, 0]]         # vedge not variable-major
    assert rc(bad) == -3
    # a check of degree 129 is the reference kernel's -1
    cptr = np.array([0, 129], np.int32)
    cidx = np.arange(129, dtype=np.int32)
    vptr = np.arange(130, dtype=np.int32)
    vedge = np.arange(129, dtype=np.int32)
    assert N.lib().atsc3_ldpc_tables_host(
        cptr.ctypes.data, cidx.ctypes.data, vptr.ctypes.data,
        vedge.ctypes.data, 129, 1, 129, 1, sizes.ctypes.data, None, None,
        None, None) == -1


def test_install_rebinds_and_restores():
    """atsc3_b200.install mirrors lab/m9_accel.py:392-433 (swap module
    attributes, restore on uninstall) for the four replaced entry points."""
    import types
    from atsc3_b200 import install as I
    m9_gpu = types.SimpleNamespace(GpuMinSum="ref")
    m16 = types.SimpleNamespace(demap_llr_fast="ref")
    m9a = types.SimpleNamespace(bch_syndrome_batch="ref", bch_syndrome="ref")
    m3 = types.SimpleNamespace(_kernel_lib="ref")
    assert I.install(m9_gpu, m16, m9a, m3) == 5
    from atsc3_b200 import bch, demap, ldpc
    assert m9_gpu.GpuMinSum is ldpc.GpuMinSum
    assert m16.demap_llr_fast is demap.demap_llr_fast
    assert m9a.bch_syndrome_batch is bch.bch_syndrome_batch
    lib = m3._kernel_lib()
    assert lib.ldpc_kernel_abi() == 1
    I.uninstall()
    assert m9_gpu.GpuMinSum == "ref" and m3._kernel_lib == "ref"
    assert m9a.bch_syndrome == "ref" and m16.demap_llr_fast == "ref"
    from atsc3_b200 import cpe
    mg = types.SimpleNamespace(sum_product_decode_batch="ref")
    ce = types.SimpleNamespace(cpe_correct="ref")
    assert I.install(m16_margin=mg, m6_cells=ce) == 2
    assert mg.sum_product_decode_batch is ldpc.sum_product_decode_batch
    assert ce.cpe_correct is cpe.cpe_correct
    I.uninstall()
    assert mg.sum_product_decode_batch == "ref" and ce.cpe_correct == "ref"


@pytest.mark.parametrize("kldpc,kpay,what", [(64801, 0, "kldpc"),
                                            (0, 0, "kldpc"),
                                            (25920, 25921, "kpayload"),
                                            (25920, -1, "kpayload")])
def test_noalloc_refuses_bch_lengths_past_the_codeword(kldpc, kpay, what):
    """The allocation-free entry point reads the first kldpc hard decisions
    of a scratch row that the LDPC step fills only up to ncell*nbits, so a
    longer kldpc (or a payload longer than kldpc) is refused with -3 before
    any plan or device access (the plan pointer here is never read)."""
    dummy = ctypes.c_void_p(1)
    rc = N.lib().atsc3_fec_decode_noalloc(
        dummy, 2, None, 0, 1, 16200, None, 4, 0, None, 0, ctypes.c_float(1.0),
        None, 50, ctypes.c_float(0.75), None, kldpc, None, kpay, None, 0,
        None, None, None, None, None, None)
    assert rc == -3
    assert what in N.lib().atsc3_last_error().decode()


def test_minsum_f32_degree_above_128_returns_minus_one_and_writes_nothing():
    """lab/ldpc_kernel.c:78-80: a check of more than MAX_ROW_DEG = 128 edges
    makes ldpc_minsum_f32 return -1 before it writes any output (the check
    runs before any device work, so this needs no GPU)."""
    import ctypes
    n = 129
    cptr = np.array([0, n], np.int32)
    cidx = np.arange(n, dtype=np.int32)
    vptr = np.arange(n + 1, dtype=np.int32)
    vedge = np.arange(n, dtype=np.int32)
    llr = np.ones((2, n), np.float32)
    bits = np.full((2, n), 7, np.uint8)
    conv = np.full(2, 7, np.uint8)
    its = np.full(2, -7, np.int32)
    bad = np.full(2, -7, np.int32)
    rc = N.lib().ldpc_minsum_f32(llr.ctypes.data, 2, n, 1, n, cptr.ctypes.data,
                                 cidx.ctypes.data, vptr.ctypes.data, vedge.ctypes.data,
                                 10, ctypes.c_float(0.75), bits.ctypes.data,
                                 conv.ctypes.data, its.ctypes.data, bad.ctypes.data, None)
    assert rc == -1
    assert (bits == 7).all() and (conv == 7).all() and (its == -7).all() and (bad == -7).all()



def test_gpuminsum_argument_checks_before_any_device_work():
    """GpuMinSum accepts the reference's four dtypes (lab/m9_gpu.py:100-101)
    and refuses others, and kernel semantics outside float32, before it
    builds a plan (so these raise without a GPU)."""
    import pytest
    from atsc3_b200 import ldpc
    with pytest.raises(ValueError):
        ldpc.GpuMinSum([[0, 1]], 2, dtype="int8")
    for dt in ("float64", "bfloat16", "float16"):
        with pytest.raises(ValueError):
            ldpc.GpuMinSum([[0, 1]], 2, dtype=dt, semantics="kernel")
    assert set(ldpc.SEMANTICS) == {"kernel", "torch", "torch_bf16", "torch_f16"}
