"""The host-pointer drop-in (ldpc_minsum_f32, the signature of
lab/ldpc_kernel.c:65) on every A/322 code and under concurrent callers.

The reference calls it from a ThreadPoolExecutor with ctypes releasing the GIL
(lab/m3_ldpc.py:409-415, lab/m9_fast.py:893-925), so the entry point must be
thread-safe; A/322 codes go to the edge-buffer quasi-cyclic decoder (the
tables are recognised by atsc3_ldpc_qc_detect2), any other matrix to the CSR
decoder.  Either way the outputs equal the oracle's field by field."""
import ctypes
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C
from atsc3_b200 import native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def minsum_f32(llr, tabs, n, iters, alpha):
    cptr, cidx, vptr, vedge = [np.ascontiguousarray(t, np.int32) for t in tabs]
    llr = np.ascontiguousarray(llr, np.float32)
    nblk = llr.shape[0]
    bits = np.full((nblk, n), 7, np.uint8)
    conv = np.full(nblk, 7, np.uint8)
    its = np.full(nblk, -7, np.int32)
    bad = np.full(nblk, -7, np.int32)
    rc = N.lib().ldpc_minsum_f32(llr.ctypes.data, nblk, n, len(cptr) - 1, len(cidx),
                                 cptr.ctypes.data, cidx.ctypes.data, vptr.ctypes.data,
                                 vedge.ctypes.data, iters, ctypes.c_float(alpha),
                                 bits.ctypes.data, conv.ctypes.data, its.ctypes.data,
                                 bad.ctypes.data, None)
    return rc, bits, conv, its, bad


def case(rate, n, seed, nblk=3):
    rng = np.random.default_rng(seed)
    llr = (rng.standard_normal((nblk, n)) * 2.5 + 1.5).astype(np.float32)
    llr[-1] = np.abs(llr[-1])                  # one clean block: its == 0
    return llr


def same(got, want):
    rc, bits, conv, its, bad = got
    return (rc == 0 and np.array_equal(bits, want[0])
            and conv.astype(bool).tolist() == want[1].tolist()
            and its.tolist() == want[2].tolist() and bad.tolist() == want[3].tolist())


@pytest.mark.parametrize("n", [16200, 64800])
def test_every_code_through_the_host_abi(n, torch):
    for rate in C.RATES:
        tabs = C.csr(rate, n)
        llr = case(rate, n, n + C.RATES.index(rate))
        want = oracle.flood(llr, tabs, n, iters=6, alpha=0.8)
        assert same(minsum_f32(llr, tabs, n, 6, 0.8), want), (rate, n)


def random_code(n=3000, nc=1500, seed=5):
    """A sparse parity-check matrix with no circulant structure (column
    degree 3, row degree about 6): the host ABI decodes it with the CSR
    kernel."""
    rng = np.random.default_rng(seed)
    checks = [[] for _ in range(nc)]
    for v in range(n):
        for c in rng.choice(nc, 3, replace=False):
            checks[c].append(v)
    return C.csr_from_checks([sorted(c) for c in checks], n)


def test_non_qc_code_through_the_host_abi(torch):
    tabs = random_code()
    llr = case("x", 3000, 9, nblk=4)
    want = oracle.flood(llr, tabs, 3000, iters=12, alpha=0.75)
    assert same(minsum_f32(llr, tabs, 3000, 12, 0.75), want)


def test_concurrent_callers(torch):
    """Eight threads, mixed codes (Type A and Type B on the edge-buffer
    decoder, a matrix without circulant structure on the CSR decoder), each
    call checked against the oracle; then the same calls again, all at
    once."""
    jobs = []
    tabs = random_code()
    llr = case("x", 3000, 77, nblk=3)
    jobs.append((llr, tabs, 3000, oracle.flood(llr, tabs, 3000, iters=8, alpha=0.75)))
    for i, (rate, n) in enumerate([("10/15", 64800), ("7/15", 64800), ("6/15", 16200),
                                   ("11/15", 16200), ("8/15", 64800), ("3/15", 16200),
                                   ("13/15", 64800), ("9/15", 16200)]):
        tabs = C.csr(rate, n)
        llr = case(rate, n, 100 + i, nblk=2 + i % 3)
        jobs.append((llr, tabs, n, oracle.flood(llr, tabs, n, iters=8, alpha=0.75)))
    with ThreadPoolExecutor(8) as ex:
        for rnd in range(3):
            res = list(ex.map(lambda j: minsum_f32(j[0], j[1], j[2], 8, 0.75), jobs * 2))
            for k, r in enumerate(res):
                assert same(r, jobs[k % len(jobs)][3]), (rnd, k)
