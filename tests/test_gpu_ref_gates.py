"""The reference receiver's own gates and callers, run on this back end
through ``atsc3_b200.install()`` -- the unmodified reference Python from
baseline/_ref (laid out by ``python oracle/build.py --ref-tree``; these
tests skip where it is absent).  Every gate is the reference's code: only
the rebound entry points are ours, and spies show that they ran.

* m9_gpu.verify (lab/m9_gpu.py:349-402): GpuMinSum on the GPU against the
  scalar float64 CPU decoder, exact equality of bits/conv/its/bad;
* m16_demap_fast.gate / gate_decoded (lab/m16_demap_fast.py:122-174):
  demap_llr_fast against the exhaustive demapper (relative 1e-12) and the
  decoded codeword of both;
* m9_accel.verify (lab/m9_accel.py:441-503): its BCH legs call the rebound
  bch_syndrome / bch_syndrome_batch against the big-integer remainder;
* build_ldpc_kernel.smoke (lab/build_ldpc_kernel.py:101-120): the
  all-erasure known answer through m3_ldpc's kernel loader;
* m3_ldpc.min_sum_decode_batch(dtype=float32) (lab/m3_ldpc.py:485-526)
  reaching libatsc3_fec.so through the rebound _kernel_lib, equal to the
  reference's own compiled kernel, numpy fallback never entered;
* m44_ldm.ldpc_batch (lab/m44_ldm.py:2497-2555) with our GpuMinSum as its
  `gpu`, equal to the same call with the reference's torch GpuMinSum.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "baseline", "_ref")
LAB = os.path.join(REF, "lab")

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not os.path.exists(os.path.join(LAB, "m9_gpu.py")),
                       reason="baseline/_ref not laid out "
                              "(python oracle/build.py --ref-tree)")]


class Count:
    """Wrap a callable and count its calls."""

    def __init__(self, fn):
        self.fn, self.n = fn, 0

    def __call__(self, *a, **k):
        self.n += 1
        return self.fn(*a, **k)


@pytest.fixture(scope="module")
def ref():
    for p in (REF, LAB):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ.pop("ATSC3_LDPC_KERNEL", None)
    os.environ.pop("ATSC3_LDM_SP", None)
    import types
    import build_ldpc_kernel
    import m3_ldpc
    import m6_bicm
    import m9_accel
    import m9_gpu
    import m16_demap_fast
    import m44_ldm
    yield types.SimpleNamespace(LD=m3_ldpc, B=m6_bicm, m9a=m9_accel,
                                m9g=m9_gpu, M16=m16_demap_fast, M44=m44_ldm,
                                BK=build_ldpc_kernel)
    m9_accel.uninstall()


@pytest.fixture
def installed():
    from atsc3_b200 import install as I
    yield I
    I.uninstall()


def test_m9_gpu_verify_on_our_gpuminsum(ref, installed, monkeypatch):
    from atsc3_b200 import ldpc
    made = []

    class Spy(ldpc.GpuMinSum):
        def __init__(self, *a, **k):
            made.append(1)
            super().__init__(*a, **k)
    monkeypatch.setattr(ldpc, "GpuMinSum", Spy)
    installed.install(m9_gpu=ref.m9g)
    assert ref.m9g.GpuMinSum is Spy
    assert ref.m9g.verify(nblk=6, verbose=False) is True
    assert len(made) == 3                     # one decoder per gate case


def test_m16_demap_gates_on_our_demapper(ref, installed, monkeypatch):
    from atsc3_b200 import demap
    spy = Count(demap.demap_f64)
    monkeypatch.setattr(demap, "demap_f64", spy)
    installed.install(m16_demap_fast=ref.M16)
    ok = ref.M16.gate(n=20000, verbose=False)
    assert ok and all(ok.values()), ok
    assert spy.n >= 3
    assert ref.M16.gate_decoded(verbose=False) is True
    assert spy.n >= 4


def test_m9_accel_verify_bch_on_our_kernel(ref, installed, monkeypatch):
    from atsc3_b200 import bch
    spy = Count(bch.bch_syndrome_batch)
    monkeypatch.setattr(bch, "bch_syndrome_batch", spy)
    installed.install(m9_accel=ref.m9a)
    assert ref.m9a.bch_syndrome_batch is spy
    assert ref.m9a.verify(verbose=False) is True
    # 26 scalar messages + the 16-row batch + its 16 scalar comparisons
    assert spy.n >= 26 + 1 + 16


def test_build_ldpc_kernel_smoke_on_our_library(ref, installed):
    from atsc3_b200 import native as N
    installed.install(m3_ldpc=ref.LD)
    assert ref.BK.smoke(N.LIB_PATH) is None
    assert os.path.samefile(ref.LD._kernel_lib()._name, N.LIB_PATH)


@pytest.mark.parametrize("rate,n,esn0", [("3/15", 16200, 1.0),
                                         ("6/15", 64800, 7.5),
                                         ("10/15", 64800, 10.5)])
def test_m3_float32_batch_reaches_our_library(ref, installed, monkeypatch,
                                              rate, n, esn0):
    import oracle
    from atsc3_b200 import codes as C
    from atsc3_b200 import native as N
    mod = "QPSK"
    pay, cells, s2 = oracle.synth_case(
        lambda p: oracle.transmit(p, n, mod, rate)[0], 5, C.kpayload(rate, n),
        C.cells_per_block(n, mod), esn0, "awgn", 3)
    q = oracle.demap(cells, C.points_for(mod, rate), C.MOD_BITS[mod], s2)
    lam = oracle.deinterleave(q, C.bicm_map(n, mod, rate), n)
    checks = ref.LD.parity_check(rate, n)
    # the reference's own compiled kernel first
    ref.LD._KERNEL_STATE["lib"] = None
    want = ref.LD.min_sum_decode_batch(lam, checks, n, iters=50, alpha=0.75,
                                       dtype=np.float32)
    assert os.path.basename(ref.LD._kernel_lib()._name) == "ldpc_kernel.so"

    def no_numpy(*a, **k):
        raise AssertionError("the numpy fallback ran")
    monkeypatch.setattr(ref.LD, "pack", no_numpy)
    installed.install(m3_ldpc=ref.LD)
    assert os.path.samefile(ref.LD._kernel_lib()._name, N.LIB_PATH)
    got = ref.LD.min_sum_decode_batch(lam, checks, n, iters=50, alpha=0.75,
                                      dtype=np.float32)
    for a, b, k in zip(got, want, ("bits", "conv", "its", "bad")):
        assert np.array_equal(a, b), k


def test_m44_ldpc_batch_with_our_gpuminsum(ref, installed):
    """m44_ldm.ldpc_batch hands its `gpu` decoder the rows to decode
    (lab/m44_ldm.py:2519-2520): ours and the reference's torch GpuMinSum
    (float64, the reference's default) give the same bits/conv/bad."""
    import oracle
    from atsc3_b200 import codes as C
    from atsc3_b200 import ldpc
    n, mod, rate = 64800, "16QAM", "6/15"
    pay, cells, s2 = oracle.synth_case(
        lambda p: oracle.transmit(p, n, mod, rate)[0], 4, C.kpayload(rate, n),
        C.cells_per_block(n, mod), 7.75, "rayleigh", 9)
    q = oracle.demap(cells, C.points_for(mod, rate), C.MOD_BITS[mod], s2)
    lam = oracle.deinterleave(q, C.bicm_map(n, mod, rate), n)
    ch = ref.B.PlpChain(n, mod, rate)
    theirs = ref.m9g.GpuMinSum(ch.checks, n, iters=50)
    want = ref.M44.ldpc_batch(lam, ch, theirs, 50, alpha=0.75)
    ours = ldpc.GpuMinSum(ch.checks, n, iters=50)
    got = ref.M44.ldpc_batch(lam, ch, ours, 50, alpha=0.75)
    for a, b, k in zip(got, want, ("bits", "conv", "bad")):
        assert np.array_equal(a, b), k


@pytest.mark.parametrize("dtype", ["bfloat16", "float16"])
@pytest.mark.parametrize("rate,n,mod,esn0,chan", [("6/15", 16200, "QPSK", 1.5, "awgn"),
                                                 ("10/15", 64800, "64QAM", 14.0, "awgn")])
def test_gpuminsum_narrow_dtypes_match_reference(ref, dtype, rate, n, mod, esn0, chan):
    """GpuMinSum(dtype="bfloat16"/"float16") (lab/m9_gpu.py:100-101): the
    reference's torch decoder in that dtype on the GPU and ours give the
    same bits/conv/its/bad (16200 6/15 at 1.5 dB: five blocks converge at
    9-13 iterations in float32 and one sticks; 64800 10/15 at 14 dB:
    17-23 iterations)."""
    import oracle
    from atsc3_b200 import codes as C
    from atsc3_b200 import ldpc
    pay, cells, s2 = oracle.synth_case(
        lambda p: oracle.transmit(p, n, mod, rate)[0], 6, C.kpayload(rate, n),
        C.cells_per_block(n, mod), esn0, chan, 21)
    q = oracle.demap(cells, C.points_for(mod, rate), C.MOD_BITS[mod], s2)
    lam = oracle.deinterleave(q, C.bicm_map(n, mod, rate), n)
    checks = ref.LD.parity_check(rate, n)
    want = ref.m9g.GpuMinSum(checks, n, iters=30, dtype=dtype).decode(lam)
    got = ldpc.GpuMinSum(checks, n, iters=30, dtype=dtype).decode(lam)
    for a, b, k in zip(got, want, ("bits", "conv", "its", "bad")):
        assert np.array_equal(a, b), k
