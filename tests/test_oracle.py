"""The oracle against the reference's golden vectors (CPU only).

Every synthetic case of tests/golden/golden.npz was produced by the
reference's own transmitter, demapper, compiled kernel and BCH helpers
(tests/golden/make_golden.py); here the oracle recomputes each stage from
the same seed and must match bit for bit.
"""
import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C
from golden_util import golden, oracle_case, sha

CASES = sorted(golden()[0]["cases"])


@pytest.mark.parametrize("name", CASES)
def test_transmitter_demap_deinterleave(name):
    c, pay, cw, cells, s2, q, lam = oracle_case(name)
    assert sha(pay) == c["payload_sha"]
    assert sha(cw) == c["cw_sha"]
    assert sha(cells) == c["cells_sha"]
    assert sha(q) == c["llr_q_sha"]
    assert sha(lam) == c["lam_sha"]


@pytest.mark.parametrize("name", CASES)
def test_decoder_and_bch(name):
    c, pay, cw, cells, s2, q, lam = oracle_case(name)
    n = c["n"]
    bits, conv, its, bad = oracle.flood(lam, C.csr(c["rate"], n), n,
                                        iters=50, alpha=0.75, semantics=0)
    assert sha(bits) == c["bits_sha"]
    assert conv.astype(int).tolist() == c["conv"]
    assert its.tolist() == c["its"]
    assert bad.tolist() == c["bad"]
    k = C.kldpc(c["rate"], n)
    assert [hex(s) for s in oracle.bch_syndrome(bits[:, :k], n)] == c["bch"]
    kp = C.kpayload(c["rate"], n)
    payload = np.packbits(bits[:, :kp] ^ C.scrambler_sequence(kp)[None, :],
                          axis=1)
    assert sha(payload) == c["payload_bytes_sha"]


@pytest.mark.parametrize("name", [k for k in CASES if k.startswith("c16")])
def test_decoder_float64_torch_semantics(name):
    c, pay, cw, cells, s2, q, lam = oracle_case(name)
    n = c["n"]
    bits, conv, its, bad = oracle.flood(lam.astype(np.float64),
                                        C.csr(c["rate"], n), n, iters=50,
                                        alpha=0.75, semantics=1,
                                        dtype=np.float64)
    assert sha(bits) == c["f64_bits_sha"]
    assert conv.astype(int).tolist() == c["f64_conv"]
    assert its.tolist() == c["f64_its"]
    assert bad.tolist() == c["f64_bad"]


@pytest.mark.parametrize("name", CASES)
def test_demap_estimated_sigma(name):
    c, pay, cw, cells, s2, q, lam = oracle_case(name)
    pts = C.points_for(c["mod"], c["rate"])
    qe = oracle.demap(cells, pts, C.MOD_BITS[c["mod"]], None)
    assert sha(qe) == c["llr_q_est_sha"]


def test_bch_messages():
    meta, arrs = golden()
    for key, want in meta["bch"].items():
        n, k = map(int, key.split(":"))
        m = np.unpackbits(arrs[f"bch_msg/{key}"], axis=1)[:, :k]
        assert [hex(s) for s in oracle.bch_syndrome(m, n)] == want


def test_bch_encode_roundtrip():
    rng = np.random.default_rng(1)
    for n in (16200, 64800):
        for rate in ("2/15", "13/15"):
            kp = C.kpayload(rate, n)
            cw = oracle.bch_encode(rng.integers(0, 2, (2, kp)), n)
            assert oracle.bch_syndrome(cw, n) == [0, 0]


def test_reference_kernel_known_answer():
    """lab/build_ldpc_kernel.py:101-120: LLR=+5 retires at iteration 0."""
    if oracle.ref_lib() is None:
        pytest.skip("reference kernel not built here")
    tabs = C.csr("3/15", 16200)
    for fn in (lambda l: oracle.flood_ref(l, tabs, 16200),
               lambda l: oracle.flood(l, tabs, 16200)):
        bits, conv, its, bad = fn(np.full((2, 16200), 5.0, np.float32))
        assert conv.all() and (its == 0).all() and (bad == 0).all()
        assert not bits.any()


def test_oracle_equals_reference_kernel_random_llr():
    """Oracle C restatement == lab/ldpc_kernel.c on random LLRs, including
    the high-degree Type A code (row degree 86)."""
    if oracle.ref_lib() is None:
        pytest.skip("reference kernel not built here")
    rng = np.random.default_rng(3)
    for rate, n, scale in (("7/15", 64800, 2.0), ("2/15", 16200, 1.5),
                           ("13/15", 16200, 4.0)):
        tabs = C.csr(rate, n)
        llr = (rng.standard_normal((2, n)) * scale + 1.0).astype(np.float32)
        a = oracle.flood(llr, tabs, n, iters=12, alpha=0.8)
        b = oracle.flood_ref(llr, tabs, n, iters=12, alpha=0.8)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_bch_fast_equals_polynomial_division():
    meta, arrs = golden()
    for key, want in meta["bch"].items():
        n, k = map(int, key.split(":"))
        m = np.unpackbits(arrs[f"bch_msg/{key}"], axis=1)[:, :k]
        assert [hex(s) for s in oracle.bch_syndrome_fast(m, n)] == want
