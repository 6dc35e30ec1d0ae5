"""Code construction (atsc3_b200/codes.py) against the reference's tables."""
import numpy as np
import pytest

from atsc3_b200 import codes as C
from golden_util import golden, sha


@pytest.mark.parametrize("n", [16200, 64800])
def test_parity_check_tables_match_reference(n):
    meta, _ = golden()
    for r in C.RATES:
        got = [sha(np.asarray(t, np.int32)) for t in C.csr(r, n)]
        assert got == meta["tables"][f"{n}:{r}"], (n, r)


def test_bicm_maps_match_reference():
    meta, _ = golden()
    assert len(meta["bicm"]) == 120
    for key, want in meta["bicm"].items():
        n, mod, rate = key.split(":")
        assert sha(C.bicm_map(int(n), mod, rate)) == want, key


def test_bicm_maps_are_permutations():
    meta, _ = golden()
    for key in meta["bicm"]:
        n, mod, rate = key.split(":")
        m = C.bicm_map(int(n), mod, rate)
        assert np.array_equal(np.sort(m), np.arange(int(n)))


def test_block_interleaver_worked_example():
    """A/322 6.2.3.1's printed example (256QAM, Ninner 64800, Type A), the
    gate of lab/m6_bicm.py:380-406."""
    v = C.blockint_map(64800, "256QAM", "2/15")
    assert list(v[:16]) == [0, 7920, 15840, 23760, 31680, 39600, 47520, 55440,
                            1, 7921, 15841, 23761, 31681, 39601, 47521, 55441]
    assert list(v[-8:]) == [63539, 63719, 63899, 64079, 64259, 64439, 64619,
                            64799]
    assert list(v[8 * 7920 - 1:8 * 7920 + 8]) == [63359, 63360, 63540, 63720,
                                                  63900, 64080, 64260, 64440,
                                                  64620]


def test_nuc_mean_power():
    """lab/spec_nuc.py:130-141 identity: every NUC has unit mean power."""
    for mod, tol in (("16QAM", 1.5e-3), ("64QAM", 2e-4), ("256QAM", 2e-4)):
        for r in C.RATES:
            p = C.points_for(mod, r)
            assert abs(np.mean(np.abs(p) ** 2) - 1) < tol


def test_standin_qam_unit_power():
    for m in (1024, 4096):
        assert abs(np.mean(np.abs(C.standin_qam(m)) ** 2) - 1) < 1e-12


def test_structure():
    """lab/m3_ldpc.py:637-674 gates: N-K checks, every column covered."""
    for n in (16200, 64800):
        for r in C.RATES:
            cptr, cidx, vptr, vedge = C.csr(r, n)
            assert len(cptr) - 1 == n - C.kldpc(r, n)
            assert (np.diff(vptr) > 0).all()


def test_encoder_satisfies_parity_checks():
    import oracle
    rng = np.random.default_rng(4)
    for n in (16200, 64800):
        for r in ("2/15", "6/15", "7/15", "13/15"):
            K = C.kldpc(r, n)
            cw = oracle.ldpc_encode(rng.integers(0, 2, (2, K)), r, n)
            cptr, cidx, _, _ = C.csr(r, n)
            syn = np.bitwise_xor.reduceat(cw[:, cidx], cptr[:-1], axis=1)
            assert not syn.any(), (n, r)


def test_bch_remainder_table_matches_polynomial_division():
    import oracle
    rng = np.random.default_rng(5)
    for n, k in ((16200, 11880), (64800, 25920)):
        R = C.bch_remainder_table(k, n)
        m = rng.integers(0, 2, (3, k)).astype(np.uint8)
        for row in m:
            words = np.bitwise_xor.reduce(R[row.astype(bool)], axis=0)
            assert C.syndrome_words_to_int(words) == oracle.bch_syndrome(row, n)[0]
