"""The weighted min-sum oracle (oracle.flood_weighted, numpy) is pinned to
the C oracle (itself pinned to lab/ldpc_kernel.c): with scale = alpha and
offset = 0 for every iteration and check degree, both decode identically,
on Type A and Type B codes, blocks that converge and blocks that do not."""
import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C


def weights_for(tables, T, alpha):
    degs = np.unique(np.diff(tables[0]))
    db = np.zeros(256, np.int64)
    db[degs] = np.arange(len(degs))
    return (np.full((T, len(degs)), alpha, np.float32),
            np.zeros((T, len(degs)), np.float32), db)


@pytest.mark.parametrize("rate,n", [("3/15", 16200), ("2/15", 16200), ("8/15", 16200),
                                    ("11/15", 16200), ("7/15", 64800)])
def test_weighted_oracle_matches_c_oracle(rate, n):
    tabs = C.csr(rate, n)
    rng = np.random.default_rng(n + C.RATES.index(rate))
    llr = (rng.standard_normal((4, n)) * 1.6 + np.array([[2.6], [2.2], [1.6], [9.0]])).astype(np.float32)
    for alpha in (0.75, 0.875):
        wa, wb, db = weights_for(tabs, 3, alpha)
        got = oracle.flood_weighted(llr, tabs, n, wa, wb, db, iters=14)
        want = oracle.flood(llr, tabs, n, iters=14, alpha=alpha)
        for g, w in zip(got, want):
            assert np.array_equal(g, w), (rate, n, alpha)


def test_row_buckets_with_equal_rows_equal_degree_buckets():
    """Per-block-row weights whose rows all carry the same (scale, offset)
    decode exactly like per-degree weights with that value."""
    from atsc3_b200 import learned as LR
    rate, n, T = "11/15", 16200, 4
    tabs = C.csr(rate, n)
    rng = np.random.default_rng(2)
    llr = (rng.standard_normal((2, n)) * 2.0 + 2.0).astype(np.float32)
    rows = LR.block_rows(rate, n)
    nr = int(rows.max()) + 1
    a_t = (0.7 + 0.2 * rng.random(T)).astype(np.float32)
    b_t = (0.1 * rng.random(T)).astype(np.float32)
    wa_r = np.repeat(a_t[:, None], nr, 1)
    wb_r = np.repeat(b_t[:, None], nr, 1)
    db = np.zeros(256, np.int64)
    got = oracle.flood_weighted(llr, tabs, n, wa_r, wb_r, db, iters=8,
                                cbucket=rows)
    want = oracle.flood_weighted(llr, tabs, n, a_t[:, None], b_t[:, None], db,
                                 iters=8)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
