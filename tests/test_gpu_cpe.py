"""GPU common phase error correction (csrc/cpe.cu) against the oracle on
the golden pools: every corrected cell and every per-symbol gain within
1e-12 (relative to the pool's scale) -- float64 sums run in other orders
than numpy's BLAS dot products -- and identical hard decisions."""
import numpy as np
import pytest

import oracle
from test_cpe_oracle import case_inputs, cases

pytestmark = pytest.mark.gpu


def _hard(z, sym, alph, region):
    h = np.zeros(len(z), np.int64)
    for rid in (0, 1):
        sel = region == rid
        h[sel] = np.abs(z[sel][:, None] - alph[rid][None, :]).argmin(1)
    return h


@pytest.mark.parametrize("name", sorted(cases()))
def test_gpu_cpe_matches_oracle(name):
    from atsc3_b200.cpe import cpe_correct
    c = cases()[name]
    pool, sym, alph, region, dummy = case_inputs(c)
    want, wg = oracle.cpe_correct(pool, sym, alph, region, dummy, iters=c["iters"])
    got, gg = cpe_correct(pool, sym, alph, region, dummy, iters=c["iters"])
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))
    for s in wg:
        assert abs(gg[s] - wg[s]) <= 1e-12 * abs(wg[s])
    assert np.array_equal(_hard(got, sym, alph, region), _hard(want, sym, alph, region))


def test_gpu_cpe_unsorted_symbols_and_no_iterations():
    """Cells of a symbol need not be contiguous (the drop-in groups them);
    iters = 0 only normalises the pool."""
    from atsc3_b200.cpe import cpe_correct
    c = cases()["cpe_64_16"]
    pool, sym, alph, region, dummy = case_inputs(c)
    perm = np.random.default_rng(0).permutation(len(pool))
    want, wg = oracle.cpe_correct(pool[perm], sym[perm], alph, region[perm],
                                  dummy[perm], iters=3)
    got, gg = cpe_correct(pool[perm], sym[perm], alph, region[perm], dummy[perm])
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))
    got0, g0 = cpe_correct(pool, sym, alph, region, dummy, iters=0)
    assert np.allclose(got0, pool / np.sqrt(np.mean(np.abs(pool) ** 2)), rtol=0, atol=1e-13)
    assert all(v == 1 for v in g0.values())
