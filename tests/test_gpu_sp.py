"""GPU exact sum-product (csrc/sp.cu) against the oracle on the golden
near-miss cases: convergence, iteration, unsatisfied count and hard
decisions equal (messages agree to float64 rounding: CUDA's tanh/log/exp/
atanh are not the host libm's, so the comparison is on decisions)."""
import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C
from test_sp_oracle import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(cases()))
def test_gpu_sum_product_matches_oracle(name):
    import torch
    from atsc3_b200 import ldpc as LDPC
    c = cases()[name]
    n = c["n"]
    lam, cw = oracle.near_miss_llr(c["rate"], n, c["nblk"], c["mu"], c["seed"])
    tabs = C.csr(c["rate"], n)
    tab = LDPC.sp_tables(tabs, n)
    o = LDPC.sp_decode(tab, torch.from_numpy(lam.astype(np.float64)).cuda(),
                       iters=c["iters"])
    torch.cuda.synchronize()
    assert o["conv"].cpu().numpy().astype(bool).tolist() == c["conv"]
    assert o["its"].cpu().numpy().tolist() == c["its"]
    assert o["bad"].cpu().numpy().tolist() == c["bad"]
    want = oracle.sum_product(lam, tabs, n, iters=c["iters"])[0]
    assert np.array_equal(o["bits"].cpu().numpy(), want)


def test_sum_product_dropin_signature():
    from atsc3_b200 import ldpc as LDPC
    c = cases()["sp_4_15"]
    lam, cw = oracle.near_miss_llr(c["rate"], c["n"], c["nblk"], c["mu"], c["seed"])
    bits, conv, its, bad = LDPC.sum_product_decode_batch(
        lam, C.parity_check(c["rate"], c["n"]), c["n"], iters=c["iters"])
    assert bits.dtype == np.uint8 and conv.dtype == bool
    assert conv.tolist() == c["conv"] and its.tolist() == c["its"]
    assert np.array_equal(bits, cw)


class TickClock:
    """A perf_counter that advances by one per reading, so a deadline of
    k - 0.5 lets iterations 0 .. k-1 start and stops at iteration k."""

    def __init__(self):
        self.t = -1.0

    def __call__(self):
        self.t += 1.0
        return self.t


@pytest.mark.parametrize("stop_at", [0, 1, 3])
def test_sum_product_deadline_stops_like_the_reference(monkeypatch, stop_at):
    """lab/m16_margin.py:364-371: after the deadline no new iteration
    starts; the iteration at which it is seen takes the syndrome, rows that
    converged there keep their verdict, the rest return their current hard
    decisions with conv False, its = that iteration, bad = the unsatisfied
    count, and stats["sp_timeout"] counts them.  That is exactly a decode
    run to iters = stop_at (the oracle), plus the count."""
    import types
    from atsc3_b200 import ldpc as LDPC
    c = cases()["sp_4_15"]
    n = c["n"]
    lam, cw = oracle.near_miss_llr(c["rate"], n, c["nblk"], c["mu"], c["seed"])
    assert min(c["its"]) > 3                 # every row is still decoding
    # the decoder's clock only (ldpc.time), not the process-wide one
    monkeypatch.setattr(LDPC, "time", types.SimpleNamespace(perf_counter=TickClock()))
    stats = {}
    bits, conv, its, bad = LDPC.sum_product_decode_batch(
        lam, C.parity_check(c["rate"], n), n, iters=c["iters"],
        deadline=stop_at - 0.5, stats=stats)
    wb, wc, wi, wd = oracle.sum_product(lam, C.csr(c["rate"], n), n, iters=stop_at)
    assert its.tolist() == [stop_at] * len(its) == wi.tolist()
    assert conv.tolist() == wc.tolist() and bad.tolist() == wd.tolist()
    assert np.array_equal(bits, wb)
    assert stats == {"sp_timeout": int((~wc).sum())} and (~wc).sum() > 0


def test_sum_product_deadline_not_reached_is_the_full_decode():
    import time as _time
    from atsc3_b200 import ldpc as LDPC
    c = cases()["sp_4_15"]
    lam, cw = oracle.near_miss_llr(c["rate"], c["n"], c["nblk"], c["mu"], c["seed"])
    stats = {}
    bits, conv, its, bad = LDPC.sum_product_decode_batch(
        lam, C.parity_check(c["rate"], c["n"]), c["n"], iters=c["iters"],
        deadline=_time.perf_counter() + 3600.0, stats=stats)
    assert conv.tolist() == c["conv"] and its.tolist() == c["its"]
    assert bad.tolist() == c["bad"] and stats == {}
    assert np.array_equal(bits, cw)


def test_rescue_replaces_min_sum_failures():
    """Blocks min-sum leaves unconverged get the sum-product; those it
    closes carry the sum-product's hard decisions (packed) and conv = 1."""
    import torch
    from atsc3_b200 import ldpc as LDPC
    c = cases()["sp_8_15_a"]
    n = c["n"]
    lam, cw = oracle.near_miss_llr(c["rate"], n, c["nblk"], c["mu"], c["seed"])
    tabs = C.csr(c["rate"], n)
    plan = LDPC.plan_for(c["rate"], n)
    x = torch.from_numpy(lam).cuda()
    o = LDPC.decode_flood(plan, x, iters=50, want_hard=True)
    assert not o["conv"].bool().any()                # min-sum fails them all
    got = LDPC.rescue_near_misses(LDPC.sp_tables(tabs, n), x, o,
                                  near_max=100000, max_blocks=8, iters=c["iters"])
    assert sorted(got.tolist()) == [b for b, ok in enumerate(c["conv"]) if ok]
    sp_bits = oracle.sum_product(lam, tabs, n, iters=c["iters"])[0]
    hard = o["hard"].cpu().numpy()[:, :n // 8]
    for b in got:
        assert np.array_equal(hard[b], np.packbits(sp_bits[b]))
        assert int(o["conv"][b]) == 1 and int(o["bad"][b]) == 0


@pytest.mark.parametrize("kind", ["auto", "csr"])
def test_gpu_ladder_matches_oracle(kind):
    """The alpha ladder on the GPU keeps, per block, the same rung, bits,
    convergence, iterations and unsatisfied count as the oracle ladder
    (which reproduces the reference's, tests/test_ladder_oracle.py)."""
    import torch
    from atsc3_b200 import ldpc as LDPC
    from test_ladder_oracle import golden
    g = golden()
    for name, c in sorted(g["cases"].items()):
        n = c["n"]
        lam, cw = oracle.near_miss_llr(c["rate"], n, c["nblk"], c["mu"], c["seed"])
        want = oracle.ladder(lam, C.csr(c["rate"], n), n, alphas=tuple(g["ladder"]),
                             iters=c["iters"])
        plan = LDPC.plan_for(c["rate"], n, kind=kind)
        o = LDPC.ladder_decode(plan, torch.from_numpy(lam).cuda(),
                               ladder=tuple(g["ladder"]), iters=c["iters"])
        assert np.array_equal(o["bits"].cpu().numpy(), want[0]), name
        assert o["conv"].cpu().numpy().astype(bool).tolist() == want[1].tolist()
        assert o["its"].cpu().numpy().tolist() == want[2].tolist()
        assert o["bad"].cpu().numpy().tolist() == want[3].tolist()
        assert np.array_equal(o["alpha"].cpu().numpy(), want[4])
        assert np.array_equal(o["hard"].cpu().numpy()[:, :n // 8],
                              np.packbits(want[0], axis=1))


def test_pipeline_ladder_and_dropin():
    """FecPipeline(ladder=...) decodes with the ladder; the host-array
    ldpc_batch drop-in returns the oracle ladder's (bits, conv, bad)."""
    import torch
    from atsc3_b200 import ldpc as LDPC
    from test_ladder_oracle import golden
    g = golden()
    c = g["cases"]["ladder_6_15"]
    n = c["n"]
    lam, cw = oracle.near_miss_llr(c["rate"], n, c["nblk"], c["mu"], c["seed"])
    want = oracle.ladder(lam, C.csr(c["rate"], n), n, alphas=tuple(g["ladder"]),
                         iters=c["iters"])
    bits, conv, bad = LDPC.ldpc_batch(lam, c["rate"], n, iters=c["iters"])
    assert np.array_equal(bits, want[0])
    assert conv.tolist() == want[1].tolist() and bad.tolist() == want[3].tolist()
