"""Layered min-sum on the GPU against the layered oracle (bit-exact), and
its convergence advantage over flooding under the same alpha."""
import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C
from golden_util import oracle_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rate", ["6/15", "8/15", "10/15", "13/15"])
def test_layered_vs_oracle_random(rate):
    import torch
    from atsc3_b200.ldpc import LayeredPlan, check_layered_error, decode_layered
    n = 64800
    rng = np.random.default_rng(len(rate) * 7)
    llr = (rng.standard_normal((4, n)) * 2.0 + 2.2).astype(np.float32)
    llr[3] = np.abs(llr[3])                          # clean block: its == 0
    want = oracle.layered(llr, rate, n, iters=12, alpha=0.75)
    plan = LayeredPlan(rate, n, ctas=3)              # fewer CTAs than blocks
    o = decode_layered(plan, torch.from_numpy(llr).cuda(), iters=12,
                       alpha=0.75, want_hard=True)
    check_layered_error(plan)
    bits = o["bits"].cpu().numpy()
    assert np.array_equal(bits, want[0])
    assert o["conv"].cpu().numpy().astype(bool).tolist() == want[1].tolist()
    assert o["its"].cpu().numpy().tolist() == want[2].tolist()
    assert o["bad"].cpu().numpy().tolist() == want[3].tolist()
    assert np.array_equal(o["hard"].cpu().numpy()[:, :n // 8],
                          np.packbits(bits, axis=1))


@pytest.mark.parametrize("name", ["c64_256qam_10_15", "c64_16qam_6_15_ray"])
def test_layered_golden_cases(name):
    import torch
    from atsc3_b200.ldpc import LayeredPlan, check_layered_error, decode_layered
    c, pay, cw, cells, s2, q, lam = oracle_case(name)
    want = oracle.layered(lam, c["rate"], c["n"], iters=50, alpha=0.75)
    plan = LayeredPlan(c["rate"], c["n"])
    o = decode_layered(plan, torch.from_numpy(lam).cuda(), iters=50, alpha=0.75)
    check_layered_error(plan)
    assert np.array_equal(o["bits"].cpu().numpy(), want[0])
    assert o["its"].cpu().numpy().tolist() == want[2].tolist()
    assert o["bad"].cpu().numpy().tolist() == want[3].tolist()
    # converged blocks decode to the transmitted codeword
    for i in np.flatnonzero(want[1]):
        assert np.array_equal(want[0][i], cw[i])


def test_layered_copy_timeout_path_reports_and_context_survives():
    """The bounded-wait error path: the test hook makes every CTA take the
    timeout branch at layer 5 of iteration 0, right after that layer's
    copies completed (nothing is in flight when the CTAs return).  The
    launch records error code 1, check_layered_error raises, and the next
    launch on the same plan decodes bit-exactly again."""
    import torch
    from atsc3_b200 import native as N
    from atsc3_b200.ldpc import LayeredPlan, check_layered_error, decode_layered
    n, rate = 64800, "8/15"
    rng = np.random.default_rng(11)
    llr = (rng.standard_normal((4, n)) * 2.0 + 1.0).astype(np.float32)
    plan = LayeredPlan(rate, n, ctas=2)
    d = torch.from_numpy(llr).cuda()
    N.call("atsc3_ldpc_layered_inject_timeout", 5)
    decode_layered(plan, d, iters=8, alpha=0.75)
    torch.cuda.synchronize()
    assert int(plan.err.item()) == 1
    with pytest.raises(N.FecError) as e:
        check_layered_error(plan)
    assert "error code 1" in str(e.value)
    assert int(plan.err.item()) == 0           # the checker clears it
    # the hook is consumed by one call: this launch runs normally
    want = oracle.layered(llr, rate, n, iters=8, alpha=0.75)
    o = decode_layered(plan, d, iters=8, alpha=0.75)
    check_layered_error(plan)
    assert np.array_equal(o["bits"].cpu().numpy(), want[0])
    assert o["its"].cpu().numpy().tolist() == want[2].tolist()
