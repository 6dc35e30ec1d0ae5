"""Pins ``oracle.flood_torch_narrow`` against the reference's own torch
decoder run on the CPU with dtype bfloat16 / float16 (lab/m9_gpu.py:84-220,
from the unmodified copy in baseline/_ref laid out by
``python oracle/build.py --ref-tree``; skipped where it is absent): bits,
conv, its and bad identical, converging and stuck blocks alike."""
import os
import sys

import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LAB = os.path.join(ROOT, "baseline", "_ref", "lab")

needs_ref = pytest.mark.skipif(
    not os.path.exists(os.path.join(LAB, "m9_gpu.py")),
    reason="baseline/_ref not laid out (python oracle/build.py --ref-tree)")


def _case(rate, n, mod, esn0, chan, nblk, seed):
    pay, cells, s2 = oracle.synth_case(
        lambda p: oracle.transmit(p, n, mod, rate)[0], nblk, C.kpayload(rate, n),
        C.cells_per_block(n, mod), esn0, chan, seed)
    q = oracle.demap(cells, C.points_for(mod, rate), C.MOD_BITS[mod], s2)
    return oracle.deinterleave(q, C.bicm_map(n, mod, rate), n)


@needs_ref
@pytest.mark.parametrize("dtype", ["bfloat16", "float16"])
@pytest.mark.parametrize("rate,esn0", [("6/15", 1.5), ("3/15", -3.75)])
def test_narrow_oracle_matches_reference_torch_cpu(dtype, rate, esn0):
    import torch
    for p in (os.path.dirname(LAB), LAB):
        if p not in sys.path:
            sys.path.insert(0, p)
    import m3_ldpc
    import m9_gpu
    n = 16200                      # 6/15 Type B, 3/15 Type A
    lam = _case(rate, n, "QPSK", esn0, "awgn", 6, 21)
    want = m9_gpu.GpuMinSum(m3_ldpc.parity_check(rate, n), n, iters=30,
                            device="cpu", dtype=dtype).decode(lam)
    tdt = torch.bfloat16 if dtype == "bfloat16" else torch.float16
    lam_n = torch.from_numpy(np.ascontiguousarray(lam, np.float64)).to(tdt).float().numpy()
    got = oracle.flood_torch_narrow(lam_n, C.csr(rate, n), n, iters=30, alpha=0.75,
                                    dtype=dtype)
    for a, b, k in zip(got, want, ("bits", "conv", "its", "bad")):
        assert np.array_equal(np.asarray(a), np.asarray(b)), k
    # the case holds converging blocks and at least one that sticks
    assert np.asarray(want[1]).any() and not np.asarray(want[1]).all()


@pytest.mark.parametrize("dtype", ["bfloat16", "float16"])
def test_narrow_rounding_matches_torch_conversion(dtype):
    """The oracle's rounding to bfloat16 / float16 equals torch's own
    float32 -> narrow conversion (round to nearest even, float16 overflowing
    to infinity) on random values, exact ties and extremes."""
    import torch
    rng = np.random.default_rng(5)
    x = np.concatenate([
        (rng.standard_normal(20000) * 10.0 ** rng.integers(-8, 6, 20000)),
        np.array([0.0, -0.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 65504.0, 65519.0,
                  65520.0, 1e30, -1e30, 3e38, 2.0 ** -130, np.inf, -np.inf])]).astype(np.float32)
    tdt = torch.bfloat16 if dtype == "bfloat16" else torch.float16
    want = torch.from_numpy(x).to(tdt).float().numpy()
    got = oracle._narrow(x, dtype)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
