"""The float64 weighted min-sum reference (the oracle of the backward
kernels) against finite differences, and against the plain normalised
min-sum oracle when the weights reduce to alpha-scaling (CPU only)."""
import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C


def _llr(n, nb, seed, scale=2.0, mean=1.5):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((nb, n)) * scale + mean).astype(np.float32)


def test_reference_equals_plain_minsum_when_unweighted():
    import torch
    from atsc3_b200.learned import reference_f64
    rate, n, T = "11/15", 16200, 4
    llr = _llr(n, 2, 1)
    nbk = len(np.unique(np.diff(C.csr(rate, n)[0])))
    a = torch.full((T, nbk), 0.75, dtype=torch.float64)
    b = torch.zeros((T, nbk), dtype=torch.float64)
    out = reference_f64(torch.from_numpy(llr), a, b, rate, n).numpy()
    # the plain oracle with float64 messages, T updates, no early stop:
    # compare hard decisions (summation order differs from float32)
    bits, conv, its, bad = oracle.flood(llr.astype(np.float64),
                                        C.csr(rate, n), n, iters=T,
                                        alpha=0.75, semantics=1,
                                        dtype=np.float64)
    if not conv.any():
        assert np.array_equal((out < 0).astype(np.uint8), bits)


def test_reference_gradient_matches_finite_differences():
    import torch
    from atsc3_b200.learned import bce_loss, reference_f64
    rate, n, T = "11/15", 16200, 3
    llr = torch.from_numpy(_llr(n, 2, 2, scale=2.5, mean=1.0))
    bits = torch.zeros((2, n), dtype=torch.float64)
    nbk = len(np.unique(np.diff(C.csr(rate, n)[0])))
    rng = np.random.default_rng(3)
    a = torch.tensor(0.6 + 0.3 * rng.random((T, nbk)), dtype=torch.float64,
                     requires_grad=True)
    b = torch.tensor(0.05 * rng.random((T, nbk)), dtype=torch.float64,
                     requires_grad=True)
    loss = bce_loss(reference_f64(llr, a, b, rate, n), bits)
    loss.backward()
    eps = 1e-6
    for P, G in ((a, a.grad), (b, b.grad)):
        for (t, d) in ((0, 0), (T - 1, nbk - 1), (1, 0)):
            with torch.no_grad():
                P[t, d] += eps
                lp = float(bce_loss(reference_f64(llr, a, b, rate, n), bits))
                P[t, d] -= 2 * eps
                lm = float(bce_loss(reference_f64(llr, a, b, rate, n), bits))
                P[t, d] += eps
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - float(G[t, d])) <= 1e-5 * max(1.0, abs(fd)) + 1e-9, (fd, float(G[t, d]))


def test_reference_gradient_fd_at_the_training_shape():
    """Config 4's shape: 4 blocks of the 64800-bit rate-8/15 code with
    64-NUC LLRs from the demapper near the MODCOD's threshold (12.6 dB),
    T = 12 unrolled iterations, per-iteration x per-check-degree (scale,
    offset).  Central differences (eps 1e-6, float64) on entries at the
    first, a middle and the last iteration agree with the autograd
    gradient to 1e-6 relative (measured: about 1e-9)."""
    import torch
    from atsc3_b200.learned import bce_loss, reference_f64
    rate, n, T, mod = "8/15", 64800, 12, "64QAM"
    pay, cells, s2 = oracle.synth_case(
        lambda p: oracle.transmit(p, n, mod, rate)[0], 4, C.kpayload(rate, n),
        C.cells_per_block(n, mod), 12.6, "awgn", 21)
    q = oracle.demap(cells, C.points_for(mod, rate), C.MOD_BITS[mod], s2)
    lam = oracle.deinterleave(q, C.bicm_map(n, mod, rate), n)
    cw = oracle.transmit(pay, n, mod, rate)[1]
    llr = torch.from_numpy(lam)
    bits = torch.from_numpy(cw).double()
    nbk = len(np.unique(np.diff(C.csr(rate, n)[0])))
    rng = np.random.default_rng(3)
    a = torch.tensor(0.6 + 0.3 * rng.random((T, nbk)), dtype=torch.float64,
                     requires_grad=True)
    b = torch.tensor(0.2 * rng.random((T, nbk)), dtype=torch.float64,
                     requires_grad=True)
    loss = bce_loss(reference_f64(llr, a, b, rate, n), bits)
    loss.backward()
    eps = 1e-6
    for P, G in ((a, a.grad), (b, b.grad)):
        for (t, d) in ((0, 0), (5, nbk - 1), (T - 1, 0), (T - 1, nbk - 1)):
            with torch.no_grad():
                P[t, d] += eps
                lp = float(bce_loss(reference_f64(llr, a, b, rate, n), bits))
                P[t, d] -= 2 * eps
                lm = float(bce_loss(reference_f64(llr, a, b, rate, n), bits))
                P[t, d] += eps
            fd = (lp - lm) / (2 * eps)
            g = float(G[t, d])
            assert g != 0.0
            assert abs(fd - g) <= 1e-6 * abs(g), (t, d, fd, g)
