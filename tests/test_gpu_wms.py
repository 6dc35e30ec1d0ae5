"""The hand-written weighted min-sum kernels (forward + backward) against the
float64 autograd reference on 4 blocks of the 64800-bit rate-8/15 code, the
plain-normalised special case, and the BF16-message variant."""
import numpy as np
import pytest

from atsc3_b200 import codes as C

pytestmark = pytest.mark.gpu


def _case(seed=5, nb=4, n=64800, rate="8/15"):
    import oracle
    c_rng = np.random.default_rng(seed)
    tx = lambda p: oracle.transmit(p, n, "64QAM", rate)[0]
    pay, cells, s2 = oracle.synth_case(tx, nb, C.kpayload(rate, n),
                                       C.cells_per_block(n, "64QAM"), 11.5,
                                       "awgn", seed)
    q = oracle.demap(cells, C.points_for("64QAM", rate), 6, s2)
    lam = oracle.deinterleave(q, C.bicm_map(n, "64QAM", rate), n)
    cw = oracle.transmit(pay, n, "64QAM", rate)[1]
    return lam, cw


def test_wms_forward_and_gradients_vs_float64_reference():
    import torch
    from atsc3_b200.learned import (WeightedMinSum, WmsCode, bce_loss,
                                    reference_f64)
    rate, n, T = "8/15", 64800, 12
    lam, cw = _case()
    code = WmsCode(rate, n)
    rng = np.random.default_rng(7)
    a0 = (0.7 + 0.2 * rng.random((T, code.nbucket))).astype(np.float32)
    b0 = (0.1 * rng.random((T, code.nbucket))).astype(np.float32)
    a = torch.tensor(a0, device="cuda", requires_grad=True)
    b = torch.tensor(b0, device="cuda", requires_grad=True)
    x = torch.from_numpy(lam).cuda()
    bits = torch.from_numpy(cw).cuda()
    out = WeightedMinSum.apply(x, a, b, code, False)
    loss = bce_loss(out, bits)
    loss.backward()
    a64 = torch.tensor(a0, dtype=torch.float64, requires_grad=True)
    b64 = torch.tensor(b0, dtype=torch.float64, requires_grad=True)
    ref = reference_f64(torch.from_numpy(lam), a64, b64, rate, n)
    lref = bce_loss(ref, torch.from_numpy(cw).double())
    lref.backward()
    o = out.detach().cpu().double().numpy()
    r = ref.detach().numpy()
    # measured on one B200 over three seeds of this case: output LLRs
    # within 3.0e-6 of max(1, |ref|), loss within 3.3e-7 relative, parameter
    # gradients within 1.8e-4 of the largest gradient entry (float32
    # messages against float64); the bars keep a margin of 5-10x
    assert (np.abs(o - r) <= 3e-5 * np.maximum(1.0, np.abs(r))).all()
    assert abs(float(loss.detach()) - float(lref.detach())) <= 3e-6 * abs(float(lref.detach()))
    for g, gr in ((a.grad, a64.grad), (b.grad, b64.grad)):
        g = g.cpu().double().numpy()
        gr = gr.numpy()
        rel = np.abs(g - gr).max() / max(np.abs(gr).max(), 1e-12)
        assert rel < 1e-3, rel


def test_wms_unweighted_equals_plain_minsum_hard_decisions():
    """alpha = 0.75, beta = 0 for T iterations is the normalised min-sum
    without early stop: same hard decisions as the float32 oracle when the
    oracle runs the same number of updates (torch semantics)."""
    import torch
    import oracle
    from atsc3_b200.learned import WeightedMinSum, WmsCode
    rate, n, T = "8/15", 64800, 6
    lam, cw = _case(seed=9)
    code = WmsCode(rate, n)
    a, b = code.init_params(T, 0.75, 0.0)
    out = WeightedMinSum.apply(torch.from_numpy(lam).cuda(), a, b, code, False)
    want = oracle.flood(lam, C.csr(rate, n), n, iters=T, alpha=0.75, semantics=1)
    got = (out.cpu().numpy() < 0).astype(np.uint8)
    for i in range(len(lam)):
        if not want[1][i]:                # no early stop happened: same T
            assert (got[i] != want[0][i]).mean() < 1e-3


def test_wms_bf16_messages_close_to_fp32():
    import torch
    from atsc3_b200.learned import WeightedMinSum, WmsCode, bce_loss
    rate, n, T = "8/15", 64800, 12
    lam, cw = _case(seed=11)
    code = WmsCode(rate, n)
    a, b = code.init_params(T, 0.8, 0.05)
    x = torch.from_numpy(lam).cuda()
    bits = torch.from_numpy(cw).cuda()
    l32 = float(bce_loss(WeightedMinSum.apply(x, a, b, code, False), bits))
    l16 = float(bce_loss(WeightedMinSum.apply(x, a, b, code, True), bits))
    assert abs(l16 - l32) <= 0.05 * abs(l32) + 1e-4


@pytest.mark.parametrize("kind", ["qce", "qc"])
def test_weighted_qc_decoder_matches_wms_forward(kind):
    """The inference decoder with learned weights (both quasi-cyclic layouts,
    torch semantics) computes the same posterior as the differentiable
    forward for blocks that run all T iterations: identical hard
    decisions."""
    import torch
    from atsc3_b200.ldpc import decode_flood, plan_for
    from atsc3_b200.learned import WeightedMinSum, WmsCode, inference_weights
    rate, n, T = "8/15", 64800, 12
    lam, cw = _case(seed=13, nb=6)
    lam[:3] *= 0.55                        # weaker blocks: no early stop
    code = WmsCode(rate, n)
    rng = np.random.default_rng(4)
    a = torch.tensor(0.7 + 0.2 * rng.random((T, code.nbucket)), dtype=torch.float32, device="cuda")
    b = torch.tensor(0.1 * rng.random((T, code.nbucket)), dtype=torch.float32, device="cuda")
    x = torch.from_numpy(lam).cuda()
    ref = (WeightedMinSum.apply(x, a, b, code, False) < 0).to(torch.uint8).cpu().numpy()
    plan = plan_for(rate, n, kind=kind)
    o = decode_flood(plan, x, iters=T, semantics="torch",
                     weights=inference_weights(a, b, code.buckets))
    its = o["its"].cpu().numpy()
    bits = o["bits"].cpu().numpy()
    ran_all = np.flatnonzero(~o["conv"].cpu().numpy().astype(bool))
    assert len(ran_all) >= 1
    for i in ran_all:
        assert its[i] == T
        assert np.array_equal(bits[i], ref[i])


@pytest.mark.parametrize("kind", ["qce", "qc"])
def test_weighted_qc_with_zero_offset_is_plain(kind):
    import torch
    from atsc3_b200.ldpc import decode_flood, plan_for
    from atsc3_b200.learned import WmsCode, inference_weights
    rate, n = "8/15", 64800
    lam, cw = _case(seed=15, nb=4)
    code = WmsCode(rate, n)
    a, b = code.init_params(5, 0.75, 0.0)
    x = torch.from_numpy(lam).cuda()
    plan = plan_for(rate, n, kind=kind)
    p = decode_flood(plan, x, iters=50)
    w = decode_flood(plan, x, iters=50, weights=inference_weights(a, b, code.buckets))
    for k in ("bits", "conv", "its", "bad"):
        assert torch.equal(p[k], w[k]), k


def test_weighted_layouts_agree():
    """Learned weights with a nonzero offset: the edge-buffer and the
    record-layout decoders give identical outputs (same arithmetic)."""
    import torch
    from atsc3_b200.ldpc import decode_flood, plan_for
    from atsc3_b200.learned import WmsCode, inference_weights
    rate, n, T = "8/15", 64800, 12
    lam, cw = _case(seed=17, nb=5)
    code = WmsCode(rate, n)
    rng = np.random.default_rng(8)
    a = torch.tensor(0.7 + 0.25 * rng.random((T, code.nbucket)), dtype=torch.float32, device="cuda")
    b = torch.tensor(0.15 * rng.random((T, code.nbucket)), dtype=torch.float32, device="cuda")
    w = inference_weights(a, b, code.buckets)
    x = torch.from_numpy(lam).cuda()
    o1 = decode_flood(plan_for(rate, n, kind="qce"), x, iters=40, weights=w)
    o2 = decode_flood(plan_for(rate, n, kind="qc"), x, iters=40, weights=w)
    for k in ("bits", "conv", "its", "bad"):
        assert torch.equal(o1[k], o2[k]), k


@pytest.mark.parametrize("rate,n", [("2/15", 16200), ("3/15", 16200), ("7/15", 64800),
                                    ("8/15", 16200), ("6/15", 64800)])
def test_weighted_edge_buffer_vs_weighted_oracle(rate, n):
    """Random per-iteration, per-check-degree scale and offset on the
    edge-buffer decoder, against the numpy weighted oracle: Type A codes with
    and without heavy accumulator rows (the loop path's weights are indexed by
    degrees up to 86), a 16200 code with two circulants in some blocks, and
    the bench code."""
    import torch
    import oracle
    from atsc3_b200.ldpc import decode_flood, plan_for
    tabs = C.csr(rate, n)
    degs = np.unique(np.diff(tabs[0]))
    db = np.zeros(256, np.int8)
    db[degs] = np.arange(len(degs))
    T = 5
    rng = np.random.default_rng(n + C.RATES.index(rate))
    wa = (0.7 + 0.25 * rng.random((T, len(degs)))).astype(np.float32)
    wb = (0.15 * rng.random((T, len(degs)))).astype(np.float32)
    llr = (rng.standard_normal((3, n)) * 1.8 + np.array([[2.4], [1.8], [8.0]])).astype(np.float32)
    want = oracle.flood_weighted(llr, tabs, n, wa, wb, db.astype(np.int64), iters=16)
    plan = plan_for(rate, n, kind="qce")
    w = (torch.from_numpy(wa).cuda(), torch.from_numpy(wb).cuda(), torch.from_numpy(db).cuda())
    o = decode_flood(plan, torch.from_numpy(llr).cuda(), iters=16, weights=w)
    assert np.array_equal(o["bits"].cpu().numpy(), want[0])
    assert o["conv"].cpu().numpy().astype(bool).tolist() == want[1].tolist()
    assert o["its"].cpu().numpy().tolist() == want[2].tolist()
    assert o["bad"].cpu().numpy().tolist() == want[3].tolist()


def test_wms_backward_recomputes_instead_of_storing_messages():
    """Config 4's batch (256 blocks of 64800 8/15, T = 12): the peak device
    memory of forward + backward stays below what storing every
    iteration's per-edge messages alone would take (T x E x 4 bytes per
    block, 3.5 GB here) -- the forward keeps a 16-byte record per check and
    iteration, and the backward recomputes each iteration's messages from
    them."""
    import torch
    from atsc3_b200 import synth
    from atsc3_b200.learned import WeightedMinSum, WmsCode, bce_loss, make_batch
    rate, n, T, nblk = "8/15", 64800, 12, 256
    code = WmsCode(rate, n)
    tx = synth.Transmitter(n, "64QAM", rate, device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    lam, cw = make_batch(tx, g, nblk, 12.1, 14.1)
    a, b = code.init_params(T, 0.8, 0.05)
    a.requires_grad_(True)
    b.requires_grad_(True)
    bits = cw.float()
    torch.cuda.synchronize()
    base = torch.cuda.memory_allocated()
    torch.cuda.reset_peak_memory_stats()
    loss = bce_loss(WeightedMinSum.apply(lam, a, b, code, False), bits)
    loss.backward()
    torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated() - base
    stored = T * code.ne * 4 * nblk
    records = T * code.nc * 16 * nblk
    assert torch.isfinite(a.grad).all() and a.grad.abs().sum() > 0
    assert peak < stored, (peak, stored, records)


@pytest.mark.parametrize("rate,n", [("6/15", 64800), ("8/15", 64800),
                                    ("7/15", 64800), ("3/15", 16200)])
def test_row_weighted_edge_buffer_vs_weighted_oracle(rate, n):
    """Learned weights per (iteration, block row) on the edge-buffer decoder
    against the numpy weighted oracle with the same per-check buckets: Type B
    codes, Type A 64800 7/15 (its heavy accumulator rows take the split
    path) and a 16200-bit Type A code."""
    import torch
    import oracle
    from atsc3_b200 import learned as LR
    from atsc3_b200.ldpc import decode_flood, plan_for
    tabs = C.csr(rate, n)
    rows = LR.block_rows(rate, n)
    nr = int(rows.max()) + 1
    T = 5
    rng = np.random.default_rng(n + nr)
    wa = (0.7 + 0.25 * rng.random((T, nr))).astype(np.float32)
    wb = (0.15 * rng.random((T, nr))).astype(np.float32)
    llr = (rng.standard_normal((3, n)) * 1.8 + np.array([[2.4], [1.8], [8.0]])).astype(np.float32)
    want = oracle.flood_weighted(llr, tabs, n, wa, wb, np.zeros(256, np.int64),
                                 iters=16, cbucket=rows)
    w = LR.inference_weights(torch.from_numpy(wa), torch.from_numpy(wb),
                             np.arange(nr), mode="row")
    o = decode_flood(plan_for(rate, n, kind="qce"), torch.from_numpy(llr).cuda(),
                     iters=16, weights=w)
    assert np.array_equal(o["bits"].cpu().numpy(), want[0])
    assert o["conv"].cpu().numpy().astype(bool).tolist() == want[1].tolist()
    assert o["its"].cpu().numpy().tolist() == want[2].tolist()
    assert o["bad"].cpu().numpy().tolist() == want[3].tolist()


def test_row_weighted_training_step_gradients():
    """The training kernels with one bucket per block row (108 buckets for
    64800 6/15).  Exact: with every row carrying its degree's (scale,
    offset), the forward is the degree-bucket forward, so the row gradients
    summed over each degree class equal the degree-bucket gradients of the
    same launch (only the reduction buckets differ; row 0 holds the one
    degree-6 check, missing its wrap edge, and 359 degree-7 checks).  And
    against the float64 autograd reference on the same row buckets (1e-2 of
    the largest entry; measured 3.3e-3: with 720 checks per parameter a
    first/second-minimum choice that float32 and float64 make differently
    weighs more than with degree buckets)."""
    import torch
    import oracle
    from atsc3_b200 import learned as LR
    from atsc3_b200.learned import WeightedMinSum, WmsCode, bce_loss, reference_f64
    rate, n, T = "6/15", 64800, 4
    pay, cells, s2 = oracle.synth_case(
        lambda p: oracle.transmit(p, n, "16QAM", rate)[0], 2, C.kpayload(rate, n),
        C.cells_per_block(n, "16QAM"), 7.0, "awgn", 4)
    q = oracle.demap(cells, C.points_for("16QAM", rate), 4, s2)
    lam = oracle.deinterleave(q, C.bicm_map(n, "16QAM", rate), n)
    cw = oracle.transmit(pay, n, "16QAM", rate)[1]
    x = torch.from_numpy(lam).cuda()
    bits = torch.from_numpy(cw).cuda()
    rcode = WmsCode(rate, n, mode="row")
    dcode = WmsCode(rate, n)
    assert rcode.nbucket == 108 and list(dcode.buckets) == [6, 7, 8]
    rng = np.random.default_rng(6)
    ad = (0.7 + 0.2 * rng.random((T, 3))).astype(np.float32)
    bd = (0.1 * rng.random((T, 3))).astype(np.float32)
    # each row's degree class (all 360 checks of a row share it, but row 0's
    # check 0, which lacks the wrap edge)
    cptr = C.csr(rate, n)[0]
    deg = np.diff(cptr)
    rows = LR.block_rows(rate, n)
    rdeg = np.array([np.bincount(deg[rows == r]).argmax() for r in range(108)])
    cls = np.searchsorted(dcode.buckets, rdeg)
    assert deg[0] == 6 and rows[0] == 0 and rdeg[0] == 7
    ga = {}
    for mode, code, a0, b0 in (("row", rcode, ad[:, cls], bd[:, cls]),
                               ("degree", dcode, ad, bd)):
        # the degree-6 check has its own bucket; give it row 0's values
        if mode == "degree":
            a0 = a0.copy(); b0 = b0.copy()
            a0[:, 0] = a0[:, 1]; b0[:, 0] = b0[:, 1]
        a = torch.tensor(a0, device="cuda", requires_grad=True)
        b = torch.tensor(b0, device="cuda", requires_grad=True)
        bce_loss(WeightedMinSum.apply(x, a, b, code, False), bits).backward()
        ga[mode] = (a.grad.double().cpu().numpy(), b.grad.double().cpu().numpy())
    for k in range(2):
        gr, gd = ga["row"][k], ga["degree"][k]
        for c in (1, 2):                     # degree 7 (+ the degree-6 check), 8
            want = gd[:, c] + (gd[:, 0] if c == 1 else 0.0)
            got = gr[:, cls == c].sum(axis=1)
            assert np.allclose(got, want, rtol=1e-4, atol=1e-9), (k, c, got, want)
    # against the float64 reference with distinct per-row values
    a0 = (0.7 + 0.2 * rng.random((T, 108))).astype(np.float32)
    b0 = (0.1 * rng.random((T, 108))).astype(np.float32)
    a = torch.tensor(a0, device="cuda", requires_grad=True)
    b = torch.tensor(b0, device="cuda", requires_grad=True)
    bce_loss(WeightedMinSum.apply(x, a, b, rcode, False), bits).backward()
    a64 = torch.tensor(a0, dtype=torch.float64, requires_grad=True)
    b64 = torch.tensor(b0, dtype=torch.float64, requires_grad=True)
    bce_loss(reference_f64(torch.from_numpy(lam), a64, b64, rate, n, mode="row"),
             torch.from_numpy(cw).double()).backward()
    for g, gr in ((a.grad, a64.grad), (b.grad, b64.grad)):
        g = g.cpu().double().numpy()
        gr = gr.numpy()
        rel = np.abs(g - gr).max() / max(np.abs(gr).max(), 1e-12)
        assert rel < 1e-2, rel
