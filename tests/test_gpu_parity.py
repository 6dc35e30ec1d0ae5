"""GPU parity: every CUDA path against the oracle / reference golden vectors.

Bar: hard decisions, iteration counts and BCH outcomes
bit-exact with float32 messages; demapper LLRs bit-exact with a supplied
sigma2 (within 1e-5 relative with the estimated sigma2).
"""
import ctypes

import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C
from golden_util import golden, oracle_case, sha

pytestmark = pytest.mark.gpu
CASES = sorted(golden()[0]["cases"])


def _torch():
    import torch
    return torch


@pytest.fixture(scope="module")
def torch():
    return _torch()


def dev_cells(cells):
    t = _torch()
    return t.from_numpy(np.ascontiguousarray(cells, np.complex64)).cuda()


def dev_sigma(s2):
    t = _torch()
    if np.ndim(s2) == 0:
        return float(s2)
    return t.from_numpy(np.ascontiguousarray(s2, np.float32)).cuda()


@pytest.mark.parametrize("name", CASES)
def test_demap_deinterleave_bit_exact(name, torch):
    from atsc3_b200 import demap as DM
    c, pay, cw, cells, s2, q, lam = oracle_case(name)
    got = DM.demap(dev_cells(cells), c["mod"], c["rate"], sigma2=dev_sigma(s2),
                   n=c["n"]).cpu().numpy()
    assert sha(got) == c["lam_sha"]
    gq = DM.demap(dev_cells(cells), c["mod"], c["rate"], sigma2=dev_sigma(s2),
                  deinterleave=False).cpu().numpy()
    assert sha(gq) == c["llr_q_sha"]


@pytest.mark.parametrize("name", CASES)
def test_demap_estimated_sigma_tolerance(name, torch):
    from atsc3_b200 import demap as DM
    c, pay, cw, cells, s2, q, lam = oracle_case(name)
    pts = C.points_for(c["mod"], c["rate"])
    ref = oracle.demap(cells, pts, C.MOD_BITS[c["mod"]], None)
    got = DM.demap(dev_cells(cells), c["mod"], c["rate"], sigma2=None,
                   deinterleave=False).cpu().numpy()
    # relative to the cell's LLR scale (|y|^2 + max|p|^2)/sigma2
    z2 = np.abs(cells) ** 2
    zz = (z2 + np.max(np.abs(pts)) ** 2)
    scale = np.repeat(zz, C.MOD_BITS[c["mod"]], axis=1)
    s2e = np.maximum(((z2.astype(np.float32)
                       + 0).mean(1)), 1e-9)[:, None]   # order of magnitude only
    tol = 1e-5 * np.maximum(np.abs(ref), scale / s2e)
    assert (np.abs(got - ref) <= tol).all()
    _, arrs = golden()
    head = arrs[f"llr_est_head/{name}"]
    assert np.allclose(got[:, :64], head, rtol=1e-5, atol=1e-5 * np.abs(head).max())


@pytest.mark.parametrize("name", CASES)
def test_flood_decode_bit_exact(name, torch):
    from atsc3_b200 import ldpc as LDPC
    c, pay, cw, cells, s2, q, lam = oracle_case(name)
    n = c["n"]
    plan = LDPC.plan_for(c["rate"], n)
    o = LDPC.decode_flood(plan, torch.from_numpy(lam).cuda(), iters=50,
                          alpha=0.75, semantics="kernel", want_hard=True)
    bits = o["bits"].cpu().numpy()
    assert sha(bits) == c["bits_sha"]
    assert o["conv"].cpu().numpy().astype(int).tolist() == c["conv"]
    assert o["its"].cpu().numpy().tolist() == c["its"]
    assert o["bad"].cpu().numpy().tolist() == c["bad"]
    hard = o["hard"].cpu().numpy()[:, :n // 8]
    assert np.array_equal(hard, np.packbits(bits, axis=1))


@pytest.mark.parametrize("name", CASES)
def test_pipeline_end_to_end(name, torch):
    from atsc3_b200.bch import syndromes_to_ints
    from atsc3_b200.pipeline import FecPipeline
    c, pay, cw, cells, s2, q, lam = oracle_case(name)
    p = FecPipeline(c["n"], c["mod"], c["rate"], iters=50, alpha=0.75)
    ws = p.decode(dev_cells(cells), dev_sigma(s2))
    assert sha(ws["payload"].cpu().numpy()) == c["payload_bytes_sha"]
    syn = syndromes_to_ints(ws["syn"].cpu().numpy())
    assert [hex(s) for s in syn] == c["bch"]
    assert ws["ok"].cpu().numpy().tolist() == [int(s == "0x0") for s in c["bch"]]
    assert ws["its"].cpu().numpy().tolist() == c["its"]
    r = p.decode_host(cells, s2)
    assert sha(r["payload"]) == c["payload_bytes_sha"]


@pytest.mark.parametrize("name", [k for k in CASES if k.startswith("c16")])
def test_gpuminsum_float64_torch_semantics(name, torch):
    from atsc3_b200.ldpc import GpuMinSum
    c, pay, cw, cells, s2, q, lam = oracle_case(name)
    g = GpuMinSum(C.parity_check(c["rate"], c["n"]), c["n"], iters=50,
                  alpha=0.75, dtype="float64")
    bits, conv, its, bad = g.decode(lam.astype(np.float64))
    assert sha(bits) == c["f64_bits_sha"]
    assert conv.astype(int).tolist() == c["f64_conv"]
    assert its.tolist() == c["f64_its"]
    assert bad.tolist() == c["f64_bad"]


def test_c_abi_ldpc_minsum_f32_matches_reference(torch):
    from atsc3_b200 import native as N
    L = N.lib()
    for name in ("c16_64qam_11_15", "c64_256qam_10_15", "c64_64qam_7_15"):
        c, pay, cw, cells, s2, q, lam = oracle_case(name)
        n = c["n"]
        cptr, cidx, vptr, vedge = [np.ascontiguousarray(t, np.int32)
                                   for t in C.csr(c["rate"], n)]
        nblk = lam.shape[0]
        bits = np.zeros((nblk, n), np.uint8)
        conv = np.zeros(nblk, np.uint8)
        its = np.zeros(nblk, np.int32)
        bad = np.zeros(nblk, np.int32)
        work = np.zeros(n + len(cidx), np.float32)
        rc = L.ldpc_minsum_f32(lam.ctypes.data, nblk, n, len(cptr) - 1,
                               len(cidx), cptr.ctypes.data, cidx.ctypes.data,
                               vptr.ctypes.data, vedge.ctypes.data, 50,
                               ctypes.c_float(0.75), bits.ctypes.data,
                               conv.ctypes.data, its.ctypes.data,
                               bad.ctypes.data, work.ctypes.data)
        assert rc == 0
        assert sha(bits) == c["bits_sha"]
        assert conv.tolist() == c["conv"] and its.tolist() == c["its"]
        assert bad.tolist() == c["bad"]


def test_c_abi_degree_limit_returns_minus_one(torch):
    from atsc3_b200 import native as N
    cptr = np.array([0, 129], np.int32)
    cidx = np.arange(129, dtype=np.int32)
    vptr = np.arange(130, dtype=np.int32)
    vedge = np.arange(129, dtype=np.int32)
    llr = np.ones((1, 129), np.float32)
    bits = np.full((1, 129), 7, np.uint8)
    conv = np.full(1, 7, np.uint8)
    its = np.full(1, 7, np.int32)
    bad = np.full(1, 7, np.int32)
    rc = N.lib().ldpc_minsum_f32(llr.ctypes.data, 1, 129, 1, 129,
                                 cptr.ctypes.data, cidx.ctypes.data,
                                 vptr.ctypes.data, vedge.ctypes.data, 5,
                                 ctypes.c_float(0.75), bits.ctypes.data,
                                 conv.ctypes.data, its.ctypes.data,
                                 bad.ctypes.data, None)
    assert rc == -1
    assert (bits == 7).all() and conv[0] == 7 and its[0] == 7 and bad[0] == 7


def test_known_answer_all_erasure(torch):
    """lab/build_ldpc_kernel.py:101-120: LLR=+5 retires at iteration 0."""
    from atsc3_b200 import ldpc as LDPC
    plan = LDPC.plan_for("3/15", 16200)
    o = LDPC.decode_flood(plan, torch.full((2, 16200), 5.0, device="cuda"))
    assert o["conv"].cpu().tolist() == [1, 1]
    assert o["its"].cpu().tolist() == [0, 0]
    assert o["bad"].cpu().tolist() == [0, 0]
    assert int(o["bits"].sum()) == 0


@pytest.mark.parametrize("n,kind", [(16200, "auto"), (64800, "auto"),
                                    (64800, "qc"), (64800, "csr")])
def test_all_codes_random_llr_vs_oracle(n, kind, torch):
    """Every A/322 rate (Type A and B), random LLRs near the waterfall,
    few iterations: the GPU decoder equals the oracle field by field.  kind
    "auto" runs the edge-buffer quasi-cyclic decoder on the Type B codes it
    accepts, "qc" the record-layout one, "csr" forces the CSR decoder on all
    of them (Type A codes always take the CSR decoder)."""
    from atsc3_b200 import ldpc as LDPC
    rng = np.random.default_rng(n)
    for rate in C.RATES:
        tabs = C.csr(rate, n)
        llr = (rng.standard_normal((3, n)) * 2.5 + 1.5).astype(np.float32)
        llr[2] = np.abs(llr[2])                    # one clean block: its == 0
        want = oracle.flood(llr, tabs, n, iters=6, alpha=0.8)
        plan = LDPC.plan_for(rate, n, kind=kind)
        o = LDPC.decode_flood(plan, torch.from_numpy(llr).cuda(), iters=6,
                              alpha=0.8)
        assert np.array_equal(o["bits"].cpu().numpy(), want[0]), rate
        assert o["conv"].cpu().numpy().astype(bool).tolist() == want[1].tolist()
        assert o["its"].cpu().numpy().tolist() == want[2].tolist(), rate
        assert o["bad"].cpu().numpy().tolist() == want[3].tolist(), rate


@pytest.mark.parametrize("cluster", [1, 2, 4, 8, 16])
def test_cluster_sizes_agree(cluster, torch):
    from atsc3_b200 import native as N
    from atsc3_b200.ldpc import Plan, decode_flood
    rng = np.random.default_rng(cluster)
    rate, n = ("10/15", 16200) if cluster <= 2 else ("10/15", 64800)
    tabs = C.csr(rate, n)
    try:
        plan = Plan(*tabs, n, cluster=cluster)
    except N.FecError as e:
        assert e.rc == -4                       # state does not fit
        pytest.skip(str(e))
    llr = (rng.standard_normal((5, n)) * 2.0 + 1.4).astype(np.float32)
    want = oracle.flood(llr, tabs, n, iters=7, alpha=0.75)
    o = decode_flood(plan, torch.from_numpy(llr).cuda(), iters=7, alpha=0.75)
    assert np.array_equal(o["bits"].cpu().numpy(), want[0])
    assert o["its"].cpu().numpy().tolist() == want[2].tolist()
    assert o["bad"].cpu().numpy().tolist() == want[3].tolist()


def test_float32_torch_semantics_vs_oracle(torch):
    from atsc3_b200.ldpc import GpuMinSum
    rng = np.random.default_rng(21)
    rate, n = "8/15", 16200
    llr = (rng.standard_normal((4, n)) * 2.0 + 1.3).astype(np.float32)
    want = oracle.flood(llr, C.csr(rate, n), n, iters=9, alpha=0.7,
                        semantics=1)
    g = GpuMinSum(C.parity_check(rate, n), n, iters=9, alpha=0.7,
                  dtype="float32")
    bits, conv, its, bad = g.decode(torch.from_numpy(llr).cuda())
    assert np.array_equal(bits, want[0])
    assert its.tolist() == want[2].tolist() and bad.tolist() == want[3].tolist()


def test_edge_cases(torch):
    from atsc3_b200 import ldpc as LDPC
    from atsc3_b200 import native as N
    plan = LDPC.plan_for("11/15", 16200)
    # empty batch
    o = LDPC.decode_flood(plan, torch.empty((0, 16200), device="cuda"))
    assert o["conv"].numel() == 0
    # ragged row stride: a view into a wider buffer
    rng = np.random.default_rng(2)
    wide = (rng.standard_normal((3, 16200 + 40)) * 2 + 1.5).astype(np.float32)
    t = torch.from_numpy(wide).cuda()[:, 8:8 + 16200]
    o = LDPC.decode_flood(plan, t, iters=5)
    want = oracle.flood(wide[:, 8:8 + 16200], C.csr("11/15", 16200), 16200,
                        iters=5)
    assert np.array_equal(o["bits"].cpu().numpy(), want[0])
    # iters = 0: syndrome only
    o = LDPC.decode_flood(plan, t, iters=0)
    want = oracle.flood(wide[:, 8:8 + 16200], C.csr("11/15", 16200), 16200,
                        iters=0)
    assert o["its"].cpu().tolist() == want[2].tolist()
    assert o["bad"].cpu().tolist() == want[3].tolist()
    # wrong dtype / shape raise before any launch
    with pytest.raises(TypeError):
        LDPC.decode_flood(plan, t.double())
    with pytest.raises(ValueError):
        LDPC.decode_flood(plan, torch.zeros((2, 100), device="cuda"))
    with pytest.raises(N.FecError):
        LDPC.decode_flood(plan, t, semantics="torch", iters=0)


def test_repeat_launch_determinism(torch):
    from atsc3_b200 import ldpc as LDPC
    c, pay, cw, cells, s2, q, lam = oracle_case("c64_16qam_6_15_ray")
    plan = LDPC.plan_for("6/15", 64800)
    x = torch.from_numpy(lam).cuda()
    ref = LDPC.decode_flood(plan, x, iters=50)
    for _ in range(3):
        o = LDPC.decode_flood(plan, x, iters=50)
        for k in ("bits", "conv", "its", "bad"):
            assert torch.equal(o[k], ref[k])


def test_bch_dropins_match_golden(torch):
    from atsc3_b200.bch import bch_syndrome, bch_syndrome_batch
    meta, arrs = golden()
    for key, want in meta["bch"].items():
        n, k = map(int, key.split(":"))
        m = np.unpackbits(arrs[f"bch_msg/{key}"], axis=1)[:, :k]
        assert [hex(s) for s in bch_syndrome_batch(m, n)] == want
        assert hex(bch_syndrome(m[0], n)) == want[0]


def _exhaustive_f64(cells, pts, nb, s2):
    """float64 max-log LLRs, |z - p|^2 exhaustively (the lab/m6_bicm.py:
    213-225 form the reference's demap_llr_fast gate compares against)."""
    d2 = np.abs(np.asarray(cells, np.complex128)[:, None] - pts[None, :]) ** 2
    if s2 is None:
        s2 = max(float(d2.min(1).mean()), 1e-9)
    m = d2.reshape(len(cells), *([2] * nb))
    out = np.empty((len(cells), nb))
    for i in range(nb):
        ax = tuple(a for a in range(1, nb + 1) if a != i + 1)
        mn = m.min(axis=ax)
        out[:, i] = (mn[:, 1] - mn[:, 0]) / (s2 if np.ndim(s2) == 0
                                              else np.asarray(s2, np.float64))
    return out.ravel()


def test_demap_llr_fast_dropin(torch):
    from atsc3_b200 import codes as C
    from atsc3_b200.demap import demap_llr_fast
    c, pay, cw, cells, s2, q, lam = oracle_case("c64_16qam_6_15_ray")
    # dtype=float32: bit-exact with the float32 reference arithmetic
    got = demap_llr_fast(cells[0], c["mod"], c["rate"], sigma2=s2[0],
                         dtype=np.float32)
    assert got.dtype == np.float64
    assert np.array_equal(got.astype(np.float32), q[0])
    c2, _, _, cells2, s22, q2, _ = oracle_case("c64_256qam_10_15")
    got = demap_llr_fast(cells2[1], c2["mod"], c2["rate"], sigma2=float(s22),
                         dtype=np.float32)
    assert np.array_equal(got.astype(np.float32), q2[1])
    # dtype=float64 (the reference's default): within the reference gate's
    # 1e-12 of the largest LLR (lab/m16_demap_fast.py:134-140) of the
    # exhaustive float64 demapper, supplied per-cell, scalar and estimated
    # sigma2
    for cc, s, mod, rate in ((cells[0], s2[0], c["mod"], c["rate"]),
                             (cells2[1], float(s22), c2["mod"], c2["rate"]),
                             (cells2[0], None, c2["mod"], c2["rate"])):
        pts = C.points_for(mod, rate)
        want = _exhaustive_f64(cc, pts, C.MOD_BITS[mod], s)
        got = demap_llr_fast(cc, mod, rate, sigma2=s)
        assert got.dtype == np.float64 and got.shape == want.shape
        rel = np.abs(got - want).max() / np.abs(want).max()
        assert rel < 1e-12, rel


@pytest.mark.parametrize("kind,cluster,threads", [
    ("qc", 4, 0), ("qc", 8, 0), ("qc", 16, 0),
    ("qce", 8, 0), ("qce", 16, 0), ("qce", 8, 512)])
@pytest.mark.parametrize("rate", ["6/15", "8/15", "9/15", "10/15", "11/15",
                                  "12/15", "13/15"])
def test_qc_decoder_vs_oracle(rate, kind, cluster, threads, torch):
    """Both quasi-cyclic decoders (record layout "qc", edge-buffer layout
    "qce"), every 64800 Type B rate, several cluster sizes and CTA sizes,
    both semantics, against the oracle (30 iterations, mixed convergence)."""
    from atsc3_b200 import native as N
    from atsc3_b200.ldpc import QcePlan, QcPlan, decode_flood
    n = 64800
    try:
        plan = (QcPlan if kind == "qc" else QcePlan)(rate, n, cluster=cluster)
    except N.FecError as e:
        assert e.rc == -4
        pytest.skip(str(e))
    rng = np.random.default_rng(cluster * 100 + len(rate))
    tabs = C.csr(rate, n)
    llr = (rng.standard_normal((6, n)) * 2.2 + 1.6).astype(np.float32)
    x = torch.from_numpy(llr).cuda()
    for sem, code in (("kernel", 0), ("torch", 1)):
        want = oracle.flood(llr, tabs, n, iters=30, alpha=0.75, semantics=code)
        o = decode_flood(plan, x, iters=30, alpha=0.75, semantics=sem,
                         want_hard=True, threads=threads)
        bits = o["bits"].cpu().numpy()
        assert np.array_equal(bits, want[0]), (rate, sem)
        assert o["conv"].cpu().numpy().astype(bool).tolist() == want[1].tolist()
        assert o["its"].cpu().numpy().tolist() == want[2].tolist(), (rate, sem)
        assert o["bad"].cpu().numpy().tolist() == want[3].tolist(), (rate, sem)
        assert np.array_equal(o["hard"].cpu().numpy()[:, :n // 8],
                              np.packbits(bits, axis=1))


@pytest.mark.parametrize("kind", ["qce", "qc", "csr"])
def test_many_codewords_per_cluster_outputs_consistent(kind, torch):
    """More codewords than resident clusters: every cluster decodes several
    codewords in turn; packed hard decisions, bits and status of every block
    must match the oracle (a retire/prologue overlap would corrupt them)."""
    from atsc3_b200 import ldpc as LDPC
    rate, n = "10/15", 64800
    rng = np.random.default_rng(31)
    nb = 100
    llr = (rng.standard_normal((nb, n)) * 1.5 + 2.5).astype(np.float32)
    plan = LDPC.plan_for(rate, n, kind=kind)
    o = LDPC.decode_flood(plan, torch.from_numpy(llr).cuda(), iters=8,
                          want_hard=True)
    bits = o["bits"].cpu().numpy()
    assert np.array_equal(o["hard"].cpu().numpy()[:, :n // 8],
                          np.packbits(bits, axis=1))
    sel = [0, 33, 66, 99]
    want = oracle.flood(llr[sel], C.csr(rate, n), n, iters=8)
    assert np.array_equal(bits[sel], want[0])
    assert o["its"].cpu().numpy()[sel].tolist() == want[2].tolist()


@pytest.mark.parametrize("rate", ["6/15", "7/15", "8/15", "9/15", "10/15", "11/15",
                                  "12/15", "13/15"])
@pytest.mark.parametrize("cluster", [2, 4])
def test_qce_16200_codes_vs_oracle(rate, cluster, torch):
    """Edge-buffer decoder on every 16200-bit Type B code (6/15, 8/15, 10/15,
    12/15 and 13/15 put two circulants in some blocks), both semantics,
    packed and unpacked outputs, against the oracle."""
    from atsc3_b200.ldpc import QcePlan, decode_flood
    n = 16200
    plan = QcePlan(rate, n, cluster=cluster)
    rng = np.random.default_rng(cluster + 7 * len(rate))
    tabs = C.csr(rate, n)
    llr = (rng.standard_normal((9, n)) * 2.0 + 1.5).astype(np.float32)
    llr[4] = np.abs(llr[4])                          # clean block: its == 0
    x = torch.from_numpy(llr).cuda()
    for sem, code in (("kernel", 0), ("torch", 1)):
        want = oracle.flood(llr, tabs, n, iters=25, alpha=0.75, semantics=code)
        o = decode_flood(plan, x, iters=25, alpha=0.75, semantics=sem,
                         want_hard=True)
        bits = o["bits"].cpu().numpy()
        assert np.array_equal(bits, want[0]), (rate, sem)
        assert o["its"].cpu().numpy().tolist() == want[2].tolist(), (rate, sem)
        assert o["bad"].cpu().numpy().tolist() == want[3].tolist(), (rate, sem)
        assert o["conv"].cpu().numpy().astype(bool).tolist() == want[1].tolist()
        assert np.array_equal(o["hard"].cpu().numpy()[:, :n // 8],
                              np.packbits(bits, axis=1))


TYPE_A = [(r, n) for n in (16200, 64800) for r in C.RATES
          if C.ldpc_params(r, n)[0] == "A"]


@pytest.mark.parametrize("rate,n", TYPE_A)
@pytest.mark.parametrize("bigger", [0, 1])
def test_qce_type_a_codes_vs_oracle(rate, n, bigger, torch):
    """Edge-buffer decoder on every Type A code: accumulator rows of high
    degree take the kernel's loop path, identity rows the register path;
    both semantics, packed and unpacked outputs, at the smallest cluster that
    holds a codeword and one CTA more, against the oracle."""
    from atsc3_b200.ldpc import QcePlan, decode_flood
    plan = QcePlan(rate, n)
    if bigger:
        plan = QcePlan(rate, n, cluster=plan.cluster + 1)
    rng = np.random.default_rng(n + C.RATES.index(rate) + 100 * bigger)
    tabs = C.csr(rate, n)
    llr = (rng.standard_normal((5, n)) * 2.0 + 1.2).astype(np.float32)
    llr[2] = np.abs(llr[2])                          # clean block: its == 0
    x = torch.from_numpy(llr).cuda()
    for sem, code in (("kernel", 0), ("torch", 1)):
        want = oracle.flood(llr, tabs, n, iters=20, alpha=0.75, semantics=code)
        o = decode_flood(plan, x, iters=20, alpha=0.75, semantics=sem,
                         want_hard=True)
        bits = o["bits"].cpu().numpy()
        assert np.array_equal(bits, want[0]), (rate, n, sem)
        assert o["its"].cpu().numpy().tolist() == want[2].tolist(), (rate, n, sem)
        assert o["bad"].cpu().numpy().tolist() == want[3].tolist(), (rate, n, sem)
        assert o["conv"].cpu().numpy().astype(bool).tolist() == want[1].tolist()
        assert np.array_equal(o["hard"].cpu().numpy()[:, :n // 8],
                              np.packbits(bits, axis=1))


def test_qce_iters_zero_and_empty_batch(torch):
    """iters=0 only evaluates the syndrome of the channel LLRs (its 0); an
    empty batch launches nothing."""
    from atsc3_b200.ldpc import QcePlan, decode_flood
    rate, n = "10/15", 64800
    plan = QcePlan(rate, n)
    rng = np.random.default_rng(5)
    llr = (rng.standard_normal((3, n)) * 2.0 + 1.0).astype(np.float32)
    llr[1] = np.abs(llr[1])
    want = oracle.flood(llr, C.csr(rate, n), n, iters=0, alpha=0.75)
    o = decode_flood(plan, torch.from_numpy(llr).cuda(), iters=0)
    assert np.array_equal(o["bits"].cpu().numpy(), want[0])
    assert o["its"].cpu().numpy().tolist() == [0, 0, 0]
    assert o["bad"].cpu().numpy().tolist() == want[3].tolist()
    e = decode_flood(plan, torch.zeros((0, n), dtype=torch.float32, device="cuda"))
    assert e["its"].numel() == 0


@pytest.mark.parametrize("rate,n", [("10/15", 64800), ("7/15", 64800), ("11/15", 16200),
                                    ("8/15", 16200), ("3/15", 16200)])
def test_qce_float64_vs_oracle(rate, n, torch):
    """The float64 edge-buffer decoder (8-byte slots, float64 arithmetic)
    against the float64 C oracle, both semantics: Type B, Type A (with heavy
    accumulator rows) and a 16200 code with two circulants in some blocks."""
    from atsc3_b200.ldpc import QcePlan, decode_flood
    plan = QcePlan(rate, n, dtype="float64")
    rng = np.random.default_rng(n + C.RATES.index(rate))
    tabs = C.csr(rate, n)
    llr = rng.standard_normal((4, n)) * 2.0 + 1.4
    llr[3] = np.abs(llr[3])
    x = torch.from_numpy(llr).cuda()
    for sem, code in (("kernel", 0), ("torch", 1)):
        want = oracle.flood(llr, tabs, n, iters=18, alpha=0.8, semantics=code,
                            dtype=np.float64)
        o = decode_flood(plan, x, iters=18, alpha=0.8, semantics=sem, want_hard=True)
        bits = o["bits"].cpu().numpy()
        assert np.array_equal(bits, want[0]), (rate, n, sem)
        assert o["its"].cpu().numpy().tolist() == want[2].tolist(), (rate, n, sem)
        assert o["bad"].cpu().numpy().tolist() == want[3].tolist(), (rate, n, sem)
        assert o["conv"].cpu().numpy().astype(bool).tolist() == want[1].tolist()
        assert np.array_equal(o["hard"].cpu().numpy()[:, :n // 8],
                              np.packbits(bits, axis=1))


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_gpuminsum_routes_a322_codes_to_the_edge_buffer_decoder(dtype, torch):
    """GpuMinSum is built from check lists; an A/322 code is recognised and
    decoded by the edge-buffer plan, with the CSR decoder's outputs."""
    from atsc3_b200.ldpc import GpuMinSum, Plan, decode_flood
    rate, n = "9/15", 16200
    g = GpuMinSum(C.parity_check(rate, n), n, dtype=dtype)
    assert g.plan.kind == "qce" and g.plan.dtype == dtype
    rng = np.random.default_rng(4)
    llr = (rng.standard_normal((5, n)) * 2.0 + 1.8).astype(dtype)
    got = g.decode(llr)
    csr = Plan(*C.csr(rate, n), n, dtype=dtype)
    want = decode_flood(csr, torch.from_numpy(llr).cuda(), iters=50, alpha=0.75,
                        semantics="torch")
    assert np.array_equal(got[0], want["bits"].cpu().numpy())
    assert got[2].tolist() == want["its"].cpu().numpy().tolist()
    assert got[3].tolist() == want["bad"].cpu().numpy().tolist()


@pytest.mark.parametrize("n", [16200, 64800])
def test_all_codes_float64_edge_buffer_equals_csr(n, torch):
    """Every A/322 code in float64 (torch semantics, GpuMinSum's default):
    the edge-buffer decoder equals the float64 CSR decoder field by field."""
    from atsc3_b200.ldpc import Plan, QcePlan, decode_flood
    rng = np.random.default_rng(n + 64)
    for rate in C.RATES:
        llr = rng.standard_normal((3, n)) * 2.2 + 1.4
        llr[2] = np.abs(llr[2])
        x = torch.from_numpy(llr).cuda()
        a = decode_flood(QcePlan(rate, n, dtype="float64"), x, iters=10, alpha=0.75,
                         semantics="torch")
        b = decode_flood(Plan(*C.csr(rate, n), n, dtype="float64"), x, iters=10,
                         alpha=0.75, semantics="torch")
        for k in ("bits", "conv", "its", "bad"):
            assert torch.equal(a[k], b[k]), (rate, n, k)
