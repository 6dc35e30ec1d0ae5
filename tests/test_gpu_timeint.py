"""Time de-interleave fused into the demapper (csrc/timeint.cu) against the
oracle: the received stream is de-interleaved on the CPU by the oracle's
restatement of lab/m6_tbi.py / lab/m10_cti.py, demapped by the oracle, and
must equal the GPU's LLRs bit for bit; erasures (cells the convolutional
interleaver had not delivered) give LLR 0.  End to end, decoding a PLP
stream through the pipeline equals decoding its de-interleaved FEC
Blocks."""
import numpy as np
import pytest

import oracle
from atsc3_b200 import codes as C

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


def _blocks(torch, n, mod, rate, nblk, esn0, seed, channel="awgn"):
    from atsc3_b200 import synth
    tx = synth.Transmitter(n, mod, rate, device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    pay = torch.randint(0, 2, (nblk, tx.kp), generator=g, device="cuda",
                        dtype=torch.uint8)
    x, _ = tx.encode(pay)
    y, s2 = synth.channel(x, esn0, channel, g)
    return y, s2


def _oracle_llr(cells2d, n, mod, rate, s2):
    q = oracle.demap(cells2d, C.points_for(mod, rate), C.MOD_BITS[mod], s2)
    return oracle.deinterleave(q, C.bicm_map(n, mod, rate), n)


@pytest.mark.parametrize("n,mod,rate,nrows_blocks,nti,nv", [
    (16200, "64QAM", "11/15", 5, 2, 0),
    (64800, "16QAM", "6/15", 4, 1, 0),
    (16200, "QPSK", "7/15", 6, 2, 2),
])
def test_hybrid_ti_demap_bit_exact(torch, n, mod, rate, nrows_blocks, nti, nv):
    from atsc3_b200 import timeint as T
    ncell = C.cells_per_block(n, mod)
    ti = T.HybridTI(ncell, nrows_blocks, nti=nti, n_virtual=nv, offset=3)
    y, s2 = _blocks(torch, n, mod, rate, ti.nblk, 9.0, 5)
    stream = ti.interleave(y)
    host = stream.cpu().numpy()
    # oracle: de-interleave each TI block with the reference's map
    rows = []
    for t in range(nti):
        seg = host[3 + t * ti.per_ti: 3 + (t + 1) * ti.per_ti]
        mem = oracle.tbi_deinterleave(seg, ncell, nrows_blocks, nv)
        rows.append(mem.reshape(nrows_blocks - nv, ncell))
    cells = np.concatenate(rows)
    want = _oracle_llr(cells, n, mod, rate, float(s2))
    for table in (False, True):
        got = T.demap_deinterleave(stream, ti, mod, rate, n, sigma2=float(s2),
                                   table=table)
        assert np.array_equal(got.cpu().numpy(), want), table


def test_convolutional_ti_demap_with_erasures(torch):
    from atsc3_b200 import timeint as T
    n, mod, rate = 16200, "16QAM", "9/15"
    ncell = C.cells_per_block(n, mod)
    nblk, nrows, start, c0 = 3, 64, 17, 5
    y, s2 = _blocks(torch, n, mod, rate, nblk, 11.0, 8, channel="rayleigh")
    pre = torch.zeros(c0 + nblk * ncell, dtype=torch.complex64, device="cuda")
    pre[c0:] = y.reshape(-1)
    sig_pre = torch.ones(c0 + nblk * ncell, dtype=torch.float32, device="cuda")
    sig_pre[c0:] = s2.reshape(-1)
    L = c0 + nblk * ncell - 40 * nrows          # the tail is not delivered yet
    ti = T.ConvolutionalTI(nrows, start, C=c0, nblk=nblk, ncell=ncell)
    stream = ti.interleave(pre, L)
    sig_stream = ti.interleave(sig_pre, L)
    got = T.demap_deinterleave(stream, ti, mod, rate, n, sigma2=sig_stream)
    # oracle: de-interleave the stream, demap the delivered cells, erase
    # the others
    out, valid = oracle.cti_deinterleave(stream.cpu().numpy(), nrows, start,
                                         c0 + nblk * ncell)
    sig, _ = oracle.cti_deinterleave(sig_stream.cpu().numpy(), nrows, start,
                                     c0 + nblk * ncell)
    cells = out[c0:].reshape(nblk, ncell)
    s2c = np.where(valid[c0:], sig[c0:], 1.0).reshape(nblk, ncell)
    q = oracle.demap(cells, C.points_for(mod, rate), C.MOD_BITS[mod], s2c)
    nb = C.MOD_BITS[mod]
    q = q.reshape(nblk, ncell, nb)
    q[~valid[c0:].reshape(nblk, ncell)] = 0.0
    want = oracle.deinterleave(q.reshape(nblk, -1), C.bicm_map(n, mod, rate), n)
    assert (~valid[c0:]).sum() > 0
    assert np.array_equal(got.cpu().numpy(), want)
    tab = T.demap_deinterleave(stream, ti, mod, rate, n, sigma2=sig_stream,
                               table=True)
    assert np.array_equal(tab.cpu().numpy(), want)


def test_pipeline_stream_equals_block_decode(torch):
    from atsc3_b200 import timeint as T
    from atsc3_b200.pipeline import FecPipeline
    n, mod, rate = 64800, "16QAM", "6/15"
    ncell = C.cells_per_block(n, mod)
    ti = T.HybridTI(ncell, 3, nti=2)
    y, s2 = _blocks(torch, n, mod, rate, ti.nblk, 8.5, 21, channel="rayleigh")
    stream = ti.interleave(y)
    s2_stream = ti.interleave(s2)
    p = FecPipeline(n, mod, rate)
    a = {k: v.clone() for k, v in p.decode(y, s2).items()}
    b = p.decode_stream(stream, ti, s2_stream)
    for k in ("payload", "conv", "its", "bad", "ok", "lam"):
        assert torch.equal(a[k], b[k]), k
