"""The multi-rank path on the CPU: two gloo ranks each decode their block
range (the oracle stands in for the GPU decode here), gather the per-block
status and take the max of their timings; the result must equal one
process decoding the whole batch."""
import os
import socket

import numpy as np
import pytest

from atsc3_b200.shard import block_range

RATE, N, MOD = "11/15", 16200, "QPSK"


def test_block_range_partitions():
    for nblk in (0, 1, 5, 75, 76, 4800):
        for world in (1, 2, 3, 4, 8):
            seen = []
            for r in range(world):
                lo, hi = block_range(nblk, r, world)
                assert 0 <= lo <= hi <= nblk
                seen.extend(range(lo, hi))
            assert seen == list(range(nblk))
            sizes = [np.subtract(*block_range(nblk, r, world)[::-1])
                     for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        block_range(5, 2, 2)


def _case(nblk):
    import oracle
    from atsc3_b200 import codes as C
    cw = []

    def tx(pay):
        cells, c = oracle.transmit(pay, N, MOD, RATE)
        cw.append(c)
        return cells

    _, cells, s2 = oracle.synth_case(tx, nblk, C.kpayload(RATE, N),
                                     C.cells_per_block(N, MOD), 2.5, "awgn", 5)
    q = oracle.demap(cells, C.points_for(MOD, RATE), C.MOD_BITS[MOD], s2)
    return oracle.deinterleave(q, C.bicm_map(N, MOD, RATE), N)


def _decode_status(lam):
    import oracle
    from atsc3_b200 import codes as C
    K = C.kldpc(RATE, N)
    bits, conv, its, bad = oracle.flood(lam, C.csr(RATE, N), N, iters=20)
    syn = oracle.bch_syndrome_fast(bits[:, :K], N)
    ok = np.array([s == 0 for s in syn], np.int32)
    return np.stack([conv.astype(np.int32), its, bad, ok], axis=1)


def _rank(rank, world, port, nblk, q):
    import torch
    import torch.distributed as dist
    from atsc3_b200 import shard
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}",
                                rank=rank, world_size=world)
        lam = _case(nblk)
        lo, hi = shard.block_range(nblk, rank, world)
        st = torch.from_numpy(_decode_status(lam[lo:hi]))
        full = shard.gather_status(st, nblk)
        mx = shard.max_over_ranks(10.0 + rank)
        errs = shard.sum_over_ranks([int((st[:, 3] == 0).sum()), hi - lo])
        q.put((rank, full.numpy(), mx, errs))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:          # reported to the parent
        q.put((rank, repr(e), None, None))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("nblk", [5])
def test_two_gloo_ranks_match_single_process(nblk):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, nblk, q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, full, mx, errs = q.get(timeout=300)
        res[r] = (full, mx, errs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        assert not isinstance(res[r][0], str), res[r][0]
    want = _decode_status(_case(nblk))
    for r in range(2):
        full, mx, errs = res[r]
        assert np.array_equal(full, want)
        assert mx == 11.0
        assert errs == [float((want[:, 3] == 0).sum()), float(nblk)]
