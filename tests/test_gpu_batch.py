"""Uneven batches: one persistent launch over mixed codes, lengths and
constellations must give exactly the per-MODCOD results, eager or replayed
from its CUDA graph, before and after autotuning."""
import numpy as np
import pytest

from atsc3_b200 import codes as C

pytestmark = pytest.mark.gpu

MIX = [(64800, "256QAM", "10/15"), (64800, "QPSK", "2/15"),
       (16200, "64QAM", "11/15"), (64800, "1024QAM", "8/15"),
       (16200, "16QAM", "5/15"), (64800, "4096QAM", "12/15"),
       (64800, "64QAM", "7/15"), (16200, "QPSK", "13/15")]
ESN0 = {"QPSK": 2.0, "16QAM": 9.0, "64QAM": 14.0, "256QAM": 20.0,
        "1024QAM": 26.0, "4096QAM": 33.0}


def _blocks(torch, specs, seed=5):
    from atsc3_b200 import synth
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    cells, s2s = [], []
    for n, m, r in specs:
        tx = synth.Transmitter(n, m, r, device="cuda")
        pay = torch.randint(0, 2, (1, tx.kp), generator=g, device="cuda",
                            dtype=torch.uint8)
        x, _ = tx.encode(pay)
        y, s2 = synth.channel(x, ESN0[m] + (0.5 if r == "2/15" else 0.0), "awgn", g)
        cells.append(y[0])
        s2s.append(float(s2))
    return cells, s2s


@pytest.mark.parametrize("hybrid", [True, False])
def test_uneven_batch_equals_per_modcod_pipelines(hybrid):
    """hybrid: Type B blocks on per-code edge-buffer launches beside the CSR
    queue; False: every block on the CSR queue."""
    import torch
    from atsc3_b200.batch import UnevenBatch
    from atsc3_b200.pipeline import FecPipeline
    rng = np.random.default_rng(2)
    specs = [MIX[i] for i in rng.integers(0, len(MIX), 20)] + MIX
    cells, s2s = _blocks(torch, specs)
    ub = UnevenBatch(specs, iters=50, alpha=0.75, hybrid=hybrid)
    assert (len(ub.groups) > 0) == hybrid
    ub.load(cells, s2s)
    ub.launch()
    got = ub.results()
    for b, (n, m, r) in enumerate(specs):
        p = FecPipeline(n, m, r, iters=50, alpha=0.75)
        ws = p.decode(cells[b][None], s2s[b])
        assert np.array_equal(got[b]["payload"], ws["payload"][0].cpu().numpy()), b
        for k in ("conv", "its", "bad", "ok"):
            assert got[b][k] == int(ws[k][0]), (b, k)
    # graph replay: same results twice
    ub.capture()
    for _ in range(2):
        ub.run()
        again = ub.results()
        for b in range(len(specs)):
            assert np.array_equal(again[b]["payload"], got[b]["payload"])
            assert again[b]["its"] == got[b]["its"]
    # autotuner picks a valid configuration with identical results
    table = ub.autotune(reps=1)
    assert len(table) >= 2 and ub.config["cluster"] >= ub.cl_min
    ub.run()
    tuned = ub.results()
    for b in range(len(specs)):
        assert np.array_equal(tuned[b]["payload"], got[b]["payload"])
        assert tuned[b]["its"] == got[b]["its"]


def test_uneven_batch_all_quasi_cyclic():
    """A batch with no CSR block at all (every code Type B)."""
    import torch
    from atsc3_b200.batch import UnevenBatch
    from atsc3_b200.pipeline import FecPipeline
    specs = [(64800, "256QAM", "10/15"), (16200, "64QAM", "11/15"),
             (64800, "4096QAM", "12/15"), (64800, "256QAM", "10/15")]
    cells, s2s = _blocks(torch, specs, seed=9)
    ub = UnevenBatch(specs, iters=50, alpha=0.75)
    assert ub.ncsr == 0 and len(ub.groups) == 3
    ub.load(cells, s2s)
    ub.capture()
    ub.run()
    got = ub.results()
    for b, (n, m, r) in enumerate(specs):
        ws = FecPipeline(n, m, r, iters=50, alpha=0.75).decode(cells[b][None], s2s[b])
        assert np.array_equal(got[b]["payload"], ws["payload"][0].cpu().numpy()), b
        assert got[b]["its"] == int(ws["its"][0])
