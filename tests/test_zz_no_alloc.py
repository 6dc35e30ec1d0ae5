"""atsc3_fec_decode_noalloc: the decode entry point for callers that cannot
allocate device memory (a real-time loop with a fixed memory budget, a host
that lends the GPU only pre-reserved buffers).  It keeps the LLR and
hard-decision intermediates in a fixed device scratch, so its results must
equal the regular three-call path (demap -> LDPC -> BCH with caller buffers)
exactly -- on two calls in a row, since every call reuses the same scratch.
This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from golden_util import oracle_case

pytestmark = pytest.mark.gpu


def _noalloc(torch, p, cells, s2):
    """Call the entry point through the C ABI with device inputs/outputs."""
    from atsc3_b200 import bch as BCH
    from atsc3_b200 import demap as DM
    from atsc3_b200 import native as N
    dev = torch.device("cuda")
    nblk, ncell = cells.shape
    c = torch.from_numpy(np.ascontiguousarray(cells, np.complex64)).to(dev)
    zf = torch.view_as_real(c)
    if np.ndim(s2) == 0:
        mode, s2t, s2s, ld_s = 0, None, float(s2), 0
    else:
        s2t = torch.from_numpy(np.ascontiguousarray(s2, np.float32)).to(dev)
        mode, s2s, ld_s = 1, 0.0, s2t.stride(0)
    out = {"payload": torch.empty((nblk, p.kpayload // 8), dtype=torch.uint8, device=dev),
           "conv": torch.empty(nblk, dtype=torch.uint8, device=dev),
           "its": torch.empty(nblk, dtype=torch.int32, device=dev),
           "bad": torch.empty(nblk, dtype=torch.int32, device=dev),
           "syn": torch.empty((nblk, 6), dtype=torch.int32, device=dev),
           "ok": torch.empty(nblk, dtype=torch.uint8, device=dev)}
    # the entry point takes CSR (0), record-layout quasi-cyclic (1) and
    # edge-buffer quasi-cyclic (2) plans
    kinds = {"csr": 0, "qc": 1, "qce": 2}
    plan_kind = getattr(p.plan, "kind", "csr")
    assert plan_kind in kinds, f"no-alloc entry point has no {plan_kind} plans"
    kind = kinds[plan_kind]
    N.call("atsc3_fec_decode_noalloc", p.plan.handle, kind, zf.data_ptr(),
           zf.stride(0) // 2, nblk, ncell,
           DM.device_points(p.mod, p.rate, dev).data_ptr(), p.nb, mode,
           N.ptr(s2t), ld_s, s2s,
           DM.device_lam_of_q(p.n, p.mod, p.rate, dev).data_ptr(), p.iters,
           ctypes.c_float(p.alpha),
           BCH.device_rtab(p.kldpc, p.n, dev).data_ptr(), p.kldpc,
           BCH.device_scrambler_bytes(p.kpayload, dev).data_ptr(), p.kpayload,
           out["payload"].data_ptr(), out["payload"].stride(0),
           out["conv"].data_ptr(), out["its"].data_ptr(), out["bad"].data_ptr(),
           out["syn"].data_ptr(), out["ok"].data_ptr(),
           torch.cuda.current_stream().cuda_stream)
    return {k: v.cpu().numpy() for k, v in out.items()}


def _kind(c):
    """Record-layout quasi-cyclic plan for Type B codes, else CSR."""
    from atsc3_b200 import codes as C
    return "qc" if C.ldpc_params(c["rate"], c["n"])[0] == "B" else "csr"


@pytest.mark.parametrize("kinds", ["qc_csr", "qce"])
def test_noalloc_matches_regular_path_twice(kinds):
    import torch
    from atsc3_b200.pipeline import FecPipeline
    # two different codes (Type B and Type A) in a row: the second call
    # reuses the scratch the first one left behind
    for name in ("c64_16qam_6_15_ray", "c64_64qam_7_15", "c64_16qam_6_15_ray"):
        c, pay, cw, cells, s2, q, lam = oracle_case(name)
        kind = _kind(c) if kinds == "qc_csr" else "qce"
        p = FecPipeline(c["n"], c["mod"], c["rate"], iters=50, alpha=0.75,
                        kind=kind)
        assert p.plan.kind == kind
        s2d = float(s2) if np.ndim(s2) == 0 else \
            torch.from_numpy(np.ascontiguousarray(s2, np.float32)).cuda()
        ws = p.decode(torch.from_numpy(cells).cuda(), s2d)
        want = {k: ws[k].cpu().numpy() for k in ("payload", "conv", "its",
                                                 "bad", "syn", "ok")}
        got = _noalloc(torch, p, cells, s2)
        for k in want:
            assert np.array_equal(got[k], want[k]), (name, k)
        assert got["its"].tolist() == c["its"]


def test_noalloc_rejects_oversize_batch():
    import torch
    from atsc3_b200 import native as N
    from atsc3_b200.pipeline import FecPipeline
    p = FecPipeline(64800, "16QAM", "6/15", kind="qc")
    cells = np.zeros((17, p.ncell), np.complex64)
    with pytest.raises(N.FecError) as e:
        _noalloc(torch, p, cells, 1.0)
    assert e.value.rc == -3 and "at most 16" in str(e.value)


def test_noalloc_rejects_float64_edge_buffer_plan():
    import torch
    from atsc3_b200 import ldpc as LDPC
    from atsc3_b200 import native as N
    from atsc3_b200.pipeline import FecPipeline
    p = FecPipeline(16200, "QPSK", "6/15", kind="qce")
    p.plan = LDPC.QcePlan("6/15", 16200, dtype="float64")
    cells = np.zeros((2, p.ncell), np.complex64)
    with pytest.raises(N.FecError) as e:
        _noalloc(torch, p, cells, 1.0)
    assert e.value.rc == -3 and "float64" in str(e.value)
