"""Empty batches through every drop-in entry point: nothing to decode gives
empty results of the reference's shapes and types and no error, as the
reference's loops over zero blocks do (lab/ldpc_kernel.c:65-146 returns 0 for
nblk = 0; the numpy paths return empty arrays)."""
import ctypes

import numpy as np
import pytest

from atsc3_b200 import codes as C
from atsc3_b200 import native as N

pytestmark = pytest.mark.gpu

RATE, N_ = "6/15", 16200


def test_ldpc_minsum_f32_zero_blocks():
    cptr, cidx, vptr, vedge = [np.ascontiguousarray(t, np.int32) for t in C.csr(RATE, N_)]
    llr = np.zeros((0, N_), np.float32)
    bits = np.zeros((0, N_), np.uint8)
    conv = np.zeros(0, np.uint8)
    its = np.zeros(0, np.int32)
    bad = np.zeros(0, np.int32)
    rc = N.lib().ldpc_minsum_f32(llr.ctypes.data, 0, N_, len(cptr) - 1, len(cidx),
                                 cptr.ctypes.data, cidx.ctypes.data, vptr.ctypes.data,
                                 vedge.ctypes.data, 50, ctypes.c_float(0.75),
                                 bits.ctypes.data, conv.ctypes.data, its.ctypes.data,
                                 bad.ctypes.data, None)
    assert rc == 0


@pytest.mark.parametrize("dtype", ["float32", "float64", "bfloat16"])
def test_gpuminsum_zero_rows(dtype):
    from atsc3_b200 import ldpc
    cptr, cidx, vptr, vedge = C.csr(RATE, N_)
    checks = [cidx[cptr[c]:cptr[c + 1]].tolist() for c in range(len(cptr) - 1)]
    bits, conv, its, bad = ldpc.GpuMinSum(checks, N_, dtype=dtype).decode(
        np.zeros((0, N_)))
    assert bits.shape == (0, N_) and bits.dtype == np.uint8
    assert conv.shape == its.shape == bad.shape == (0,)
    assert conv.dtype == bool and its.dtype == np.int32 and bad.dtype == np.int32


def test_demap_and_bch_zero_cells():
    from atsc3_b200 import bch, demap
    for s2 in (0.1, None):
        for dt in (np.float64, np.float32):
            q = demap.demap_llr_fast(np.zeros(0, np.complex128), "16QAM", RATE, sigma2=s2,
                                     dtype=dt)
            assert q.shape == (0,) and q.dtype == np.float64
    assert bch.bch_syndrome_batch(np.zeros((0, C.ldpc_params(RATE, N_)[1]), np.uint8),
                                  N_) == []


def test_sum_product_zero_rows():
    from atsc3_b200 import ldpc
    cptr, cidx, vptr, vedge = C.csr(RATE, N_)
    checks = [cidx[cptr[c]:cptr[c + 1]].tolist() for c in range(len(cptr) - 1)]
    stats = {}
    bits, conv, its, bad = ldpc.sum_product_decode_batch(np.zeros((0, N_)), checks, N_,
                                                         iters=10, stats=stats)
    assert bits.shape == (0, N_) and conv.shape == its.shape == bad.shape == (0,)
    assert stats.get("sp_timeout", 0) == 0


@pytest.mark.parametrize("sigma2", [0.1, None])
def test_pipeline_zero_blocks(sigma2):
    import torch
    from atsc3_b200.pipeline import FecPipeline
    p = FecPipeline(N_, "16QAM", RATE, device=torch.device("cuda"))
    cells = torch.zeros((0, C.cells_per_block(N_, "16QAM")), dtype=torch.complex64,
                        device="cuda")
    ws = p.decode(cells, sigma2)
    torch.cuda.synchronize()
    for k in ("conv", "its", "bad", "ok"):
        assert ws[k].shape[0] == 0, k
