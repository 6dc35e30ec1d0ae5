"""Common phase error correction on the GPU (csrc/cpe.cu).

``cpe_correct`` keeps the signature and results of
``lab/m6_cells.py:176-209`` (the reference's decision-directed per-symbol
complex gain, also ``lab/m9_gpu.py:283-299`` ``GpuBicm.cpe``): numpy in,
numpy out, float64.  ``cpe_correct_device`` runs on device tensors.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import native as N


def _torch():
    import torch
    return torch


def cpe_correct_device(pool, sym_ptr, region, alphabets, dummy=None, iters=3,
                       out=None, stream=None):
    """pool (n,) complex128 CUDA tensor whose OFDM symbols are the contiguous
    ranges sym_ptr[s] .. sym_ptr[s+1] (int32 CUDA tensor); region (n,) uint8
    (0 / 1: alphabets[0] / [1], 2: dummy); alphabets: one or two complex128
    CUDA tensors; dummy (n,) complex128 or None.  Returns (out, gains)."""
    torch = _torch()
    if pool.dtype != torch.complex128 or pool.device.type != "cuda" or pool.dim() != 1:
        raise TypeError("pool must be a 1-D CUDA complex128 tensor")
    if not 1 <= len(alphabets) <= 2:
        raise ValueError("one or two alphabets")
    pool = pool.resolve_conj().contiguous()
    n = pool.numel()
    nsym = sym_ptr.numel() - 1
    dev = pool.device
    out = out if out is not None else torch.empty_like(pool)
    gains = torch.empty(max(nsym, 0), dtype=torch.complex128, device=dev)
    nbytes = ctypes.c_int64()
    N.call("atsc3_cpe_workspace", ctypes.byref(nbytes))
    work = torch.empty(nbytes.value // 8, dtype=torch.float64, device=dev)
    a0 = alphabets[0].contiguous()
    a1 = alphabets[1].contiguous() if len(alphabets) > 1 else None
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    N.call("atsc3_cpe_correct", torch.view_as_real(pool).data_ptr(), n,
           sym_ptr.data_ptr(), nsym, region.data_ptr(),
           torch.view_as_real(a0).data_ptr(), a0.numel(),
           torch.view_as_real(a1).data_ptr() if a1 is not None else None,
           a1.numel() if a1 is not None else 0,
           torch.view_as_real(dummy).data_ptr() if dummy is not None else None,
           int(iters), torch.view_as_real(out).data_ptr(),
           torch.view_as_real(gains).data_ptr(), work.data_ptr(), st)
    out._cpe_work = work
    return out, gains


def cpe_correct(pool, symbol_of, alphabets, region, dummy_values, iters=3):
    """Drop-in for ``lab/m6_cells.py:176`` ``cpe_correct``: returns (out
    complex128 numpy, {symbol: total complex gain}).  Cells are grouped by
    symbol on the host (stable order) and put back afterwards."""
    torch = _torch()
    pool = np.asarray(pool, np.complex128)
    symbol_of = np.asarray(symbol_of)
    region = np.asarray(region, np.uint8)
    order = np.argsort(symbol_of, kind="stable")
    srt = symbol_of[order]
    syms, starts = np.unique(srt, return_index=True)
    sym_ptr = np.concatenate([starts, [len(srt)]]).astype(np.int32)
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    dummy = (np.zeros(len(pool), np.complex128) if dummy_values is None
             else np.asarray(dummy_values, np.complex128))
    out_d, gains_d = cpe_correct_device(
        t(pool[order]), t(sym_ptr), t(region[order]),
        [t(np.asarray(a, np.complex128)) for a in alphabets[:2]],
        t(dummy[order]), iters=iters)
    out = np.empty(len(pool), np.complex128)
    out[order] = out_d.cpu().numpy()
    g = gains_d.cpu().numpy()
    return out, {int(s): complex(g[i]) for i, s in enumerate(syms)}
