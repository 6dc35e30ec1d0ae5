"""Soft demapper on the GPU (+ the fused bit de-interleaver).

``demap`` is the batched device entry point; ``demap_llr_fast`` keeps the
signature of ``lab/m16_demap_fast.py:80-119`` (and of
``lab/m6_bicm.py:213`` ``demap_llr``) so the reference's callers can use it.

Arithmetic: float32, the operation order of ``lab/m44_ldm.py:2431-2451``
(``_point_metric``) and the per-bit minima of ``:2483-2486``.  With a
supplied sigma2 the LLRs are bit-identical to that float32 reference; the
estimated-sigma2 path accumulates the mean in float64 (within 1e-5 relative
of the reference, not bit-identical: numpy's float32 pairwise mean has no
GPU-side restatement).
"""
from __future__ import annotations

import functools

import numpy as np

from . import codes as C
from . import native as N


def _torch():
    import torch
    return torch


@functools.lru_cache(maxsize=None)
def _host_points(mod, rate):
    pr, pi, p2 = C.point_tables_f32(C.alphabet(mod, rate))
    return np.concatenate([pr, pi, p2]).astype(np.float32)


_DEV = {}


def device_points(mod, rate, device):
    torch = _torch()
    key = ("pts", mod, rate, str(device))
    t = _DEV.get(key)
    if t is None:
        t = torch.from_numpy(_host_points(mod, rate)).to(device)
        _DEV[key] = t
    return t


def device_lam_of_q(n, mod, rate, device):
    torch = _torch()
    key = ("lq", n, mod, rate, str(device))
    t = _DEV.get(key)
    if t is None:
        t = torch.from_numpy(np.array(C.bicm_map(n, mod, rate), np.int32)).to(device)
        _DEV[key] = t
    return t


def _as_float_pairs(cells):
    torch = _torch()
    if cells.dtype == torch.complex64:
        # a lazily conjugated tensor (x.conj()) has no real view: resolve it
        return torch.view_as_real(cells.resolve_conj())
    if cells.dtype == torch.complex128:
        return torch.view_as_real(cells.resolve_conj().to(torch.complex64))
    raise TypeError("cells must be complex64 (or complex128)")


def demap(cells, mod, rate, sigma2=None, n=None, deinterleave=True, out=None,
          stream=None):
    """(nblk, ncell) complex64 CUDA cells -> float32 LLRs.

    sigma2: None (per-row estimate), a Python float (one value), a (nblk,)
    tensor (per row) or a (nblk, ncell) tensor (per cell).  With
    ``deinterleave`` the LLRs land in LDPC codeword order (``lam``, shape
    (nblk, n)); otherwise in q order (nblk, ncell*nbits)."""
    torch = _torch()
    if cells.dim() == 1:
        cells = cells[None]
    if cells.device.type != "cuda":
        raise TypeError("cells must be a CUDA tensor")
    cells = cells.contiguous() if cells.stride(-1) != 1 else cells
    nblk, ncell = cells.shape
    nb = C.MOD_BITS[mod]
    dev = cells.device
    pts = device_points(mod, rate, dev)
    zf = _as_float_pairs(cells)
    if deinterleave:
        n = n or ncell * nb
        if n != ncell * nb:
            raise ValueError("ncell * nbits must equal Ninner")
        lq = device_lam_of_q(n, mod, rate, dev)
    else:
        lq = None
    width = ncell * nb
    if out is None:
        out = torch.empty((nblk, width), dtype=torch.float32, device=dev)
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    s2t = None
    s2s = 0.0
    ld_s = 0
    if sigma2 is None:
        s2t = torch.empty(nblk, dtype=torch.float32, device=dev)
        N.call("atsc3_demap_row_sigma2", zf.data_ptr(), zf.stride(0) // 2,
               nblk, ncell, pts.data_ptr(), nb, s2t.data_ptr(), st)
        mode = 2
    elif isinstance(sigma2, (float, int, np.floating)):
        mode, s2s = 0, float(np.float32(sigma2))
    else:
        s2t = sigma2.to(device=dev, dtype=torch.float32)
        if s2t.dim() == 1 and s2t.shape[0] == nblk:
            mode = 2
        else:
            s2t = s2t.reshape(nblk, ncell)
            if s2t.stride(1) != 1:
                s2t = s2t.contiguous()
            mode, ld_s = 1, s2t.stride(0)
    N.call("atsc3_demap", zf.data_ptr(), zf.stride(0) // 2, nblk, ncell,
           pts.data_ptr(), nb, mode, N.ptr(s2t), ld_s, s2s, N.ptr(lq),
           out.data_ptr(), out.stride(0), st)
    return out


@functools.lru_cache(maxsize=None)
def _host_points_f64(mod, rate):
    # |p|^2 as lab/m16_demap_fast.py:103 forms it: np.abs(pts) ** 2
    pts = np.asarray(C.alphabet(mod, rate), np.complex128)
    return np.concatenate([pts.real, pts.imag, np.abs(pts) ** 2])


def demap_f64(cells, mod, rate, sigma2=None, n=None, deinterleave=False,
              out=None, stream=None):
    """Float64 demapper: (nblk, ncell) complex128 CUDA cells -> float64
    LLRs, the double-precision arithmetic of the reference's default
    ``demap_llr_fast`` (lab/m16_demap_fast.py:80-119).  sigma2: None
    (per-row float64 estimate), a float, or a (nblk, ncell) tensor."""
    torch = _torch()
    if cells.dim() == 1:
        cells = cells[None]
    if cells.device.type != "cuda" or cells.dtype != torch.complex128:
        raise TypeError("cells must be a complex128 CUDA tensor")
    cells = cells.resolve_conj().contiguous()
    nblk, ncell = cells.shape
    nb = C.MOD_BITS[mod]
    dev = cells.device
    key = ("pts64", mod, rate, str(dev))
    pts = _DEV.get(key)
    if pts is None:
        pts = _DEV[key] = torch.from_numpy(_host_points_f64(mod, rate)).to(dev)
    zf = torch.view_as_real(cells)
    lq = None
    if deinterleave:
        n = n or ncell * nb
        lq = device_lam_of_q(n, mod, rate, dev)
    if out is None:
        out = torch.empty((nblk, ncell * nb), dtype=torch.float64, device=dev)
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    s2t, s2s, ld_s = None, 0.0, 0
    if sigma2 is None:
        s2t = torch.empty(nblk, dtype=torch.float64, device=dev)
        N.call("atsc3_demap_row_sigma2_f64", zf.data_ptr(), zf.stride(0) // 2,
               nblk, ncell, pts.data_ptr(), nb, s2t.data_ptr(), st)
        mode = 2
    elif isinstance(sigma2, (float, int, np.floating)):
        mode, s2s = 0, float(sigma2)
    else:
        s2t = sigma2.to(device=dev, dtype=torch.float64).reshape(nblk, ncell)
        s2t = s2t.contiguous()
        mode, ld_s = 1, s2t.stride(0)
    N.call("atsc3_demap_f64", zf.data_ptr(), zf.stride(0) // 2, nblk, ncell,
           pts.data_ptr(), nb, mode, N.ptr(s2t), ld_s, s2s, N.ptr(lq),
           out.data_ptr(), out.stride(0), st)
    return out


def demap_llr_fast(cells, mod, rate, sigma2=None, dtype=np.float64, ex=None,
                   chunk=20_000):
    """Drop-in for ``m16_demap_fast.demap_llr_fast``: one row of cells ->
    float64 (ncell*nbits,) LLRs in q order.  ``dtype`` picks the GPU
    arithmetic as it picks the reference's: float64 (the default) runs the
    float64 demapper, float32 the float32 one (the lab/m44_ldm.py:2431-2451
    operation order).  ``ex`` and ``chunk`` are accepted for signature
    compatibility.  ``sigma2`` may also be a per-cell array (divided after
    the minima)."""
    torch = _torch()
    if np.size(cells) == 0:         # nothing to demap (no sigma2 estimate either)
        return np.zeros(0, np.float64)
    if np.dtype(dtype) == np.float64:
        z = np.ascontiguousarray(np.asarray(cells), np.complex128).reshape(1, -1)
        s2 = sigma2
        if sigma2 is not None and np.ndim(sigma2) > 0:
            s2 = torch.from_numpy(np.asarray(sigma2, np.float64).reshape(1, -1)).cuda()
        elif sigma2 is not None:
            s2 = float(sigma2)
        q = demap_f64(torch.from_numpy(z).cuda(), mod, rate, sigma2=s2)
        return q.cpu().numpy().ravel()
    z = np.ascontiguousarray(np.asarray(cells), np.complex64).reshape(1, -1)
    t = torch.from_numpy(z).cuda()
    s2 = sigma2
    if sigma2 is not None and np.ndim(sigma2) > 0:
        s2 = torch.from_numpy(np.asarray(sigma2, np.float32).reshape(1, -1)).cuda()
    q = demap(t, mod, rate, sigma2=s2, deinterleave=False)
    return q.cpu().numpy().ravel().astype(np.float64)
