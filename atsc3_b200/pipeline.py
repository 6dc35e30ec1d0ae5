"""The fused FEC back end: cells -> demap + de-interleave -> min-sum LDPC ->
BCH + descramble -> Baseband Packet bytes, all on one GPU stream.

This is the batched path the reference runs as ``m44_ldm.decode_blocks``
(``lab/m44_ldm.py:2348-2390``: demap_batch_qam, ``lam[:, lam_of_q] = q``,
ldpc_batch, bch_syndrome_batch, descramble) and ``m9_fast._decode_frame``
(``lab/m9_fast.py:1117-1154``).  Three launches: the demapper (writes LLRs
in codeword order), the cluster LDPC decoder (packed hard decisions +
per-block conv/its/bad), the BCH check (syndrome, ok flag, payload bytes).
"""
from __future__ import annotations

import os

import numpy as np

from . import bch as BCH
from . import codes as C
from . import demap as DM
from . import ldpc as LDPC


def _torch():
    import torch
    return torch


class _Range:
    """An NVTX range around a stage when ATSC3_NVTX=1 (for nsys/ncu
    timelines); nothing otherwise."""

    on = os.environ.get("ATSC3_NVTX", "0") not in ("", "0")

    def __init__(self, name):
        self.name = name

    def __enter__(self):
        if self.on:
            _torch().cuda.nvtx.range_push(self.name)

    def __exit__(self, *exc):
        if self.on:
            _torch().cuda.nvtx.range_pop()


class FecPipeline:
    """One (Ninner, constellation, rate) PLP configuration.  kind selects the
    LDPC decoder ("auto", "qce", "qc" or "csr"; see ldpc.plan_for).
    rescue: None (off, as the reference's default) or a dict of
    ldpc.rescue_near_misses arguments (near_max, max_blocks, iters): blocks
    min-sum leaves a few checks short get the exact sum-product before BCH
    (this adds a host read of the flags).  ladder: None (the single `alpha`,
    as the configs pin it) or a tuple of alphas tried in turn on the blocks
    that did not converge (ldpc.ladder_decode; the reference's default
    ladder is ldpc.ALPHA_LADDER)."""

    def __init__(self, n, mod, rate, iters=50, alpha=0.75, semantics="kernel",
                 cluster=0, threads=0, device="cuda", kind="auto",
                 rescue=None, ladder=None):
        torch = _torch()
        self.n, self.mod, self.rate = int(n), mod, rate
        self.nb = C.MOD_BITS[mod]
        self.ncell = C.cells_per_block(n, mod)
        self.kldpc = C.kldpc(rate, n)
        self.kpayload = C.kpayload(rate, n)
        self.iters, self.alpha = iters, alpha
        self.semantics = semantics
        self.threads = threads
        self.device = torch.device(device)
        with torch.cuda.device(self.device):
            self.plan = LDPC.plan_for(rate, n, "float32", cluster, kind=kind)
            self.rescue = dict(rescue) if rescue else None
            self.ladder = tuple(ladder) if ladder else None
            self.sp_tab = (LDPC.sp_tables(C.csr(rate, n), n, self.device)
                           if self.rescue else None)
        self._ws = {}

    def _buffers(self, nblk):
        torch = _torch()
        ws = self._ws.get(nblk)
        if ws is None:
            d = self.device
            ws = {"lam": torch.empty((nblk, self.n), dtype=torch.float32, device=d),
                  "hard": torch.empty((nblk, (self.n + 31) // 32 * 4),
                                      dtype=torch.uint8, device=d),
                  "conv": torch.empty(nblk, dtype=torch.uint8, device=d),
                  "its": torch.empty(nblk, dtype=torch.int32, device=d),
                  "bad": torch.empty(nblk, dtype=torch.int32, device=d),
                  "syn": torch.empty((nblk, 6), dtype=torch.int32, device=d),
                  "ok": torch.empty(nblk, dtype=torch.uint8, device=d),
                  "payload": torch.empty((nblk, self.kpayload // 8),
                                         dtype=torch.uint8, device=d)}
            self._ws[nblk] = ws
        return ws

    def decode(self, cells, sigma2=None, iters=None, alpha=None, out=None,
               weights=None):
        """cells: (nblk, ncell) complex64 CUDA tensor; sigma2: float, (nblk,)
        or (nblk, ncell) tensor, or None (per-row estimate).  Returns a dict
        of device tensors: the workspace (reused by the next call of the same
        batch size) overridden by any caller-owned buffers in `out` (keys
        conv, its, bad, syn, ok, payload).  `weights`: learned per-iteration,
        per-check-degree scale/offset tables (``learned.inference_weights``)
        in place of the single `alpha`.  All launches go to the current
        stream."""
        nblk = cells.shape[0]
        ws = dict(self._buffers(nblk))
        if out:
            ws.update(out)
        with _Range("atsc3.demap"):
            DM.demap(cells, self.mod, self.rate, sigma2=sigma2, n=self.n,
                     deinterleave=True, out=ws["lam"])
        with _Range("atsc3.ldpc"):
            self._ldpc(ws, iters, alpha, weights)
        if self.rescue:
            with _Range("atsc3.sp_rescue"):
                LDPC.rescue_near_misses(self.sp_tab, ws["lam"], ws, **self.rescue)
        with _Range("atsc3.bch"):
            BCH.bch_check(ws["hard"], self.kldpc, self.n, self.kpayload,
                          want_payload=True, out=ws)
        return ws

    def _ldpc(self, ws, iters, alpha, weights):
        if self.ladder and alpha is None and weights is None:
            o = LDPC.ladder_decode(self.plan, ws["lam"], ladder=self.ladder,
                                   iters=iters or self.iters,
                                   semantics=self.semantics, want_bits=False,
                                   threads=self.threads)
            for k in ("hard", "conv", "its", "bad"):
                ws[k].copy_(o[k])
            return
        LDPC.decode_flood(self.plan, ws["lam"], iters=iters or self.iters,
                          alpha=self.alpha if alpha is None else alpha,
                          semantics=self.semantics, want_bits=False,
                          want_hard=True, threads=self.threads, out=ws,
                          weights=weights)

    def decode_stream(self, stream, ti, sigma2, iters=None, alpha=None,
                      out=None, weights=None):
        """As decode, from a received PLP cell stream instead of FEC Block
        rows: ``ti`` (timeint.HybridTI / ConvolutionalTI) is de-interleaved
        inside the demapper's cell load (the reference de-interleaves on
        the host first, lab/m9_fast.py:1087-1093, lab/m10_cti.py:126-141).
        sigma2: float, per received cell, or per FEC Block."""
        from . import timeint as TI
        nblk = ti.nblk
        ws = dict(self._buffers(nblk))
        if out:
            ws.update(out)
        TI.demap_deinterleave(stream, ti, self.mod, self.rate, self.n,
                              sigma2=sigma2, out=ws["lam"])
        self._ldpc(ws, iters, alpha, weights)
        if self.rescue:
            LDPC.rescue_near_misses(self.sp_tab, ws["lam"], ws, **self.rescue)
        BCH.bch_check(ws["hard"], self.kldpc, self.n, self.kpayload,
                      want_payload=True, out=ws)
        return ws

    def decode_host(self, cells, sigma2=None):
        """End-to-end from host memory: numpy (or pinned torch) cells in,
        numpy results out (payload bytes, conv, its, bad, bch ok)."""
        torch = _torch()
        if isinstance(cells, np.ndarray):
            cells = torch.from_numpy(np.ascontiguousarray(cells, np.complex64))
        c = cells.to(self.device, non_blocking=True)
        s2 = sigma2
        if isinstance(sigma2, np.ndarray):
            sigma2 = torch.from_numpy(np.ascontiguousarray(sigma2, np.float32))
        if hasattr(sigma2, "to"):
            s2 = sigma2.to(self.device, non_blocking=True)
        ws = self.decode(c, s2)
        return {k: ws[k].cpu().numpy() for k in ("payload", "conv", "its",
                                                  "bad", "ok")}
