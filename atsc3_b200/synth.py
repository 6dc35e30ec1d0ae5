"""Seeded synthetic FEC blocks for benches and training (torch, any device).

The transmit chain of ``lab/m6_bicm.py:367-373`` (``PlpChain.encode``) --
scramble, BCH encode, LDPC encode, bit interleave, constellation map --
written with batched tensor ops so thousands of blocks are produced on the
GPU in milliseconds:

* LDPC (A/322 6.1.3): the accumulator parities are the information part of
  H applied to the message (an index_add over H's information edges), then a
  prefix XOR over the dual diagonal; Type A codes feed the M1 parity bits back
  through their edges into the M2 part.
* BCH (A/322 6.1.2.1): parity = message x R mod 2 with R the remainder rows
  x^(K-1-pos) mod g(x), as a float matmul (exact: counts < 2^24).
* channels: AWGN with scalar N0, or a per-cell Rayleigh gain |CN(0,1)|
  equalised away with sigma2_cell = N0/h^2.

Checked bit-exact against the oracle transmitter in the CPU tests.
"""
from __future__ import annotations

import functools

import numpy as np

from . import codes as C


def _torch():
    import torch
    return torch


@functools.lru_cache(maxsize=None)
def _encoder_tables(rate, n):
    typ, K, M1, M2, Q1, Q2 = C.ldpc_params(rate, n)
    r, c, M = C._parity_edges(rate, n)
    info = c < K
    fb = (c >= K) & (c < K + M1) & (r >= M1) if typ == "A" else np.zeros_like(info)
    a = np.arange(M, dtype=np.int64)
    s1, t1 = np.divmod(a, max(Q1, 1))
    s2, t2 = np.divmod(a - M1, Q2)
    pi = np.where(a < M1, K + 360 * t1 + s1, K + M1 + 360 * t2 + s2)
    return dict(typ=typ, K=K, M1=M1, M=M, info_r=r[info].astype(np.int64),
                info_c=c[info].astype(np.int64), fb_r=r[fb].astype(np.int64),
                fb_c=(c[fb] - K).astype(np.int64), pi=pi)


class Transmitter:
    """payload bits (nblk, K_payload) uint8 -> cells (nblk, ncell) complex64."""

    def __init__(self, n, mod, rate, device="cpu", chunk=128):
        torch = _torch()
        self.n, self.mod, self.rate = n, mod, rate
        self.dev = torch.device(device)
        self.nb = C.MOD_BITS[mod]
        self.ncell = C.cells_per_block(n, mod)
        self.K = C.kldpc(rate, n)
        self.kp = C.kpayload(rate, n)
        self.chunk = chunk
        t = _encoder_tables(rate, n)
        self.t = {k: (torch.from_numpy(v).to(self.dev) if isinstance(v, np.ndarray)
                      else v) for k, v in t.items()}
        R = C.bch_remainder_table(self.K, n)[:self.kp]
        bits = np.unpackbits(R.view(np.uint8), axis=1, bitorder="little")
        self.rbits = torch.from_numpy(bits[:, :C.MOUTER[n]].astype(np.float32)).to(self.dev)
        self.scr = torch.from_numpy(C.scrambler_sequence(self.kp).copy()).to(self.dev)
        self.lam_of_q = torch.from_numpy(C.bicm_map(n, mod, rate).astype(np.int64)).to(self.dev)
        pts = C.alphabet(mod, rate)
        self.pts = torch.from_numpy(np.asarray(pts, np.complex64)).to(self.dev)
        self.shift = torch.tensor([1 << (self.nb - 1 - i) for i in range(self.nb)],
                                  dtype=torch.int64, device=self.dev)

    def bch_encode(self, info):
        torch = _torch()
        deg = C.MOUTER[self.n]
        par = (info.float() @ self.rbits).to(torch.int64) & 1
        # remainder word bit b = coefficient of x^b; codeword bit Kp+i is the
        # coefficient of x^(deg-1-i)
        par = torch.flip(par, dims=[1]).to(torch.uint8)
        return torch.cat([info, par[:, :deg]], dim=1)

    def ldpc_encode(self, s):
        torch = _torch()
        t = self.t
        nblk = s.shape[0]
        lam = torch.zeros((nblk, self.n), dtype=torch.uint8, device=self.dev)
        lam[:, :self.K] = s
        acc = torch.zeros((nblk, t["M"]), dtype=torch.int32, device=self.dev)
        acc.index_add_(1, t["info_r"], s[:, t["info_c"]].to(torch.int32))
        acc &= 1
        M1 = t["M1"]
        if t["typ"] == "A":
            p1 = torch.cumsum(acc[:, :M1], dim=1) & 1
            lam[:, t["pi"][:M1]] = p1.to(torch.uint8)
            fbv = torch.zeros_like(acc)
            fbv.index_add_(1, t["fb_r"],
                           lam[:, self.K:self.K + M1][:, t["fb_c"]].to(torch.int32))
            p2 = (acc[:, M1:] + fbv[:, M1:]) & 1
            lam[:, t["pi"][M1:]] = p2.to(torch.uint8)
        else:
            p = torch.cumsum(acc, dim=1) & 1
            lam[:, t["pi"]] = p.to(torch.uint8)
        return lam

    def encode(self, payload):
        """payload (nblk, K_payload) uint8 -> (cells complex64, codewords)."""
        torch = _torch()
        payload = payload.to(self.dev, torch.uint8)
        cells, cws = [], []
        for lo in range(0, payload.shape[0], self.chunk):
            p = payload[lo:lo + self.chunk]
            nouter = self.bch_encode(p ^ self.scr[None, :])
            cw = self.ldpc_encode(nouter)
            q = cw[:, self.lam_of_q].to(torch.int64)
            k = (q.view(q.shape[0], self.ncell, self.nb) * self.shift).sum(-1)
            cells.append(self.pts[k])
            cws.append(cw)
        return torch.cat(cells), torch.cat(cws)


def channel(x, esn0_db, kind, gen):
    """x complex64 (nblk, ncell) on any device; returns (y complex64,
    sigma2: float for AWGN, (nblk, ncell) float32 for Rayleigh)."""
    torch = _torch()
    n0 = 10.0 ** (-float(esn0_db) / 10.0)
    shape = x.shape

    def cn():
        re = torch.randn(shape, generator=gen, device=x.device)
        im = torch.randn(shape, generator=gen, device=x.device)
        return torch.complex(re, im) / np.sqrt(2.0)

    if kind == "awgn":
        return (x + cn() * np.sqrt(n0)).to(torch.complex64), n0
    if kind == "rayleigh":
        h = cn().abs()
        y = (h * x + cn() * np.sqrt(n0)) / h
        return y.to(torch.complex64), (n0 / h ** 2).to(torch.float32)
    raise ValueError(kind)
