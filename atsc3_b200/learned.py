"""Differentiable unrolled weighted min-sum and its learned weights.

``WeightedMinSum`` (a ``torch.autograd.Function``) runs the forward and the
hand-written backward kernels of ``csrc/wms.cu``: T flooding iterations with
per-iteration, per-check-degree scale ``alpha[t, d]`` and offset
``beta[t, d]`` (messages ``sgn * relu(alpha * mu - beta)``), checkpointing one
16-byte record per check per iteration and recomputing messages in the
backward.  ``reference_f64`` is the same forward in float64 torch ops whose
autograd gradient (and finite differences) check the kernels.

``train`` fits the weights on LLRs produced by this package's own demapper
from seeded synthetic blocks (mean BCE of the output LLRs against the
transmitted bits, LLR > 0 meaning bit 0); ``save_weights`` / ``load_weights``
keep them with a manifest (code, iterations, degree buckets, seed, step) so
training resumes by step.
"""
from __future__ import annotations

import ctypes
import functools
import json
import os

import numpy as np

from . import codes as C
from . import native as N


def _torch():
    import torch
    return torch


def block_rows(rate, n):
    """Block row of every check of an A/322 code: accumulator checks
    r + QA*k (k = 0..359) are row r; a Type A code's identity checks
    360*QA + (r - QA) + QB*k are row r (QA <= r < QA + QB)."""
    typ, K, M1, M2, Q1, Q2 = C.ldpc_params(rate, n)
    nc = n - K
    c = np.arange(nc)
    if typ == "A":
        qa, qb = Q1, Q2
        return np.where(c < 360 * qa, c % qa,
                        qa + (c - 360 * qa) % max(qb, 1)).astype(np.int64)
    return (c % Q2).astype(np.int64)


@functools.lru_cache(maxsize=None)
def host_tables(rate, n, mode="degree"):
    """CSR tables + per variable-major edge (check, position) + per-check
    bucket.  mode "degree": buckets = the code's distinct check degrees,
    ascending; "row": one bucket per block row (at most 127)."""
    cptr, cidx, vptr, vedge = C.csr(rate, n)
    deg = np.diff(cptr)
    if deg.max() > 32:
        raise ValueError("weighted min-sum serves check degrees <= 32")
    chk = np.repeat(np.arange(len(deg), dtype=np.int32), deg)
    pos = (np.arange(len(cidx)) - cptr[chk]).astype(np.int32)
    if mode == "row":
        rows = block_rows(rate, n)
        buckets = np.arange(int(rows.max()) + 1)
        if len(buckets) > 127:
            raise ValueError("per-row weights serve codes of at most 127 block rows")
        cb = rows.astype(np.int8)
    elif mode == "degree":
        buckets = np.unique(deg)
        cb = np.searchsorted(buckets, deg).astype(np.int8)
    else:
        raise ValueError(f"unknown bucket mode {mode}")
    return dict(cptr=cptr, cidx=cidx, vptr=vptr, vedge=vedge,
                vchk=chk[vedge].astype(np.int32), vpos=pos[vedge],
                cbucket=cb, buckets=buckets, n=n, nc=len(deg), ne=len(cidx),
                mode=mode)


class WmsCode:
    """Device copy of host_tables for one code; mode "degree" (weights per
    iteration and check degree) or "row" (per iteration and block row)."""

    def __init__(self, rate, n, device="cuda", mode="degree"):
        torch = _torch()
        h = host_tables(rate, n, mode)
        self.rate, self.n, self.mode = rate, n, mode
        self.nc, self.ne = h["nc"], h["ne"]
        self.buckets = h["buckets"]
        self.nbucket = len(self.buckets)
        self.dev = torch.device(device)
        self.t = {k: torch.from_numpy(np.array(h[k])).to(self.dev)
                  for k in ("cptr", "cidx", "vptr", "vedge", "vchk", "vpos",
                            "cbucket")}

    def ptrs(self):
        t = self.t
        return [t[k].data_ptr() for k in ("cptr", "cidx", "vptr", "vedge",
                                          "vchk", "vpos", "cbucket")]

    def init_params(self, iters, alpha=0.75, beta=0.0):
        torch = _torch()
        a = torch.full((iters, self.nbucket), float(alpha), device=self.dev)
        b = torch.full((iters, self.nbucket), float(beta), device=self.dev)
        return a, b


class WeightedMinSum:
    """torch.autograd.Function wrapper: out = WeightedMinSum.apply(llr,
    alpha, beta, code, bf16).  llr (nblk, n) float32 CUDA (not
    differentiated: it is data); alpha, beta (T, nbucket) float32."""

    @staticmethod
    def _fn():
        torch = _torch()

        class _F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, llr, alpha, beta, code, bf16):
                iters = alpha.shape[0]
                nblk = llr.shape[0]
                llr = llr.contiguous()
                a = alpha.detach().contiguous().float()
                b = beta.detach().contiguous().float()
                rec = torch.empty((iters, nblk, code.nc, 16), dtype=torch.uint8,
                                  device=llr.device)
                out = torch.empty_like(llr)
                N.call("atsc3_wms_forward", *code.ptrs(), code.n, code.nc,
                       code.ne, code.nbucket, nblk, iters, llr.data_ptr(),
                       a.data_ptr(), b.data_ptr(), int(bool(bf16)),
                       rec.data_ptr(), out.data_ptr(),
                       torch.cuda.current_stream(llr.device).cuda_stream)
                ctx.save_for_backward(llr, a, b, rec)
                ctx.code = code
                return out

            @staticmethod
            def backward(ctx, g):
                llr, a, b, rec = ctx.saved_tensors
                code = ctx.code
                iters, nblk = a.shape[0], llr.shape[0]
                gt = g.contiguous().float().clone()
                ga = torch.zeros_like(a)
                gb = torch.zeros_like(b)
                work = torch.empty(nblk * code.n + 2 * nblk * code.ne,
                                   dtype=torch.float32, device=llr.device)
                N.call("atsc3_wms_backward", *code.ptrs(), code.n, code.nc,
                       code.ne, code.nbucket, nblk, iters, llr.data_ptr(),
                       a.data_ptr(), b.data_ptr(), rec.data_ptr(),
                       gt.data_ptr(), ga.data_ptr(), gb.data_ptr(),
                       work.data_ptr(),
                       torch.cuda.current_stream(llr.device).cuda_stream)
                return None, ga, gb, None, None

        return _F

    _F = None

    @classmethod
    def apply(cls, llr, alpha, beta, code, bf16=False):
        if cls._F is None:
            cls._F = cls._fn()
        return cls._F.apply(llr, alpha, beta, code, bf16)


def reference_f64(llr, alpha, beta, rate, n, mode="degree"):
    """The weighted min-sum forward in float64 torch ops (CPU), for autograd
    and finite-difference checks.  Same rules as csrc/wms.cu: first-minimum
    arg-min, sign(x) = -1 iff x < 0, relu(alpha*mu - beta)."""
    torch = _torch()
    h = host_tables(rate, n, mode)
    cptr, cidx = h["cptr"], h["cidx"]
    deg = np.diff(cptr)
    nc, dmax = len(deg), int(deg.max())
    idx = np.full((nc, dmax), n, np.int64)
    mask = np.zeros((nc, dmax), bool)
    for c in range(nc):
        idx[c, :deg[c]] = cidx[cptr[c]:cptr[c + 1]]
        mask[c, :deg[c]] = True
    idx_t = torch.from_numpy(idx)
    mask_t = torch.from_numpy(mask)
    cb = torch.from_numpy(h["cbucket"].astype(np.int64))
    llr = llr.double()
    nb = llr.shape[0]
    iters = alpha.shape[0]
    ar = torch.arange(dmax)
    inf = torch.tensor(float("inf"), dtype=torch.float64)
    m = torch.zeros((nb, nc, dmax), dtype=torch.float64)
    tot = llr
    for t in range(iters):
        tp = torch.cat([tot, torch.zeros((nb, 1), dtype=torch.float64)], 1)
        x = tp[:, idx_t] - m
        sx = (x < 0) & mask_t
        par = (sx.sum(-1) % 2).bool()
        mag = torch.where(mask_t, x.abs(), inf)
        mn = mag.detach()
        min1v = mn.min(-1, keepdim=True).values
        first = ((mn == min1v).long() * (dmax - ar)).argmax(-1, keepdim=True)
        mn2 = mn.scatter(-1, first, float("inf"))
        min2v = mn2.min(-1, keepdim=True).values
        second = ((mn2 == min2v).long() * (dmax - ar)).argmax(-1, keepdim=True)
        min1 = mag.gather(-1, first)
        min2 = mag.gather(-1, second)
        mu = torch.where(ar == first, min2, min1)
        a = alpha[t][cb].double()[None, :, None] * mu - beta[t][cb].double()[None, :, None]
        sgn = torch.where(par[..., None] ^ sx, -1.0, 1.0).double()
        m = torch.where(mask_t, sgn * torch.relu(a), torch.zeros((), dtype=torch.float64))
        s = torch.zeros((nb, n + 1), dtype=torch.float64)
        s = s.index_add(1, idx_t.reshape(-1), m.reshape(nb, -1))
        tot = llr + s[:, :n]
    return tot


def bce_loss(out_llr, bits):
    """Mean BCE of output LLRs against the true bits (LLR > 0 = bit 0)."""
    torch = _torch()
    return torch.nn.functional.binary_cross_entropy_with_logits(
        -out_llr, bits.to(out_llr.dtype))


# ---------------------------------------------------------------------------
# training on the package's own demapper output
# ---------------------------------------------------------------------------

def make_batch(tx, gen, nblk, esn0_lo, esn0_hi, channel="awgn", device="cuda"):
    """Seeded blocks -> (llr (nblk, n) float32 codeword order, codewords).

    Es/N0 is drawn per block uniformly in [esn0_lo, esn0_hi]; channel
    "awgn", "rayleigh" (per-cell |CN(0,1)| gain, equalised, per-cell sigma2)
    or "mixed" (odd blocks Rayleigh).  LLRs come from this package's
    demapper with the per-cell noise variance."""
    torch = _torch()
    from . import demap as DM
    pay = torch.randint(0, 2, (nblk, tx.kp), generator=gen, device=device,
                        dtype=torch.uint8)
    x, cw = tx.encode(pay)
    esn0 = torch.rand(nblk, 1, generator=gen, device=device) * (esn0_hi - esn0_lo) + esn0_lo
    n0 = torch.pow(10.0, -esn0 / 10.0)

    def cn():
        re = torch.randn(x.shape, generator=gen, device=device)
        im = torch.randn(x.shape, generator=gen, device=device)
        return torch.complex(re, im) / np.sqrt(2.0)

    if channel == "awgn":
        h = torch.ones(x.shape, device=device)
    else:
        h = cn().abs()
        if channel == "mixed":
            odd = (torch.arange(nblk, device=device) % 2 == 1)[:, None]
            h = torch.where(odd, h, torch.ones_like(h))
    y = ((h * x + cn() * torch.sqrt(n0)) / h).to(torch.complex64)
    s2 = (n0 / h ** 2).to(torch.float32)
    lam = DM.demap(y, tx.mod, tx.rate, sigma2=s2, n=tx.n)
    return lam, cw


def save_weights(path, alpha, beta, manifest):
    torch = _torch()
    torch.save({"alpha": alpha.detach().cpu(), "beta": beta.detach().cpu(),
                "manifest": manifest}, path)


def load_weights(path, device="cuda"):
    torch = _torch()
    d = torch.load(path, map_location="cpu")
    return d["alpha"].to(device), d["beta"].to(device), d["manifest"]


def train(rate, n, mod, steps=200, nblk=64, iters=12, lr=0.02, esn0=(0.0, 2.0),
          channel="awgn", seed=1, bf16=False, log_every=50, resume=None,
          device="cuda", depths=None, mode="degree"):
    """Adam on (alpha, beta) of the unrolled decoder; returns (alpha, beta,
    history).  Fresh seeded blocks every step.  depths: None (the loss is the
    BCE of the output after all `iters` iterations) or a list of unrolled
    depths t <= iters whose output BCEs are averaged (each depth uses the
    first t rows of the weights), which rewards being right early."""
    torch = _torch()
    from . import synth
    code = WmsCode(rate, n, device, mode)
    tx = synth.Transmitter(n, mod, rate, device=device)
    alpha, beta = code.init_params(iters)
    start = 0
    if resume is not None:
        a0, b0, man = load_weights(resume, device)
        alpha.copy_(a0)
        beta.copy_(b0)
        start = int(man.get("step", 0))
    alpha.requires_grad_(True)
    beta.requires_grad_(True)
    opt = torch.optim.Adam([alpha, beta], lr=lr)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed + start)
    hist = []
    for step in range(start, start + steps):
        lam, cw = make_batch(tx, gen, nblk, esn0[0], esn0[1], channel, device)
        if depths:
            loss = sum(bce_loss(WeightedMinSum.apply(lam, alpha[:t], beta[:t],
                                                     code, bf16), cw)
                       for t in depths) / len(depths)
        else:
            out = WeightedMinSum.apply(lam, alpha, beta, code, bf16)
            loss = bce_loss(out, cw)
        opt.zero_grad()
        loss.backward()
        opt.step()
        with torch.no_grad():
            beta.clamp_(min=0.0)
        if step % log_every == 0 or step == start + steps - 1:
            hist.append((step, float(loss.detach())))
    manifest = {"rate": rate, "n": n, "mod": mod, "iters": iters,
                "buckets": [int(x) for x in code.buckets], "mode": mode,
                "seed": seed,
                "step": start + steps, "esn0": list(esn0), "channel": channel,
                "bf16": bool(bf16), "depths": list(depths) if depths else None}
    return alpha.detach(), beta.detach(), hist, manifest


def inference_weights(alpha, beta, buckets, device="cuda", mode="degree"):
    """(walpha, wbeta, dbucket) device tensors for the quasi-cyclic decoder:
    dbucket[degree] = bucket index of that check degree; mode "row":
    (walpha, wbeta, rbucket, "row") with rbucket[block row] = its bucket
    (the edge-buffer decoder's per-row weights)."""
    torch = _torch()
    db = np.zeros(256, np.int8)          # every check degree the decoders take (<= 250)
    for i, d in enumerate(buckets):
        db[int(d)] = i
    w = (alpha.detach().float().contiguous().to(device),
         beta.detach().float().contiguous().to(device),
         torch.from_numpy(db).to(device))
    return w + ("row",) if mode == "row" else w
