"""Uneven batches: blocks of different code lengths, rates and constellations
decoded together -- one launch per stage, replayed as a CUDA graph, with the
launch shape chosen by an autotuner.

The reference decodes one PLP configuration at a time (``m9_fast`` and
``m44_ldm`` loop per MODCOD, ``lab/m9_fast.py:1117-1154``,
``lab/m44_ldm.py:2348-2390``).  ``UnevenBatch`` takes any list of
``(n, mod, rate)`` blocks and runs

    mixed demap + de-interleave  (atsc3_demap_batch, 256-cell chunks)
    LDPC, concurrently on forked streams:
      one edge-buffer quasi-cyclic launch per Type B code it accepts
                                 (atsc3_ldpc_qce_decode over that code's
                                  blocks, which sit contiguously inside)
      one persistent CSR launch for every other block
                                 (atsc3_ldpc_batch_decode: clusters pull
                                  blocks from a device queue, most work first)
    mixed BCH + descramble        (atsc3_bch_batch)

``capture()`` records the launches (queue reset, fork and join included)
into a CUDA graph; ``autotune()`` times the graph for each cluster size of
the CSR launch (1..16 CTAs per codeword, as far as every CSR code fits) and
CTA size (512 or 1024 threads) and keeps the fastest; results are cached per
batch signature.  Blocks are stored grouped by decoder; ``load`` takes and
``results`` returns them in the caller's order.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import bch as BCH
from . import codes as C
from . import demap as DM
from . import ldpc as LDPC
from . import native as N


def _torch():
    import torch
    return torch


_TUNED = {}
_CSR = {}


def csr_plan(rate, n, cluster):
    key = (rate, n, cluster)
    p = _CSR.get(key)
    if p is None:
        p = LDPC.Plan(*C.csr(rate, n), n, dtype="float32", cluster=cluster)
        _CSR[key] = p
    return p


def min_cluster(rate, n):
    for cl in (1, 2, 4, 8, 16):
        try:
            csr_plan(rate, n, cl)
            return cl
        except N.FecError as e:
            if e.rc != -4:
                raise
    raise RuntimeError(f"code {n} {rate} does not fit 16 CTAs")


_QCE = {}


def qce_plan(rate, n, cluster=0):
    """The edge-buffer quasi-cyclic plan of a code (every A/322 code) at a
    cluster size (0: the smallest that holds a codeword), or None if that
    decoder does not take it at that size."""
    key = (rate, n, cluster)
    if key not in _QCE:
        p = None
        try:
            p = LDPC.QcePlan(rate, n, cluster=cluster)
        except N.FecError as e:
            if e.rc != -4:
                raise
        _QCE[key] = p
    return _QCE[key]


class UnevenBatch:
    """A fixed list of blocks ``specs = [(n, mod, rate), ...]``.  hybrid:
    decode the blocks with the edge-buffer quasi-cyclic decoder (one launch
    per code, concurrent; the CSR persistent launch keeps any code it does
    not take); False puts every block on the CSR persistent launch."""

    def __init__(self, specs, iters=50, alpha=0.75, device="cuda", hybrid=True):
        torch = _torch()
        user = [tuple(s) for s in specs]
        self.iters, self.alpha = iters, alpha
        self.dev = torch.device(device)
        d = self.dev
        # internal order: quasi-cyclic groups (by code), then the CSR blocks
        with torch.cuda.device(d):
            qp = {(r, n): (qce_plan(r, n) if hybrid else None)
                  for n, m, r in user}
        qcodes = sorted({(r, n) for n, m, r in user if qp[(r, n)] is not None},
                        key=lambda c: (c[1], c[0]))
        perm = []
        for code in qcodes:
            perm += [i for i, (n, m, r) in enumerate(user) if (r, n) == code]
        rest = [i for i, (n, m, r) in enumerate(user) if qp[(r, n)] is None]
        perm += rest
        self.perm = np.array(perm, np.int64)         # internal -> caller index
        self.specs = [user[i] for i in perm]
        self.user_specs = user
        self.groups = []                             # (plan, first, count, n)
        first = 0
        for code in qcodes:
            cnt = sum(1 for n, m, r in user if (r, n) == code)
            self.groups.append((qp[code], first, cnt, code[1]))
            first += cnt
        self.csr_ids = list(range(first, len(user)))
        # launch shape of each edge-buffer group: (cluster, CTA threads),
        # (0, 0) = the plan's own choice; autotune() moves them
        self.gshape = [(0, 0)] * len(self.groups)
        nb = len(self.specs)
        self.nblk = nb
        ncell = [C.cells_per_block(n, m) for n, m, r in self.specs]
        nbits = [C.MOD_BITS[m] for n, m, r in self.specs]
        self.ncell = ncell
        # alphabets, de-interleavers, BCH tables: one copy per distinct key
        pts, pts_off, pkey = [], [], {}
        lq, lq_off, lkey = [], [], {}
        rt, rt_off, rkey = [], [], {}
        o_p = o_l = o_r = 0
        for (n, m, r) in self.specs:
            if (m, r) not in pkey:
                a = DM._host_points(m, r)
                pkey[(m, r)] = o_p
                pts.append(a)
                o_p += len(a)
            pts_off.append(pkey[(m, r)])
            if (n, m, r) not in lkey:
                a = np.asarray(C.bicm_map(n, m, r), np.int32)
                lkey[(n, m, r)] = o_l
                lq.append(a)
                o_l += len(a)
            lq_off.append(lkey[(n, m, r)])
            k = C.kldpc(r, n)
            if (k, n) not in rkey:
                a = np.asarray(C.bch_remainder_table(k, n)).ravel()
                rkey[(k, n)] = o_r
                rt.append(a)
                o_r += len(a)
            rt_off.append(rkey[(k, n)])
        T = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt)).to(d)
        self.t_pts = T(np.concatenate(pts), np.float32)
        self.t_lq = T(np.concatenate(lq), np.int32)
        self.t_rt = T(np.concatenate(rt), np.uint32)
        kpays = [C.kpayload(r, n) for n, m, r in self.specs]
        self.t_scr = T(np.packbits(np.array(C.scrambler_sequence(max(kpays)))), np.uint8)
        cell_off = np.concatenate([[0], np.cumsum(ncell)[:-1]]).astype(np.int64)
        ns = [n for n, m, r in self.specs]
        llr_off = np.concatenate([[0], np.cumsum(ns)[:-1]]).astype(np.int64)
        hb = [(n + 31) // 32 * 4 for n in ns]
        hard_off = np.concatenate([[0], np.cumsum(hb)[:-1]]).astype(np.int64)
        pb = [k // 8 for k in kpays]
        pay_off = np.concatenate([[0], np.cumsum(pb)[:-1]]).astype(np.int64)
        self.cell_off, self.llr_off = cell_off, llr_off
        self.hard_off, self.pay_off = hard_off, pay_off
        self.kpays = kpays
        chunk_blk, chunk_start = [], []
        for b, c in enumerate(ncell):
            for s in range(0, c, 256):
                chunk_blk.append(b)
                chunk_start.append(s)
        self.nchunks = len(chunk_blk)
        self.max_nbits = max(nbits)
        self.a = {
            "cell_off": T(cell_off, np.int64), "ncell": T(ncell, np.int32),
            "nbits": T(nbits, np.int32), "pts_off": T(pts_off, np.int64),
            "lq_off": T(lq_off, np.int64), "llr_off": T(llr_off, np.int64),
            "hard_off": T(hard_off, np.int64), "pay_off": T(pay_off, np.int64),
            "kldpc": T([C.kldpc(r, n) for n, m, r in self.specs], np.int32),
            "rt_off": T(rt_off, np.int64), "kpay": T(kpays, np.int32),
            "chunk_blk": T(chunk_blk, np.int32),
            "chunk_start": T(chunk_start, np.int32),
        }
        # CSR queue: its blocks, most edges first
        edges = np.array([len(C.csr(r, n)[1]) for n, m, r in self.specs])
        ids = np.array(self.csr_ids, np.int64)
        self.a["order"] = T(ids[np.argsort(-edges[ids], kind="stable")]
                            if len(ids) else np.zeros(1, np.int64), np.int32)
        self.ncsr = len(ids)
        self.hb = hb
        self.side = [torch.cuda.Stream(d) for _ in range(len(self.groups) + 1)]
        # buffers
        self.cells = torch.empty(int(sum(ncell)), dtype=torch.complex64, device=d)
        self.sigma2 = torch.ones(nb, dtype=torch.float32, device=d)
        self.llr = torch.empty(int(sum(ns)), dtype=torch.float32, device=d)
        self.hard = torch.empty(int(sum(hb)), dtype=torch.uint8, device=d)
        self.payload = torch.empty(int(sum(pb)), dtype=torch.uint8, device=d)
        self.conv = torch.empty(nb, dtype=torch.uint8, device=d)
        self.its = torch.empty(nb, dtype=torch.int32, device=d)
        self.bad = torch.empty(nb, dtype=torch.int32, device=d)
        self.syn = torch.empty((nb, 6), dtype=torch.int32, device=d)
        self.ok = torch.empty(nb, dtype=torch.uint8, device=d)
        self.counter = torch.zeros(1, dtype=torch.int32, device=d)
        # CSR plans for the codes of the CSR blocks (one if there are none,
        # so the launch configuration stays defined)
        self.codes = sorted({(self.specs[b][2], self.specs[b][0])
                             for b in self.csr_ids}) or [(self.specs[0][2],
                                                          self.specs[0][0])]
        self.cl_min = max(min_cluster(r, n) for r, n in self.codes)
        self.graph = None
        self.config = None
        self.set_config(self.cl_min, 1024)

    # -- inputs -----------------------------------------------------------
    def load(self, cells_list, sigma2_list):
        """Copy per-block cells (complex64 tensors) and scalar sigma2, in the
        caller's block order."""
        torch = _torch()
        for b, u in enumerate(self.perm):
            o = int(self.cell_off[b])
            self.cells[o:o + self.ncell[b]].copy_(cells_list[u].reshape(-1))
        s2 = np.asarray(sigma2_list, np.float32)[self.perm]
        self.sigma2.copy_(torch.as_tensor(s2))

    # -- launch configuration ----------------------------------------------
    def set_config(self, cluster, threads):
        torch = _torch()
        self.plans = [csr_plan(r, n, cluster) for r, n in self.codes]
        idx = {code: i for i, code in enumerate(self.codes)}
        bplan = [idx.get((r, n), 0) for n, m, r in self.specs]   # CSR blocks only
        self.a["bplan"] = torch.tensor(bplan, dtype=torch.int32, device=self.dev)
        nbytes = ctypes.c_int64()
        N.call("atsc3_ldpc_batch_desc_bytes", len(self.plans), ctypes.byref(nbytes))
        self.desc = torch.empty(nbytes.value, dtype=torch.uint8, device=self.dev)
        arr = (ctypes.c_void_p * len(self.plans))(*[p.handle.value for p in self.plans])
        cl, sm = ctypes.c_int32(), ctypes.c_int32()
        N.call("atsc3_ldpc_batch_prepare", arr, len(self.plans),
               self.desc.data_ptr(), ctypes.byref(cl), ctypes.byref(sm))
        self.cluster, self.smem, self.threads = cl.value, sm.value, threads
        self.config = {"cluster": self.cluster, "threads": threads,
                       "smem_bytes": self.smem}
        self.graph = None

    # -- the three launches -------------------------------------------------
    def launch(self, stream=None):
        torch = _torch()
        st = stream if stream is not None else torch.cuda.current_stream(self.dev).cuda_stream
        a = self.a
        zf = torch.view_as_real(self.cells)
        self.counter.zero_()
        main = torch.cuda.current_stream(self.dev) if stream is None else None
        N.call("atsc3_demap_batch", zf.data_ptr(), a["cell_off"].data_ptr(),
               a["ncell"].data_ptr(), a["nbits"].data_ptr(),
               self.t_pts.data_ptr(), a["pts_off"].data_ptr(),
               self.sigma2.data_ptr(), self.t_lq.data_ptr(),
               a["lq_off"].data_ptr(), self.llr.data_ptr(),
               a["llr_off"].data_ptr(), a["chunk_blk"].data_ptr(),
               a["chunk_start"].data_ptr(), self.nchunks, self.max_nbits, st)
        # fork: one stream per quasi-cyclic group and one for the CSR queue
        if main is not None and self.groups:
            for s_ in self.side:
                s_.wait_stream(main)
        for gi, (plan, first, cnt, n) in enumerate(self.groups):
            gst = self.side[gi].cuda_stream if main is not None else st
            N.call("atsc3_ldpc_qce_decode", plan.handle,
                   self.llr.data_ptr() + 4 * int(self.llr_off[first]), n, cnt,
                   int(self.iters), float(self.alpha), 0, None, 0,
                   self.hard.data_ptr() + int(self.hard_off[first]),
                   self.hb[first], self.conv.data_ptr() + first,
                   self.its.data_ptr() + 4 * first, self.bad.data_ptr() + 4 * first,
                   int(self.gshape[gi][1]), gst)
        if self.ncsr:
            cst = self.side[-1].cuda_stream if (main is not None and self.groups) else st
            N.call("atsc3_ldpc_batch_decode", self.desc.data_ptr(), self.cluster,
                   self.smem, a["bplan"].data_ptr(), a["order"].data_ptr(),
                   self.ncsr, self.llr.data_ptr(), a["llr_off"].data_ptr(),
                   self.hard.data_ptr(), a["hard_off"].data_ptr(),
                   self.conv.data_ptr(), self.its.data_ptr(), self.bad.data_ptr(),
                   int(self.iters), float(self.alpha), self.counter.data_ptr(),
                   self.threads, 0, cst)
        if main is not None and self.groups:
            for s_ in self.side:
                main.wait_stream(s_)
        N.call("atsc3_bch_batch", self.hard.data_ptr(), a["hard_off"].data_ptr(),
               a["kldpc"].data_ptr(), self.t_rt.data_ptr(), a["rt_off"].data_ptr(),
               self.t_scr.data_ptr(), a["kpay"].data_ptr(),
               self.payload.data_ptr(), a["pay_off"].data_ptr(),
               self.syn.data_ptr(), self.ok.data_ptr(), self.nblk, st)

    def capture(self):
        torch = _torch()
        self.launch()                     # warm: attributes, occupancy cache
        torch.cuda.synchronize(self.dev)
        s = torch.cuda.Stream(self.dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.launch()
        torch.cuda.synchronize(self.dev)
        self.graph = g
        return g

    def run(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def set_group_shape(self, gi, cluster, threads):
        """Launch shape of edge-buffer group gi: cluster size (0 = the
        smallest that holds a codeword) and CTA threads (0 = default, 512 or
        1024).  Raises FecError (-4) when the code does not fit that shape."""
        plan, first, cnt, n = self.groups[gi]
        rate = self.specs[first][2]
        p = qce_plan(rate, n, cluster)
        if p is None:
            raise N.FecError("atsc3_ldpc_qce_plan_create2", -4,
                             f"{n} {rate} does not fit {cluster} CTAs")
        self.groups[gi] = (p, first, cnt, n)
        self.gshape[gi] = (cluster, threads)
        self.graph = None

    def _time(self, reps):
        torch = _torch()
        self.capture()
        self.graph.replay()
        torch.cuda.synchronize(self.dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            self.graph.replay()
        e1.record()
        torch.cuda.synchronize(self.dev)
        return e0.elapsed_time(e1) / reps

    def signature(self):
        return (tuple(sorted(self.specs)), self.iters, len(self.groups))

    def autotune(self, reps=3, clusters=None, threads=(512, 1024), shapes=None):
        """Time the captured graph over the launch knobs and keep the
        fastest; returns the table of timings (ms), keyed ("csr", cluster,
        threads) for the persistent CSR launch and (code, cluster, threads)
        for each edge-buffer group.  The CSR launch (when it has blocks) is
        swept over cluster x threads; then each edge-buffer group, most edges
        first, over its cluster size (the smallest that holds a codeword and
        the next two) x threads with the others fixed (coordinate descent).
        Results are cached per batch signature."""
        torch = _torch()
        key = self.signature()
        if key in _TUNED:
            (csr_best, gbest), table = _TUNED[key]
            self.set_config(*csr_best)
            for gi, shp in enumerate(gbest):
                self.set_group_shape(gi, *shp)
            self.capture()
            return table
        table = {}
        if self.ncsr:
            clusters = clusters or [c for c in (1, 2, 4, 8, 16) if c >= self.cl_min]
            for cl in clusters:
                for th in threads:
                    try:
                        self.set_config(cl, th)
                        table[("csr", cl, th)] = self._time(reps)
                    except N.FecError:
                        continue
            best = min((k for k in table if k[0] == "csr"), key=table.get)
            self.set_config(best[1], best[2])
        csr_best = (self.cluster, self.threads)
        base = self._time(reps)
        order = sorted(range(len(self.groups)),
                       key=lambda g: -self.groups[g][2] * self.groups[g][3])
        for gi in order:
            plan, first, cnt, n = self.groups[gi]
            code = f"{n} {self.specs[first][2]}"
            c0 = int(plan.info["cluster"])
            cur = self.gshape[gi]
            cands = shapes or [(c, t) for c in (c0, c0 + 1, c0 + 2)
                               for t in threads]
            best_t, best_s = base, cur
            for cl, th in cands:
                try:
                    self.set_group_shape(gi, cl, th)
                    t = self._time(reps)
                except N.FecError:
                    continue
                table[(code, cl, th)] = t
                if t < best_t:
                    best_t, best_s = t, (cl, th)
            self.set_group_shape(gi, *best_s)
            base = best_t
        _TUNED[key] = ((csr_best, list(self.gshape)), table)
        self.capture()
        return table

    # -- results -------------------------------------------------------------
    def results(self):
        """Per block: payload bytes, conv, its, bad, ok (numpy)."""
        pay = self.payload.cpu().numpy()
        out = [None] * self.nblk
        conv, its, bad, ok = (t.cpu().numpy() for t in (self.conv, self.its,
                                                        self.bad, self.ok))
        for b in range(self.nblk):
            o = int(self.pay_off[b])
            out[int(self.perm[b])] = {"payload": pay[o:o + self.kpays[b] // 8],
                                      "conv": int(conv[b]), "its": int(its[b]),
                                      "bad": int(bad[b]), "ok": int(ok[b])}
        return out
