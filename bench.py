#!/usr/bin/env python3
"""Throughput of the B200 FEC back end on the frame-scale workload.

Workload (one step = one frame): 1,216,939 complex64 cells per frame, 16-NUC
with the 64800-bit rate-6/15 LDPC code, i.e. 75 whole FEC blocks of 16,200
cells (the remaining 1,939 cells of the frame do not fill a block).  Each
cell has a Rayleigh channel gain |CN(0,1)| that the equaliser removed, so the
noise variance N0/h^2 is passed per cell.  Frame f is at Es/N0 =
4.0 + 0.5*(f mod 9) dB (the 4..8 dB sweep), normalised min-sum alpha 0.75,
at most 50 iterations, early stop on a zero syndrome, then BCH + descramble.
Payload bits are seeded uniform random, encoded by the package's GPU
transmitter; every step reads a different frame (1.87 GB of distinct frames
for the default 128 steps, far above the 126 MB L2).

metric = decoded info Mbit/s = 75 * 25728 payload bits per frame / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  `--impl reference` times the reference's own
CPU path on the host cores instead (demap + de-interleave in numpy, the
reference's compiled lab/ldpc_kernel.c, BCH), on a bounded sample per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

N_INNER, MOD, RATE = 64800, "16QAM", "6/15"
CELLS_PER_FRAME = 1_216_939
ESN0 = [4.0 + 0.5 * i for i in range(9)]
ITERS, ALPHA = 50, 0.75
METRIC = ("decoded info Mbit/s on 1 B200 at FER<=1e-4; mean iterations, "
          "learned vs plain min-sum")
PEAKS = os.path.join(HERE, "MEASURED_PEAKS.json")


def peaks():
    try:
        with open(PEAKS) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_frames(nframes, seed, device):
    """Seeded frames: cells (F, 75, 16200) complex64, sigma2 same shape f32."""
    import torch
    from atsc3_b200 import codes as C
    from atsc3_b200 import synth
    nblk = CELLS_PER_FRAME // C.cells_per_block(N_INNER, MOD)
    tx = synth.Transmitter(N_INNER, MOD, RATE, device=device, chunk=128)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    cells = torch.empty((nframes, nblk, tx.ncell), dtype=torch.complex64,
                        device=device)
    sig = torch.empty((nframes, nblk, tx.ncell), dtype=torch.float32,
                      device=device)
    for f in range(nframes):
        pay = torch.randint(0, 2, (nblk, tx.kp), generator=g, device=device,
                            dtype=torch.uint8)
        x, _ = tx.encode(pay)
        y, s2 = synth.channel(x, ESN0[f % len(ESN0)], "rayleigh", g)
        cells[f] = y
        sig[f] = s2
    return cells, sig, nblk, tx.kp


def cpu_reference_decode(cells, sig, threads, mod=None, rate=None, n=None,
                         full=False):
    """The reference's CPU path on host cores, through the oracle: float32
    demap (numpy, the lab/m44_ldm.py:2431-2494 arithmetic) with per-cell
    sigma2, de-interleave, the reference's own lab/ldpc_kernel.c compiled
    into oracle/_ref (thread sub-batches, as lab/m44_ldm.py:2558-2576), BCH
    as a packed GF(2) product (lab/m9_accel.py:212-236).  Returns
    (#blocks BCH-clean, its), or with full=True the dict of every output
    (bits, conv, its, bad, ok, payload)."""
    import oracle
    from concurrent.futures import ThreadPoolExecutor
    from atsc3_b200 import codes as C
    mod, rate, n = mod or MOD, rate or RATE, n or N_INNER
    pts = C.points_for(mod, rate)
    nb = C.MOD_BITS[mod]
    lq = C.bicm_map(n, mod, rate)
    tabs = C.csr(rate, n)
    K = C.kldpc(rate, n)
    nblk = cells.shape[0]
    scalar = np.ndim(sig) == 0
    with ThreadPoolExecutor(threads) as ex:
        q = np.concatenate(list(ex.map(
            lambda b: oracle.demap(cells[b:b + 1], pts, nb,
                                   sig if scalar else sig[b:b + 1]),
            range(nblk))))
    lam = oracle.deinterleave(q, lq, n)
    bits, conv, its, bad = oracle.flood_ref(lam, tabs, n, iters=ITERS,
                                            alpha=ALPHA, threads=threads)
    syn = oracle.bch_syndrome_fast(bits[:, :K], n)
    if not full:
        return sum(1 for s in syn if s == 0), its
    kp = C.kpayload(rate, n)
    pay = np.packbits(bits[:, :kp] ^ C.scrambler_sequence(kp)[None, :], axis=1)
    return {"bits": bits, "conv": np.asarray(conv, bool), "its": its,
            "bad": bad, "ok": np.array([s == 0 for s in syn]),
            "payload": pay}


REF_TREE = os.path.join(HERE, "baseline", "_ref")


class ReferenceCpuPath:
    """The reference receiver's own CPU FEC path, imported from the
    unmodified copy in baseline/_ref (laid out by `python oracle/build.py
    --ref-tree`; absent -> RuntimeError):

    * m44_ldm._point_metric (lab/m44_ldm.py:2431-2451), the float32 point
      metric, and the per-bit minima of demap_batch_qam (:2483-2486), with
      the raw minima difference divided by the per-cell sigma2 (the
      lab/m9_fast.py:1096-1115 convention; demap_batch_qam itself only
      estimates a per-row sigma2);
    * lam[:, ch.lam_of_q] = q (lab/m44_ldm.py:2363), ch = m6_bicm.PlpChain;
    * m44_ldm.ldpc_batch (:2497-2555) at the single rung alpha = 0.75: the
      compiled lab/ldpc_kernel.c over thread sub-batches (SP rescue off);
    * m9_accel.bch_syndrome_batch (lab/m9_accel.py:212-236) and the
      descramble + pack of lab/m44_ldm.py:2374-2377.
    """

    def __init__(self, threads, mod=None, rate=None, n=None):
        from concurrent.futures import ThreadPoolExecutor
        lab = os.path.join(REF_TREE, "lab")
        if not (os.path.exists(os.path.join(lab, "m44_ldm.py")) and
                os.path.exists(os.path.join(lab, "ldpc_kernel.so"))):
            raise RuntimeError("baseline/_ref is not laid out "
                               "(python oracle/build.py --ref-tree)")
        os.environ.pop("ATSC3_LDM_SP", None)        # SP rescue off (default)
        os.environ.pop("ATSC3_LDPC_KERNEL", None)   # compiled kernel on
        for pth in (REF_TREE, lab):
            if pth not in sys.path:
                sys.path.insert(0, pth)
        import m3_ldpc
        import m4_scrambler
        import m6_bicm
        import m9_accel
        import m44_ldm
        if m3_ldpc._kernel_lib() is None:
            raise RuntimeError("the reference's compiled ldpc_kernel.so did "
                               "not load (its numpy fallback would run)")
        if m44_ldm.SP_RESCUE:
            raise RuntimeError("ATSC3_LDM_SP rescue is on")
        self.M44, self.BCH = m44_ldm, m9_accel
        mod, rate, n = mod or MOD, rate or RATE, n or N_INNER
        self.ch = ch = m6_bicm.PlpChain(n, mod, rate, iters=ITERS)
        pts = m6_bicm.points_for(mod, rate)
        self.pr = np.asarray(pts.real, np.float32)
        self.pi = np.asarray(pts.imag, np.float32)
        self.p2 = (pts.real ** 2 + pts.imag ** 2).astype(np.float32)
        self.nb = ch.mod_bits
        self.threads = threads
        self.ex = ThreadPoolExecutor(threads)
        self.seq = m4_scrambler.sequence(ch.kpayload)
        # BCH tables built before any clock starts (lab/m9_accel.py:169-194)
        m9_accel.bch_syndrome_batch(np.zeros((1, ch.kldpc), np.uint8),
                                    ch.ninner)

    def _demap(self, cells, sig, out, lo, hi):
        k, ncell = hi - lo, cells.shape[1]
        z = cells[lo:hi]
        zr = np.asarray(z.real, np.float32)
        zi = np.asarray(z.imag, np.float32)
        q = self.M44._point_metric(zr.ravel(), zi.ravel(), self.pr, self.pi,
                                   self.p2)
        m = q.shape[1]
        s2 = sig[lo:hi] if np.ndim(sig) else sig
        for i in range(self.nb):
            # label bit i (MSB first) splits the m points into 2^i runs of
            # (m >> i) labels: the first half of each run has the bit 0
            qb = q.reshape(k, ncell, 1 << i, 2, m >> (i + 1))
            one = qb[:, :, :, 1, :].min(axis=(2, 3))
            zero = qb[:, :, :, 0, :].min(axis=(2, 3))
            out[lo:hi, :, i] = (one - zero) / s2

    def decode(self, cells, sig, chunk=4):
        """(nblk, ncell) complex64 cells, per-cell float32 sigma2 (or a
        scalar) -> dict(bits, conv, bad, ok, payload) of numpy arrays."""
        ch = self.ch
        nblk, ncell = cells.shape
        q = np.empty((nblk, ncell, self.nb), np.float32)
        jobs = [(lo, min(nblk, lo + chunk)) for lo in range(0, nblk, chunk)]
        list(self.ex.map(lambda j: self._demap(cells, sig, q, *j), jobs))
        lam = np.empty((nblk, ch.ninner), np.float32)
        lam[:, ch.lam_of_q] = q.reshape(nblk, -1)
        bits, conv, bad = self.M44.ldpc_batch(lam, ch, None, ITERS, self.ex,
                                              self.threads, alpha=ALPHA)
        nouter = bits[:, :ch.kldpc]
        syn = self.BCH.bch_syndrome_batch(nouter, ch.ninner)
        pay = np.packbits(nouter[:, :ch.kpayload] ^ self.seq[None, :], axis=1)
        return {"bits": bits, "conv": np.asarray(conv, bool), "bad": bad,
                "ok": np.array([s == 0 for s in syn]), "payload": pay}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path on the host cores, rank 0
    only, on the same frames (same seed) as rank 0 of the GPU arm, every
    step one whole 75-block frame.  The reference receiver's own Python
    from baseline/_ref (ReferenceCpuPath) when it is laid out, else the
    oracle route around the reference's compiled kernel (oracle/_ref)."""
    if rank != 0:
        return None
    import torch
    from atsc3_b200 import codes as C
    threads = os.cpu_count() or 1
    kp = C.kpayload(RATE, N_INNER)
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    nsteps = args.steps + args.warmup
    cells, sig, nblk, _ = make_frames(nsteps, args.seed, dev)
    cells = cells.cpu().numpy()
    sig = sig.cpu().numpy()
    try:
        path = ReferenceCpuPath(threads)
        what = (f"the reference receiver's own Python from baseline/_ref: "
                f"m44_ldm._point_metric + per-bit minima / per-cell sigma2, "
                f"lam[:, lam_of_q] = q, m44_ldm.ldpc_batch (lab/ldpc_kernel.c "
                f"compiled -O3 -ffp-contract=off, {threads} thread "
                f"sub-batches), m9_accel.bch_syndrome_batch, descramble")

        def dec(c, g):
            return path.decode(c, g)
    except RuntimeError as e:
        what = (f"oracle route ({e}): numpy float32 demap, lab/ldpc_kernel.c "
                f"compiled -O3 -ffp-contract=off over {threads} threads "
                f"(oracle/_ref), packed BCH")

        def dec(c, g):
            return cpu_reference_decode(c, g, threads, full=True)
    times, ok, conv = [], 0, 0
    for s in range(nsteps):
        t0 = time.perf_counter()
        o = dec(cells[s], sig[s])
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
            ok += int(np.sum(o["ok"]))
            conv += int(np.sum(o["conv"]))
    tot = sum(times)
    value = args.steps * nblk * kp / tot / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value,
            "unit": "Mbit/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": config(nblk),
            "cpu_baseline": {"value": value, "unit": "Mbit/s",
                             "cores": threads, "kind": "reference",
                             "sample": f"every step one whole frame ({nblk} "
                                       f"blocks, the GPU arm's frames); "
                                       + what},
            "e2e": {"value": value, "unit": "Mbit/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "bch_ok_blocks": ok, "converged_frac": conv / (args.steps * nblk)}
    return line


def config(blocks):
    return {"workload": "frame-scale plain decode: 64800-bit LDPC rate 6/15, "
                        "16-NUC, 1,216,939 cells/frame -> 75 FEC blocks, "
                        "Rayleigh |CN(0,1)| gain with per-cell sigma2, "
                        "Es/N0 4..8 dB step 0.5 cycling per frame",
            "code": "64800 6/15 (Type B)", "constellation": "NUC_16_6/15",
            "blocks_per_step": blocks, "cells_per_frame": CELLS_PER_FRAME,
            "esn0_db": ESN0, "alpha": ALPHA, "iters_max": ITERS,
            "early_stop": "zero syndrome", "sigma2": "per cell",
            "parallelism": "blocks sharded per GPU (no exchange)",
            "l2": "inputs larger than L2: a distinct 14.6 MB frame per step "
                  "(1.87 GB over the default 128 steps)"}


def decode_frame(pipe, cells, sig, out, stream, weights=None):
    """One frame on one stream: demap -> LDPC -> BCH into `out` (3 launches)."""
    from atsc3_b200 import bch as BCH
    from atsc3_b200 import demap as DM
    from atsc3_b200 import ldpc as LDPC
    nblk = cells.shape[0]
    ws = pipe._buffers(nblk)
    st = stream.cuda_stream
    DM.demap(cells, MOD, RATE, sigma2=sig, n=N_INNER, out=ws["lam"], stream=st)
    o = dict(ws)
    o.update(out)
    LDPC.decode_flood(pipe.plan, ws["lam"], iters=ITERS, alpha=ALPHA,
                      want_bits=False, want_hard=True, threads=pipe.threads,
                      out=o, stream=st, weights=weights)
    BCH.bch_check(ws["hard"], pipe.kldpc, N_INNER, pipe.kpayload, out=o,
                  stream=st)


def learned_weights(dev):
    """Committed learned weights for this code, if any: (weights, manifest)."""
    path = os.path.join(HERE, "atsc3_b200", "data",
                        f"weights_{RATE.replace('/', '_')}_{MOD}.pt")
    if not os.path.exists(path):
        return None, None
    from atsc3_b200 import learned as LR
    al, be, man = LR.load_weights(path, dev)
    code = LR.WmsCode(RATE, N_INNER, dev)
    return LR.inference_weights(al, be, code.buckets, dev), man


def run_gpu(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from atsc3_b200 import codes as C
    from atsc3_b200 import shard
    from atsc3_b200.pipeline import FecPipeline
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    K, W = args.steps, args.warmup
    nframes = K + W
    cells, sig, nblk, kp = make_frames(nframes, args.seed + 1000 * rank, dev)
    S = max(1, args.streams)
    # one pipeline (workspace) per stream; they share the decoder plan
    pipes = [FecPipeline(N_INNER, MOD, RATE, iters=ITERS, alpha=ALPHA,
                         cluster=args.cluster, threads=args.threads, device=dev,
                         kind=args.decoder)
             for _ in range(S)]
    streams = [torch.cuda.Stream(dev) for _ in range(S)]

    def new_out():
        return {"conv": torch.empty(nblk, dtype=torch.uint8, device=dev),
                "its": torch.empty(nblk, dtype=torch.int32, device=dev),
                "bad": torch.empty(nblk, dtype=torch.int32, device=dev),
                "ok": torch.empty(nblk, dtype=torch.uint8, device=dev),
                "syn": torch.empty((nblk, 6), dtype=torch.int32, device=dev),
                "payload": torch.empty((nblk, kp // 8), dtype=torch.uint8,
                                       device=dev)}
    outs = [new_out() for _ in range(nframes)]
    main = torch.cuda.current_stream(dev)
    for f in range(W):
        decode_frame(pipes[f % S], cells[f], sig[f], outs[f], streams[f % S])
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ends = [torch.cuda.Event() for _ in range(S)]
    clk = Clocks(local_rank) if rank == 0 else None
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if clk:
        clk.start()
    e0.record(main)
    for st in streams:
        st.wait_event(e0)
    for s in range(K):
        f = W + s
        decode_frame(pipes[f % S], cells[f], sig[f], outs[f], streams[f % S])
    for st, ev in zip(streams, ends):
        ev.record(st)
        main.wait_event(ev)
    e1.record(main)
    torch.cuda.synchronize()
    clocks = clk.stop() if clk else None
    ms = e0.elapsed_time(e1)
    if world > 1:
        ms = shard.max_over_ranks(ms, device=dev)
        dist.barrier()
    conv = torch.stack([outs[W + s]["conv"] for s in range(K)]).cpu().numpy()
    its = torch.stack([outs[W + s]["its"] for s in range(K)]).cpu().numpy()
    ok = torch.stack([outs[W + s]["ok"] for s in range(K)]).cpu().numpy()
    total_bits = world * K * nblk * kp
    value = total_bits / (ms / 1e3) / 1e6
    # ---- per-stage device time, one stream, no overlap (roofline) ---------
    nprof = min(K, 9)
    stage_its, stage_hard, stage_flags = [], [], []
    E = [[torch.cuda.Event(enable_timing=True) for _ in range(4)]
         for _ in range(nprof)]
    from atsc3_b200 import bch as BCH, demap as DM, ldpc as LDPC
    p0 = pipes[0]
    ws = p0._buffers(nblk)
    # keep the GPU busy while the host enqueues the stage launches and their
    # events, so each interval is kernel time, not host launch gaps
    torch.cuda.synchronize()
    torch.cuda._sleep(200_000_000)
    for s in range(nprof):
        f = W + s
        E[s][0].record(main)
        DM.demap(cells[f], MOD, RATE, sigma2=sig[f], n=N_INNER, out=ws["lam"])
        E[s][1].record(main)
        o = dict(ws)
        LDPC.decode_flood(p0.plan, ws["lam"], iters=ITERS, alpha=ALPHA,
                          want_bits=False, want_hard=True, threads=p0.threads,
                          out=o)
        E[s][2].record(main)
        BCH.bch_check(ws["hard"], p0.kldpc, N_INNER, kp, out=o)
        E[s][3].record(main)
        stage_its.append(int(o["its"].sum()))
        # kept for the parity check: the full hard decisions of this frame
        # and its flags from this second, untimed decode
        stage_hard.append(ws["hard"][:, :N_INNER // 8].clone())
        stage_flags.append(torch.stack([o["conv"].int(), o["its"], o["bad"],
                                        o["ok"].int()]))
    torch.cuda.synchronize()
    stage = np.array([[E[s][0].elapsed_time(E[s][1]), E[s][1].elapsed_time(E[s][2]),
                       E[s][2].elapsed_time(E[s][3])] for s in range(nprof)])
    # ---- e2e: host buffers through the public API -------------------------
    e2e = run_e2e(pipes, streams, cells, sig, W, K, nblk, kp, dev, world)
    # ---- learned weights on the same frames (same decoder, early stop) -----
    learned = None
    w, man = learned_weights(dev)
    if w is not None:
        louts = [new_out() for _ in range(K)]
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
            torch.cuda.synchronize()
        e0.record(main)
        for st in streams:
            st.wait_event(e0)
        for s in range(K):
            f = W + s
            decode_frame(pipes[f % S], cells[f], sig[f], louts[s], streams[f % S],
                         weights=w)
        for st, ev in zip(streams, ends):
            ev.record(st)
            main.wait_event(ev)
        e1.record(main)
        torch.cuda.synchronize()
        lms = e0.elapsed_time(e1)
        if world > 1:
            lms = shard.max_over_ranks(lms, device=dev)
        lits = torch.stack([o["its"] for o in louts]).cpu().numpy()
        lok = torch.stack([o["ok"] for o in louts]).cpu().numpy()
        learned = {"value": world * K * nblk * kp / (lms / 1e3) / 1e6,
                   "unit": "Mbit/s", "mean_iters": float(lits.mean()),
                   "bch_fer": float((lok == 0).mean()),
                   "weights": {k: man[k] for k in ("rate", "mod", "iters",
                                                   "step", "seed")}}
    # ---- roofline of the dominant kernel (the LDPC decoder) ---------------
    ldpc_ms = float(stage[:, 1].mean())
    # on-chip exchange of the edge-buffer decoder: per edge and iteration one
    # 4-byte load of the variable-to-check value and one 4-byte store of the
    # message through distributed shared memory (the iterations of the
    # stage-timing frames, read from their outputs)
    nedges = int(C.csr(RATE, N_INNER)[1].shape[0])
    its_stage = float(np.mean(stage_its)) if stage_its else 0.0
    onchip = {"unit": "GB/s", "bytes_per_launch": 8 * nedges * its_stage,
              "achieved": 8 * nedges * its_stage / (ldpc_ms / 1e3) / 1e9,
              "what": "edge-slot exchange of the edge-buffer decoder, 8 B "
                      "per edge per iteration (a 4-byte load and a 4-byte "
                      "store); about half is served by the CTA's own shared "
                      "memory (columns placed with their rows), the rest "
                      "crosses the cluster's xbar",
              "peak_ncu": 9350.0,
              "peak_note": "xbar-to-L1 distributed shared memory bytes at "
                           "23.7% of peak = 2.22 TB/s (7.55 GB per launch) "
                           "in one ncu capture of this workload, i.e. about "
                           "9.35 TB/s (capture-derived peak)"}
    onchip["frac"] = onchip["achieved"] / onchip["peak_ncu"]
    # instruction issue, the decoder's actual bound (ncu: issue active ~60%,
    # not_selected and math-pipe throttle the leading stalls): warp
    # instructions per codeword-iteration from one ncu capture x the
    # iterations of the timed launch, against 4 schedulers per occupied SM
    issue = None
    if p0.plan.info.get("kind") == "qce" and its_stage:
        from atsc3_b200 import native as N
        cfg = np.zeros(4, np.int32)
        N.call("atsc3_ldpc_qce_config", p0.plan._h, 0, 0, cfg.ctypes.data)
        sms = int(cfg[0]) * int(cfg[1])
        mhz = float((clocks or {}).get("sm_mhz") or 1965.0)
        instr = INSTR_PER_BLOCK_ITER * its_stage
        ach = instr / (ldpc_ms / 1e3) / 1e9
        peak = sms * 4 * mhz / 1e3
        issue = {"unit": "G warp instructions/s", "achieved": ach, "peak": peak,
                 "frac": ach / peak, "sms": sms, "instructions_per_launch": instr,
                 "instructions_source": "warp instructions per "
                                        "codeword-iteration, " + CAPTURE_NOTE,
                 "what": "warp instructions per codeword-iteration (one ncu "
                         "capture) x the launch's iterations / launch time; "
                         "peak = 4 schedulers x SM clock x the SMs the "
                         "clusters occupy"}
    b_ldpc = nblk * (4 * N_INNER + N_INNER // 8 + 9)
    hbm, peak_kind = peaks()
    achieved = b_ldpc / (ldpc_ms / 1e3) / 1e9
    fer = {f"{e:.1f}": [0, 0] for e in ESN0}
    for s in range(K):
        d = fer[f"{ESN0[(W + s) % len(ESN0)]:.1f}"]
        d[0] += int((ok[s] == 0).sum())
        d[1] += nblk
    if world > 1:   # block errors of every rank's frames
        keys = sorted(fer)
        tot = shard.sum_over_ranks([v for k in keys for v in fer[k]], device=dev)
        fer = {k: [tot[2 * i], tot[2 * i + 1]] for i, k in enumerate(keys)}
    # ---- what the parity check needs: the first nprof timed frames (one
    # per Es/N0 point), their cells and the GPU outputs of the timed run ---
    parity = None
    if rank == 0 and world == 1:
        fr = list(range(W, W + nprof))
        parity = {"frames": fr,
                  "esn0_db": [ESN0[f % len(ESN0)] for f in fr],
                  "cells": cells[W:W + nprof].cpu().numpy(),
                  "sig": sig[W:W + nprof].cpu().numpy(),
                  "conv": conv[:nprof].astype(bool), "its": its[:nprof],
                  "bad": torch.stack([outs[f]["bad"] for f in fr]).cpu().numpy(),
                  "ok": ok[:nprof].astype(bool),
                  "payload": torch.stack([outs[f]["payload"] for f in fr]).cpu().numpy(),
                  "hard": torch.stack(stage_hard).cpu().numpy(),
                  "stage_flags": torch.stack(stage_flags).cpu().numpy()}
    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Mbit/s",
                "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms / K,
                "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config(nblk),
                "roofline": {"bound": "hbm", "achieved": achieved,
                             "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm,
                             "traffic": (TRAFFIC_PER_BLOCK * nblk
                                         if TRAFFIC_PER_BLOCK else None),
                             "traffic_source": "dram__bytes_read.sum + "
                                               "dram__bytes_write.sum, "
                                               + CAPTURE_NOTE,
                             "kernel": KERNEL_NAMES.get(p0.plan.info.get("kind"),
                                                        "ldpc_flood_kernel (CSR flooding)"),
                             "peak_kind": peak_kind,
                             "bytes_per_launch": b_ldpc,
                             "ms_per_launch": ldpc_ms,
                             "onchip": onchip,
                             "issue": issue},
                "stage_ms": {"demap": float(stage[:, 0].mean()),
                             "ldpc": ldpc_ms,
                             "bch": float(stage[:, 2].mean())},
                "streams": S,
                "gpu_launches": 3 * K,
                "clocks": clocks, "e2e": e2e,
                "mean_iters": float(its.mean()),
                "converged_frac": float(conv.mean()),
                "fer_bch_by_esn0": {k: v[0] / v[1] for k, v in sorted(fer.items())
                                    if v[1]},
                "learned": learned,
                "plan": p0.plan.info}
    return line, parity


KERNEL_NAMES = {"qce": "ldpc_qce_kernel (quasi-cyclic flooding, edge-buffer layout)",
                "qc": "ldpc_qc_kernel (quasi-cyclic flooding, record layout)"}

# Constants taken from one ncu capture of the edge-buffer decoder on this
# workload (one 75-block launch of the 64800 6/15 frame, --clock-control
# none); the bench line labels them as capture-derived, and they are
# re-taken whenever the kernel changes.
# DRAM bytes (read + write) per 64800-bit block of the LDPC launch:
# dram__bytes_read.sum + dram__bytes_write.sum / 75.
TRAFFIC_PER_BLOCK = 19_602_688 / 75
# warp instructions (smsp__inst_executed.sum) per codeword-iteration:
# the launch's count / (75 blocks x its 50 iterations).
INSTR_PER_BLOCK_ITER = 1_664_781_981 / 3750
CAPTURE_NOTE = ("constant from one ncu capture of a 75-block launch of this "
                "workload (not measured by this run)")


def run_e2e(pipes, streams, cells, sig, W, K, nblk, kp, dev, world):
    """Same metric through FecPipeline.decode with pinned host buffers: per
    step the H2D copy of its cells + sigma2, the decode, and the D2H copy of
    the payload bytes and per-block flags, all on the step's stream (steps
    alternate over the pipelines' streams, so one step's copies overlap the
    other's decode)."""
    import torch
    S = len(pipes)
    nh = min(8, K)
    hc = [cells[W + s].cpu().pin_memory() for s in range(nh)]
    hs = [sig[W + s].cpu().pin_memory() for s in range(nh)]
    hp = torch.empty((K, nblk, kp // 8), dtype=torch.uint8).pin_memory()
    hf = torch.empty((K, 4, nblk), dtype=torch.int32).pin_memory()
    dc = [torch.empty_like(cells[0]) for _ in range(S)]
    ds = [torch.empty_like(sig[0]) for _ in range(S)]
    flags = [torch.empty((4, nblk), dtype=torch.int32, device=dev)
             for _ in range(S)]
    main = torch.cuda.current_stream(dev)

    def step(s):
        i = s % S
        with torch.cuda.stream(streams[i]):
            dc[i].copy_(hc[s % nh], non_blocking=True)
            ds[i].copy_(hs[s % nh], non_blocking=True)
            ws = pipes[i].decode(dc[i], ds[i])
            f = flags[i]
            f[0].copy_(ws["conv"])
            f[1].copy_(ws["its"])
            f[2].copy_(ws["bad"])
            f[3].copy_(ws["ok"])
            hp[s].copy_(ws["payload"], non_blocking=True)
            hf[s].copy_(f, non_blocking=True)

    for s in range(2 * S):   # warm the pinned path
        step(s % K)
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ends = [torch.cuda.Event() for _ in range(S)]
    e0.record(main)
    for st in streams:
        st.wait_event(e0)
    for s in range(K):
        step(s)
    for st, ev in zip(streams, ends):
        ev.record(st)
        main.wait_event(ev)
    e1.record(main)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:                      # the slowest rank's time, as for `value`
        from atsc3_b200 import shard
        ms = shard.max_over_ranks(ms, device=dev)
    h2d = nblk * pipes[0].ncell * (8 + 4)
    d2h = nblk * (kp // 8) + 4 * nblk * 4
    return {"value": world * K * nblk * kp / (ms / 1e3) / 1e6, "unit": "Mbit/s",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "ms_per_step": ms / K, "streams": S,
            "bch_ok_blocks": int(hf[:, 3].sum())}


def cpu_baseline(par):
    """The reference CPU path timed on the host cores over the parity
    frames (the first timed frames, one whole 75-block frame per Es/N0
    point, 675 blocks): the reference receiver's own Python from
    baseline/_ref when laid out, else the oracle route around the
    reference's compiled kernel.  Returns (cpu_baseline dict, outputs)."""
    from atsc3_b200 import codes as C
    threads = os.cpu_count() or 1
    kp = C.kpayload(RATE, N_INNER)
    c = par["cells"].reshape(-1, par["cells"].shape[-1])
    g = par["sig"].reshape(-1, par["sig"].shape[-1])
    try:
        path = ReferenceCpuPath(threads)
        what = ("the reference receiver's own Python from baseline/_ref "
                "(m44_ldm._point_metric + per-bit minima / per-cell sigma2, "
                "m44_ldm.ldpc_batch over lab/ldpc_kernel.c compiled -O3 "
                "-ffp-contract=off, m9_accel.bch_syndrome_batch, descramble)")
    except RuntimeError as e:
        path = None
        what = (f"oracle route ({e}): numpy float32 demap + lab/ldpc_kernel.c "
                f"(-O3 -ffp-contract=off, oracle/_ref) + packed BCH")
    t0 = time.perf_counter()
    out = (path.decode(c, g) if path is not None else
           cpu_reference_decode(c, g, threads, full=True))
    dt = time.perf_counter() - t0
    nf = par["cells"].shape[0]
    return ({"value": c.shape[0] * kp / dt / 1e6, "unit": "Mbit/s",
             "cores": threads, "kind": "reference",
             "sample": f"{c.shape[0]} blocks: the first {nf} timed frames "
                       f"(one whole frame per Es/N0 point "
                       f"{par['esn0_db'][0]:g}..{par['esn0_db'][-1]:g} dB), "
                       f"{what}, {threads} threads; {dt:.1f} s wall"},
            out)


def parity_check(par, ref_py):
    """GPU outputs of the timed frames against the reference on the same
    blocks: the oracle route around the reference's compiled kernel
    (bits, conv, its, bad, BCH ok, payload bytes) and, where it ran, the
    reference's own Python path (all of those but its, which ldpc_batch
    does not return).  Mismatch counts are blocks."""
    threads = os.cpu_count() or 1
    c = par["cells"].reshape(-1, par["cells"].shape[-1])
    g = par["sig"].reshape(-1, par["sig"].shape[-1])
    nb = c.shape[0]
    gpu = {"bits": par["hard"].reshape(nb, -1),
           "conv": par["conv"].reshape(-1), "its": par["its"].reshape(-1),
           "bad": par["bad"].reshape(-1), "ok": par["ok"].reshape(-1),
           "payload": par["payload"].reshape(nb, -1)}
    sf = par["stage_flags"]                    # (frames, 4, blocks)
    rerun = int((sf[:, 0].astype(bool).reshape(-1) != gpu["conv"]).sum() +
                (sf[:, 1].reshape(-1) != gpu["its"]).sum() +
                (sf[:, 2].reshape(-1) != gpu["bad"]).sum() +
                (sf[:, 3].astype(bool).reshape(-1) != gpu["ok"]).sum())

    def mism(ref, keys):
        out = {}
        for k in keys:
            r = ref[k]
            if k == "bits":
                r = np.packbits(r, axis=1)
            a, b = gpu[k], r
            out[k] = int((a != b).reshape(nb, -1).any(axis=1).sum())
        return out
    o = cpu_reference_decode(c, g, threads, full=True)
    res = {"blocks": nb, "frames": par["frames"], "esn0_db": par["esn0_db"],
           "vs_reference_kernel": mism(o, ("bits", "conv", "its", "bad",
                                            "ok", "payload")),
           "gpu_rerun_flag_mismatch": rerun,
           "reference_kernel": "lab/ldpc_kernel.c compiled -O3 "
                               "-ffp-contract=off (oracle/_ref), float32 "
                               "demap with per-cell sigma2, packed BCH"}
    if ref_py is not None and "its" not in ref_py:
        res["vs_reference_python"] = mism(ref_py, ("bits", "conv", "bad",
                                                   "ok", "payload"))
    tot = sum(res["vs_reference_kernel"].values()) + rerun
    tot += sum(res.get("vs_reference_python", {}).values())
    res["mismatch"] = tot
    res["mean_iters"] = float(gpu["its"].mean())
    res["converged_blocks"] = int(gpu["conv"].sum())
    return res


def run_uneven(args):
    """Config 3: 512 seeded blocks with random code length, rate and
    constellation (1024/4096 points: uniform-QAM stand-ins), Es/N0 = the
    measured threshold + 1 dB (atsc3_b200/data/thresholds.json), AWGN.  One
    persistent launch per stage replayed as a CUDA graph with the autotuned
    launch shape, against per-MODCOD sequential launches of FecPipeline."""
    import torch
    from atsc3_b200 import codes as C
    from atsc3_b200 import synth, thresholds
    from atsc3_b200.batch import UnevenBatch
    from atsc3_b200.pipeline import FecPipeline
    rng = np.random.default_rng(args.seed)
    mcs = thresholds.modcods()
    specs = [mcs[i] for i in rng.integers(0, len(mcs), args.blocks)]
    g = torch.Generator(device="cuda")
    g.manual_seed(args.seed)
    cells, s2s = [], []
    for n, m, r in specs:
        tx = synth.Transmitter(n, m, r, device="cuda")
        pay = torch.randint(0, 2, (1, tx.kp), generator=g, device="cuda",
                            dtype=torch.uint8)
        x, _ = tx.encode(pay)
        y, s2 = synth.channel(x, thresholds.lookup(n, m, r) + 1.0, "awgn", g)
        cells.append(y[0])
        s2s.append(float(s2))
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)

    def timed(ub):
        for _ in range(args.warmup):
            ub.run()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            ub.run()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    # every block on the CSR queue (one persistent launch)
    ub_csr = UnevenBatch(specs, iters=ITERS, alpha=ALPHA, hybrid=False)
    ub_csr.load(cells, s2s)
    ub_csr.autotune(reps=2)
    ms_csr = timed(ub_csr)
    # per-code edge-buffer launches (every A/322 code) beside the CSR queue
    ub = UnevenBatch(specs, iters=ITERS, alpha=ALPHA)
    ub.load(cells, s2s)
    ms_default = timed(ub)
    table = ub.autotune(reps=2)
    ms = timed(ub)
    tuned_shapes = {f"{ub.groups[g][3]} {ub.specs[ub.groups[g][1]][2]}": list(ub.gshape[g])
                    for g in range(len(ub.groups))}
    res = ub.results()
    # every code on one shared launch shape (the largest cluster any code
    # needs, 512 threads: what one launch over all codes would have to use)
    cl_all = max(int(g[0].info["cluster"]) for g in ub.groups) if ub.groups else 0
    ms_shared = None
    if ub.groups:
        for g in range(len(ub.groups)):
            ub.set_group_shape(g, cl_all, 512)
        ms_shared = timed(ub)
    bits = sum(C.kpayload(r, n) for n, m, r in specs)
    # per-MODCOD sequential launches (eager)
    groups = {}
    for b, sp in enumerate(specs):
        groups.setdefault(sp, []).append(b)
    pipes = {sp: FecPipeline(*sp, iters=ITERS, alpha=ALPHA) for sp in groups}
    stacks = {sp: torch.stack([cells[b] for b in idx]) for sp, idx in groups.items()}

    def seq():
        for sp, idx in groups.items():
            pipes[sp].decode(stacks[sp], s2s[idx[0]])
    for _ in range(args.warmup):
        seq()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        seq()
    e1.record()
    torch.cuda.synchronize()
    ms_seq = e0.elapsed_time(e1) / args.steps
    return {"metric": "uneven batch decoded info Mbit/s (CUDA graph, autotuned; per-code edge-buffer launches + one persistent CSR launch)",
            "value": bits / (ms / 1e3) / 1e6, "unit": "Mbit/s",
            "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
            "csr_only_mbit_s": bits / (ms_csr / 1e3) / 1e6,
            "quasi_cyclic_blocks": int(sum(g[2] for g in ub.groups)),
            "sequential_mbit_s": bits / (ms_seq / 1e3) / 1e6,
            "sequential_ms_per_step": ms_seq, "speedup_vs_sequential": ms_seq / ms,
            "blocks": len(specs), "distinct_modcods": len(groups),
            "untuned_mbit_s": bits / (ms_default / 1e3) / 1e6,
            "shared_shape_mbit_s": (bits / (ms_shared / 1e3) / 1e6) if ms_shared else None,
            "shared_shape": {"cluster": cl_all, "threads": 512},
            "tuned_shapes": tuned_shapes,
            "autotune_ms": {f"{k[0]} cl{k[1]} t{k[2]}": v for k, v in table.items()},
            "config": ub.config,
            "bch_ok": int(sum(r["ok"] for r in res)),
            "mean_iters": float(np.mean([r["its"] for r in res])),
            "data": "synthetic", "dtype": "f32"}


def run_frame_ti(args):
    """The frame workload received through a hybrid time interleaver (3 TI
    blocks of 25 FEC Blocks, A/322 7.1.5.4 twisted block interleaver): each
    step decodes one PLP cell stream with the de-interleave fused into the
    demapper's load (FecPipeline.decode_stream), against the same frames
    decoded from de-interleaved rows (FecPipeline.decode), frames alternating
    over --streams streams as in the frame bench (one-stream figures beside);
    per-stage device times of the gather demap and the row demap."""
    import torch
    from atsc3_b200 import demap as DM
    from atsc3_b200 import timeint as TI
    from atsc3_b200.pipeline import FecPipeline
    dev = torch.device("cuda")
    K, W = args.steps, args.warmup
    cells, sig, nblk, kp = make_frames(K + W, args.seed, dev)
    ti = TI.HybridTI(cells.shape[2], 25, nti=nblk // 25)
    streams = [ti.interleave(cells[f]) for f in range(K + W)]
    sstreams = [ti.interleave(sig[f]) for f in range(K + W)]
    p = FecPipeline(N_INNER, MOD, RATE, iters=ITERS, alpha=ALPHA, device=dev)
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)

    def timed(fn):
        for f in range(W):
            fn(f)
        torch.cuda.synchronize()
        e0.record()
        for s_ in range(K):
            fn(W + s_)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / K

    # frames alternate over S streams with a pipeline (workspace) each, as in
    # the frame bench: one LDPC launch's last round overlaps the next frame
    S = max(1, args.streams)
    pipes = [p] + [FecPipeline(N_INNER, MOD, RATE, iters=ITERS, alpha=ALPHA, device=dev)
                   for _ in range(S - 1)]
    sts = [torch.cuda.Stream(device=dev) for _ in range(S)]

    def timed_s(fn):
        main = torch.cuda.current_stream(dev)
        for f in range(W):
            fn(f, pipes[f % S])
        torch.cuda.synchronize()
        e0.record(main)
        for st in sts:
            st.wait_stream(main)
        for k in range(K):
            with torch.cuda.stream(sts[k % S]):
                fn(W + k, pipes[k % S])
        for st in sts:
            main.wait_stream(st)
        e1.record(main)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / K

    ok = []
    ms_ti = timed_s(lambda f, q: ok.append(q.decode_stream(streams[f], ti, sstreams[f])["ok"].sum()))
    ms_rows = timed_s(lambda f, q: q.decode(cells[f], sig[f]))
    ms_ti1 = timed(lambda f: p.decode_stream(streams[f], ti, sstreams[f]))
    ms_rows1 = timed(lambda f: p.decode(cells[f], sig[f]))
    dg = timed(lambda f: TI.demap_deinterleave(streams[f], ti, MOD, RATE, N_INNER,
                                               sigma2=sstreams[f]))
    dr = timed(lambda f: DM.demap(cells[f], MOD, RATE, sigma2=sig[f], n=N_INNER))
    return {"metric": "decoded info Mbit/s, time-interleaved frame stream "
                      "(hybrid TI de-interleave fused into the demap load)",
            "value": nblk * kp / (ms_ti / 1e3) / 1e6, "unit": "Mbit/s",
            "ms_per_step": ms_ti, "steps": K, "warmup": W,
            "rows_mbit_s": nblk * kp / (ms_rows / 1e3) / 1e6, "streams": S,
            "one_stream_mbit_s": nblk * kp / (ms_ti1 / 1e3) / 1e6,
            "one_stream_rows_mbit_s": nblk * kp / (ms_rows1 / 1e3) / 1e6,
            "gather_demap_ms": dg, "row_demap_ms": dr,
            "ti": {"nrows": ti.nrows, "ncols": ti.ncols, "nti": ti.nti},
            "bch_ok_blocks": int(sum(int(x) for x in ok[W:])),
            "data": "synthetic", "dtype": "f32"}


def run_plain(args):
    """The reference's own CPU-runnable plain case: 32 blocks of 64800-bit
    rate 10/15 with 256-NUC, AWGN at Es/N0 = 20 dB, the noise variance
    supplied (scalar), alpha 0.75, at most 50 iterations.  The GPU pipeline
    (demap -> LDPC -> BCH) on device-resident cells, and the same blocks
    through the reference's CPU path on the host cores (float32 demap,
    lab/ldpc_kernel.c over all threads, packed BCH)."""
    import time
    import torch
    from atsc3_b200 import codes as C
    from atsc3_b200 import synth
    from atsc3_b200.pipeline import FecPipeline
    n, mod, rate, nblk = 64800, "256QAM", "10/15", 32
    tx = synth.Transmitter(n, mod, rate, device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(args.seed)
    pay = torch.randint(0, 2, (nblk, tx.kp), generator=g, device="cuda", dtype=torch.uint8)
    x, _ = tx.encode(pay)
    y, s2 = synth.channel(x, 20.0, "awgn", g)
    s2 = float(s2)
    pipe = FecPipeline(n, mod, rate, iters=ITERS, alpha=ALPHA)
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    for _ in range(args.warmup):
        pipe.decode(y, sigma2=s2)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        o = pipe.decode(y, sigma2=s2)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    ok = int(o["ok"].sum())
    same = bool(torch.equal(o["payload"][:, :tx.kp // 8],
                            torch.from_numpy(np.packbits(pay.cpu().numpy(), axis=1)).cuda()))
    its = o["its"].float().mean().item()
    kp = C.kpayload(rate, n)
    threads = os.cpu_count() or 1
    cells = y.cpu().numpy()
    t0 = time.perf_counter()
    nok_cpu, its_cpu = cpu_reference_decode(cells, s2, threads, mod=mod, rate=rate, n=n)
    cpu_s = time.perf_counter() - t0
    return {"metric": "decoded info Mbit/s, plain case (32 blocks 64800 10/15 256-NUC, 20 dB AWGN)",
            "value": nblk * kp / (ms / 1e3) / 1e6, "unit": "Mbit/s", "ms_per_step": ms,
            "steps": args.steps, "warmup": args.warmup, "bch_ok": ok,
            "payload_equals_sent": same, "mean_iters": its,
            "cpu_reference": {"value": nblk * kp / cpu_s / 1e6, "unit": "Mbit/s",
                              "cores": threads, "bch_ok": int(nok_cpu),
                              "mean_iters": float(np.mean(its_cpu)),
                              "what": "float32 demap numpy + lab/ldpc_kernel.c over all host threads + packed BCH, same 32 blocks"},
            "data": "synthetic", "dtype": "f32"}


def run_codes(args):
    """Every A/322 code (16200 and 64800, rates 2/15..13/15): the LDPC launch
    alone on 16-NUC blocks at the code's measured threshold + 1 dB (AWGN,
    atsc3_b200/data/thresholds.json), three blocks per resident cluster, on
    the edge-buffer decoder and on the CSR decoder; kernel semantics in
    float32, torch semantics in float64 (--dtype), at most 50 iterations,
    alpha 0.75.  Outputs of the two decoders must agree."""
    import torch
    from atsc3_b200 import codes as C
    from atsc3_b200 import demap as DM
    from atsc3_b200 import ldpc as LDPC
    from atsc3_b200 import native as N
    from atsc3_b200 import synth, thresholds
    g = torch.Generator(device="cuda")
    g.manual_seed(args.seed)
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    steps = max(1, min(args.steps, 8))

    f64 = args.dtype == "float64"
    sem = "torch" if f64 else "kernel"   # the float64 decoders run torch semantics

    def timed(plan, lam):
        for _ in range(args.warmup):
            LDPC.decode_flood(plan, lam, iters=ITERS, alpha=ALPHA, semantics=sem)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            o = LDPC.decode_flood(plan, lam, iters=ITERS, alpha=ALPHA, semantics=sem)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, o

    rows = []
    only = {x.strip() for x in args.only.split(",")} if args.only else None
    for n in (16200, 64800):
        for r in C.RATES:
            if only and f"{n} {r}" not in only:
                continue
            qce = LDPC.plan_for(r, n, kind="qce", dtype=args.dtype)
            csr = LDPC.plan_for(r, n, kind="csr", dtype=args.dtype)
            cfg = np.zeros(4, np.int32)
            N.call("atsc3_ldpc_qce_config", qce._h, 0, 0, cfg.ctypes.data)
            nblk = 3 * int(cfg[0])
            tx = synth.Transmitter(n, "16QAM", r, device="cuda")
            pay = torch.randint(0, 2, (nblk, tx.kp), generator=g, device="cuda",
                                dtype=torch.uint8)
            x, _ = tx.encode(pay)
            esn0 = thresholds.lookup(n, "16QAM", r) + 1.0
            y, s2 = synth.channel(x, esn0, "awgn", g)
            lam = DM.demap(y, "16QAM", r, sigma2=float(s2), n=n)
            if f64:
                lam = lam.double()
            ms_q, oq = timed(qce, lam)
            ms_c, oc = timed(csr, lam)
            same = all(torch.equal(oq[k], oc[k]) for k in ("bits", "conv", "its", "bad"))
            kp = C.kpayload(r, n)
            rows.append({"code": f"{n} {r}", "type": C.ldpc_params(r, n)[0],
                         "esn0_db": esn0, "blocks": nblk,
                         "cluster": int(cfg[1]), "resident_clusters": int(cfg[0]),
                         "mean_iters": float(oq["its"].float().mean()),
                         "qce_ms": ms_q, "qce_mbit_s": nblk * kp / (ms_q / 1e3) / 1e6,
                         "csr_ms": ms_c, "csr_mbit_s": nblk * kp / (ms_c / 1e3) / 1e6,
                         "outputs_equal": bool(same)})
    return {"metric": "per-code LDPC decoded info Mbit/s (edge-buffer vs CSR decoder)",
            "unit": "Mbit/s", "steps": steps, "warmup": args.warmup,
            "data": "synthetic", "dtype": "f64" if f64 else "f32",
            "semantics": sem, "codes": rows}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="frame",
                    choices=["frame", "uneven", "frame_ti", "codes", "plain"])
    ap.add_argument("--blocks", type=int, default=512)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=128)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cluster", type=int, default=0)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--streams", type=int, default=2)
    ap.add_argument("--decoder", default="auto", choices=["auto", "qce", "qc", "csr"],
                    help="LDPC decoder (auto = edge-buffer quasi-cyclic)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dtype", default="float32", choices=["float32", "float64"],
                    help="--workload codes: decoder arithmetic")
    ap.add_argument("--only", default="",
                    help="--workload codes: comma-separated codes, e.g. '64800 7/15'")
    a = ap.parse_args(argv)
    if a.warmup < 3:
        a.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if a.workload == "uneven":
        if rank == 0:
            print(json.dumps(run_uneven(a)), flush=True)
        return 0
    if a.workload == "frame_ti":
        if rank == 0:
            print(json.dumps(run_frame_ti(a)), flush=True)
        return 0
    if a.workload == "codes":
        if rank == 0:
            print(json.dumps(run_codes(a)), flush=True)
        return 0
    if a.workload == "plain":
        if rank == 0:
            print(json.dumps(run_plain(a)), flush=True)
        return 0
    if a.impl == "reference":
        line = run_reference(a, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0
    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    line, par = run_gpu(a, rank, world, local_rank)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"], ref_out = cpu_baseline(par)
        line["parity"] = parity_check(par, ref_out)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
