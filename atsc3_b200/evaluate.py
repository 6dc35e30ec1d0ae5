"""Learned vs plain normalised min-sum: thresholds, training, FER and
iteration sweeps (all on the GPU, BCH as the arbiter).

    python -m atsc3_b200.evaluate [--steps 2000] [--batch 256] [--blocks 100000]
    python -m atsc3_b200.evaluate --compare 6/15 16QAM 8.25 --blocks 11111

For each MODCOD (64800-bit rate 6/15 with 16-NUC, 8/15 with 64-NUC, 10/15
with 256-NUC):
1. threshold: the lowest Es/N0 (0.1 dB grid) at which the plain decoder
   (alpha 0.75, at most 50 iterations, AWGN) reaches a block error rate of
   1e-2 on 2000 seeded blocks -- the "3/3"-style search the reference uses
   for its LDM thresholds, run with this decoder;
2. training: per-iteration, per-check-degree scale/offset of the unrolled
   12-iteration weighted min-sum (``learned.train``) on fresh seeded blocks
   at Es/N0 uniform in [thr-0.5, thr+1.5], half AWGN, half Rayleigh gain;
3. the same threshold search for the learned decoder (the gain in dB at a
   block error rate of 1e-2 is the difference);
4. evaluation on held-out seeded blocks over an Es/N0 sweep from 0.5 dB below
   the plain threshold in 0.25 dB steps: block errors
   (BCH syndrome nonzero or information bits wrong), mean iterations and
   decoded Mbit/s for the plain and the learned decoder, both the same
   flooding schedule with early stop (iterations past 12 reuse the last
   learned row).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import bch as BCH
from . import codes as C
from . import demap as DM
from . import ldpc as LDPC
from . import learned as LR
from . import native as N
from . import synth

MODCODS = (("6/15", "16QAM"), ("8/15", "64QAM"), ("10/15", "256QAM"))
HERE = os.path.dirname(os.path.abspath(__file__))


def _torch():
    import torch
    return torch


def blocks(tx, gen, nblk, esn0, channel="awgn"):
    """Seeded blocks at one Es/N0: (lam float32 codeword order, codewords)."""
    torch = _torch()
    pay = torch.randint(0, 2, (nblk, tx.kp), generator=gen, device=tx.dev,
                        dtype=torch.uint8)
    x, cw = tx.encode(pay)
    y, s2 = synth.channel(x, esn0, channel, gen)
    lam = DM.demap(y, tx.mod, tx.rate, sigma2=s2 if channel == "rayleigh" else float(s2),
                   n=tx.n)
    return lam, cw


def decode_count(plan, lam, cw, kldpc, n, weights=None, iters=50, alpha=0.75):
    """(block errors, sum of iterations, GPU ms) for one batch."""
    torch = _torch()
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    e0.record()
    o = LDPC.decode_flood(plan, lam, iters=iters, alpha=alpha, want_bits=True,
                          want_hard=True, weights=weights)
    e1.record()
    chk = BCH.bch_check(o["hard"], kldpc, n, want_payload=False)
    wrong = (o["bits"][:, :kldpc] != cw[:, :kldpc]).any(dim=1)
    err = wrong | (chk["ok"] == 0)
    torch.cuda.synchronize()
    return int(err.sum()), int(o["its"].sum()), e0.elapsed_time(e1)


def threshold(rate, mod, n=64800, target=1e-2, nblk=2000, seed=11, lo=-2.0,
              hi=24.0, step=0.1, weights=None):
    """Lowest Es/N0 on a `step` grid in (lo, hi] where the decoder's block
    error rate over `nblk` seeded blocks is <= target (bisection); the plain
    decoder, or the weighted one when `weights` is given."""
    torch = _torch()
    tx = synth.Transmitter(n, mod, rate, device="cuda")
    plan = LDPC.plan_for(rate, n)
    K = C.kldpc(rate, n)

    def fer(e):
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed)
        errs = 0
        for lo_ in range(0, nblk, 500):
            lam, cw = blocks(tx, gen, min(500, nblk - lo_), e)
            errs += decode_count(plan, lam, cw, K, n, weights=weights)[0]
        return errs / nblk

    while hi - lo > step + 1e-9:
        mid = round((lo + hi) / 2 / step) * step
        if mid <= lo or mid >= hi:
            break
        if fer(mid) <= target:
            hi = mid
        else:
            lo = mid
    return round(hi, 2)


def sweep(rate, mod, weights, esn0s, nblk, n=64800, seed=99, chunk=2000):
    torch = _torch()
    tx = synth.Transmitter(n, mod, rate, device="cuda")
    plan = LDPC.plan_for(rate, n)
    K = C.kldpc(rate, n)
    kp = C.kpayload(rate, n)
    out = []
    for e in esn0s:
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed + int(round(e * 10)))
        acc = {"plain": [0, 0, 0.0], "learned": [0, 0, 0.0]}
        for lo in range(0, nblk, chunk):
            lam, cw = blocks(tx, gen, min(chunk, nblk - lo), e)
            for name, w in (("plain", None), ("learned", weights)):
                er, it, ms = decode_count(plan, lam, cw, K, n, weights=w)
                acc[name][0] += er
                acc[name][1] += it
                acc[name][2] += ms
        row = {"esn0_db": e, "blocks": nblk}
        for name, (er, it, ms) in acc.items():
            row[name] = {"fer": er / nblk, "block_errors": er,
                         "mean_iters": it / nblk,
                         "mbit_s": nblk * kp / (ms / 1e3) / 1e6}
        out.append(row)
    return out


def run(steps=2000, batch=256, nblk=100000, points=9, out_dir=None, seed=1,
        iters=12, window=(-0.5, 1.5), tag="", depths=None, mode="degree"):
    """iters: unrolled depth of the training decoder; window: training Es/N0
    range relative to the plain threshold (dB); tag: weights file infix."""
    report = {}
    out_dir = out_dir or os.path.join(HERE, "data")
    for rate, mod in MODCODS:
        t0 = time.time()
        thr = threshold(rate, mod)
        al, be, hist, man = LR.train(rate, 64800, mod, steps=steps, nblk=batch,
                                     iters=iters,
                                     esn0=(thr + window[0], thr + window[1]),
                                     channel="mixed", seed=seed,
                                     log_every=max(1, steps // 10),
                                     depths=depths, mode=mode)
        man["threshold_db"] = thr
        name = f"weights_{tag + '_' if tag else ''}{rate.replace('/', '_')}_{mod}.pt"
        path = os.path.join(out_dir, name)
        LR.save_weights(path, al, be, man)
        code = LR.WmsCode(rate, 64800, mode=mode)
        w = LR.inference_weights(al, be, code.buckets, mode=mode)
        lthr = threshold(rate, mod, lo=thr - 3.0, hi=thr, weights=w)
        esn0s = [round(thr - 0.5 + 0.25 * i, 2) for i in range(points)]
        rows = sweep(rate, mod, w, esn0s, nblk // points)
        report[f"{rate} {mod}"] = {"threshold_db": thr,
                                   "learned_threshold_db": lthr,
                                   "gain_db_at_fer_1e-2": round(thr - lthr, 2),
                                   "train_loss": hist,
                                   "weights": os.path.basename(path),
                                   "sweep": rows, "operating_point": summary(rows),
                                   "seconds": time.time() - t0}
    return report


def summary(rows, target=1e-4):
    """The plain decoder's operating point: the lowest Es/N0 of the sweep
    where its block error rate is <= target; the learned decoder's block
    error rate and mean iterations there."""
    for r in rows:
        if r["plain"]["fer"] <= target:
            p, l = r["plain"], r["learned"]
            return {"esn0_db": r["esn0_db"], "plain_fer": p["fer"],
                    "learned_fer": l["fer"], "plain_mean_iters": p["mean_iters"],
                    "learned_mean_iters": l["mean_iters"],
                    "iteration_reduction": 1 - l["mean_iters"] / p["mean_iters"],
                    "plain_mbit_s": p["mbit_s"], "learned_mbit_s": l["mbit_s"]}
    return None


def compare_decoders(rate, mod, esn0, nblk, weights_path=None, n=64800,
                     seed=99, chunk=2000, iters=50, alpha=0.75):
    """Mean iterations of four decoders on the same held-out seeded AWGN
    blocks at one Es/N0 (the blocks ``sweep`` draws at that point): the plain
    flooding min-sum, the learned flooding min-sum, the layered min-sum
    (Type B codes) and the float64 log-tanh sum-product flooding decoder
    (the exact message update a scale/offset min-sum approximates).
    Iterations count message updates up to the zero syndrome (the
    sum-product count is the update after which its syndrome vanished, the
    same count).  A block error is a wrong information bit or no zero
    syndrome within ``iters``."""
    torch = _torch()
    tx = synth.Transmitter(n, mod, rate, device="cuda")
    plan = LDPC.plan_for(rate, n)
    K = C.kldpc(rate, n)
    if weights_path is None:
        weights_path = os.path.join(
            HERE, "data", f"weights_fast_{rate.replace('/', '_')}_{mod}.pt")
    al, be, _ = LR.load_weights(weights_path)
    w = LR.inference_weights(al, be, LR.WmsCode(rate, n).buckets)
    try:
        lplan = LDPC.LayeredPlan(rate, n)
    except (ValueError, N.FecError):
        lplan = None
    sptab = LDPC.sp_tables(C.csr(rate, n), n)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed + int(round(esn0 * 10)))
    acc = {}

    def add(name, o, cw, ms):
        wrong = (o["bits"][:, :K] != cw[:, :K]).any(dim=1) | (o["conv"] == 0)
        a = acc.setdefault(name, [0, 0, 0.0])
        a[0] += int(wrong.sum())
        a[1] += int(o["its"].sum())
        a[2] += ms

    for lo in range(0, nblk, chunk):
        lam, cw = blocks(tx, gen, min(chunk, nblk - lo), esn0)
        runs = [("plain flooding min-sum",
                 lambda: LDPC.decode_flood(plan, lam, iters=iters, alpha=alpha)),
                ("learned flooding min-sum",
                 lambda: LDPC.decode_flood(plan, lam, iters=iters, alpha=alpha,
                                           weights=w)),
                ("float64 sum-product flooding",
                 lambda: LDPC.sp_decode(sptab, lam.double(), iters=iters))]
        if lplan is not None:
            runs.append(("plain layered min-sum",
                         lambda: LDPC.decode_layered(lplan, lam, iters=iters,
                                                     alpha=alpha)))
        for name, fn in runs:
            e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
            e0.record()
            o = fn()
            e1.record()
            torch.cuda.synchronize()
            add(name, o, cw, e0.elapsed_time(e1))
        if lplan is not None:
            LDPC.check_layered_error(lplan)
    return {"rate": rate, "mod": mod, "n": n, "esn0_db": esn0, "blocks": nblk,
            "channel": "awgn", "weights": os.path.basename(weights_path),
            "decoders": {k: {"block_errors": er, "mean_iters": it / nblk,
                             "gpu_ms": round(ms, 1)}
                         for k, (er, it, ms) in acc.items()}}


# ---------------------------------------------------------------------------
# settling the target: thresholds of every decoder and a large sample at the
# plain decoder's FER 1e-4 point, AWGN and Rayleigh
# ---------------------------------------------------------------------------

def clopper_pearson(k, n, conf=0.95):
    """Exact two-sided binomial confidence interval for k events in n."""
    from scipy.stats import beta
    a = 1.0 - conf
    lo = 0.0 if k == 0 else float(beta.ppf(a / 2, k, n - k + 1))
    hi = 1.0 if k == n else float(beta.ppf(1 - a / 2, k + 1, n - k))
    return [lo, hi]


def load_decoder_weights(path, n=64800):
    """Inference weights of a saved set (degree or row buckets) + manifest."""
    al, be, man = LR.load_weights(path)
    mode = man.get("mode", "degree")
    code = LR.WmsCode(man["rate"], n, mode=mode)
    return LR.inference_weights(al, be, code.buckets, mode=mode), man


def _decoders(rate, n, weight_sets, alphas=(0.75,), sp=False):
    """name -> callable(lam) -> device dict with bits, conv, its."""
    plan = LDPC.plan_for(rate, n)
    out = {}
    for a in alphas:
        out[f"plain alpha {a:g}"] = (lambda lam, a=a: LDPC.decode_flood(
            plan, lam, iters=50, alpha=a))
    for name, w in weight_sets.items():
        out[name] = (lambda lam, w=w: LDPC.decode_flood(
            plan, lam, iters=50, alpha=0.75, weights=w))
    if sp:
        tab = LDPC.sp_tables(C.csr(rate, n), n)
        out["float64 sum-product"] = (lambda lam: LDPC.sp_decode(
            tab, lam.double(), iters=50))
    return out


def _errors(o, cw, K, n, arbiter="bch"):
    """Block errors of one decode: a wrong information bit, or (arbiter
    "bch", the judge the evaluation names) a nonzero BCH syndrome of the
    K_ldpc decoded bits, or (arbiter "conv", the reference receiver's
    delivery rule: lab/m44_ldm.py:2380-2382 drops a block whose LDPC did not
    converge) no zero LDPC syndrome within the iteration cap."""
    torch = _torch()
    wrong = (o["bits"][:, :K] != cw[:, :K]).any(dim=1)
    if arbiter == "conv":
        return wrong | (o["conv"] == 0)
    bits = o["bits"]
    nblk = bits.shape[0]
    syn = torch.empty((nblk, 6), dtype=torch.int32, device=bits.device)
    N.call("atsc3_bch_syndrome_bits", bits.data_ptr(), bits.stride(0), nblk, K,
           BCH.device_rtab(K, n, bits.device).data_ptr(), syn.data_ptr(),
           torch.cuda.current_stream(bits.device).cuda_stream)
    return wrong | (syn != 0).any(dim=1)


def threshold_of(rate, mod, fn, channel="awgn", n=64800, target=1e-2,
                 nblk=2000, seed=11, lo=-2.0, hi=24.0, step=0.1, chunk=500,
                 arbiter="bch"):
    """Lowest Es/N0 (on a `step` grid, bisection in (lo, hi]) at which the
    decoder `fn` has a block error rate <= target over `nblk` seeded blocks
    (errors as `_errors` counts them)."""
    torch = _torch()
    tx = synth.Transmitter(n, mod, rate, device="cuda")
    K = C.kldpc(rate, n)

    def fer(e):
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed)
        errs = 0
        for lo_ in range(0, nblk, chunk):
            lam, cw = blocks(tx, gen, min(chunk, nblk - lo_), e, channel)
            errs += int(_errors(fn(lam), cw, K, n, arbiter).sum())
        return errs / nblk

    while hi - lo > step + 1e-9:
        mid = round((lo + hi) / 2 / step) * step
        if mid <= lo or mid >= hi:
            break
        if fer(mid) <= target:
            hi = mid
        else:
            lo = mid
    return round(hi, 2)


def op_eval(rate, mod, esn0, nblk, decoders, channel="awgn", n=64800, seed=7,
            chunk=2000, arbiter="bch"):
    """Every decoder on the same `nblk` held-out seeded blocks at one Es/N0:
    block errors with their 95% Clopper-Pearson interval, mean iterations
    (a failing block counts 50) and decoded Mbit/s over the decode-only GPU
    time."""
    torch = _torch()
    tx = synth.Transmitter(n, mod, rate, device="cuda")
    K = C.kldpc(rate, n)
    kp = C.kpayload(rate, n)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed + int(round(esn0 * 100)) + (0 if channel == "awgn" else 1))
    acc = {k: [0, 0, 0.0] for k in decoders}
    for lo in range(0, nblk, chunk):
        lam, cw = blocks(tx, gen, min(chunk, nblk - lo), esn0, channel)
        for name, fn in decoders.items():
            e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
            e0.record()
            o = fn(lam)
            e1.record()
            err = _errors(o, cw, K, n, arbiter)
            torch.cuda.synchronize()
            a = acc[name]
            a[0] += int(err.sum())
            a[1] += int(o["its"].sum())
            a[2] += e0.elapsed_time(e1)
    return {name: {"block_errors": er, "fer": er / nblk,
                   "fer_cp95": clopper_pearson(er, nblk),
                   "mean_iters": it / nblk,
                   "mbit_s": nblk * kp / (ms / 1e3) / 1e6}
            for name, (er, it, ms) in acc.items()}


def settle(rate, mod, weight_paths, channel="awgn", nblk=100000, n=64800,
           max_points=8, arbiter="bch", start=0.25):
    """Thresholds (FER 1e-2, 2000 blocks) of plain min-sum at alpha 0.75,
    0.85 and 1.0, of each learned set and of the float64 sum-product
    decoder; then the plain (alpha 0.75) decoder's FER 1e-4 point: from
    `start` dB above its threshold in 0.25 dB steps, `nblk` held-out blocks at
    each point until plain reaches <= 1e-4, with every decoder on the same
    blocks.  Block errors as `_errors` counts them under `arbiter`."""
    sets, mans = {}, {}
    for pth in weight_paths:
        w, man = load_decoder_weights(pth, n)
        name = f"learned {os.path.basename(pth)}"
        sets[name], mans[name] = w, man
    dec = _decoders(rate, n, sets, alphas=(0.75, 0.85, 1.0), sp=True)
    thr = {name: threshold_of(rate, mod, fn, channel, arbiter=arbiter)
           for name, fn in dec.items()}
    base = thr["plain alpha 0.75"]
    evald = {k: v for k, v in dec.items() if k != "float64 sum-product"}
    points = []
    for i in range(max_points):
        e = round(base + start + 0.25 * i, 2)
        res = op_eval(rate, mod, e, nblk, evald, channel, n, arbiter=arbiter)
        points.append({"esn0_db": e, "blocks": nblk, "decoders": res})
        if res["plain alpha 0.75"]["fer"] <= 1e-4:
            break
    op = points[-1]
    plain = op["decoders"]["plain alpha 0.75"]
    gains = {name: {"iteration_reduction": 1 - r["mean_iters"] / plain["mean_iters"],
                    "mbit_s_ratio": r["mbit_s"] / plain["mbit_s"]}
             for name, r in op["decoders"].items() if name.startswith("learned")}
    return {"rate": rate, "mod": mod, "n": n, "channel": channel,
            "arbiter": arbiter, "thresholds_db_fer_1e-2": thr, "points": points,
            "operating_point_db": op["esn0_db"],
            "operating_point_reached": plain["fer"] <= 1e-4,
            "learned_vs_plain_at_op": gains,
            "weights": {k: {kk: m.get(kk) for kk in ("iters", "esn0", "channel",
                                                     "step", "mode")}
                        for k, m in mans.items()}}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--blocks", type=int, default=100000)
    ap.add_argument("--points", type=int, default=9)
    ap.add_argument("--out", default=None)
    ap.add_argument("--iters", type=int, default=12,
                    help="unrolled iterations of the training decoder")
    ap.add_argument("--window", type=float, nargs=2, default=(-0.5, 1.5),
                    help="training Es/N0 range relative to the plain threshold")
    ap.add_argument("--tag", default="", help="weights file infix")
    ap.add_argument("--depths", type=int, nargs="*", default=None,
                    help="average the output BCE over these unrolled depths")
    ap.add_argument("--compare", nargs=3, metavar=("RATE", "MOD", "ESN0"),
                    default=None,
                    help="only compare the mean iterations of the plain, learned, "
                         "layered and sum-product decoders at one Es/N0 on "
                         "--blocks held-out blocks")
    ap.add_argument("--weights", default=None, help="weights file for --compare")
    ap.add_argument("--buckets", default="degree", choices=["degree", "row"],
                    help="learned parameters per (iteration, check degree) or "
                         "per (iteration, block row)")
    ap.add_argument("--settle", nargs="+", metavar="RATE MOD WEIGHTS...",
                    default=None,
                    help="thresholds of every decoder and --blocks held-out "
                         "blocks at the plain decoder's FER 1e-4 point, for "
                         "one MODCOD and the given weight files")
    ap.add_argument("--channel", default="awgn", choices=["awgn", "rayleigh"])
    ap.add_argument("--arbiter", default="bch", choices=["bch", "conv"],
                    help="--settle block errors: BCH syndrome (default) or no "
                         "LDPC convergence (the receiver's delivery rule)")
    ap.add_argument("--start", type=float, default=0.25,
                    help="--settle: first point above the plain threshold (dB)")
    a = ap.parse_args(argv)
    if a.settle:
        rate, mod, *paths = a.settle
        print(json.dumps(settle(rate, mod, paths, a.channel, a.blocks,
                                arbiter=a.arbiter, start=a.start)), flush=True)
        return
    if a.compare:
        rate, mod, e = a.compare
        print(json.dumps(compare_decoders(rate, mod, float(e), a.blocks,
                                          weights_path=a.weights)), flush=True)
        return
    print(json.dumps(run(a.steps, a.batch, a.blocks, a.points, a.out,
                         iters=a.iters, window=tuple(a.window), tag=a.tag,
                         depths=a.depths, mode=a.buckets)),
          flush=True)


if __name__ == "__main__":
    main()
