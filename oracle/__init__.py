"""The parity oracle -- TEST INFRASTRUCTURE ONLY.

A CPU restatement of the Felbs/atsc3 FEC back end, used as the checker by
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py``.  The product (``atsc3_b200``) never imports it and has no CPU
fallback.

Pinning: every function here is checked by ``tests/test_oracle.py`` against
golden vectors produced by the reference itself (``tests/golden/``, made by
``tests/golden/make_golden.py``), and the C decoder is additionally checked
against the reference's own ``lab/ldpc_kernel.c`` compiled into
``oracle/_ref/`` by ``oracle/build.py`` wherever that file is present.

Contents (reference file:line each restates):
* ``transmit`` / ``ldpc_encode`` / ``bch_encode`` / ``map_cells`` --
  lab/m6_bicm.py:367-373 (``PlpChain.encode``), lab/m3_ldpc.py:119-159
  (A/322 6.1.3 encoder), lab/m6_bicm.py:283-290, :228-236.
* ``demap`` -- lab/m44_ldm.py:2431-2494 (float32 point metric and per-bit
  minima), with a supplied scalar or per-cell sigma2 (lab/m9_fast.py:
  1096-1115) or the per-row estimate.
* ``bch_syndrome`` -- lab/m6_bicm.py:269-280 (polynomial remainder).
* ``flood`` -- ``ldpc_oracle.c`` (lab/ldpc_kernel.c semantics and the
  float64 / torch semantics); ``flood_ref`` -- the reference kernel itself;
  ``flood_weighted`` -- the same kernel semantics with per-iteration,
  per-check-degree scale/offset minima (the learned decoder), numpy;
  ``flood_torch_narrow`` -- lab/m9_gpu.py:138-220 in bfloat16 / float16.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from atsc3_b200 import codes as C          # noqa: E402  (tables + H, data only)

_LIBS = {}


def _load(path, name):
    if name not in _LIBS:
        if not os.path.exists(path):
            from . import build as _b
            _b.build()
        _LIBS[name] = ctypes.CDLL(path)
    return _LIBS[name]


def oracle_lib():
    from . import build as _b
    L = _load(_b.ORACLE_SO, "oracle")
    vp, i32 = ctypes.c_void_p, ctypes.c_int32
    L.oracle_flood_f32.restype = i32
    L.oracle_flood_f32.argtypes = [vp, i32, i32, i32, vp, vp, vp, vp, i32,
                                   ctypes.c_float, i32, vp, vp, vp, vp]
    L.oracle_flood_f64.restype = i32
    L.oracle_flood_f64.argtypes = [vp, i32, i32, i32, vp, vp, vp, vp, i32,
                                   ctypes.c_double, i32, vp, vp, vp, vp]
    L.oracle_layered_f32.restype = i32
    L.oracle_layered_f32.argtypes = [vp, i32, i32, i32, vp, vp, vp, vp, i32,
                                     ctypes.c_float, vp, vp, vp, vp]
    return L


def ref_lib():
    """The reference's own compiled kernel, or None where it was not built."""
    from . import build as _b
    if not os.path.exists(_b.REF_SO):
        try:
            _b.build()
        except Exception:
            return None
        if not os.path.exists(_b.REF_SO):
            return None
    L = _load(_b.REF_SO, "ref")
    vp, i32 = ctypes.c_void_p, ctypes.c_int32
    L.ldpc_minsum_f32.restype = i32
    L.ldpc_minsum_f32.argtypes = [vp, i32, i32, i32, i32, vp, vp, vp, vp, i32,
                                  ctypes.c_float, vp, vp, vp, vp, vp]
    return L


def _p(a):
    return a.ctypes.data


def flood(llr, tables, n, iters=50, alpha=0.75, semantics=0, dtype=np.float32):
    """Oracle flooding decode: (bits, conv bool, its, bad)."""
    cptr, cidx, vptr, vedge = [np.ascontiguousarray(t, np.int32) for t in tables]
    llr = np.ascontiguousarray(llr, dtype)
    nblk = llr.shape[0]
    bits = np.zeros((nblk, n), np.uint8)
    conv = np.zeros(nblk, np.uint8)
    its = np.zeros(nblk, np.int32)
    bad = np.zeros(nblk, np.int32)
    L = oracle_lib()
    fn = L.oracle_flood_f32 if dtype == np.float32 else L.oracle_flood_f64
    rc = fn(_p(llr), nblk, n, len(cptr) - 1, _p(cptr), _p(cidx), _p(vptr),
            _p(vedge), int(iters), float(alpha), int(semantics), _p(bits),
            _p(conv), _p(its), _p(bad))
    if rc != 0:
        raise RuntimeError(f"oracle decode returned {rc}")
    return bits, conv.astype(bool), its, bad


def flood_weighted(llr, tables, n, walpha, wbeta, dbucket, iters=50,
                   cbucket=None):
    """Weighted flooding min-sum, kernel semantics (lab/ldpc_kernel.c:95-142
    with the check messages of the learned decoder): per iteration t and
    check of degree d, the minima become relu(min * walpha[min(t, T-1),
    dbucket[d]] - wbeta[...]) (each float32 op rounded once, no fused
    multiply-add); first minimum by strict <, sign = parity ^ (v < 0);
    variable sums from +0 in vedge order, then + llr.  numpy float32,
    vectorised per check degree and per variable degree.  With walpha = alpha
    and wbeta = 0 it is ``flood(..., alpha)`` bit for bit (tests pin that).
    cbucket (optional, one entry per check) replaces dbucket[degree] by a
    bucket per check (the per-block-row weights).
    Returns (bits, conv bool, its, bad)."""
    cptr, cidx, vptr, vedge = [np.asarray(t, np.int64) for t in tables]
    walpha = np.asarray(walpha, np.float32)
    wbeta = np.asarray(wbeta, np.float32)
    dbucket = np.asarray(dbucket, np.int64)
    T = walpha.shape[0]
    nc, ne = len(cptr) - 1, len(cidx)
    cdeg = np.diff(cptr)
    chk = np.repeat(np.arange(nc), cdeg)
    vdeg = np.diff(vptr)
    cgroups = [(d, np.nonzero(cdeg == d)[0]) for d in np.unique(cdeg)]
    vgroups = [(d, np.nonzero(vdeg == d)[0]) for d in np.unique(vdeg)]
    nblk = llr.shape[0]
    bits = np.zeros((nblk, n), np.uint8)
    conv = np.zeros(nblk, bool)
    its = np.zeros(nblk, np.int32)
    bad = np.zeros(nblk, np.int32)
    f32 = np.float32
    for b in range(nblk):
        lam = np.asarray(llr[b], f32)
        tot = lam.copy()
        m = np.zeros(ne, f32)
        for it in range(iters + 1):
            hard = (tot < 0).astype(np.int64)
            par = np.bitwise_xor.reduceat(hard[cidx], cptr[:-1]) if ne else np.zeros(nc, np.int64)
            badct = int(par.sum())
            if badct == 0:
                conv[b], its[b], bad[b] = True, it, 0
                break
            if it == iters:
                its[b], bad[b] = iters, badct
                break
            v = (tot[cidx] - m).astype(f32)
            newm = np.empty(ne, f32)
            ti = min(it, T - 1)
            for d, cs in cgroups:
                idx = cptr[cs][:, None] + np.arange(d)[None, :]
                vv = v[idx]
                mag = np.abs(vv)
                first = np.argmin(mag, axis=1)
                rows = np.arange(len(cs))
                min1 = mag[rows, first]
                mag2 = mag.copy()
                mag2[rows, first] = np.inf
                min2 = mag2.min(axis=1) if d > 1 else np.full(len(cs), np.inf, f32)
                if cbucket is None:
                    wa = walpha[ti, dbucket[d]]
                    wb = wbeta[ti, dbucket[d]]
                else:
                    wa = walpha[ti, np.asarray(cbucket)[cs]]
                    wb = wbeta[ti, np.asarray(cbucket)[cs]]
                A = np.maximum(f32(min1 * wa) - wb, f32(0)).astype(f32)
                B = np.maximum(f32(min2 * wa) - wb, f32(0)).astype(f32)
                ng = vv < 0
                parity = np.bitwise_xor.reduce(ng.astype(np.int64), axis=1)
                mg = np.where(np.arange(d)[None, :] == first[:, None], B[:, None], A[:, None])
                sg = (parity[:, None] ^ ng.astype(np.int64)).astype(bool)
                newm[idx] = np.where(sg, -mg, mg).astype(f32)
            m = newm
            s = np.zeros(n, f32)
            for d, vs in vgroups:
                acc = np.zeros(len(vs), f32)
                for k in range(d):
                    acc = (acc + m[vedge[vptr[vs] + k]]).astype(f32)
                s[vs] = acc
            tot = (lam + s).astype(f32)
        bits[b] = (tot < 0)
    return bits, conv, its, bad


def _narrow(x, dtype):
    """Round float32 values to bfloat16 / float16 (round to nearest even) and
    back: the result of a torch operation in that dtype."""
    x = np.asarray(x, np.float32)
    if dtype == "float16":
        with np.errstate(over="ignore"):        # overflow to +-inf is the result
            return x.astype(np.float16).astype(np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def flood_torch_narrow(llr, tables, n, iters=50, alpha=0.75, dtype="bfloat16"):
    """The reference's torch min-sum decoder run with dtype bfloat16 / float16
    (lab/m9_gpu.py:138-220): every elementwise operation computed in float32
    and its result rounded to the narrow type.  Per-edge messages m in the
    CSR edge order; each iteration v = tot[cidx] - m, first/second minimum of
    |v| per check (first position wins ties), m = round(round(alpha) * out)
    with the sign parity ^ (v < 0), then tot = llr + m summed over each bit's
    edges in edge order (bits of lower degree add 0.0, as the reference's
    padded table does), hard decisions and the syndrome of tot; a block
    freezes at its first zero syndrome with its = it + 1 (no iteration-0
    retire).  llr: (nblk, n) already in the narrow type (float64 input is
    rounded by the caller, as the reference's ``.to(dtype)``).  Checks of
    degree 1 are assumed absent (the reference pads with a large finite
    value, here infinity).  Returns (bits uint8, conv bool, its int32,
    bad int32)."""
    cptr, cidx, vptr, vedge = [np.asarray(t) for t in tables]
    lam = np.asarray(llr, np.float32)
    nb = lam.shape[0]
    nc = len(cptr) - 1
    deg = np.diff(cptr)
    dmax = int(deg.max())
    E = len(cidx)
    echk = np.repeat(np.arange(nc), deg)
    eslot = np.arange(E) - cptr[echk]
    vdeg = np.diff(vptr)
    ar = _narrow(np.float32(alpha), dtype)
    m = np.zeros((nb, E), np.float32)
    tot = lam.copy()
    out_bits = np.zeros((nb, n), np.uint8)
    out_its = np.full(nb, iters, np.int32)
    out_bad = np.zeros(nb, np.int32)
    frozen = np.zeros(nb, bool)
    bad = np.zeros(nb, np.int32)
    bits = (tot < 0).astype(np.uint8)
    rows = np.arange(nb)[:, None]
    for it in range(iters):
        v = _narrow(tot[:, cidx] - m, dtype)
        sg = v < 0
        par = np.zeros((nb, nc), np.int64)
        np.add.at(par, (slice(None), echk), sg.astype(np.int64))
        par &= 1
        mag = np.full((nb, nc, dmax), np.inf, np.float32)
        mag[:, echk, eslot] = np.abs(v)
        m1 = mag.min(2)
        first = np.argmax(mag == m1[:, :, None], axis=2)
        mag[rows, np.arange(nc)[None, :], first] = np.inf
        m2 = mag.min(2)
        outv = np.where(eslot[None, :] == first[:, echk], m2[:, echk], m1[:, echk])
        mm = _narrow(ar * outv, dtype)
        m = np.where((par[:, echk] == 1) ^ sg, -mm, mm).astype(np.float32)
        tot = lam.copy()
        for k in range(int(vdeg.max())):
            add = np.zeros((nb, n), np.float32)
            sel = vdeg > k
            add[:, sel] = m[:, vedge[vptr[:-1][sel] + k]]
            tot = _narrow(tot + add, dtype)
        bits = (tot < 0).astype(np.uint8)
        syn = np.zeros((nb, nc), np.int64)
        np.add.at(syn, (slice(None), echk), bits[:, cidx].astype(np.int64))
        bad = (syn & 1).sum(1).astype(np.int32)
        newly = ~frozen & (bad == 0)
        out_bits[newly] = bits[newly]
        out_its[newly] = it + 1
        frozen |= newly
        if frozen.all():
            break
    live = ~frozen
    out_bits[live] = bits[live]
    out_bad[live] = bad[live]
    return out_bits, frozen, out_its, out_bad


def flood_ref(llr, tables, n, iters=50, alpha=0.75, threads=1):
    """The reference kernel (lab/ldpc_kernel.c) itself, sub-batched over
    `threads` host threads the way lab/m44_ldm.py:2558-2576 drives it."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference kernel not built here")
    cptr, cidx, vptr, vedge = [np.ascontiguousarray(t, np.int32) for t in tables]
    llr = np.ascontiguousarray(llr, np.float32)
    nblk = llr.shape[0]
    ne = len(cidx)
    bits = np.zeros((nblk, n), np.uint8)
    conv = np.zeros(nblk, np.uint8)
    its = np.zeros(nblk, np.int32)
    bad = np.zeros(nblk, np.int32)

    def one(lo, hi):
        work = np.empty(n + ne, np.float32)
        rc = L.ldpc_minsum_f32(
            llr[lo:].ctypes.data, hi - lo, n, len(cptr) - 1, ne, _p(cptr),
            _p(cidx), _p(vptr), _p(vedge), int(iters), float(alpha),
            bits[lo:].ctypes.data, conv[lo:].ctypes.data,
            its[lo:].ctypes.data, bad[lo:].ctypes.data, _p(work))
        if rc != 0:
            raise RuntimeError(f"reference kernel returned {rc}")

    threads = max(1, min(threads, nblk))
    if threads == 1:
        one(0, nblk)
    else:
        from concurrent.futures import ThreadPoolExecutor
        step = (nblk + threads - 1) // threads
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(lambda i: one(i * step, min(nblk, (i + 1) * step)),
                        range(threads)))
    return bits, conv.astype(bool), its, bad


# ---------------------------------------------------------------------------
# transmitter (synthetic inputs)
# ---------------------------------------------------------------------------

def _addr(x, mm, M1, M2, Q1, Q2):
    # A/322 6.1.3.1 step ii, lab/m3_ldpc.py:63-66
    x = np.asarray(x, np.int64)
    mm = np.asarray(mm, np.int64)
    return np.where(x < M1, (x + mm * Q1) % max(M1, 1),
                    M1 + (x - M1 + mm * Q2) % M2)


def _pi_of(M1, M2, Q1, Q2, K):
    # accumulator -> codeword index (lab/m3_ldpc.py:69-82, "standard")
    a = np.arange(M1 + M2, dtype=np.int64)
    s1, t1 = np.divmod(a, max(Q1, 1))
    s2, t2 = np.divmod(a - M1, Q2)
    return np.where(a < M1, K + 360 * t1 + s1, K + M1 + 360 * t2 + s2)


def _accumulate(bits, rowptr, addr, row0, M1, M2, Q1, Q2, M):
    """XOR of the table addresses hit by the set bits (lab/m3_ldpc.py:
    129-135), vectorised over all bits of all blocks: (nblk, nbits) ->
    (nblk, M)."""
    nb = bits.shape[1]
    bit = np.arange(nb)
    row = row0 + bit // 360
    cnt = (rowptr[row + 1] - rowptr[row]).astype(np.int64)
    rep = np.repeat(bit, cnt)
    first = np.repeat(rowptr[row].astype(np.int64), cnt)
    within = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    acc = _addr(addr[first + within], rep % 360, M1, M2, Q1, Q2)
    out = np.zeros((bits.shape[0], M), np.uint8)
    for b in range(bits.shape[0]):
        sel = bits[b, rep].astype(bool)
        out[b] = (np.bincount(acc[sel], minlength=M) & 1).astype(np.uint8)
    return out


def ldpc_encode(s, rate, n):
    """(nblk, K) info bits -> (nblk, n) codewords, A/322 6.1.3.1 / 6.1.3.2."""
    s = np.atleast_2d(np.asarray(s, np.uint8))
    typ, K, M1, M2, Q1, Q2 = C.ldpc_params(rate, n)
    rowptr, addr = C.address_rows(rate, n)
    M = M1 + M2
    pi = _pi_of(M1, M2, Q1, Q2, K)
    lam = np.zeros((s.shape[0], n), np.uint8)
    lam[:, :K] = s
    p = _accumulate(s, rowptr, addr, 0, M1, M2, Q1, Q2, M)
    if typ == "A":
        p[:, :M1] = np.bitwise_xor.accumulate(p[:, :M1], axis=1)
        lam[:, pi[:M1]] = p[:, :M1]
        fb = _accumulate(lam[:, K:K + M1], rowptr, addr, K // 360, M1, M2,
                         Q1, Q2, M)
        p ^= fb
        lam[:, pi[M1:]] = p[:, M1:]
    else:
        p = np.bitwise_xor.accumulate(p, axis=1)
        lam[:, pi] = p
    return lam


def bch_encode(info, n):
    """(nblk, K_ldpc - Mouter) -> (nblk, K_ldpc) systematic BCH codewords
    (lab/m6_bicm.py:283-290)."""
    info = np.atleast_2d(np.asarray(info, np.uint8))
    g = C.bch_generator(n)
    deg = C.MOUTER[n]
    out = np.zeros((info.shape[0], info.shape[1] + deg), np.uint8)
    out[:, :info.shape[1]] = info
    for b in range(info.shape[0]):
        v = int.from_bytes(np.packbits(info[b]).tobytes(), "big") >> (
            (-info.shape[1]) % 8)
        r = _poly_mod(v << deg, g, deg)
        out[b, info.shape[1]:] = [(r >> (deg - 1 - i)) & 1 for i in range(deg)]
    return out


def _poly_mod(v, g, gd):
    # lab/m6_bicm.py:269-273
    while v and v.bit_length() - 1 >= gd:
        v ^= g << ((v.bit_length() - 1) - gd)
    return v


def bch_syndrome(bits, n):
    """Python-int syndrome of each row (0 = clean), lab/m6_bicm.py:276-280."""
    bits = np.atleast_2d(np.asarray(bits, np.uint8))
    g = C.bch_generator(n)
    deg = C.MOUTER[n]
    out = []
    for row in bits:
        v = int.from_bytes(np.packbits(row).tobytes(), "big") >> ((-len(row)) % 8)
        out.append(_poly_mod(v, g, deg))
    return out


def map_cells(q, pts, nb):
    """(nblk, ncell*nb) bits in q order -> complex cells (lab/m6_bicm.py:228)."""
    q = np.asarray(q, np.uint8)
    b = q.reshape(q.shape[0], -1, nb)
    k = np.zeros(b.shape[:2], np.int64)
    for i in range(nb):
        k |= b[:, :, i].astype(np.int64) << (nb - 1 - i)
    return np.asarray(pts)[k]


def transmit(payload, n, mod, rate, pts=None):
    """PlpChain.encode for a batch: payload bits -> complex128 cells."""
    payload = np.atleast_2d(np.asarray(payload, np.uint8))
    kp = payload.shape[1]
    scr = payload ^ C.scrambler_sequence(kp)[None, :]
    nouter = bch_encode(scr, n)
    cw = ldpc_encode(nouter, rate, n)
    q = cw[:, C.bicm_map(n, mod, rate)]
    pts = C.alphabet(mod, rate) if pts is None else pts
    return map_cells(q, pts, C.MOD_BITS[mod]), cw


# ---------------------------------------------------------------------------
# demapper
# ---------------------------------------------------------------------------

def point_metric(zr, zi, pr, pi, p2):
    # lab/m44_ldm.py:2447-2451, float32, same operation order
    q = zr[:, None] * pr[None, :]
    q += zi[:, None] * pi[None, :]
    q *= np.float32(-2.0)
    q += p2[None, :]
    return q


def demap(cells2d, pts, nb, sigma2=None):
    """(nblk, ncell) complex -> (nblk, ncell*nb) float32 LLRs in q order.

    sigma2 None: per-row estimate (lab/m44_ldm.py:2480); a scalar; or a
    (nblk, ncell) per-cell array (divide after the minima, lab/m9_fast.py:
    1114)."""
    cells2d = np.atleast_2d(cells2d)
    nblk, ncell = cells2d.shape
    pr, pi, p2 = C.point_tables_f32(pts)
    zr = np.asarray(cells2d.real, np.float32)
    zi = np.asarray(cells2d.imag, np.float32)
    q = point_metric(zr.ravel(), zi.ravel(), pr, pi, p2).reshape(nblk, ncell, -1)
    if sigma2 is None:
        z2 = zr * zr + zi * zi
        s2 = np.maximum((z2 + q.min(2)).mean(1), 1e-9)[:, None]
    elif np.ndim(sigma2) == 0:
        s2 = np.float32(sigma2)
    else:
        s2 = np.asarray(sigma2, np.float32).reshape(nblk, ncell)
    qr = q.reshape(nblk, ncell, *([2] * nb))
    sub = tuple(range(2, 2 + nb - 1))
    out = np.empty((nblk, ncell, nb), np.float32)
    head = (slice(None), slice(None))
    for i in range(nb):
        a = qr[head + (slice(None),) * i + (1,)].min(axis=sub)
        b = qr[head + (slice(None),) * i + (0,)].min(axis=sub)
        out[:, :, i] = (a - b) / s2
    return out.reshape(nblk, ncell * nb)


def deinterleave(q2d, lam_of_q, n):
    lam = np.empty((q2d.shape[0], n), np.float32)
    lam[:, lam_of_q] = q2d
    return lam


def awgn(cells, esn0_db, rng):
    """complex64 cells + complex Gaussian noise of variance N0 = 10^(-Es/N0/10)
    (unit-power alphabet): the draw order of lab/m6_bicm.py:436-438."""
    n0 = 10 ** (-esn0_db / 10.0)
    nz = (rng.standard_normal(cells.shape)
          + 1j * rng.standard_normal(cells.shape)) / np.sqrt(2)
    return (cells + nz * np.sqrt(n0)).astype(np.complex64), n0


def synth_case(tx, nblk, kpay, ncell, esn0_db, channel, seed):
    """The seeded synthetic-case procedure shared by the golden generator
    (with the reference transmitter) and the tests (with ``transmit``):

    payload bits (one rng.integers draw for the batch) -> tx -> complex64
    cells through AWGN (scalar sigma2 = N0) or a per-cell Rayleigh gain
    h = |CN(0,1)| equalised away, y = (h x + n)/h, sigma2_cell = N0/h^2.
    Returns (payload, cells complex64 (nblk, ncell), sigma2)."""
    rng = np.random.default_rng(seed)
    pay = rng.integers(0, 2, (nblk, kpay), dtype=np.uint8)
    x = np.asarray(tx(pay), np.complex128).reshape(nblk, ncell)
    n0 = 10 ** (-esn0_db / 10.0)
    if channel == "awgn":
        nz = (rng.standard_normal((nblk, ncell))
              + 1j * rng.standard_normal((nblk, ncell))) / np.sqrt(2)
        y = (x + nz * np.sqrt(n0)).astype(np.complex64)
        return pay, y, np.float32(n0)
    if channel == "rayleigh":
        h = np.abs(rng.standard_normal((nblk, ncell))
                   + 1j * rng.standard_normal((nblk, ncell))) / np.sqrt(2)
        nz = (rng.standard_normal((nblk, ncell))
              + 1j * rng.standard_normal((nblk, ncell))) / np.sqrt(2)
        y = ((h * x + nz * np.sqrt(n0)) / h).astype(np.complex64)
        return pay, y, (n0 / h ** 2).astype(np.float32)
    raise ValueError(channel)


_BCH_MASKS = {}


def _bch_masks(k, n):
    """Packed (deg, k/64) uint64 masks: bit i of row j set iff x^(k-1-i)
    mod g has x^j -- the table of lab/m9_accel.py:169-194."""
    key = (k, n)
    if key not in _BCH_MASKS:
        R = C.bch_remainder_table(k, n)                      # (k, 6) u32
        deg = C.MOUTER[n]
        cols = np.unpackbits(R.view(np.uint8), axis=1,
                             bitorder="little")[:, :deg]     # (k, deg)
        pad = (-k) % 64
        if pad:
            cols = np.concatenate([cols, np.zeros((pad, deg), np.uint8)])
        masks = np.ascontiguousarray(np.packbits(cols.T, axis=1)).view(np.uint64)
        _BCH_MASKS[key] = (masks, pad)
    return _BCH_MASKS[key]


def bch_syndrome_fast(bits2d, n):
    """Batch syndromes as a packed GF(2) matrix product (the evaluation of
    lab/m9_accel.py:212-236); returns a list of Python ints."""
    a = np.atleast_2d(np.asarray(bits2d, np.uint8))
    nblk, k = a.shape
    masks, pad = _bch_masks(k, n)
    if pad:
        a = np.concatenate([a, np.zeros((nblk, pad), np.uint8)], axis=1)
    v = np.ascontiguousarray(np.packbits(a, axis=1)).view(np.uint64)
    par = (np.bitwise_count(v[:, None, :] & masks[None, :, :]).sum(2)
           & 1).astype(np.uint8)                              # (nblk, deg)
    out = []
    for row in par:
        x = 0
        for j in range(len(row) - 1, -1, -1):
            x = (x << 1) | int(row[j])
        out.append(x)
    return out


def qc_row_slots(rate, n):
    """Block-row slot lists of a quasi-cyclic Type B code, built from the
    Annex A address rows: (Q, rptr, col, u, wrap).  Row r, in position
    order: its information circulants by block column (column g, shift
    x // Q for entry x with x % Q == r), then the dual-diagonal parity slots
    (columns K/360 + r - 1 and K/360 + r; row 0: K/360 and the wrap slot
    K/360 + Q - 1 with shift 1)."""
    typ, K, M1, M2, Q1, Q = C.ldpc_params(rate, n)
    if typ != "B":
        raise ValueError("layered oracle: Type B codes only")
    rowptr, addr = C.address_rows(rate, n)
    nbi = K // 360
    rows = [[] for _ in range(Q)]
    for g in range(nbi):
        for x in addr[rowptr[g]:rowptr[g + 1]]:
            rows[x % Q].append((g, x // Q, 0))
    rp, col, u, wrap = [0], [], [], []
    for r in range(Q):
        sl = sorted(rows[r])
        if len(set(g for g, _, _ in sl)) != len(sl):
            raise ValueError("two circulants share a block: not layerable")
        sl += [(nbi + r - 1, 0, 0), (nbi + r, 0, 0)] if r else \
              [(nbi, 0, 0), (nbi + Q - 1, 1, 1)]
        for g, uu, w in sl:
            col.append(g)
            u.append(uu)
            wrap.append(w)
        rp.append(len(col))
    return (Q,) + tuple(np.asarray(a, np.int32) for a in (rp, col, u, wrap))


def layered(llr, rate, n, iters=50, alpha=0.75):
    """Oracle layered decode (the GPU layered schedule): (bits, conv, its, bad)."""
    Q, rp, col, u, wrap = qc_row_slots(rate, n)
    llr = np.ascontiguousarray(llr, np.float32)
    nblk = llr.shape[0]
    bits = np.zeros((nblk, n), np.uint8)
    conv = np.zeros(nblk, np.uint8)
    its = np.zeros(nblk, np.int32)
    bad = np.zeros(nblk, np.int32)
    rc = oracle_lib().oracle_layered_f32(
        _p(llr), nblk, n, Q, _p(rp), _p(col), _p(u), _p(wrap), int(iters),
        float(alpha), _p(bits), _p(conv), _p(its), _p(bad))
    if rc != 0:
        raise RuntimeError(f"oracle layered decode returned {rc}")
    return bits, conv.astype(bool), its, bad


# ---------------------------------------------------------------------------
# time de-interleavers (checkers of csrc/timeint.cu)
# ---------------------------------------------------------------------------

def tbi_read_order(nrows, ncols, n_virtual=0):
    """Memory index of each transmitted cell of a twisted-block TI block,
    virtual positions dropped.  Follows lab/m6_tbi.py:46-58 (A/322 7.1.5.4):
    R = i mod Nr, C = ((R mod Nc) + i div Nr) mod Nc, theta = Nr*C + R."""
    out = []
    for i in range(nrows * ncols):
        r = i % nrows
        c = ((r % ncols) + i // nrows) % ncols
        theta = nrows * c + r
        if theta >= n_virtual * nrows:
            out.append(theta - n_virtual * nrows)
    return np.array(out, np.int64)


def tbi_deinterleave(cells, nrows, ncols, n_virtual=0):
    """Transmitted order -> memory order (FEC Block major); follows
    lab/m6_tbi.py:61-68."""
    order = tbi_read_order(nrows, ncols, n_virtual)
    out = np.empty_like(np.asarray(cells))
    out[order] = cells
    return out


def cti_deinterleave(recv, nrows, start_row, n_out):
    """Pre-interleaver cells from the received stream, and the valid mask;
    follows lab/m10_cti.py:97-100 and :126-141 (out[i] = recv[q(i)],
    q(i) = i + Nrows*((start_row + i) mod Nrows))."""
    recv = np.asarray(recv)
    i = np.arange(n_out, dtype=np.int64)
    q = i + nrows * ((start_row + i) % nrows)
    valid = q < len(recv)
    out = np.zeros(n_out, recv.dtype)
    out[valid] = recv[q[valid]]
    return out, valid


# ---------------------------------------------------------------------------
# exact sum-product (checker of csrc/sp.cu)
# ---------------------------------------------------------------------------

def sum_product(lam2d, tables, n, iters=100):
    """Float64 log-tanh belief propagation with the stopping rule of
    lab/m16_margin.py:325-390 (sum_product_decode_batch, deadline None):
    padded (check, slot) view of the CSR tables as lab/m3_ldpc.py:228-242
    `pack` builds it, syndrome before each update, messages
    +-2 atanh(exp(clip(sum log|tanh(v/2)| - own, -700, -1e-16))), totals
    rebuilt as llr + messages accumulated in (check, slot) order.
    Returns (bits uint8, conv bool, its int32, bad int32)."""
    cptr, cidx = np.asarray(tables[0]), np.asarray(tables[1])
    nc = len(cptr) - 1
    deg = np.diff(cptr)
    dmax = int(deg.max())
    idx = np.full((nc, dmax), n, np.int64)
    mask = np.zeros((nc, dmax), bool)
    for c in range(nc):
        idx[c, :deg[c]] = cidx[cptr[c]:cptr[c + 1]]
        mask[c, :deg[c]] = True
    lam2d = np.asarray(lam2d, np.float64)
    nblk = lam2d.shape[0]
    tot = np.zeros((nblk, n + 1))
    tot[:, :n] = lam2d
    m = np.zeros((nblk, nc, dmax))
    bits = (lam2d < 0).astype(np.uint8)
    conv = np.zeros(nblk, bool)
    its = np.full(nblk, iters, np.int32)
    bad_out = np.full(nblk, -1, np.int32)
    act = np.arange(nblk)
    for it in range(iters + 1):
        gg = tot[:, idx]
        syn = np.bitwise_xor.reduce((gg < 0) & mask, axis=2)
        bad = syn.sum(axis=1, dtype=np.int32)
        done = bad == 0
        if done.any():
            sel = act[done]
            bits[sel] = tot[done, :n] < 0
            conv[sel] = True
            its[sel] = it
            bad_out[sel] = 0
            keep = ~done
            if not keep.any():
                return bits, conv, its, bad_out
            act, tot, m, gg, bad = act[keep], tot[keep], m[keep], gg[keep], bad[keep]
        if it == iters:
            bits[act] = tot[:, :n] < 0
            bad_out[act] = bad
            its[act] = it
            break
        v = gg - m
        t = np.tanh(np.clip(v, -38.0, 38.0) * 0.5)
        sg = t < 0
        parity = np.bitwise_xor.reduce(sg & mask, axis=2)
        lt = np.log(np.clip(np.abs(t), 1e-300, 1.0))
        lt[:, ~mask] = 0.0
        lsum = lt.sum(axis=2, keepdims=True)
        le = np.clip(lsum - lt, -700.0, -1e-16)
        mnew = 2.0 * np.arctanh(np.clip(np.exp(le), 0.0, 1.0 - 1e-16))
        sgn = np.where(parity[:, :, None] ^ sg, -1.0, 1.0)
        m = np.where(mask, sgn * mnew, 0.0)
        na = len(act)
        tot[:, :n] = lam2d[act]
        tot[:, n] = 0.0
        np.add.at(tot, (np.arange(na)[:, None, None], idx[None, :, :]), m)
        tot[:, n] = 0.0
    return bits, conv, its, bad_out


def near_miss_llr(rate, n, nblk, mu, seed):
    """Consistent-Gaussian LLRs of random codewords (llr = (1 - 2c)*mu +
    N(0, 2*mu)): the seeded input of the sum-product checks."""
    rng = np.random.default_rng(seed)
    K = C.kldpc(rate, n)
    info = rng.integers(0, 2, (nblk, K)).astype(np.uint8)
    cw = ldpc_encode(info, rate, n)
    lam = (1.0 - 2.0 * cw) * mu + rng.standard_normal(cw.shape) * np.sqrt(2.0 * mu)
    return lam.astype(np.float32), cw


# ---------------------------------------------------------------------------
# common phase error correction (checker of csrc/cpe.cu)
# ---------------------------------------------------------------------------

def cpe_correct(pool, symbol_of, alphabets, region, dummy_values, iters=3):
    """Per-OFDM-symbol decision-directed complex gain, lab/m6_cells.py:176-209:
    normalise the pool to unit mean power, then per symbol `iters` times:
    hard decisions (nearest point of the cell's region alphabet, region 2 =
    known dummy values), c = <hard, z> / max(<hard, hard>, 1e-12), z /= c.
    Returns (out complex128, {symbol: total gain})."""
    out = pool / np.sqrt(np.mean(np.abs(pool) ** 2))
    gains = {}
    for sym in np.unique(symbol_of):
        m = np.flatnonzero(symbol_of == sym)
        z = out[m]
        r = region[m]
        c_tot = 1.0 + 0j
        for _ in range(iters):
            hard = np.empty_like(z)
            for rid, pts in enumerate(alphabets):
                sel = r == rid
                if sel.any():
                    d = np.abs(z[sel][:, None] - pts[None, :])
                    hard[sel] = pts[d.argmin(1)]
            sel = r == 2
            if sel.any():
                hard[sel] = dummy_values[m[sel]]
            c = np.vdot(hard, z) / max(np.vdot(hard, hard).real, 1e-12)
            z = z / c
            c_tot *= c
        out[m] = z
        gains[int(sym)] = complex(c_tot)
    return out, gains


def cpe_pool(nsym, per_sym, mods, seed, esn0_db=18.0):
    """Seeded synthetic cell pool for the CPE checks: per symbol a block of
    region-0 cells (alphabet mods[0]), region-1 cells (mods[1]) and known
    +-1 dummy cells, each symbol rotated by its own complex gain, AWGN.
    Returns (pool, symbol_of, alphabets, region, dummy_values)."""
    rng = np.random.default_rng(seed)
    alph = [np.asarray(C.points_for(m, r), np.complex128) for m, r in mods]
    n = nsym * per_sym
    symbol_of = np.repeat(np.arange(nsym), per_sym)
    region = rng.choice(np.array([0, 0, 0, 1, 2], np.uint8), n)
    x = np.empty(n, np.complex128)
    for rid in (0, 1):
        sel = region == rid
        x[sel] = alph[rid][rng.integers(0, len(alph[rid]), sel.sum())]
    dummy = np.zeros(n, np.complex128)
    sel = region == 2
    dummy[sel] = 1.0 - 2.0 * rng.integers(0, 2, sel.sum())
    x[sel] = dummy[sel]
    g = (1.0 + 0.1 * rng.standard_normal(nsym)) * np.exp(1j * rng.uniform(-0.3, 0.3, nsym))
    n0 = 10 ** (-esn0_db / 10.0)
    nz = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * np.sqrt(n0 / 2)
    pool = x * g[symbol_of] * 1.7 + nz
    return pool, symbol_of, alph, region, dummy


def ladder(llr, tables, n, alphas=(1.0, 0.85, 0.75), iters=50):
    """The alpha ladder of lab/m9_fast.py:843-885 / lab/m44_ldm.py:2497-2526
    over the oracle's flooding decoder: blocks that did not converge are
    decoded again at the next alpha; a block keeps the first converged rung,
    else the rung with the fewest unsatisfied checks.  Returns (bits, conv,
    its, bad, alpha_kept)."""
    llr = np.asarray(llr, np.float32)
    nb = llr.shape[0]
    bits = np.zeros((nb, n), np.uint8)
    conv = np.zeros(nb, bool)
    its = np.zeros(nb, np.int32)
    bad = np.full(nb, 1 << 30, np.int32)
    kept = np.full(nb, -1.0, np.float32)
    todo = np.arange(nb)
    for a in alphas:
        if not len(todo):
            break
        b, c, it, d = flood(llr[todo], tables, n, iters=iters, alpha=a)
        take = c | (d < bad[todo])
        sel = todo[take]
        bits[sel], conv[sel], its[sel], bad[sel] = b[take], c[take], it[take], d[take]
        kept[sel] = a
        todo = todo[~c]
    return bits, conv, its, bad, kept
