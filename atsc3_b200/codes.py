"""ATSC A/322 code construction for the FEC back end (host side, numpy).

Everything the GPU kernels need about a (Ninner, rate, constellation) triple
is derived here from the standard's numeric tables in ``data/a322_tables.npz``:

* ``parity_check(rate, n)``  -- the LDPC parity-check matrix as per-check
  column lists, built from the Annex A address tables by the accumulator rule
  of A/322 6.1.3.1 (Type A) / 6.1.3.2 (Type B).  Same matrix, same check order
  and same ascending column order as ``lab/m3_ldpc.py:166-212``
  (``parity_check``; ``_addr`` :63, ``_pi`` :69, ``_params`` :85), including
  the GF(2) cancellation of a column listed twice in one check (:199-211).
* ``csr(rate, n)``  -- the check-major CSR (``cptr``, ``cidx``) and the
  variable-major edge lists (``vptr``, ``vedge``) exactly as
  ``lab/m3_ldpc.py:459-482`` (``_kernel_tables``) builds them for the
  ``ldpc_minsum_f32`` C ABI: ``vedge`` is the stable argsort of ``cidx``.
* ``bicm_map(n, mod, rate)``  -- ``lam_of_q``, the composite bit
  de-interleaver permutation of ``lab/m6_bicm.py:185-190`` (parity
  interleaver identity :76, group-wise :137, block interleaver :152).
* ``points_for(mod, rate)``  -- the constellation alphabet with index =
  label, y0 = MSB (``lab/m6_bicm.py:197-210``; NUC quadrant rule
  ``lab/spec_nuc.py:77-80``).  1024- and 4096-point alphabets have no NUC
  table in the data; ``points_for`` raises for them and ``standin_qam``
  gives the uniform square QAM stand-in (``lab/spec_nuc.py:169``).
* BCH generator polynomials (``lab/m6_bicm.py:243-266``) and the Baseband
  Packet scrambling sequence (``lab/m4_scrambler.py:148``).

All builders are vectorised; results are cached per key.
"""
from __future__ import annotations

import functools
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLES = os.path.join(HERE, "data", "a322_tables.npz")

RATES = ("2/15", "3/15", "4/15", "5/15", "6/15", "7/15", "8/15", "9/15",
         "10/15", "11/15", "12/15", "13/15")
MOD_BITS = {"QPSK": 2, "16QAM": 4, "64QAM": 6, "256QAM": 8, "1024QAM": 10,
            "4096QAM": 12}
MOUTER = {16200: 168, 64800: 192}
ALPHA_LADDER = (1.0, 0.85, 0.75)          # lab/m6_bicm.py:313
MAX_ROW_DEG = 128                          # lab/ldpc_kernel.c:48


@functools.lru_cache(maxsize=1)
def _tables():
    z = np.load(TABLES)
    arrs = {k: z[k] for k in z.files}
    meta = json.loads(str(arrs.pop("meta_json")))
    return meta, arrs


def _check_n(n):
    if n not in (16200, 64800):
        raise ValueError(f"Ninner must be 16200 or 64800, got {n!r}")


def _check_rate(rate):
    if rate not in RATES:
        raise ValueError(f"unknown code rate {rate!r}")


def ldpc_params(rate, n=16200):
    """(type, K, M1, M2, Q1, Q2) for (rate, Ninner) -- lab/m3_ldpc.py:85-112."""
    _check_n(n)
    _check_rate(rate)
    meta, _ = _tables()
    P = meta["ldpc"][f"{n}:{rate}"]
    K = int(P["Kldpc"])
    if P["type"] == "A":
        M1, M2, Q1, Q2 = (int(P["M1"]), int(P["M2"]), int(P["Q1"]),
                          int(P["Q2"]))
    else:
        M1, M2, Q1 = 0, n - K, 0
        Q2 = int(P["Qldpc"] or (n - K) // 360)
    return P["type"], K, M1, M2, Q1, Q2


def kldpc(rate, n=16200):
    return ldpc_params(rate, n)[1]


def kpayload(rate, n=16200):
    """K_payload = K_ldpc - Mouter (lab/m6_bicm.py:265,324)."""
    return kldpc(rate, n) - MOUTER[n]


def address_rows(rate, n=16200):
    """Annex A address table rows as (rowptr, addr) int32 arrays."""
    _, arrs = _tables()
    key = f"{n}:{rate}"
    return arrs[f"ldpc_rowptr/{key}"], arrs[f"ldpc_addr/{key}"]


def _addr(x, mm, M1, M2, Q1, Q2):
    """Accumulator address of table entry x for bit mm of its 360-group
    (A/322 6.1.3.1 step ii; lab/m3_ldpc.py:63-66).  Vectorised."""
    x = np.asarray(x, np.int64)
    mm = np.asarray(mm, np.int64)
    lo = (x + mm * Q1) % max(M1, 1)
    hi = M1 + (x - M1 + mm * Q2) % M2
    return np.where(x < M1, lo, hi)


def _pi(a, M1, M2, Q1, Q2, K):
    """Accumulator index -> codeword index of the parity bit it becomes
    (A/322 6.1.3.1 steps vi/viii, the "standard" bijection of
    lab/m3_ldpc.py:69-82).  Vectorised."""
    a = np.asarray(a, np.int64)
    s1, t1 = np.divmod(a, max(Q1, 1))
    b = a - M1
    s2, t2 = np.divmod(b, Q2)
    return np.where(a < M1, K + 360 * t1 + s1, K + M1 + 360 * t2 + s2)


def _expand_rows(rowptr, addr, row_lo, nbits):
    """Edges (accumulator, bit-offset) contributed by `nbits` consecutive bits
    that use table rows row_lo.. (one row per 360 bits)."""
    bit = np.arange(nbits, dtype=np.int64)
    row = row_lo + bit // 360
    mm = bit % 360
    cnt = (rowptr[row + 1] - rowptr[row]).astype(np.int64)
    rep_bit = np.repeat(bit, cnt)
    first = np.repeat(rowptr[row].astype(np.int64), cnt)
    within = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    x = addr[first + within]
    return x, np.repeat(mm, cnt), rep_bit


@functools.lru_cache(maxsize=None)
def _parity_edges(rate, n):
    """(check, column) pairs of H after GF(2) cancellation, sorted
    check-major / column-minor."""
    typ, K, M1, M2, Q1, Q2 = ldpc_params(rate, n)
    rowptr, addr = address_rows(rate, n)
    rows, cols = [], []
    # information bits: every table entry of the bit's 360-group row
    x, mm, bit = _expand_rows(rowptr, addr, 0, K)
    rows.append(_addr(x, mm, M1, M2, Q1, Q2))
    cols.append(bit)
    M = M1 + M2
    if typ == "A":
        # step (vii): the M1 dual-diagonal parity bits, in codeword order
        # K + i, are fed back through the Q1 extra rows
        x, mm, bit = _expand_rows(rowptr, addr, K // 360, M1)
        rows.append(_addr(x, mm, M1, M2, Q1, Q2))
        cols.append(K + bit)
        a = np.arange(M1)
        rows += [a, a[1:]]
        cols += [_pi(a, M1, M2, Q1, Q2, K), _pi(a[1:] - 1, M1, M2, Q1, Q2, K)]
        a2 = np.arange(M1, M)
        rows.append(a2)
        cols.append(_pi(a2, M1, M2, Q1, Q2, K))
    else:
        a = np.arange(M)
        rows += [a, a[1:]]
        cols += [_pi(a, M1, M2, Q1, Q2, K), _pi(a[1:] - 1, M1, M2, Q1, Q2, K)]
    r = np.concatenate(rows).astype(np.int64)
    c = np.concatenate(cols).astype(np.int64)
    key = r * n + c
    key.sort()
    # a column listed an even number of times in one check cancels
    uniq, cnt = np.unique(key, return_counts=True)
    keep = uniq[(cnt & 1) == 1]
    return (keep // n).astype(np.int32), (keep % n).astype(np.int32), M


def parity_check(rate, n=16200):
    """H as a list of ascending column lists, one per check equation."""
    r, c, M = _parity_edges(rate, n)
    ptr = np.searchsorted(r, np.arange(M + 1))
    return [c[ptr[i]:ptr[i + 1]].tolist() for i in range(M)]


@functools.lru_cache(maxsize=None)
def csr(rate, n=16200):
    """(cptr, cidx, vptr, vedge) int32, the ``ldpc_minsum_f32`` tables."""
    r, c, M = _parity_edges(rate, n)
    cptr = np.searchsorted(r, np.arange(M + 1)).astype(np.int32)
    cidx = c.astype(np.int32)
    vedge = np.argsort(cidx, kind="stable").astype(np.int32)
    counts = np.bincount(cidx, minlength=n)
    vptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    for a in (cptr, cidx, vptr, vedge):
        a.setflags(write=False)
    return cptr, cidx, vptr, vedge


def csr_from_checks(checks, n):
    """CSR tables from an arbitrary per-check column list (any code)."""
    cn = np.array([len(x) for x in checks], np.int32)
    cptr = np.concatenate([[0], np.cumsum(cn)]).astype(np.int32)
    cidx = (np.concatenate([np.asarray(x, np.int32) for x in checks])
            if len(checks) else np.zeros(0, np.int32)).astype(np.int32)
    vedge = np.argsort(cidx, kind="stable").astype(np.int32)
    counts = np.bincount(cidx, minlength=n)
    vptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return cptr, cidx, vptr, vedge


# ---------------------------------------------------------------------------
# A/322 6.2 bit interleaver as index permutations
# ---------------------------------------------------------------------------

def cells_per_block(n, mod):
    meta, _ = _tables()
    v = meta["demux"].get(f"{n}:{mod}")
    if v is None or v[1] is None:
        raise ValueError(f"no ({n}, {mod}) pairing in A/322 Table 6.14")
    return int(v[1])


def groupwise_map(n, mod, rate, invert=False):
    """u_of_v (lab/m6_bicm.py:137-149): output group j carries input group
    pi(j)."""
    _, arrs = _tables()
    key = f"groupwise/{n}:{mod}:{rate}"
    if key not in arrs:
        raise ValueError(f"no group-wise table for ({n}, {mod}, {rate})")
    p = arrs[key].astype(np.int64)
    if invert:
        p = np.argsort(p)
    return (360 * p[:, None] + np.arange(360)[None, :]).ravel()


def blockint_map(n, mod, rate):
    """v_of_q (lab/m6_bicm.py:152-182), Type A column-twist-free block
    interleaver or Type B part-1/part-2 interleaver of A/322 6.2.3."""
    meta, _ = _tables()
    nc = MOD_BITS[mod]
    typ = meta["bi_type"][f"{n}:{nc}:{rate}"]
    q_of_v = np.empty(n, np.int64)
    if typ == "A":
        nr1, nr2, nc2 = meta["type_a"][f"{n}:{mod}"]
        if nr1 is None or nc2 != nc or nr1 + nr2 != n // nc:
            raise ValueError(f"no Type A block interleaver for ({n}, {mod})")
        i = np.arange(nc * nr1)
        cc, rr = i // nr1, i % nr1
        q_of_v[:nc * nr1] = rr * nc + cc
        if nr2:
            i2 = np.arange(n - nc * nr1)
            c2, r2 = i2 // nr2, nr1 + i2 % nr2
            q_of_v[nc * nr1:] = r2 * nc + c2
    else:
        nq, np1, np2 = meta["type_b"][f"{n}:{mod}"]
        if np1 is None or nq != nc or np1 + np2 != n:
            raise ValueError(f"no Type B block interleaver for ({n}, {mod})")
        blk = nq * 360
        row, col = np.divmod(np.arange(blk), 360)
        within = col * nq + row
        base = (np.arange(np1 // blk) * blk)[:, None]
        q_of_v[:np1] = (base + within[None, :]).ravel()
        q_of_v[np1:] = np.arange(np1, n)
    v_of_q = np.empty(n, np.int64)
    v_of_q[q_of_v] = np.arange(n)
    return v_of_q


@functools.lru_cache(maxsize=None)
def bicm_map(n, mod, rate, gw_invert=False):
    """lam_of_q[j] = LDPC codeword bit carried by q_j, int32.

    The A/322 6.2.1 parity interleaver is the identity in this codeword
    ordering (lab/m6_bicm.py:76-107), so the composite is group-wise after
    block interleaver."""
    u_of_v = groupwise_map(n, mod, rate, gw_invert)
    v_of_q = blockint_map(n, mod, rate)
    out = u_of_v[v_of_q].astype(np.int32)
    out.setflags(write=False)
    return out


# ---------------------------------------------------------------------------
# A/322 6.3 constellations
# ---------------------------------------------------------------------------

QPSK_POINTS = np.array([1 + 1j, -1 + 1j, 1 - 1j, -1 - 1j]) / np.sqrt(2)
_NUC_M = {"16QAM": 16, "64QAM": 64, "256QAM": 256}


def points_for(mod, rate):
    """Alphabet (complex128, index = label, y0 = MSB)."""
    if mod == "QPSK":
        return QPSK_POINTS
    if mod not in _NUC_M:
        raise ValueError(f"no NUC table for {mod}; use standin_qam()")
    _, arrs = _tables()
    return arrs[f"nuc/{_NUC_M[mod]}:{rate}"]


def standin_qam(m):
    """Uniform square QAM of order m at unit power, index -> point as
    lab/spec_nuc.py:169-174.  A labelled STAND-IN for the 1024/4096 NUCs,
    whose position vectors the data does not hold."""
    r = int(round(np.sqrt(m)))
    lv = np.arange(-(r - 1), r, 2)
    p = np.array([complex(i, q) for i in lv for q in lv])
    return p / np.sqrt(np.mean(np.abs(p) ** 2))


def alphabet(mod, rate):
    """points_for, falling back to the uniform QAM stand-in for 1024/4096."""
    if mod in ("1024QAM", "4096QAM"):
        return standin_qam(1 << MOD_BITS[mod])
    return points_for(mod, rate)


def point_tables_f32(pts):
    """(pr, pi, p2) float32 exactly as lab/m44_ldm.py:2476-2478 derive them:
    p2 is |p|^2 in float64, rounded once to float32."""
    pts = np.asarray(pts, np.complex128)
    pr = np.asarray(pts.real, np.float32)
    pi = np.asarray(pts.imag, np.float32)
    p2 = (pts.real ** 2 + pts.imag ** 2).astype(np.float32)
    return pr, pi, p2


def bit_masks(nbits):
    """masks[i, k] = bit i of label k, y0 = MSB (lab/m6_bicm.py:203-210)."""
    k = np.arange(1 << nbits)
    return np.array([((k >> (nbits - 1 - i)) & 1).astype(bool)
                     for i in range(nbits)])


# ---------------------------------------------------------------------------
# BCH (A/322 6.1.2.1) and the Baseband Packet scrambler
# ---------------------------------------------------------------------------

def _gf2_mul(a, b):
    r = 0
    while b:
        if b & 1:
            r ^= a
        a <<= 1
        b >>= 1
    return r


@functools.lru_cache(maxsize=None)
def bch_generator(n):
    """g(x) as a Python int (bit k = coefficient of x^k): the product of the
    twelve A/322 factors for this Ninner."""
    _check_n(n)
    meta, _ = _tables()
    g = 1
    for p in meta["bch_polys"][str(n)]:
        g = _gf2_mul(g, sum(1 << e for e in p))
    if g.bit_length() - 1 != MOUTER[n]:
        raise AssertionError("BCH generator degree mismatch")
    return g


@functools.lru_cache(maxsize=None)
def bch_remainder_table(k, n):
    """R[pos] = x^(k-1-pos) mod g(x) as (k, 6) uint32 words, word w holding
    coefficients 32w..32w+31 (bit b = x^(32w+b)).  The BCH syndrome of a
    k-bit MSB-first message is the XOR of R[pos] over its set bits."""
    g = bch_generator(n)
    deg = MOUTER[n]
    out = np.zeros((k, 6), np.uint32)
    r = 1
    mask32 = (1 << 32) - 1
    rows = [0] * k
    for j in range(k):
        rows[k - 1 - j] = r
        r <<= 1
        if (r >> deg) & 1:
            r ^= g
    for w in range(6):
        out[:, w] = np.array([(v >> (32 * w)) & mask32 for v in rows],
                             np.uint64).astype(np.uint32)
    out.setflags(write=False)
    return out


def syndrome_words_to_int(words):
    """(6,) uint32 remainder words -> the Python int m9_accel returns."""
    v = 0
    for w in range(5, -1, -1):
        v = (v << 32) | int(words[w])
    return v


@functools.lru_cache(maxsize=None)
def scrambler_sequence(nbits):
    """Baseband Packet scrambling bits, MSB-first (lab/m4_scrambler.py:148)."""
    meta, arrs = _tables()
    if nbits > meta["scrambler_nbits"]:
        raise ValueError("scrambling sequence longer than the stored table")
    out = np.unpackbits(arrs["scrambler_bits"])[:nbits].astype(np.uint8)
    out.setflags(write=False)
    return out
