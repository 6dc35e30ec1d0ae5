"""LDPC decoding on the GPU: plans, the flooding decoder and the
``GpuMinSum`` drop-in.

``GpuMinSum`` keeps the constructor and ``decode`` signature of
``lab/m9_gpu.py:84-220`` (Felbs/atsc3) so the reference's callers
(``lab/m9_fast.py:872-874``, ``lab/m44_ldm.py:2519-2520``) can use it
unchanged.  Decoding runs in ``libatsc3_fec.so`` (one thread-block cluster per
codeword, state in distributed shared memory); nothing here falls back to a
CPU decoder.

Two bit-exact semantics are offered (``semantics=``):

* ``"torch"`` -- the reference GpuMinSum / numpy float64 decoders
  (``lab/m9_gpu.py:168-211``, ``lab/m3_ldpc.py:560-630``): message update
  first, ``its`` >= 1, variable sums accumulated onto the channel LLR.  The
  default of ``GpuMinSum``, in float64 or float32.
* ``"kernel"`` -- ``lab/ldpc_kernel.c`` and the numpy float32 fast path
  (``lab/m3_ldpc.py:336-397``): syndrome before each update, ``its`` may be
  0, variable sums from +0 then added to the channel LLR.  float32 only.
"""
from __future__ import annotations

import ctypes
import threading
import time

import numpy as np

from . import codes as C
from . import native as N

# torch_bf16 / torch_f16: lab/m9_gpu.py with dtype bfloat16 / float16 (every
# operation computed in float32 and rounded to the narrow type), on float32
# CSR plans only
SEMANTICS = {"kernel": 0, "torch": 1, "torch_bf16": 2, "torch_f16": 3}
_DTYPES = {"float32": 0, "float64": 1}


def _torch():
    import torch
    return torch


class Plan:
    """Device tables of one code for one message dtype and cluster size
    (the CSR decoder of csrc/ldpc_flood.cu, any code)."""

    kind = "csr"

    def __init__(self, cptr, cidx, vptr, vedge, n, dtype="float32",
                 cluster=0):
        self.n = int(n)
        self.nc = len(cptr) - 1
        self.nedges = int(len(cidx))
        self.dtype = dtype
        arrs = [np.ascontiguousarray(a, np.int32)
                for a in (cptr, cidx, vptr, vedge)]
        h = ctypes.c_void_p()
        N.call("atsc3_ldpc_plan_create", *[a.ctypes.data for a in arrs],
               self.n, self.nc, self.nedges, _DTYPES[dtype], int(cluster),
               ctypes.byref(h))
        self._h = h
        info = np.zeros(10, np.int64)
        N.call("atsc3_ldpc_plan_info", h, info.ctypes.data)
        self.info = dict(zip(("n", "nc", "nedges", "cluster", "smem_bytes",
                              "record_bytes", "dmax_c", "dmax_v",
                              "table_bytes", "dtype"), info.tolist()))
        self.cluster = self.info["cluster"]

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                N.lib().atsc3_ldpc_plan_destroy(h)
            except Exception:       # interpreter shutdown
                pass
            self._h = None


class QcPlan:
    """Quasi-cyclic plan of an A/322 Type B code (float32 messages): the
    decoder of csrc/ldpc_qc.cu, driven by circulant descriptors built from
    the Annex A address rows."""

    kind = "qc"

    def __init__(self, rate, n, cluster=0):
        typ, K, M1, M2, Q1, Q2 = C.ldpc_params(rate, n)
        if typ != "B":
            raise ValueError("the quasi-cyclic decoder serves Type B codes")
        rowptr, addr = C.address_rows(rate, n)
        rowptr = np.ascontiguousarray(rowptr, np.int32)
        addr = np.ascontiguousarray(addr, np.int32)
        h = ctypes.c_void_p()
        N.call("atsc3_ldpc_qc_plan_create", n, K, Q2, rowptr.ctypes.data,
               addr.ctypes.data, int(cluster), ctypes.byref(h))
        self._h = h
        self.n, self.nc, self.dtype = n, n - K, "float32"
        info = np.zeros(10, np.int64)
        N.call("atsc3_ldpc_qc_plan_info", h, info.ctypes.data)
        self.info = dict(zip(("n", "K", "Q", "cluster", "smem_bytes",
                              "dr_max", "dc_max", "table_bytes",
                              "rows_per_cta", "cols_per_cta"), info.tolist()))
        self.info["kind"] = "qc"
        self.cluster = self.info["cluster"]

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                N.lib().atsc3_ldpc_qc_plan_destroy(h)
            except Exception:
                pass
            self._h = None


class QcePlan(QcPlan):
    """Quasi-cyclic plan with the edge-buffer state layout (csrc/ldpc_qce.cu):
    one float32 slot per edge in the distributed shared memory of the edge's
    column owner, no per-check records.  Serves every A/322 code (Type A and
    Type B, where QcPlan takes Type B codes with one circulant per block);
    same semantics and outputs; cluster 0 picks the smallest cluster that
    holds a codeword."""

    kind = "qce"

    def __init__(self, rate=None, n=None, cluster=0, dtype="float32", tables=None):
        """rate, n: an A/322 code; or tables = (n, K, qa, qb, rowptr, addr)
        as atsc3_ldpc_qc_detect2 recovers them from CSR tables.  dtype
        float32 or float64 (the float64 build: 8-byte slots, float64
        arithmetic, no learned weights)."""
        if dtype not in ("float32", "float64"):
            raise ValueError("dtype must be float32 or float64")
        if tables is None:
            typ, K, M1, M2, Q1, Q2 = C.ldpc_params(rate, n)
            # accumulator / identity block rows: (Q, 0) for Type B, (Q1, Q2)
            # for Type A
            qa, qb = (Q2, 0) if typ == "B" else (Q1, Q2)
            rowptr, addr = C.address_rows(rate, n)
        else:
            n, K, qa, qb, rowptr, addr = tables
        rowptr = np.ascontiguousarray(rowptr, np.int32)
        addr = np.ascontiguousarray(addr, np.int32)
        h = ctypes.c_void_p()
        fn = ("atsc3_ldpc_qce_plan_create_f64" if dtype == "float64"
              else "atsc3_ldpc_qce_plan_create2")
        N.call(fn, n, K, qa, qb, rowptr.ctypes.data, addr.ctypes.data, int(cluster),
               ctypes.byref(h))
        self._h = h
        self.n, self.nc, self.dtype = n, n - K, dtype
        info = np.zeros(10, np.int64)
        N.call("atsc3_ldpc_qce_plan_info", h, info.ctypes.data)
        self.info = dict(zip(("n", "K", "Q", "cluster", "smem_bytes",
                              "dr_max", "dc_max", "table_bytes",
                              "max_slots_per_cta", "cols_cta0"),
                             info.tolist()))
        self.info["kind"] = "qce"
        self.cluster = self.info["cluster"]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                N.lib().atsc3_ldpc_qce_plan_destroy(h)
            except Exception:
                pass
            self._h = None


_PLANS = {}
_PLANS_LOCK = threading.Lock()


def plan_for(rate, n, dtype="float32", cluster=0, kind="auto"):
    """Cached plan of an A/322 code.  kind "auto" picks the edge-buffer
    quasi-cyclic decoder (every code, float32 or float64), then in float32
    the record-layout one (Type B codes with one circulant per block),
    whichever first accepts the code; else the CSR decoder.  kind "qce" or
    "qc" asks for that decoder (raising if it rejects a code in its reach);
    codes outside its reach (float64 or Type A for "qc") get the CSR
    decoder."""
    torch = _torch()
    key = (rate, n, dtype, cluster, kind, torch.cuda.current_device())
    with _PLANS_LOCK:
        p = _PLANS.get(key)
        if p is None:
            f32 = dtype == "float32"
            type_b = C.ldpc_params(rate, n)[0] == "B"
            for k, cls, ok in (("qce", QcePlan, True), ("qc", QcPlan, f32 and type_b)):
                if p is None and kind in ("auto", k) and ok:
                    try:
                        p = (cls(rate, n, cluster=cluster, dtype=dtype) if k == "qce"
                             else cls(rate, n, cluster=cluster))
                    except N.FecError as e:
                        if kind == k or e.rc != -4:
                            raise
            if p is None:
                p = Plan(*C.csr(rate, n), n, dtype=dtype, cluster=cluster)
            _PLANS[key] = p
    return p


def decode_flood(plan, llr, iters=50, alpha=0.75, semantics="kernel",
                 want_bits=True, want_hard=False, threads=0, out=None,
                 stream=None, weights=None):
    """Decode (nblk, n) device LLRs.  Returns a dict of device tensors:
    bits (uint8, nblk x n) and/or hard (packed, nblk x ceil(n/32)*4 bytes),
    conv (uint8), its (int32), bad (int32).  weights: optional learned
    (walpha, wbeta, dbucket) device tensors (quasi-cyclic plans only), or
    (walpha, wbeta, rbucket, "row") for weights per block row (the
    edge-buffer plan only; ``learned.inference_weights``)."""
    torch = _torch()
    want_t = torch.float64 if plan.dtype == "float64" else torch.float32
    if llr.dtype != want_t or llr.device.type != "cuda":
        raise TypeError(f"llr must be a CUDA {want_t} tensor")
    if llr.dim() != 2 or llr.shape[1] != plan.n or (llr.shape[0] and llr.stride(1) != 1):
        raise ValueError("llr must be (nblk, n) with unit column stride")
    nblk = llr.shape[0]
    dev = llr.device
    o = out if out is not None else {}
    if want_bits and "bits" not in o:
        o["bits"] = torch.empty((nblk, plan.n), dtype=torch.uint8, device=dev)
    if want_hard and "hard" not in o:
        o["hard"] = torch.empty((nblk, (plan.n + 31) // 32 * 4),
                                dtype=torch.uint8, device=dev)
    for k, dt in (("conv", torch.uint8), ("its", torch.int32),
                  ("bad", torch.int32)):
        if k not in o:
            o[k] = torch.empty(nblk, dtype=dt, device=dev)
    bits = o.get("bits") if want_bits else None
    hard = o.get("hard") if want_hard else None
    if nblk == 0:                  # nothing to launch (empty tensors' strides are arbitrary)
        return o
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    kind = getattr(plan, "kind", "csr")
    if weights is not None and kind not in ("qc", "qce"):
        raise ValueError("learned weights run on the quasi-cyclic decoders")
    if kind == "qce" and plan.dtype == "float64":
        if weights is not None:
            raise ValueError("learned weights run on the float32 decoders")
        N.call("atsc3_ldpc_qce_decode_f64", plan.handle, llr.data_ptr(),
               llr.stride(0), nblk, int(iters), float(alpha), SEMANTICS[semantics],
               N.ptr(bits), bits.stride(0) if bits is not None else 0, N.ptr(hard),
               hard.stride(0) if hard is not None else 0, o["conv"].data_ptr(),
               o["its"].data_ptr(), o["bad"].data_ptr(), int(threads), st)
        return o
    if kind in ("qc", "qce"):
        wa = wb = db = None
        wT = wnb = 0
        rows = False
        if weights is not None:
            wa, wb, db = weights[:3]
            rows = len(weights) > 3 and weights[3] == "row"
            wT, wnb = wa.shape
        if rows and kind != "qce":
            raise ValueError("per-row weights run on the edge-buffer decoder")
        fn = ("atsc3_ldpc_qc_decode_weighted" if kind == "qc"
              else "atsc3_ldpc_qce_decode_weighted_rows" if rows
              else "atsc3_ldpc_qce_decode_weighted")
        N.call(fn, plan.handle, llr.data_ptr(),
               llr.stride(0), nblk, int(iters), float(alpha),
               SEMANTICS[semantics], N.ptr(wa), N.ptr(wb), wT, wnb, N.ptr(db),
               N.ptr(bits),
               bits.stride(0) if bits is not None else 0, N.ptr(hard),
               hard.stride(0) if hard is not None else 0,
               o["conv"].data_ptr(), o["its"].data_ptr(), o["bad"].data_ptr(),
               int(threads), st)
        return o
    N.call("atsc3_ldpc_decode_flood", plan.handle, llr.data_ptr(),
           llr.stride(0), nblk, int(iters), float(alpha),
           SEMANTICS[semantics], N.ptr(bits),
           bits.stride(0) if bits is not None else 0, N.ptr(hard),
           hard.stride(0) if hard is not None else 0, o["conv"].data_ptr(),
           o["its"].data_ptr(), o["bad"].data_ptr(), int(threads), st)
    return o


def qce_plan_from_csr(tables, n, dtype="float32", cluster=0):
    """The edge-buffer plan of the A/322 code whose CSR tables these are
    (atsc3_ldpc_qc_detect2: circulant structure, accumulator and identity
    parity, reference edge order), or None for any other matrix or a code
    the decoder does not take."""
    cptr, cidx, vptr, vedge = [np.ascontiguousarray(t, np.int32) for t in tables]
    nc, ne = len(cptr) - 1, len(cidx)
    kq = np.zeros(3, np.int32)
    rowptr = np.zeros(n // 360 + 1, np.int32)
    addr = np.zeros(max(ne, 1), np.int32)
    rc = N.lib().atsc3_ldpc_qc_detect2(cptr.ctypes.data, cidx.ctypes.data,
                                       vptr.ctypes.data, vedge.ctypes.data, n, nc, ne,
                                       kq.ctypes.data, rowptr.ctypes.data,
                                       addr.ctypes.data)
    if rc == -4:
        return None
    N.check("atsc3_ldpc_qc_detect2", rc)
    K, qa, qb = (int(x) for x in kq)
    nrows = K // 360 + (qa if qb else 0)
    try:
        return QcePlan(dtype=dtype, cluster=cluster,
                       tables=(n, K, qa, qb, rowptr[:nrows + 1], addr[:rowptr[nrows]]))
    except N.FecError as e:
        if e.rc != -4:
            raise
        return None


class GpuMinSum:
    """Batched normalised min-sum for ONE (rate, Ninner) code -- drop-in for
    ``lab/m9_gpu.py:84-220``.

    ``checks`` is the per-check column list (``m3_ldpc.parity_check``).
    ``decode(llr2d)`` takes (nblk, n) LLRs as numpy or a CUDA tensor and
    returns numpy ``(bits uint8, converged bool, iters int32, bad int32)``.
    """

    BIG = 1e9

    def __init__(self, checks, n, iters=50, alpha=0.75, device="cuda",
                 dtype="float64", semantics="torch", cluster=0):
        torch = _torch()
        if dtype not in ("float64", "float32", "bfloat16", "float16"):
            raise ValueError("dtype must be float64, float32, bfloat16 or float16")
        if semantics == "kernel" and dtype != "float32":
            raise ValueError("kernel semantics are float32 only")
        narrow = dtype in ("bfloat16", "float16")
        self.n, self.iters, self.alpha = int(n), iters, alpha
        self.dev = torch.device(device)
        # bfloat16/float16 (lab/m9_gpu.py:100-101): the LLRs are rounded to
        # that type as the reference's .to(dtype) does, and the CSR decoder
        # rounds every operation's result to it (semantics torch_bf16 /
        # torch_f16), holding the values in float32
        self.dt = {"float64": torch.float64, "float32": torch.float32,
                   "bfloat16": torch.bfloat16, "float16": torch.float16}[dtype]
        self.dtype_name = dtype
        self.semantics = semantics
        if narrow:
            self.semantics = "torch_bf16" if dtype == "bfloat16" else "torch_f16"
        with torch.cuda.device(self.dev):
            tabs = C.csr_from_checks(checks, n)
            pdt = "float32" if narrow else dtype
            # an A/322 code (recognised from its CSR tables) takes the
            # edge-buffer decoder, any other matrix (and the narrow types)
            # the CSR decoder
            self.plan = None if narrow else qce_plan_from_csr(tabs, n, dtype=pdt,
                                                              cluster=cluster)
            if self.plan is None:
                self.plan = Plan(*tabs, n, dtype=pdt, cluster=cluster)
        self.nc = self.plan.nc
        self.stats = dict(calls=0, iters=0, blocks=0)

    def decode(self, llr2d, iters=None, alpha=None):
        torch = _torch()
        iters = iters or self.iters
        alpha = self.alpha if alpha is None else alpha
        if isinstance(llr2d, torch.Tensor):
            llr = llr2d.to(self.dev, dtype=self.dt).contiguous()
        else:
            a = np.ascontiguousarray(np.asarray(llr2d, np.float64))
            llr = torch.from_numpy(a).to(self.dev, dtype=self.dt)
        if self.dt in (torch.bfloat16, torch.float16):
            llr = llr.float()           # exact: the decoder holds float32
        if llr.dim() != 2 or llr.shape[1] != self.n:
            raise ValueError(f"expected (nblk, {self.n}) LLRs")
        nb = llr.shape[0]
        with torch.cuda.device(self.dev):
            o = decode_flood(self.plan, llr, iters=iters, alpha=alpha,
                             semantics=self.semantics)
        self.stats["calls"] += 1
        self.stats["blocks"] += nb
        its = o["its"].cpu().numpy()
        self.stats["iters"] += int(its.max(initial=0))
        return (o["bits"].cpu().numpy(), o["conv"].cpu().numpy().astype(bool),
                its, o["bad"].cpu().numpy())


class LayeredPlan:
    """Layered min-sum plan of an A/322 Type B code (csrc/ldpc_layered.cu).

    Not bit-comparable with the flooding decoders (different schedule);
    bit-exact with oracle.layered.  ``ctas`` = resident CTAs (codewords in
    flight); the scratch workspace is allocated once per plan for them."""

    kind = "layered"

    def __init__(self, rate, n, ctas=0, device=None):
        torch = _torch()
        typ, K, M1, M2, Q1, Q2 = C.ldpc_params(rate, n)
        if typ != "B":
            raise ValueError("the layered decoder serves Type B codes")
        rowptr, addr = [np.ascontiguousarray(a, np.int32)
                        for a in C.address_rows(rate, n)]
        h = ctypes.c_void_p()
        N.call("atsc3_ldpc_layered_plan_create", n, K, Q2, rowptr.ctypes.data,
               addr.ctypes.data, ctypes.byref(h))
        self._h = h
        self.n, self.rate, self.dtype = n, rate, "float32"
        self.device = torch.device(device or "cuda")
        if not ctas:
            sms = torch.cuda.get_device_properties(self.device).multi_processor_count
            ctas = 2 * sms
        self.ctas = int(ctas)
        nbytes = ctypes.c_int64()
        N.call("atsc3_ldpc_layered_workspace", h, self.ctas, ctypes.byref(nbytes))
        self.ws = torch.empty(nbytes.value, dtype=torch.uint8, device=self.device)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                N.lib().atsc3_ldpc_layered_plan_destroy(h)
            except Exception:
                pass
            self._h = None


def decode_layered(plan, llr, iters=50, alpha=0.75, want_bits=True,
                   want_hard=False, out=None, stream=None):
    """Layered decode of (nblk, n) float32 CUDA LLRs; same outputs as
    decode_flood.  Raises if a staged copy timed out (bounded waits)."""
    torch = _torch()
    if llr.dtype != torch.float32 or llr.device.type != "cuda":
        raise TypeError("llr must be a CUDA float32 tensor")
    if llr.dim() != 2 or llr.shape[1] != plan.n or (llr.shape[0] and llr.stride(1) != 1):
        raise ValueError("llr must be (nblk, n) with unit column stride")
    nblk = llr.shape[0]
    dev = llr.device
    o = out if out is not None else {}
    if want_bits and "bits" not in o:
        o["bits"] = torch.empty((nblk, plan.n), dtype=torch.uint8, device=dev)
    if want_hard and "hard" not in o:
        o["hard"] = torch.empty((nblk, (plan.n + 31) // 32 * 4),
                                dtype=torch.uint8, device=dev)
    for k, dt in (("conv", torch.uint8), ("its", torch.int32),
                  ("bad", torch.int32)):
        if k not in o:
            o[k] = torch.empty(nblk, dtype=dt, device=dev)
    bits = o.get("bits") if want_bits else None
    hard = o.get("hard") if want_hard else None
    if nblk == 0:                  # nothing to launch (empty tensors' strides are arbitrary)
        return o
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    N.call("atsc3_ldpc_layered_decode", plan.handle, llr.data_ptr(),
           llr.stride(0), nblk, int(iters), float(alpha), N.ptr(bits),
           bits.stride(0) if bits is not None else 0, N.ptr(hard),
           hard.stride(0) if hard is not None else 0, o["conv"].data_ptr(),
           o["its"].data_ptr(), o["bad"].data_ptr(), plan.ws.data_ptr(),
           plan.ctas, plan.err.data_ptr(), st)
    return o


def check_layered_error(plan):
    """Raise if a layered launch recorded a copy timeout (syncs).  Code 1:
    a wait ran out and the CTA returned after its copies completed; code 2:
    the second wait ran out as well, so copies may have been in flight when
    the CTA returned."""
    code = int(plan.err.item())
    if code != 0:
        plan.err.zero_()
        what = ("a staged copy did not complete in time (bounded wait); the "
                "CTA returned after its copies landed" if code == 1 else
                "a staged copy did not complete within two bounded waits; "
                "copies may have been in flight when the CTA returned")
        raise N.FecError("atsc3_ldpc_layered_decode", -2,
                         f"{what} (error code {code})")


# ---------------------------------------------------------------------------
# exact sum-product: the near-miss rescue (csrc/sp.cu)
# ---------------------------------------------------------------------------

_SP_TABLES = {}
_SP_LOCK = threading.Lock()


def sp_tables(tables, n, device="cuda"):
    """Device copies of CSR tables (cptr, cidx, vptr, vedge) for sp_decode,
    cached by content."""
    torch = _torch()
    arrs = [np.ascontiguousarray(t, np.int32) for t in tables]
    key = (n, str(torch.device(device)), tuple(hash(a.tobytes()) for a in arrs))
    with _SP_LOCK:
        d = _SP_TABLES.get(key)
        if d is None:
            d = {"n": int(n), "nc": len(arrs[0]) - 1, "nedges": len(arrs[1]),
                 "t": [torch.from_numpy(np.array(a)).to(device) for a in arrs]}
            _SP_TABLES[key] = d
    return d


def sp_decode(tab, llr, iters=100, out=None, stream=None):
    """Float64 log-tanh belief propagation of (nblk, n) CUDA float64 LLRs
    (lab/m16_margin.py:325-390 semantics: syndrome before each update, its
    = the iteration the syndrome vanished, else iters with bad = the
    unsatisfied count).  Returns device tensors bits, conv, its, bad."""
    torch = _torch()
    if llr.dtype != torch.float64 or llr.device.type != "cuda" or \
            llr.dim() != 2 or llr.shape[1] != tab["n"] or \
            (llr.shape[0] and llr.stride(1) != 1):
        raise TypeError("llr must be a (nblk, n) CUDA float64 tensor")
    nblk, n = llr.shape
    dev = llr.device
    o = out if out is not None else {}
    o.setdefault("bits", torch.empty((nblk, n), dtype=torch.uint8, device=dev))
    o.setdefault("conv", torch.empty(nblk, dtype=torch.uint8, device=dev))
    o.setdefault("its", torch.empty(nblk, dtype=torch.int32, device=dev))
    o.setdefault("bad", torch.empty(nblk, dtype=torch.int32, device=dev))
    if nblk == 0:
        return o
    nbytes = ctypes.c_int64()
    N.call("atsc3_ldpc_sp_workspace", n, tab["nedges"], nblk, ctypes.byref(nbytes))
    work = torch.empty(max(8, nbytes.value), dtype=torch.uint8, device=dev)
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    c, ci, v, ve = tab["t"]
    N.call("atsc3_ldpc_sp_decode", c.data_ptr(), ci.data_ptr(), v.data_ptr(),
           ve.data_ptr(), n, tab["nc"], tab["nedges"], llr.data_ptr(),
           llr.stride(0), nblk, int(iters), o["bits"].data_ptr(),
           o["bits"].stride(0), o["conv"].data_ptr(), o["its"].data_ptr(),
           o["bad"].data_ptr(), work.data_ptr(), st)
    o["_work"] = work            # alive until the stream has run the launches
    return o


def sp_decode_deadline(tab, llr, iters=100, deadline=None, out=None,
                       stream=None):
    """sp_decode one iteration at a time, honouring a wall-clock
    ``deadline`` (a ``time.perf_counter()`` value) as lab/m16_margin.py:
    364-371 does: no new iteration starts after it; the iteration at which
    it is found passed takes the syndrome and retires every block still
    decoding with its current decisions (conv False unless the syndrome is
    zero, its = that iteration, bad = the unsatisfied count).  Each
    iteration waits for the GPU, so the clock is read after the work it
    follows.  Returns (device tensors bits/conv/its/bad, the number of
    blocks stopped by the deadline)."""
    torch = _torch()
    nblk, n = llr.shape
    dev = llr.device
    o = out if out is not None else {}
    o.setdefault("bits", torch.empty((nblk, n), dtype=torch.uint8, device=dev))
    o.setdefault("conv", torch.empty(nblk, dtype=torch.uint8, device=dev))
    o.setdefault("its", torch.empty(nblk, dtype=torch.int32, device=dev))
    o.setdefault("bad", torch.empty(nblk, dtype=torch.int32, device=dev))
    if nblk == 0:
        return o, 0
    nbytes = ctypes.c_int64()
    N.call("atsc3_ldpc_sp_workspace", n, tab["nedges"], nblk, ctypes.byref(nbytes))
    work = torch.empty(max(8, nbytes.value), dtype=torch.uint8, device=dev)
    counts = torch.zeros(2, dtype=torch.int32, device=dev)
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    c, ci, v, ve = tab["t"]
    shed = 0
    for it in range(iters + 1):
        last = it == iters or (deadline is not None and
                               time.perf_counter() > deadline)
        N.call("atsc3_ldpc_sp_step", c.data_ptr(), ci.data_ptr(), v.data_ptr(),
               ve.data_ptr(), n, tab["nc"], tab["nedges"], llr.data_ptr(),
               llr.stride(0), nblk, it, int(last), o["bits"].data_ptr(),
               o["bits"].stride(0), o["conv"].data_ptr(), o["its"].data_ptr(),
               o["bad"].data_ptr(), work.data_ptr(), counts.data_ptr(), st)
        active, stopped = (int(x) for x in counts.cpu())   # waits for the step
        if last:
            shed = stopped if it < iters else 0
            break
        if active == 0:
            break
    return o, shed


def sum_product_decode_batch(lam2d, checks, n, iters=100, deadline=None,
                             stats=None):
    """Drop-in for ``lab/m16_margin.py:325`` ``sum_product_decode_batch``:
    numpy (bits uint8, conv bool, its int32, bad int32).  ``deadline``: a
    ``time.perf_counter()`` value after which no new iteration starts
    (sp_decode_deadline); the blocks it stops are counted in
    ``stats["sp_timeout"]``, as the reference counts them.  Without a
    deadline every iteration is queued at once (sp_decode)."""
    torch = _torch()
    tab = sp_tables(C.csr_from_checks(checks, n), n)
    llr = torch.from_numpy(np.ascontiguousarray(lam2d, np.float64)).cuda()
    if deadline is None:
        o = sp_decode(tab, llr, iters=iters)
        torch.cuda.synchronize()
    else:
        o, shed = sp_decode_deadline(tab, llr, iters=iters, deadline=deadline)
        if shed and stats is not None:
            stats["sp_timeout"] = stats.get("sp_timeout", 0) + shed
    return (o["bits"].cpu().numpy(), o["conv"].cpu().numpy().astype(bool),
            o["its"].cpu().numpy(), o["bad"].cpu().numpy())


def rescue_near_misses(tab, lam, out, near_max=1500, max_blocks=8, iters=100,
                       budget_s=None, stats=None):
    """The near-miss rescue of ``lab/m44_ldm.py:2527-2554``: the blocks a
    min-sum decode left unconverged with at most ``near_max`` unsatisfied
    checks (the ``max_blocks`` closest ones) are decoded again with the
    exact float64 sum-product; those that converge replace their packed
    hard decisions (``out["hard"]``) and flags (conv = 1, bad = 0; ``its``
    keeps the min-sum count).  ``lam``: the (nblk, n) float32 LLRs of that
    decode.  Selecting the blocks reads conv/bad on the host (as the
    reference does).  ``budget_s``: the rescue's wall-clock budget from the
    call (lab/m44_ldm.py:2544-2545 with SP_BUDGET_S of :135; None = run to
    ``iters``); blocks it stops are added to ``stats["sp_timeout"]``.
    Returns the indices of the rescued blocks."""
    torch = _torch()
    conv = out["conv"].cpu().numpy()
    bad = out["bad"].cpu().numpy()
    near = np.flatnonzero((conv == 0) & (bad <= near_max))
    if len(near) > max_blocks:
        near = near[np.argsort(bad[near], kind="stable")[:max_blocks]]
    if not len(near):
        return near
    dev = lam.device
    idx = torch.from_numpy(near.astype(np.int64)).to(dev)
    sub = lam.index_select(0, idx).double()
    if budget_s is None:
        o = sp_decode(tab, sub, iters=iters)
    else:
        o, shed = sp_decode_deadline(tab, sub, iters=iters,
                                     deadline=time.perf_counter() + budget_s)
        if shed and stats is not None:
            stats["sp_timeout"] = stats.get("sp_timeout", 0) + shed
    ok = o["conv"].bool()
    sel = idx[ok]
    if sel.numel():
        n = tab["n"]
        w = torch.tensor([128, 64, 32, 16, 8, 4, 2, 1], dtype=torch.int32, device=dev)
        packed = (o["bits"][ok][:, :n // 8 * 8].view(-1, n // 8, 8).int() * w).sum(-1)
        out["hard"][sel, :n // 8] = packed.to(torch.uint8)
        out["conv"][sel] = 1
        out["bad"][sel] = 0
    return near[ok.cpu().numpy()]


# ---------------------------------------------------------------------------
# the alpha ladder
# ---------------------------------------------------------------------------

ALPHA_LADDER = (1.0, 0.85, 0.75)


def ladder_decode(plan, llr, ladder=ALPHA_LADDER, iters=50, semantics="kernel",
                  want_bits=True, threads=0):
    """Normalised min-sum with the reference's alpha ladder
    (``lab/m6_bicm.py:313,341-355`` ``decode_llr``; batched as
    ``lab/m9_fast.py:843-885`` / ``lab/m44_ldm.py:2497-2526``): every block
    is decoded at the first alpha; the blocks that did not converge are
    decoded again at the next one, and so on.  A block keeps the first rung
    that converges, else the rung with the fewest unsatisfied checks (ties
    keep the earlier rung).  Returns device tensors bits (if want_bits),
    hard (packed), conv, its, bad, alpha (the rung kept).  Each rung after the
    first reads the convergence flags on the host (as the reference does)."""
    torch = _torch()
    nb, n = llr.shape
    dev = llr.device
    out = {"hard": torch.zeros((nb, (n + 31) // 32 * 4), dtype=torch.uint8, device=dev),
           "conv": torch.zeros(nb, dtype=torch.uint8, device=dev),
           "its": torch.zeros(nb, dtype=torch.int32, device=dev),
           "bad": torch.full((nb,), 1 << 30, dtype=torch.int32, device=dev),
           "alpha": torch.full((nb,), -1.0, dtype=torch.float32, device=dev)}
    if want_bits:
        out["bits"] = torch.zeros((nb, n), dtype=torch.uint8, device=dev)
    todo = torch.arange(nb, device=dev)
    for a in ladder:
        if todo.numel() == 0:
            break
        sub = llr if todo.numel() == nb else llr.index_select(0, todo)
        o = decode_flood(plan, sub, iters=iters, alpha=a, semantics=semantics,
                         want_bits=want_bits, want_hard=True, threads=threads)
        c = o["conv"].bool()
        take = c | (o["bad"] < out["bad"][todo])
        sel = todo[take]
        for k in ("hard", "conv", "its", "bad") + (("bits",) if want_bits else ()):
            out[k][sel] = o[k][take]
        out["alpha"][sel] = float(a)
        todo = todo[~c]
    return out


def ldpc_batch(lam2d, rate, n, iters=50, alpha=None, ladder=ALPHA_LADDER,
               sp_rescue=None):
    """Host-array form of ``lab/m44_ldm.py:2497`` ``ldpc_batch``: numpy
    (bits uint8, conv bool, bad int32) of (nblk, n) LLRs decoded with the
    single ``alpha`` if given, else the alpha ladder; ``sp_rescue`` (a dict
    of rescue_near_misses arguments) adds the near-miss sum-product, as the
    reference does when ATSC3_LDM_SP is set."""
    torch = _torch()
    plan = plan_for(rate, n)
    x = torch.from_numpy(np.ascontiguousarray(lam2d, np.float32)).cuda()
    o = ladder_decode(plan, x, ladder=(alpha,) if alpha else tuple(ladder),
                      iters=iters, want_bits=True)
    if sp_rescue:
        got = rescue_near_misses(sp_tables(C.csr(rate, n), n), x, o, **sp_rescue)
        if len(got):       # unpack the rescued blocks' packed decisions
            idx = torch.from_numpy(got.astype(np.int64)).cuda()
            h = o["hard"].index_select(0, idx)[:, :n // 8]
            bits = ((h.unsqueeze(-1) >> torch.arange(7, -1, -1, device=h.device)) & 1)
            o["bits"][idx] = bits.reshape(len(got), -1)[:, :n].to(torch.uint8)
    torch.cuda.synchronize()
    return (o["bits"].cpu().numpy(), o["conv"].cpu().numpy().astype(bool),
            o["bad"].cpu().numpy())
