"""BCH zero-syndrome check on the GPU, and the ``m9_accel`` drop-ins.

``bch_syndrome_batch(bits2d, ninner)`` and ``bch_syndrome(bits, ninner)``
keep the signatures and return values of ``lab/m9_accel.py:197-236``
(Python ints, 0 = clean).  ``bch_check`` is the device entry point used by
the pipeline: packed hard decisions in, (syndrome words, ok flag,
descrambled payload bytes) out.
"""
from __future__ import annotations

import numpy as np

from . import codes as C
from . import native as N


def _torch():
    import torch
    return torch


_RT = {}


def device_rtab(k, ninner, device):
    torch = _torch()
    key = (k, ninner, str(device))
    t = _RT.get(key)
    if t is None:
        t = torch.from_numpy(np.array(C.bch_remainder_table(k, ninner))).to(device)
        _RT[key] = t
    return t


def device_scrambler_bytes(kpay, device):
    torch = _torch()
    key = ("scr", kpay, str(device))
    t = _RT.get(key)
    if t is None:
        t = torch.from_numpy(np.packbits(np.array(C.scrambler_sequence(kpay)))).to(device)
        _RT[key] = t
    return t


def bch_check(hard, kldpc, ninner, kpayload=None, want_payload=True, out=None,
              stream=None):
    """hard: (nblk, ld) uint8 CUDA packed hard decisions (first kldpc bits
    = BCH codeword).  Returns dict(syn (nblk,6) int32 view of uint32 words,
    ok (nblk,) uint8, payload (nblk, kpayload/8) uint8)."""
    torch = _torch()
    nblk = hard.shape[0]
    dev = hard.device
    o = out if out is not None else {}
    if "syn" not in o:
        o["syn"] = torch.empty((nblk, 6), dtype=torch.int32, device=dev)
    if "ok" not in o:
        o["ok"] = torch.empty(nblk, dtype=torch.uint8, device=dev)
    rt = device_rtab(kldpc, ninner, dev)
    scr = pay = None
    kp = kpayload if kpayload is not None else kldpc - C.MOUTER[ninner]
    if want_payload:
        scr = device_scrambler_bytes(kp, dev)
        if "payload" not in o:
            o["payload"] = torch.empty((nblk, kp // 8), dtype=torch.uint8,
                                       device=dev)
        pay = o["payload"]
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    N.call("atsc3_bch_check", hard.data_ptr(), hard.stride(0), nblk, kldpc,
           rt.data_ptr(), o["syn"].data_ptr(), o["ok"].data_ptr(), N.ptr(scr),
           kp, N.ptr(pay), pay.stride(0) if pay is not None else 0, st)
    return o


def syndromes_to_ints(syn_words):
    w = np.asarray(syn_words).astype(np.uint32)
    return [C.syndrome_words_to_int(row) for row in w]


def bch_syndrome_batch(bits2d, ninner=16200):
    """Drop-in for ``m9_accel.bch_syndrome_batch``: (nblk, n) {0,1} -> list
    of Python-int syndromes of the n-bit messages."""
    torch = _torch()
    a = np.array(bits2d, np.uint8, ndmin=2)      # fresh C-contiguous copy
    nblk, n = a.shape
    if nblk == 0:
        return []
    dev = torch.device("cuda")
    t = torch.from_numpy(a).to(dev)
    rt = device_rtab(n, ninner, dev)
    syn = torch.empty((nblk, 6), dtype=torch.int32, device=dev)
    N.call("atsc3_bch_syndrome_bits", t.data_ptr(), t.stride(0), nblk, n,
           rt.data_ptr(), syn.data_ptr(),
           torch.cuda.current_stream(dev).cuda_stream)
    return syndromes_to_ints(syn.cpu().numpy())


def bch_syndrome(bits, ninner=16200):
    """Drop-in for ``m9_accel.bch_syndrome`` (one message)."""
    return bch_syndrome_batch(np.asarray(bits, np.uint8)[None], ninner)[0]
