"""Rebind the Felbs/atsc3 receiver's decode entry points to this back end.

The reference swaps module attributes in place and restores them
(``lab/m9_accel.py:392-433``, ``install`` / ``uninstall``); this does the same
for the four entry points the FEC back end replaces, so the receiver's own
callers and gates run on the GPU unchanged:

* ``m9_gpu.GpuMinSum``              -> ``atsc3_b200.ldpc.GpuMinSum``
* ``m16_demap_fast.demap_llr_fast`` -> ``atsc3_b200.demap.demap_llr_fast``
* ``m9_accel.bch_syndrome_batch`` / ``bch_syndrome``
                                    -> ``atsc3_b200.bch`` drop-ins
* ``m3_ldpc._kernel_lib``           -> ``libatsc3_fec.so`` (same C ABI as
  ``lab/ldpc_kernel.c``, bound with the reference's own argtypes,
  ``lab/m3_ldpc.py:439-446``)
* ``m16_margin.sum_product_decode_batch``
                                    -> ``atsc3_b200.ldpc`` (float64 on the GPU)
* ``m6_cells.cpe_correct``          -> ``atsc3_b200.cpe.cpe_correct``

Pass the already-imported reference modules (any subset); nothing here
imports the receiver.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import native as N

_SAVED = []


def _kernel_lib_factory():
    lib = ctypes.CDLL(N.LIB_PATH)
    lib.ldpc_kernel_abi.restype = ctypes.c_int32
    i32 = np.ctypeslib.ndpointer(np.int32, flags="C")
    f32 = np.ctypeslib.ndpointer(np.float32, flags="C")
    u8 = np.ctypeslib.ndpointer(np.uint8, flags="C")
    lib.ldpc_minsum_f32.restype = ctypes.c_int32
    lib.ldpc_minsum_f32.argtypes = [
        f32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
        i32, i32, i32, i32, ctypes.c_int32, ctypes.c_float, u8, u8, i32, i32,
        f32]
    return lib


def install(m9_gpu=None, m16_demap_fast=None, m9_accel=None, m3_ldpc=None,
            m16_margin=None, m6_cells=None):
    """Patch the given reference modules; returns the number of bindings."""
    from . import bch, cpe, demap, ldpc

    def patch(mod, name, value):
        _SAVED.append((mod, name, getattr(mod, name)))
        setattr(mod, name, value)

    if m9_gpu is not None:
        patch(m9_gpu, "GpuMinSum", ldpc.GpuMinSum)
    if m16_demap_fast is not None:
        patch(m16_demap_fast, "demap_llr_fast", demap.demap_llr_fast)
    if m9_accel is not None:
        patch(m9_accel, "bch_syndrome_batch", bch.bch_syndrome_batch)
        patch(m9_accel, "bch_syndrome", bch.bch_syndrome)
    if m3_ldpc is not None:
        lib = _kernel_lib_factory()
        patch(m3_ldpc, "_kernel_lib", lambda: lib)
    if m16_margin is not None:
        patch(m16_margin, "sum_product_decode_batch", ldpc.sum_product_decode_batch)
    if m6_cells is not None:
        patch(m6_cells, "cpe_correct", cpe.cpe_correct)
    return len(_SAVED)


def uninstall():
    """Restore every attribute install() replaced, newest first."""
    while _SAVED:
        mod, name, old = _SAVED.pop()
        setattr(mod, name, old)
