"""ctypes binding of libatsc3_fec.so (the C ABI declared in include/atsc3_fec.h).

The library is built in tree by ``atsc3_b200/csrc/build.py`` into
``atsc3_b200/_lib/``.  Loading never falls back to anything: a missing or
stale library raises, and every nonzero return code of the C ABI raises
``FecError`` with the library's own message.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libatsc3_fec.so")

_LOCK = threading.Lock()
_LIB = None

c_i32, c_i64, c_f32, c_f64, c_vp = (ctypes.c_int32, ctypes.c_int64,
                                    ctypes.c_float, ctypes.c_double,
                                    ctypes.c_void_p)

# name -> (restype, argtypes); every symbol include/atsc3_fec.h declares
SIGNATURES = {
    "ldpc_kernel_abi": (c_i32, []),
    "ldpc_minsum_f32": (c_i32, [c_vp, c_i32, c_i32, c_i32, c_i32, c_vp, c_vp,
                                c_vp, c_vp, c_i32, c_f32, c_vp, c_vp, c_vp,
                                c_vp, c_vp]),
    "atsc3_last_error": (ctypes.c_char_p, []),
    "atsc3_device_info": (c_i32, [c_vp]),
    "atsc3_ldpc_plan_create": (c_i32, [c_vp, c_vp, c_vp, c_vp, c_i32, c_i32,
                                       c_i32, c_i32, c_i32, c_vp]),
    "atsc3_ldpc_plan_destroy": (None, [c_vp]),
    "atsc3_ldpc_plan_info": (c_i32, [c_vp, c_vp]),
    "atsc3_ldpc_tables_host": (c_i32, [c_vp, c_vp, c_vp, c_vp, c_i32, c_i32,
                                       c_i32, c_i32, c_vp, c_vp, c_vp, c_vp,
                                       c_vp]),
    "atsc3_ldpc_decode_flood": (c_i32, [c_vp, c_vp, c_i64, c_i32, c_i32,
                                        c_f64, c_i32, c_vp, c_i64, c_vp,
                                        c_i64, c_vp, c_vp, c_vp, c_i32,
                                        c_vp]),
    "atsc3_ldpc_flood_config": (c_i32, [c_vp, c_i32, c_i32, c_vp]),
    "atsc3_ldpc_qc_plan_create": (c_i32, [c_i32, c_i32, c_i32, c_vp, c_vp,
                                          c_i32, c_vp]),
    "atsc3_ldpc_qc_plan_destroy": (None, [c_vp]),
    "atsc3_ldpc_qc_plan_info": (c_i32, [c_vp, c_vp]),
    "atsc3_ldpc_qc_tables_host": (c_i32, [c_i32, c_i32, c_i32, c_vp, c_vp,
                                          c_i32, c_vp, c_vp, c_vp, c_vp,
                                          c_vp, c_vp]),
    "atsc3_ldpc_qc_config": (c_i32, [c_vp, c_i32, c_i32, c_vp]),
    "atsc3_ldpc_qc_decode": (c_i32, [c_vp, c_vp, c_i64, c_i32, c_i32, c_f32,
                                     c_i32, c_vp, c_i64, c_vp, c_i64, c_vp,
                                     c_vp, c_vp, c_i32, c_vp]),
    "atsc3_ldpc_qce_plan_create": (c_i32, [c_i32, c_i32, c_i32, c_vp, c_vp,
                                           c_i32, c_vp]),
    "atsc3_ldpc_qce_plan_destroy": (None, [c_vp]),
    "atsc3_ldpc_qce_plan_create2": (c_i32, [c_i32, c_i32, c_i32, c_i32, c_vp,
                                            c_vp, c_i32, c_vp]),
    "atsc3_ldpc_qce_plan_create_f64": (c_i32, [c_i32, c_i32, c_i32, c_i32, c_vp,
                                               c_vp, c_i32, c_vp]),
    "atsc3_ldpc_qce_decode_f64": (c_i32, [c_vp, c_vp, c_i64, c_i32, c_i32, c_f64,
                                          c_i32, c_vp, c_i64, c_vp, c_i64, c_vp,
                                          c_vp, c_vp, c_i32, c_vp]),
    "atsc3_ldpc_qce_bins_host": (c_i32, [c_i32, c_i32, c_i32, c_i32, c_vp, c_vp, c_i32,
                                         c_vp]),
    "atsc3_ldpc_qce_tables_host2": (c_i32, [c_i32, c_i32, c_i32, c_i32, c_vp,
                                            c_vp, c_i32, c_vp, c_vp, c_vp,
                                            c_vp, c_vp, c_vp, c_vp, c_vp,
                                            c_vp]),
    "atsc3_ldpc_qce_plan_info": (c_i32, [c_vp, c_vp]),
    "atsc3_ldpc_qce_tables_host": (c_i32, [c_i32, c_i32, c_i32, c_vp, c_vp,
                                           c_i32, c_vp, c_vp, c_vp, c_vp,
                                           c_vp, c_vp]),
    "atsc3_ldpc_qc_detect": (c_i32, [c_vp, c_vp, c_vp, c_vp, c_i32, c_i32,
                                     c_i32, c_vp, c_vp, c_vp]),
    "atsc3_ldpc_qc_detect2": (c_i32, [c_vp, c_vp, c_vp, c_vp, c_i32, c_i32,
                                      c_i32, c_vp, c_vp, c_vp]),
    "atsc3_ldpc_qce_config": (c_i32, [c_vp, c_i32, c_i32, c_vp]),
    "atsc3_ldpc_qce_decode": (c_i32, [c_vp, c_vp, c_i64, c_i32, c_i32, c_f32,
                                      c_i32, c_vp, c_i64, c_vp, c_i64, c_vp,
                                      c_vp, c_vp, c_i32, c_vp]),
    "atsc3_ldpc_qce_decode_weighted": (c_i32, [c_vp, c_vp, c_i64, c_i32,
                                               c_i32, c_f32, c_i32, c_vp,
                                               c_vp, c_i32, c_i32, c_vp, c_vp,
                                               c_i64, c_vp, c_i64, c_vp, c_vp,
                                               c_vp, c_i32, c_vp]),
    "atsc3_ldpc_qce_decode_weighted_rows": (c_i32, [c_vp, c_vp, c_i64, c_i32,
                                               c_i32, c_f32, c_i32, c_vp,
                                               c_vp, c_i32, c_i32, c_vp, c_vp,
                                               c_i64, c_vp, c_i64, c_vp, c_vp,
                                               c_vp, c_i32, c_vp]),
    "atsc3_ldpc_sp_workspace": (c_i32, [c_i32, c_i32, c_i32, c_vp]),
    "atsc3_ldpc_sp_decode": (c_i32, [c_vp, c_vp, c_vp, c_vp, c_i32, c_i32,
                                     c_i32, c_vp, c_i64, c_i32, c_i32, c_vp,
                                     c_i64, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "atsc3_ldpc_sp_step": (c_i32, [c_vp, c_vp, c_vp, c_vp, c_i32, c_i32, c_i32,
                                   c_vp, c_i64, c_i32, c_i32, c_i32, c_vp,
                                   c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "atsc3_cpe_workspace": (c_i32, [c_vp]),
    "atsc3_cpe_correct": (c_i32, [c_vp, c_i64, c_vp, c_i32, c_vp, c_vp, c_i32,
                                  c_vp, c_i32, c_vp, c_i32, c_vp, c_vp, c_vp,
                                  c_vp]),
    "atsc3_ldpc_layered_plan_create": (c_i32, [c_i32, c_i32, c_i32, c_vp,
                                               c_vp, c_vp]),
    "atsc3_ldpc_layered_plan_destroy": (None, [c_vp]),
    "atsc3_ldpc_layered_workspace": (c_i32, [c_vp, c_i32, c_vp]),
    "atsc3_ldpc_layered_decode": (c_i32, [c_vp, c_vp, c_i64, c_i32, c_i32,
                                          c_f32, c_vp, c_i64, c_vp, c_i64,
                                          c_vp, c_vp, c_vp, c_vp, c_i32, c_vp,
                                          c_vp]),
    "atsc3_ldpc_layered_inject_timeout": (c_i32, [c_i32]),
    "atsc3_wms_forward": (c_i32, [c_vp] * 7 + [c_i32] * 6 + [c_vp, c_vp, c_vp,
                                                             c_i32, c_vp, c_vp,
                                                             c_vp]),
    "atsc3_wms_backward": (c_i32, [c_vp] * 7 + [c_i32] * 6 + [c_vp] * 9),
    "atsc3_ldpc_qc_decode_weighted": (c_i32, [c_vp, c_vp, c_i64, c_i32, c_i32,
                                              c_f32, c_i32, c_vp, c_vp, c_i32,
                                              c_i32, c_vp, c_vp, c_i64, c_vp,
                                              c_i64, c_vp, c_vp, c_vp, c_i32,
                                              c_vp]),
    "atsc3_demap_batch": (c_i32, [c_vp] * 13 + [c_i32, c_i32, c_vp]),
    "atsc3_ldpc_batch_desc_bytes": (c_i32, [c_i32, c_vp]),
    "atsc3_ldpc_batch_prepare": (c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp]),
    "atsc3_ldpc_batch_decode": (c_i32, [c_vp, c_i32, c_i32, c_vp, c_vp, c_i32,
                                        c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                        c_vp, c_i32, c_f32, c_vp, c_i32,
                                        c_i32, c_vp]),
    "atsc3_bch_batch": (c_i32, [c_vp] * 11 + [c_i32, c_vp]),
    "atsc3_demap": (c_i32, [c_vp, c_i64, c_i32, c_i32, c_vp, c_i32, c_i32,
                            c_vp, c_i64, c_f32, c_vp, c_vp, c_i64, c_vp]),
    "atsc3_demap_gather": (c_i32, [c_vp, c_i64, c_i32, c_i32, c_vp, c_i32,
                                   c_i32, c_vp, c_i64, c_i64, c_i64, c_i32,
                                   c_vp, c_f32, c_vp, c_vp, c_i64, c_vp]),
    "atsc3_demap_row_sigma2": (c_i32, [c_vp, c_i64, c_i32, c_i32, c_vp,
                                       c_i32, c_vp, c_vp]),
    "atsc3_demap_f64": (c_i32, [c_vp, c_i64, c_i32, c_i32, c_vp, c_i32, c_i32,
                                c_vp, c_i64, c_f64, c_vp, c_vp, c_i64, c_vp]),
    "atsc3_demap_row_sigma2_f64": (c_i32, [c_vp, c_i64, c_i32, c_i32, c_vp,
                                           c_i32, c_vp, c_vp]),
    "atsc3_bch_check": (c_i32, [c_vp, c_i64, c_i32, c_i32, c_vp, c_vp, c_vp,
                                c_vp, c_i32, c_vp, c_i64, c_vp]),
    "atsc3_bch_syndrome_bits": (c_i32, [c_vp, c_i64, c_i32, c_i32, c_vp,
                                        c_vp, c_vp]),
    "atsc3_fec_decode_noalloc": (c_i32, [c_vp, c_i32, c_vp, c_i64, c_i32,
                                         c_i32, c_vp, c_i32, c_i32, c_vp,
                                         c_i64, c_f32, c_vp, c_i32, c_f32,
                                         c_vp, c_i32, c_vp, c_i32, c_vp,
                                         c_i64, c_vp, c_vp, c_vp, c_vp, c_vp,
                                         c_vp]),
}


class FecError(RuntimeError):
    """A nonzero return code of the C ABI."""

    def __init__(self, fn, rc, msg):
        super().__init__(f"{fn} returned {rc}: {msg}")
        self.rc = rc


def lib():
    """The loaded library (raises if it was never built)."""
    global _LIB
    with _LOCK:
        if _LIB is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with "
                    "python atsc3_b200/csrc/build.py (no CPU fallback exists)")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            if int(L.ldpc_kernel_abi()) != 1:
                raise ImportError("libatsc3_fec ABI mismatch")
            _LIB = L
        return _LIB


def check(name, rc):
    if rc != 0:
        msg = lib().atsc3_last_error()
        raise FecError(name, rc, msg.decode() if msg else "")
    return rc


def call(name, *args):
    return check(name, getattr(lib(), name)(*args))


def ptr(t):
    """Device/host address of a torch tensor or numpy array (None -> NULL)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


def stream_of(torch_mod, device=None):
    return torch_mod.cuda.current_stream(device).cuda_stream
