"""atsc3_b200 -- a B200 (sm_100a) FEC back end for ATSC 3.0 receivers.

Drop-in replacements for the Felbs/atsc3 decode entry points:

* ``ldpc.GpuMinSum``             <- lab/m9_gpu.py GpuMinSum
* ``demap.demap_llr_fast``       <- lab/m16_demap_fast.py demap_llr_fast
* ``bch.bch_syndrome_batch``     <- lab/m9_accel.py bch_syndrome_batch
* ``libatsc3_fec.so`` C ABI      <- lab/ldpc_kernel.c (ldpc_minsum_f32)

plus the fused pipeline (``pipeline.FecPipeline``).  All compute runs in
hand-written CUDA kernels in ``csrc/``; there is no CPU fallback.
"""
from . import codes  # noqa: F401

__all__ = ["codes"]
__version__ = "0.1.0"
