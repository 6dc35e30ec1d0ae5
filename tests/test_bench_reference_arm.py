"""bench.py's two CPU decodes of the headline workload agree: the reference
receiver's own Python path (``ReferenceCpuPath``: m44_ldm._point_metric and
per-bit minima with the per-cell sigma2 divide, m44_ldm.ldpc_batch over the
compiled lab/ldpc_kernel.c, m9_accel.bch_syndrome_batch, descramble) run
from the unmodified copy in baseline/_ref, and the oracle route
(``cpu_reference_decode``) that the bench's parity check compares the GPU
with.  Skipped where baseline/_ref has not been laid out."""
import os

import numpy as np
import pytest

import bench

pytestmark = pytest.mark.skipif(
    not os.path.exists(os.path.join(bench.REF_TREE, "lab", "ldpc_kernel.so")),
    reason="baseline/_ref not laid out (python oracle/build.py --ref-tree)")


@pytest.mark.parametrize("esn0,channel", [(7.5, "rayleigh"), (6.0, "rayleigh"),
                                          (9.0, "awgn")])
def test_reference_arm_equals_oracle_route(esn0, channel):
    import oracle
    from atsc3_b200 import codes as C
    n, mod, rate = bench.N_INNER, bench.MOD, bench.RATE
    pay, cells, s2 = oracle.synth_case(
        lambda p: oracle.transmit(p, n, mod, rate)[0], 3, C.kpayload(rate, n),
        C.cells_per_block(n, mod), esn0, channel, 5)
    ref = bench.ReferenceCpuPath(threads=3).decode(cells, s2)
    want = bench.cpu_reference_decode(cells, s2, 3, full=True)
    for k in ("bits", "conv", "bad", "ok", "payload"):
        assert np.array_equal(ref[k], want[k]), k
    # converged, BCH-clean blocks carry the transmitted (descrambled) payload
    for i in np.flatnonzero(ref["ok"] & ref["conv"]):
        assert np.array_equal(np.unpackbits(ref["payload"][i])[:pay.shape[1]],
                              pay[i])
