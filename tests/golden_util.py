"""Helpers shared by the tests: the golden file and the oracle cases."""
import functools
import hashlib
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "golden.npz")


@functools.lru_cache(maxsize=1)
def golden():
    z = np.load(GOLDEN)
    arrs = {k: z[k] for k in z.files}
    meta = json.loads(str(arrs.pop("meta_json")))
    return meta, arrs


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@functools.lru_cache(maxsize=None)
def oracle_case(name):
    """Regenerate a golden case with the oracle: (meta, payload, cw, cells,
    sigma2, q, lam)."""
    import oracle
    from atsc3_b200 import codes as C
    meta, _ = golden()
    c = meta["cases"][name]
    n, mod, rate = c["n"], c["mod"], c["rate"]
    cw_out = []

    def tx(pay):
        cells, cw = oracle.transmit(pay, n, mod, rate)
        cw_out.append(cw)
        return cells

    pay, cells, s2 = oracle.synth_case(tx, c["nblk"], C.kpayload(rate, n),
                                       C.cells_per_block(n, mod), c["esn0"],
                                       c["channel"], c["seed"])
    pts = C.points_for(mod, rate)
    q = oracle.demap(cells, pts, C.MOD_BITS[mod], s2)
    lam = oracle.deinterleave(q, C.bicm_map(n, mod, rate), n)
    return c, pay, cw_out[0], cells, s2, q, lam
