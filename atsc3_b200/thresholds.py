"""Per-MODCOD Es/N0 thresholds measured with this decoder (AWGN).

The reference has no threshold table; it has a procedure (bisection on the
decoded outcome, ``lab/m15_ldm_llr.py:682-697``).  ``measure`` runs that
procedure for every (Ninner, constellation, rate) the A/322 tables pair:
the lowest Es/N0 on a 0.25 dB grid at which the plain normalised min-sum
(alpha 0.75, at most 50 iterations, BCH arbiter) loses at most 10% of 256
seeded blocks.  Results are written to ``data/thresholds.json`` and read by
the uneven-batch workload (Es/N0 = threshold + 1 dB).  The 1024/4096 points
use the uniform-QAM stand-in alphabets.

    python -m atsc3_b200.thresholds
"""
from __future__ import annotations

import json
import os

from . import codes as C

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "data", "thresholds.json")


def modcods():
    out = []
    for n in (16200, 64800):
        for mod in C.MOD_BITS:
            try:
                C.cells_per_block(n, mod)
            except ValueError:
                continue
            for r in C.RATES:
                out.append((n, mod, r))
    return out


def key(n, mod, rate):
    return f"{n}|{mod}|{rate}"


def lookup(n, mod, rate):
    with open(PATH) as f:
        return json.load(f)[key(n, mod, rate)]


def measure(nblk=256, target=0.1, step=0.25, seed=7):
    from . import evaluate as EV
    out = {}
    for n, mod, r in modcods():
        out[key(n, mod, r)] = EV.threshold(r, mod, n=n, target=target,
                                           nblk=nblk, seed=seed, step=step,
                                           lo=-4.0, hi=40.0)
    return out


if __name__ == "__main__":
    res = measure()
    os.makedirs(os.path.dirname(PATH), exist_ok=True)
    with open(PATH, "w") as f:
        json.dump(res, f, indent=0, sort_keys=True)
    print(len(res), "thresholds ->", PATH)
