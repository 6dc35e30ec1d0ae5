#!/usr/bin/env python3
"""Write ``a322_tables.npz``: the ATSC A/322 numeric tables the FEC back end needs.

The numbers are facts of the standard (Annex A LDPC address tables, Section 6
parameters, Tables 6.8-6.14 and Annex B bit-interleaver tables, Annex C NUC
position vectors, the BCH generator factors and the Baseband Packet scrambling
sequence).  The Felbs/atsc3 receiver ships them as Python modules extracted
from the standard's text (``lab/spec_ldpc.py``, ``lab/spec_ldpc64k.py``,
``lab/spec_bitint.py``, ``lab/spec_nuc.py`` + ``lab/spec_bank/nuc_a322.npz``,
``lab/spec_bicm.py``, ``lab/m4_scrambler.py``).  This script reads those
modules once, on a machine that has the receiver checked out, and stores the
numbers in a compact archive so the package needs no receiver source at run
time.  No code is taken from them: only the tables.

Usage:  python tests/golden/extract_a322.py /path/to/atsc3/checkout
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(os.path.dirname(os.path.dirname(HERE)), "atsc3_b200", "data",
                   "a322_tables.npz")


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    root = argv[0] if argv else os.environ.get("ATSC3_REFERENCE", "")
    lab = os.path.join(root, "lab")
    if not os.path.isdir(lab):
        raise SystemExit(f"no receiver checkout at {root!r}")
    os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
    sys.dont_write_bytecode = True
    sys.path.insert(0, root)
    sys.path.insert(0, lab)
    import spec_ldpc as SL            # noqa: E402
    import spec_ldpc64k as SL64       # noqa: E402
    import spec_bitint as BI          # noqa: E402
    import spec_nuc as NU             # noqa: E402
    import spec_bicm as BC            # noqa: E402
    import m4_scrambler as SC         # noqa: E402

    arrs = {}
    meta = {"rates": list(BI.RATES), "mod_bits": dict(BI.MOD_BITS),
            "ldpc": {}, "type_a": {}, "type_b": {}, "demux": {},
            "bi_type": {}, "groupwise": []}
    for n in (16200, 64800):
        for r in BI.RATES:
            if n == 16200:
                P = dict(SL.LDPC_PARAMS[r])
                rows = SL.LDPC_16200[r]["rows"]
            else:
                P = dict(SL64.LDPC_64800[r])
                rows = P.pop("rows")
            key = f"{n}:{r}"
            meta["ldpc"][key] = {k: P[k] for k in
                                 ("Kldpc", "type", "M1", "M2", "Q1", "Q2",
                                  "Qldpc")}
            lens = np.array([len(x) for x in rows], np.int32)
            arrs[f"ldpc_rowptr/{key}"] = np.concatenate(
                [[0], np.cumsum(lens)]).astype(np.int32)
            arrs[f"ldpc_addr/{key}"] = np.array(
                [a for x in rows for a in x], np.int32)
    for (n, mod), v in BI.TYPE_A.items():
        meta["type_a"][f"{n}:{mod}"] = list(v)
    for (n, mod), v in BI.TYPE_B.items():
        meta["type_b"][f"{n}:{mod}"] = list(v)
    for (n, mod), v in BI.DEMUX.items():
        meta["demux"][f"{n}:{mod}"] = list(v)
    for (n, nc, r), v in BI.BI_TYPE.items():
        meta["bi_type"][f"{n}:{nc}:{r}"] = v
    for (n, mod, r), perm in BI.GROUPWISE.items():
        key = f"{n}:{mod}:{r}"
        meta["groupwise"].append(key)
        arrs[f"groupwise/{key}"] = np.asarray(perm, np.int32)
    for m in (16, 64, 256):
        for r in BI.RATES:
            arrs[f"nuc/{m}:{r}"] = np.asarray(NU.get(m, r), np.complex128)
    meta["bch_polys"] = {"16200": [list(p) for p in BC.BCH_16200_GEN_POLYS],
                         "64800": [list(p) for p in BC.BCH_64800_GEN_POLYS]}
    nseq = 64800 - 192        # longer than any K_payload
    arrs["scrambler_bits"] = np.packbits(SC.sequence(nseq))
    meta["scrambler_nbits"] = nseq
    arrs["meta_json"] = np.array(json.dumps(meta, sort_keys=True))
    np.savez_compressed(OUT, **arrs)
    print(f"wrote {OUT}: {len(arrs)} arrays, "
          f"{os.path.getsize(OUT) / 1024:.1f} KiB")


if __name__ == "__main__":
    main()
