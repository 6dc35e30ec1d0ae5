#!/usr/bin/env python3
"""Build the oracle's native parts.  TEST INFRASTRUCTURE ONLY.

* ``oracle/liboracle.so`` -- our C restatement (``ldpc_oracle.c``).
* ``oracle/_ref/ldpc_kernel.so`` -- the Felbs/atsc3 reference kernel compiled
  from its own source, ``lab/ldpc_kernel.c`` of a reference checkout, with
  the reference's flags (``-O3 -ffp-contract=off -shared -fPIC``,
  lab/build_ldpc_kernel.py:36,93).  Built only where the checkout exists
  (``ATSC3_REFERENCE`` or /root/reference); the product never loads it.

    python oracle/build.py
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "ldpc_kernel.so")
REF_ROOT = os.environ.get("ATSC3_REFERENCE", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "lab", "ldpc_kernel.c")


def _cc():
    for c in ("gcc", "cc"):
        if shutil.which(c):
            return c
    raise RuntimeError("no C compiler")


def _stale(out, src):
    return not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src)


def build(verbose=False):
    src = os.path.join(HERE, "ldpc_oracle.c")
    if _stale(ORACLE_SO, src):
        cmd = [_cc(), "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-o",
               ORACLE_SO, src, "-lm"]
        subprocess.run(cmd, check=True)
    if os.path.exists(REF_SRC) and _stale(REF_SO, REF_SRC):
        os.makedirs(REF_DIR, exist_ok=True)
        cmd = [_cc(), "-O3", "-ffp-contract=off", "-shared", "-fPIC", "-o",
               REF_SO, REF_SRC]
        subprocess.run(cmd, check=True)
    if verbose:
        print(ORACLE_SO, os.path.exists(ORACLE_SO))
        print(REF_SO, os.path.exists(REF_SO))
    return ORACLE_SO


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
