#!/usr/bin/env python3
"""Build the oracle's native parts.  TEST INFRASTRUCTURE ONLY.

* ``oracle/liboracle.so`` -- our C restatement (``ldpc_oracle.c``).
* ``oracle/_ref/ldpc_kernel.so`` -- the Felbs/atsc3 reference kernel compiled
  from its own source, ``lab/ldpc_kernel.c`` of a reference checkout, with
  the reference's flags (``-O3 -ffp-contract=off -shared -fPIC``,
  lab/build_ldpc_kernel.py:36,93).  Built only where the checkout exists
  (``ATSC3_REFERENCE`` or /root/reference); the product never loads it.
* ``baseline/_ref/`` (``--ref-tree``) -- a runnable, unmodified copy of the
  reference receiver's Python (``lab/*.py``, ``lab/spec_bank/``, the
  ``atsc3`` package) with ``lab/ldpc_kernel.so`` compiled there from the
  checkout's own ``lab/ldpc_kernel.c`` as above: the reference's own CPU
  path for ``bench.py --impl reference`` and the drop-in gate test
  (``tests/test_gpu_ref_gates.py``), which run where no checkout exists.
  The folder is git-ignored (reference code is never committed here).

    python oracle/build.py [--ref-tree]
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


REPO = os.path.dirname(HERE)
REF_TREE = os.path.join(REPO, "baseline", "_ref")


def build_ref_tree(verbose=False):
    """Lay out baseline/_ref/ from the reference checkout (see the module
    docstring).  Returns the tree's path, or None without a checkout."""
    lab = os.path.join(REF_ROOT, "lab")
    if not os.path.exists(os.path.join(lab, "m44_ldm.py")):
        return None
    dst_lab = os.path.join(REF_TREE, "lab")
    os.makedirs(dst_lab, exist_ok=True)
    for name in sorted(os.listdir(lab)):
        src = os.path.join(lab, name)
        if name.endswith(".py") and _stale(os.path.join(dst_lab, name), src):
            shutil.copyfile(src, os.path.join(dst_lab, name))
    for sub in ("spec_bank",):
        src = os.path.join(lab, sub)
        if os.path.isdir(src):
            shutil.copytree(src, os.path.join(dst_lab, sub), dirs_exist_ok=True)
    pkg = os.path.join(REF_ROOT, "atsc3")
    if os.path.isdir(pkg):
        shutil.copytree(pkg, os.path.join(REF_TREE, "atsc3"),
                        dirs_exist_ok=True)
    so = os.path.join(dst_lab, "ldpc_kernel.so")
    if _stale(so, REF_SRC):
        cmd = [_cc(), "-O3", "-ffp-contract=off", "-shared", "-fPIC", "-o",
               so, REF_SRC]
        subprocess.run(cmd, check=True)
    # the copies keep the checkout's read-only mode bits; make them
    # replaceable by the next run of this recipe
    for root, _dirs, files in os.walk(REF_TREE):
        for f in files:
            os.chmod(os.path.join(root, f), 0o644)
        os.chmod(root, 0o755)
    if verbose:
        print(REF_TREE, len(os.listdir(dst_lab)), "files in lab/")
    return REF_TREE


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
    if "--ref-tree" in sys.argv:
        build_ref_tree(verbose=True)
    sys.exit(0)
