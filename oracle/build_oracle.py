"""Build recipe for the CPU checkers (test infrastructure only).

* ``oracle/_ref/libaxref.so``: the reference's own hot-path sources
  (AsterX/src/{fluxes,source,rhs,computeBfromA,con2prim,tmunu}.cxx and the ReconX,
  Con2PrimFactory, EOSX and AsterUtils headers they include), compiled
  unmodified from where they lie in the reference checkout against the
  stand-in headers in ``oracle/refshim`` plus the harness
  ``oracle/refshim/axref_harness.cpp``.  Built only when the reference
  checkout is present; the shared object then travels with the repository.
* ``oracle/_build/libaxo.so``: the oracle restatement ``oracle/axo.cpp``.

Both use ``-ffp-contract=off`` so that every product, sum and difference is
rounded exactly as written (no fused multiply-add), which is what makes the
restatement bit-comparable with the reference code.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
# The reference checkout is named by the caller (argument or the
# AXB_REFERENCE_ROOT environment variable); there is no built-in default.
REF_ROOT = os.environ.get("AXB_REFERENCE_ROOT", "")
REF_TUS = ["fluxes", "source", "rhs", "computeBfromA", "con2prim", "tmunu"]
# -DNDEBUG: the reference's device asserts (NaN checks in fluxes.cxx:769,
# rhs.cxx:206) compile out, as in an optimised build, instead of aborting
# the test process.
CXXFLAGS = ["-std=c++17", "-O3", "-fPIC", "-fopenmp", "-ffp-contract=off",
            "-fno-fast-math", "-DNDEBUG", "-w"]


def _run(cmd):
    subprocess.run(cmd, check=True)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_ref(force=False, ref_root=None):
    """Compile the reference hot path through the shim; returns the .so path
    or None when the reference checkout is not available.  `ref_root` (or
    AXB_REFERENCE_ROOT) names the checkout."""
    out_dir = os.path.join(HERE, "_ref")
    so = os.path.join(out_dir, "libaxref.so")
    REF_ROOT = ref_root or globals()["REF_ROOT"]
    if not REF_ROOT or not os.path.isdir(os.path.join(REF_ROOT, "AsterX", "src")):
        return so if os.path.exists(so) else None
    os.makedirs(out_dir, exist_ok=True)
    shim = os.path.join(HERE, "refshim")
    inc = ["-I" + shim] + ["-I" + os.path.join(REF_ROOT, d, "src") for d in
                           ("ReconX", "EOSX", "Con2PrimFactory", "AsterUtils",
                            "AsterX")]
    srcs = [os.path.join(REF_ROOT, "AsterX", "src", t + ".cxx") for t in REF_TUS]
    harness = os.path.join(shim, "axref_harness.cpp")
    deps = srcs + [harness] + [os.path.join(shim, f) for f in os.listdir(shim)]
    deps.append(os.path.join(REPO, "include", "asterx_b200.h"))
    if not force and not _stale(so, deps):
        return so
    objs = []
    for s in srcs + [harness]:
        o = os.path.join(out_dir, os.path.splitext(os.path.basename(s))[0] + ".o")
        _run(["g++", *CXXFLAGS, *inc, "-c", s, "-o", o])
        objs.append(o)
    _run(["g++", "-shared", "-fopenmp", "-o", so, *objs])
    for o in objs:
        os.remove(o)
    return so


def build_restatement(force=False):
    out_dir = os.path.join(HERE, "_build")
    so = os.path.join(out_dir, "libaxo.so")
    src = os.path.join(HERE, "axo.cpp")
    if not os.path.exists(src):
        return None
    deps = [src, os.path.join(HERE, "axo.h"),
            os.path.join(REPO, "include", "asterx_b200.h")]
    if not force and not _stale(so, deps):
        return so
    os.makedirs(out_dir, exist_ok=True)
    _run(["g++", *CXXFLAGS, "-I" + os.path.join(REPO, "include"), "-shared",
          "-o", so, src])
    return so


def build(force=False, ref_root=None):
    return build_restatement(force), build_ref(force, ref_root)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
