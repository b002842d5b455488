"""Build the engine's shared library for sm_100a (nvcc, in-tree).

Every ``asterx_b200/csrc/*.cu`` file is compiled in parallel with
``-gencode arch=compute_100a,code=sm_100a`` and linked into
``asterx_b200/_lib/libasterx_b200.so``, which the tests, ``bench.py`` and
``__graft_entry__`` load.  nvcc cross-compiles, so this runs without a GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
SO = os.path.join(LIBDIR, "libasterx_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I" + os.path.join(REPO, "include")]
# Per-file flags.  The recovery is compiled without multiply-add contraction:
# every FP64 operation is rounded on its own, as written, so the same cell
# gives the same bits whichever kernel (single box, fast pass, deferred
# pass, batched level) inlines the recovery -- contraction choices depend on
# the surrounding code, and the Brent bracket amplifies a last-bit
# difference to the root-finder tolerance.  It also follows the per-operation
# rounding of the reference's CPU build.
# The recovery is split over three translation units (single box, batched,
# independent cells) that share axb_c2p_box.cuh, so they compile in parallel.
# The stress-energy tensor and the regrid error follow the reference's
# operation order without contraction as well, which makes them bit-equal to
# the reference's CPU build.
FILE_FLAGS = {"axb_poststep.cu": ["-fmad=false"], "axb_c2p_batch.cu": ["-fmad=false"],
              "axb_c2p_cells.cu": ["-fmad=false"], "axb_tmunu.cu": ["-fmad=false"]}


def _includes(path, seen=None):
    """The quoted #include files a source reaches, transitively."""
    import re
    seen = set() if seen is None else seen
    with open(path) as fh:
        for m in re.finditer(r'^\s*#\s*include\s+"([^"]+)"', fh.read(), re.M):
            dep = os.path.normpath(os.path.join(os.path.dirname(path), m.group(1)))
            if os.path.exists(dep) and dep not in seen:
                seen.add(dep)
                _includes(dep, seen)
    return seen


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, obj, extra):
    cmd = [NVCC, *ARCH, *FLAGS, *FILE_FLAGS.get(os.path.basename(src), []), *extra, "-c",
           src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    return r.stderr


def build(force=False, verbose=False, extra=()):
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s, *_includes(s), os.path.abspath(__file__)]):
            jobs.append((s, o))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            futs = {ex.submit(_compile, s, o, list(extra)): s for s, o in jobs}
            for fu in cf.as_completed(futs):
                log = fu.result()
                if verbose and log:
                    print(f"== {os.path.basename(futs[fu])}\n{log}")
    if force or jobs or _stale(SO, objs):
        # (NCCL, for the halo exchange of axb_halo.cu, is looked up at run
        # time: whichever libnccl the process has loaded, else libnccl.so.2)
        cmd = [NVCC, *ARCH, "-shared", "-o", SO, *objs, "-lcudart", "-ldl"]
        subprocess.run(cmd, check=True)
    return SO


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if v else []
    print(build(force="--force" in sys.argv, verbose=v, extra=extra))
