"""Build ``libsinvb.so`` in-tree with nvcc for sm_100a (B200).

    python -m sinv_b200.build            # incremental (rebuilds when a source is newer)
    python -m sinv_b200.build --force    # full rebuild
    python -m sinv_b200.build --verbose  # also print ptxas register / spill report

Each ``csrc/*.cu`` compiles to an object under ``_build/``; the objects link
into ``sinv_b200/libsinvb.so`` with the CUDA runtime linked statically, so
the library needs only the driver at run time.
"""

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libsinvb.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", os.path.join(ROOT, "include")]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return _sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) \
        + glob.glob(os.path.join(ROOT, "include", "*.h"))


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


MAX_STACK_FRAME = 16384  # bytes per thread; the persistent kernels use 2-8 KB


def stack_check(src, ptxas_log):
    """Fails the build on a kernel whose stack size ptxas cannot determine
    statically, or whose frame exceeds MAX_STACK_FRAME."""
    import re
    if "cannot be statically determined" in ptxas_log:
        raise RuntimeError("%s: a kernel needs a dynamic stack (recursion):\n%s" % (src, ptxas_log))
    frames = [int(x) for x in re.findall(r"(\d+) bytes stack frame", ptxas_log)]
    if frames and max(frames) > MAX_STACK_FRAME:
        raise RuntimeError("%s: stack frame of %d bytes exceeds %d" % (src, max(frames), MAX_STACK_FRAME))


def build(force=False, verbose=False):
    """Compile every CUDA source and link the shared library.  Returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    dep_time = _newest(_deps())
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= dep_time:
        return LIB
    # ptxas reports every kernel's stack frame; stack_check refuses a kernel
    # whose stack size it cannot determine statically (recursion), which would
    # run with the per-thread stack limit instead of a frame sized at launch
    extra = ["-Xptxas", "-v"]

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= dep_time:
            return obj, ""
        cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
        stack_check(src, r.stderr)
        return obj, r.stderr

    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(compile_one, srcs))
    if verbose:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
