"""Build libsphb.so (the sm_100a engine behind include/sphb.h) in-tree.

    python -m pysph_b200.build [--force]

Every .cu under csrc/ is compiled by nvcc for sm_100a only, in parallel, and
linked into pysph_b200/_lib/libsphb.so with the CUDA runtime linked
statically, so the library carries no dependency beyond the driver.  The
benchmark's FMA-rate probe (probe/) is built into its own
_lib/libsphb_probe.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libsphb.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-fvisibility=hidden",
                     "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers():
    return (sorted(glob.glob(os.path.join(CSRC, "*.cuh")))
            + [os.path.join(INCLUDE, "sphb.h")])


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, extra):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if _stale(obj, [src] + _headers() + [__file__]):
        cmd = [nvcc(), "-c", src, "-o", obj + ".tmp"] + NVCC_FLAGS + list(extra)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        os.replace(obj + ".tmp", obj)
        return obj, r.stderr
    return obj, ""


PROBE_SRC = os.path.join(HERE, "probe", "sphb_fma_probe.cu")
PROBE_LIB = os.path.join(LIBDIR, "libsphb_probe.so")


def build_probe(force: bool = False) -> str:
    """The benchmark's FMA-rate probe, a library of its own (not part of
    libsphb.so)."""
    os.makedirs(LIBDIR, exist_ok=True)
    if force or _stale(PROBE_LIB, [PROBE_SRC, __file__]):
        cmd = [nvcc(), "-shared", PROBE_SRC, "-o", PROBE_LIB + ".tmp"] + ARCH + [
            "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
            "-cudart", "static"]
        subprocess.check_call(cmd)
        os.replace(PROBE_LIB + ".tmp", PROBE_LIB)
    return PROBE_LIB


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = _sources()
    if force:
        for o in glob.glob(os.path.join(OBJ, "*.o")):
            os.remove(o)
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, extra), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log, file=sys.stderr)
    if _stale(LIB, objs):
        cmd = [nvcc(), "-shared", "-o", LIB + ".tmp"] + ARCH + objs + [
            "-cudart", "static", "-Xcompiler", "-fPIC"]
        subprocess.check_call(cmd)
        os.replace(LIB + ".tmp", LIB)
    build_probe(force)
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    verbose = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force=force, verbose=verbose or bool(extra), extra=extra))
