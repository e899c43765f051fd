"""Build recipe for libndlgpu.so (sm_100a), in-tree.

nvcc compiles every ``csrc/*.cu`` and ``csrc/*.cpp`` for
``-gencode arch=compute_100a,code=sm_100a`` with ``-lineinfo``; the objects
are linked into ``ndl_b200/lib/libndlgpu.so`` with the CUDA runtime linked
statically, so the library loads on a machine without a GPU (the CPU tests
check its exported symbols) and carries no dependency on a particular
libcudart.  Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(HERE, "lib", "libndlgpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
          "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]


def _headers():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hs += glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    return hs


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def _compile(src, extra):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    hdr_t = _newest(_headers())
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_t):
        return obj, None
    cmd = [NVCC] + ARCH + COMMON + extra + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + COMMON + extra + ["-x", "cu", "-c", src, "-o", obj] + ARCH
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        return obj, "%s\n%s\n%s" % (" ".join(cmd), res.stdout, res.stderr)
    return obj, None


def build(verbose=False, ptxas_info=False):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    objs = []
    errors = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        futs = {ex.submit(_compile, s, extra): s for s in srcs}
        for f in cf.as_completed(futs):
            obj, err = f.result()
            objs.append(obj)
            if err:
                errors.append(err)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n\n".join(errors))
    objs.sort()
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (res.stdout, res.stderr))
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas-info" in sys.argv)
