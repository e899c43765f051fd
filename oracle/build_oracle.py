"""Build recipe for the oracle libraries (test infrastructure only).

* ``oracle/libndloracle.so``  -- the plain-C FP64 restatement (ndl_oracle.c).
* ``oracle/_ref/libndlref.so`` -- ref_shim.cpp compiled against the UNMODIFIED
  ndl reference headers, with the reference's own default Release flags
  (``-O3 -DNDEBUG``, no ``-march``; CMakeLists.txt:8-11 picks Release, and
  NDL_NATIVE_ARCH defaults to OFF at CMakeLists.txt:86).  Built only where the
  reference source tree exists; elsewhere the prebuilt file is used as is.

Nothing from the reference is copied: the headers are reached through an
include directory, created in a temporary folder, holding one symlink
``ndl -> <reference root>`` so that ``#include <ndl/...>`` resolves.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("NDL_REFERENCE_ROOT", "/root/reference")
ORACLE_SO = os.path.join(HERE, "libndloracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "libndlref.so")


def _run(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("command failed: %s\n%s\n%s" % (" ".join(cmd), res.stdout, res.stderr))


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_restatement(force=False):
    src = os.path.join(HERE, "ndl_oracle.c")
    if force or _stale(ORACLE_SO, [src]):
        _run(["gcc", "-std=gnu11", "-O2", "-fPIC", "-shared", "-o", ORACLE_SO, src, "-lm"])
    return ORACLE_SO


def build_reference(force=False):
    """Compile the reference shim; returns the .so path or None if the
    reference tree is absent and no prebuilt library exists."""
    src = os.path.join(HERE, "ref_shim.cpp")
    if not os.path.isdir(REF_ROOT) or not os.path.exists(os.path.join(REF_ROOT, "processing", "convolution.h")):
        return REF_SO if os.path.exists(REF_SO) else None
    if not (force or _stale(REF_SO, [src])):
        return REF_SO
    os.makedirs(REF_DIR, exist_ok=True)
    inc = tempfile.mkdtemp(prefix="ndlref_inc_")
    try:
        os.symlink(REF_ROOT, os.path.join(inc, "ndl"))
        _run(["g++", "-std=c++17", "-O3", "-DNDEBUG", "-fPIC", "-shared", "-I", inc,
              "-o", REF_SO, src])
    finally:
        shutil.rmtree(inc, ignore_errors=True)
    return REF_SO


DROPIN_BIN = os.path.join(REF_DIR, "dropin_check")


def build_dropin_check(force=False):
    """tests/cpp/dropin_check.cpp (the C++ drop-in header checked against the
    reference's own calls) -> oracle/_ref/dropin_check, linked with
    libndlgpu.so.  Needs the reference tree and a built libndlgpu.so."""
    repo = os.path.dirname(HERE)
    src = os.path.join(repo, "tests", "cpp", "dropin_check.cpp")
    lib_dir = os.path.join(repo, "ndl_b200", "lib")
    hdrs = [os.path.join(repo, "include", "ndlgpu_dropin.h"), os.path.join(repo, "include", "ndlgpu.h")]
    if not os.path.isdir(REF_ROOT) or not os.path.exists(os.path.join(lib_dir, "libndlgpu.so")):
        return DROPIN_BIN if os.path.exists(DROPIN_BIN) else None
    if not (force or _stale(DROPIN_BIN, [src] + hdrs)):
        return DROPIN_BIN
    os.makedirs(REF_DIR, exist_ok=True)
    inc = tempfile.mkdtemp(prefix="ndlref_inc_")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    try:
        os.symlink(REF_ROOT, os.path.join(inc, "ndl"))
        _run(["g++", "-std=c++17", "-O2", "-I", inc, "-I", os.path.join(repo, "include"),
              "-I", os.path.join(cuda, "include"), "-o", DROPIN_BIN, src,
              "-L", lib_dir, "-lndlgpu", "-Wl,-rpath,$ORIGIN/../../ndl_b200/lib",
              "-L", os.path.join(cuda, "lib64"), "-lcudart_static", "-ldl", "-lrt", "-lpthread"])
    finally:
        shutil.rmtree(inc, ignore_errors=True)
    return DROPIN_BIN


def build(force=False):
    build_restatement(force)
    ref = build_reference(force)
    build_dropin_check(force)
    return ref


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
