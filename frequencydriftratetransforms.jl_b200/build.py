"""Build libfdrb200.so in-tree with nvcc for sm_100a.

Usage: python build.py [--force]
The shared library is written next to this file (frequencydriftratetransforms.jl_b200/).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import hashlib

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.normpath(os.path.join(HERE, "..", "include"))
LIB = os.path.join(HERE, "libfdrb200.so")
LIB_DEBUG = os.path.join(HERE, "libfdrb200_debug.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _digest(extra=()):
    h = hashlib.sha256()
    files = sources() + sorted(
        os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h")))
    files.append(os.path.join(INCLUDE, "fdr_b200.h"))
    for f in files:
        h.update(f.encode())
        with open(f, "rb") as fh:
            h.update(fh.read())
    h.update(" ".join(NVCC_FLAGS + list(extra)).encode())
    return h.hexdigest()


def nvcc_path():
    p = shutil.which("nvcc")
    if p:
        return p
    cand = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(cand):
        return cand
    raise RuntimeError("nvcc not found")


def _build_one(lib, objdir, extra, force, verbose):
    stamp = lib + ".sha256"
    dig = _digest(extra)
    if not force and os.path.exists(lib) and os.path.exists(stamp):
        with open(stamp) as fh:
            if fh.read().strip() == dig:
                return lib
    os.makedirs(objdir, exist_ok=True)
    nvcc = nvcc_path()
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc, *NVCC_FLAGS, *extra, "-I", INCLUDE, "-c", src, "-o", obj]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"nvcc failed for {src}:\n{out.decode()}\n")
        elif verbose and out:
            sys.stderr.write(out.decode())
    if failed:
        raise RuntimeError("CUDA build failed")
    tmp = lib + ".tmp"
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp,
           "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, lib)
    with open(stamp, "w") as fh:
        fh.write(dig)
    return lib


def build(force=False, verbose=True, debug=True):
    """libfdrb200.so, and (debug=True) libfdrb200_debug.so compiled with FDR_DEBUG: the same
    kernels with their global-memory indices checked (a violation is recorded in a device
    fault word that fdr_synchronize reports; FDR_B200_DEBUG=1 makes the package load it)."""
    _build_one(LIB, os.path.join(HERE, "_build"), (), force, verbose)
    if debug:
        _build_one(LIB_DEBUG, os.path.join(HERE, "_build_debug"), ("-DFDR_DEBUG",), force, verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(LIB)
