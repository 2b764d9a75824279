"""Build the sm_100a shared library ``minicombust_app_b200/lib/libmcflow.so``.

Usage: ``python -m minicombust_app_b200.build`` (also called by
``__graft_entry__.build()``).  nvcc cross-compiles without a GPU.  The
assembly kernels are compiled with ``-fmad=false`` so that their FP64
arithmetic is the plain IEEE sequence of the reference's C++; the host-side
geometry is compiled with FMA contraction off for the same reason.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(LIBDIR, "libmcflow.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
                      "-I", CSRC]

# (source, extra nvcc flags)
CUDA_SOURCES = [
    ("flow_kernels.cu", ["-fmad=false"]),
    ("krylov.cu", []),
    ("amg.cu", []),
    ("flow_api.cu", []),
    ("solve_noalloc.cu", []),
    ("exchange.cu", ["-fmad=false"]),
    ("gnn.cu", []),
    ("gnn_umma.cu", []),
    ("gnn_api.cu", []),
]
CXX_SOURCES = [("mesh_setup.cpp", ["-ffp-contract=off", "-fno-fast-math"])]


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout)
    return r.stdout


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    nvcc = _nvcc()
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "minicombust_flow.h"))
    headers.append(os.path.join(ROOT, "include", "minicombust_gnn.h"))
    objs = []
    for src, flags in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + headers):
            out = _run([nvcc] + NVCC_COMMON + flags + ["-c", s, "-o", o])
            if verbose and out:
                print(out)
        objs.append(o)
    for src, flags in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + headers):
            _run(["g++", "-O2", "-fPIC", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", CSRC] + flags
                 + ["-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
