"""Build the in-tree shared library ``specfempp_b200/_lib/libspecfem_b200.so``.

Host C++ is compiled with g++, CUDA with nvcc for sm_100a; both are linked by
nvcc into one shared object exporting the C ABI of ``include/specfem_b200.h``.
Object files are cached under ``specfempp_b200/_build`` keyed on source
timestamps.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libspecfem_b200.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall", "-Wno-unused-function"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
           "--expt-relaxed-constexpr"] + ARCH


def _sources():
    host = sorted(os.path.join(CSRC, "host", f) for f in os.listdir(os.path.join(CSRC, "host"))
                  if f.endswith(".cpp"))
    cuda = sorted(os.path.join(CSRC, "cuda", f) for f in os.listdir(os.path.join(CSRC, "cuda"))
                  if f.endswith(".cu"))
    return host, cuda


def _headers():
    out = [os.path.join(ROOT, "include", "specfem_b200.h")]
    for sub in ("host", "cuda"):
        d = os.path.join(CSRC, sub)
        out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".hpp", ".cuh", ".h"))]
    return out


def _stale(obj, src, headers):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + headers)


def _compile(src, obj, cuda, extra):
    if cuda:
        cmd = [NVCC] + NVFLAGS + extra + ["-c", src, "-o", obj]
    else:
        cmd = [CXX] + CXXFLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stderr


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    host, cuda = _sources()
    headers = _headers()
    jobs = []
    objs = []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in host + cuda:
        is_cuda = src.endswith(".cu")
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if ptxas_info and is_cuda or _stale(obj, src, headers):
            jobs.append((src, obj, is_cuda))
    logs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            futs = [ex.submit(_compile, s, o, c, extra) for s, o, c in jobs]
            for f in futs:
                logs.append(f.result())
    if jobs or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s" % (r.stdout, r.stderr))
    if verbose:
        for l in logs:
            if l:
                sys.stderr.write(l)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
