"""Build the in-tree shared libraries under ``specfempp_b200/_lib``.

``libspecfem_b200.so`` is the product: host C++ compiled with g++, CUDA with
nvcc for sm_100a, linked by nvcc into one shared object exporting the C ABI
of ``include/specfem_b200.h`` (FP32, the reference's type_real).

``libspecfem_b200_fp64.so`` is the verification build: the same device
driver and generic kernels compiled with ``-DSFB_FP64`` (every wavefield,
geometry and per-step quantity in FP64), for parity tests against the FP64
oracle at FP64 rounding level.  It is test infrastructure, not a product
path; the FP32-only kernels and the allocation-free entry point are not in
it.

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
LIB64 = os.path.join(LIBDIR, "libspecfem_b200_fp64.so")
# CUDA sources of the FP64 verification build (the device driver and kernels)
FP64_CUDA = ("context.cu", "kernels.cu")

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
    out = [os.path.join(ROOT, "include", h) for h in ("specfem_b200.h", "specfem_b200_3d.h")]
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


def _link(out, objs):
    cmd = [NVCC] + ARCH + ["-shared", "-o", out] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed: %s\n%s" % (r.stdout, r.stderr))


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    host, cuda = _sources()
    headers = _headers()
    jobs = []
    objs, objs64 = [], []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in host + cuda:
        is_cuda = src.endswith(".cu")
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if ptxas_info and is_cuda or _stale(obj, src, headers):
            jobs.append((src, obj, is_cuda, extra))
        if not is_cuda:
            objs64.append(obj)
        elif os.path.basename(src) in FP64_CUDA:
            obj64 = os.path.join(BUILD, os.path.basename(src) + ".fp64.o")
            objs64.append(obj64)
            if _stale(obj64, src, headers):
                jobs.append((src, obj64, True, ["-DSFB_FP64"]))
    logs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            futs = [ex.submit(_compile, s, o, c, e) for s, o, c, e in jobs]
            for f in futs:
                logs.append(f.result())
    if jobs or not os.path.exists(LIB):
        _link(LIB, objs)
    if jobs or not os.path.exists(LIB64):
        _link(LIB64, objs64)
    if verbose:
        for l in logs:
            if l:
                sys.stderr.write(l)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
