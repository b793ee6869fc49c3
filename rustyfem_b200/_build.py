"""Build of the native libraries, in-tree (``rustyfem_b200/_lib``).

* ``librustyfem_gpu.so`` — the product: the C interface of RustyFEM's sparse
  solver (``rustyfem_*``) and its extensions (``rfg_*``), host symbolic stage in
  C++ and the numeric phase as CUDA kernels for sm_100a;
* ``librfgmesh.so``      — the synthetic workload generator (host only).

The build is plain nvcc/g++ invocations; nothing is JIT-compiled at import.
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
REPO = os.path.dirname(HERE)
INCLUDE = os.path.join(REPO, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

GPU_LIB = os.path.join(LIBDIR, "librustyfem_gpu.so")
MESH_LIB = os.path.join(LIBDIR, "librfgmesh.so")

# host C++ sources of the product library and its CUDA sources
GPU_CXX = ["symbolic.cpp", "hostmem.cpp", "plan.cpp", "autotune.cpp", "devmem.cpp", "capi.cpp"]
GPU_CU = ["numeric.cu", "solve.cu", "chain.cu", "kernels_tc.cu", "indef.cu", "devutil.cu", "assembly.cu", "lu.cu"]
# the indefinite and LU kernels and the assembly of K round every product and sum separately,
# as the reference does
NO_FMAD = {"indef.cu", "assembly.cu", "lu.cu"}


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout)
    return r.stdout


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def build_mesh(force: bool = False) -> str:
    src = os.path.join(CSRC, "meshgen.cpp")
    os.makedirs(LIBDIR, exist_ok=True)
    if force or _stale(MESH_LIB, [src]):
        _run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", src, "-o", MESH_LIB])
    return MESH_LIB


def build_gpu(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    srcs = [os.path.join(CSRC, f) for f in GPU_CXX + GPU_CU if os.path.exists(os.path.join(CSRC, f))]
    hdrs = _headers()
    if not (force or _stale(GPU_LIB, srcs + hdrs)):
        return GPU_LIB
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        objs.append(o)
        if not (force or _stale(o, [s] + hdrs)):
            continue
        if s.endswith(".cu"):
            cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC,
                   "--expt-relaxed-constexpr", "-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            if os.path.basename(s) in NO_FMAD:
                cmd.insert(1, "-fmad=false")
        else:
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-pthread", "-I", INCLUDE, "-I", CSRC,
                   "-I", "/usr/local/cuda/include", "-c", s, "-o", o]
        out = _run(cmd)
        if verbose and out:
            print(out)
    _run([NVCC, *ARCH, "-shared", "-o", GPU_LIB, *objs, "-lcuda", "-Xcompiler", "-pthread"])
    return GPU_LIB


def mesh_library() -> str:
    if not os.path.exists(MESH_LIB):
        if shutil.which("g++") is None:
            raise RuntimeError(f"{MESH_LIB} is missing and no compiler is available")
        build_mesh()
    return MESH_LIB


def gpu_library() -> str:
    if not os.path.exists(GPU_LIB):
        raise RuntimeError(f"{GPU_LIB} is missing: run __graft_entry__.build() (or rustyfem_b200._build.build_gpu())")
    return GPU_LIB
