"""Builds libsdc_b200.so (sm_100a) in-tree: sdc_b200/_lib/libsdc_b200.so.

nvcc -gencode arch=compute_100a,code=sm_100a for the CUDA sources, g++ for the host
C++; objects are rebuilt when a source or header is newer.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(HERE, "_lib", "obj")
LIB = os.path.join(OUT_DIR, "libsdc_b200.so")
DRIVER = os.path.join(OUT_DIR, "rbc_run")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-I" + INCLUDE, "-I" + CSRC]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-I" + INCLUDE, "-I" + CSRC, "-I/usr/local/cuda/include"]

CU_SOURCES = ["api.cu", "peak_fp64.cu", "nonlinear_static.cu", "fno.cu"]
CPP_SOURCES = ["galerkin.cpp", "dump_io.cpp"]


def _deps():
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hdrs.append(os.path.join(INCLUDE, "rbc.h"))
    return max(os.path.getmtime(h) for h in hdrs)


def _stale(src, obj, hdr_time):
    return not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_time)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force=False, verbose=False, extra_nvflags=()):
    os.makedirs(OBJ_DIR, exist_ok=True)
    hdr_time = _deps()
    jobs = []
    objs = []
    for f in CU_SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ_DIR, f + ".o")
        objs.append(obj)
        if force or _stale(src, obj, hdr_time):
            jobs.append([NVCC] + ARCH + NVFLAGS + list(extra_nvflags) + ["-c", src, "-o", obj])
    for f in CPP_SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ_DIR, f + ".o")
        objs.append(obj)
        if force or _stale(src, obj, hdr_time):
            jobs.append(["g++"] + CXXFLAGS + ["-c", src, "-o", obj])
    if jobs:
        with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
            list(ex.map(lambda c: _run(c, verbose), jobs))
    if jobs or force or not os.path.exists(LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"], verbose)
    drv_src = os.path.join(CSRC, "rbc_run.cpp")
    if force or not os.path.exists(DRIVER) or os.path.getmtime(DRIVER) < max(os.path.getmtime(drv_src),
                                                                              os.path.getmtime(LIB)):
        _run(["g++", "-O2", "-std=c++17", "-I" + INCLUDE, drv_src, "-o", DRIVER, "-L" + OUT_DIR, "-lsdc_b200",
              "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
