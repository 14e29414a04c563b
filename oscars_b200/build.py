"""Build recipe of liboscars_b200.so (sm_100a kernels + C++ host core + C ABI), in-tree.

    python -m oscars_b200.build [--force]

CUDA sources are compiled with ``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo``; the
host C++ is compiled with ``-ffp-contract=off`` so its double arithmetic rounds like the
reference's x86-64 build.  Objects go to oscars_b200/_build/, the library to
oscars_b200/liboscars_b200.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liboscars_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_FLAGS = ["-O3", "-fPIC", "-ffp-contract=off", "-fvisibility=hidden", "-pthread"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xptxas=-v"] + \
    sum([["-Xcompiler", f] for f in HOST_FLAGS], [])

CU_SOURCES = ["kernels_fp64.cu", "kernels_mixed.cu", "kernels_stl.cu", "engine.cu", "stl.cu", "noalloc.cu", "batch.cu", "adjoint.cu"]
CC_SOURCES = ["host_core.cc", "capi.cc"]
HEADERS = ["host_core.h", "engine.h", "kernels.h", "batch.h", "device_common.cuh", "fd_common.cuh"]


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def _compile(args, log):
    r = subprocess.run(args, capture_output=True, text=True)
    with open(log, "w") as f:
        f.write(" ".join(args) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("compile failed:\n" + " ".join(args) + "\n" + r.stdout + r.stderr)
    return args[-1]


def build(force: bool = False, verbose: bool = False) -> str:
    if shutil.which(NVCC) is None and not os.path.exists(NVCC):
        raise RuntimeError("nvcc not found at %s" % NVCC)
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "oscars_b200.h")]
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _newer([src] + headers, obj):
            jobs.append(([NVCC] + NVCC_FLAGS + ["-I" + INCLUDE, "-c", src, "-o", obj], obj + ".log"))
    for s in CC_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _newer([src] + headers, obj):
            jobs.append((["g++", "-std=c++17"] + HOST_FLAGS + ["-I" + INCLUDE, "-I" + os.path.join(CUDA_HOME, "include"),
                                                               "-c", src, "-o", obj], obj + ".log"))
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for f in [ex.submit(_compile, a, l) for a, l in jobs]:
            f.result()
    if jobs or not os.path.exists(LIB):
        tmp = LIB + ".tmp"
        _compile([NVCC] + ARCH + ["-shared", "-cudart", "static", "-Xcompiler", "-pthread"] + objs + ["-o", tmp],
                 os.path.join(BUILD, "link.log"))
        os.replace(tmp, LIB)
    if verbose:
        for s in CU_SOURCES:
            log = os.path.join(BUILD, s + ".o.log")
            if os.path.exists(log):
                print(open(log).read())
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
