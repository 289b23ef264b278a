"""Builds the engine's shared libraries in-tree (they travel with the repo).

  lib/libnsparse_b200.so    CUDA kernels (sm_100a) + C++ API + C ABI
  synth/libnsp_synth.so     seeded synthetic corpus generator (plain C; the
                            benchmark's and tests' input data, not the engine)

Usage: python neural-sparse-cpp_b200/build.py [--force]
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(HERE, "lib", "obj")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = [f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}"]
LIBGOMP_CANDIDATES = [
    "/usr/lib/x86_64-linux-gnu/libgomp.so.1",
]


def _host_compiler():
    # Some wrappers in this image lack libgomp on their link path; the system
    # g++ is used when present.
    for c in ("/usr/bin/g++", "g++"):
        if os.path.exists(c) or c == "g++":
            return c
    return "g++"


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(ROOT, "include", "**", "*.h"), recursive=True))


def build_engine(force=False, jobs=8):
    os.makedirs(OBJ, exist_ok=True)
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    hdrs = _headers()
    cxx = _host_compiler()
    tasks = []
    objs = []
    for src in cu:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            tasks.append([NVCC, *ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                          "-ccbin", cxx, *INCLUDES, "-c", src, "-o", obj])
    for src in cpp:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            # ref_order.cpp makes the reference's C++20 library calls
            std = "-std=c++20" if os.path.basename(src) == "ref_order.cpp" else "-std=c++17"
            tasks.append([cxx, "-O3", std, "-fPIC", "-Wall", "-Wno-unused-function",
                          f"-I{CUDA}/include", *INCLUDES, "-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        list(ex.map(_run, tasks))
    so = os.path.join(LIB, "libnsparse_b200.so")
    if force or tasks or _stale(so, objs):
        _run([NVCC, *ARCH, "-shared", "-ccbin", cxx, "-o", so, *objs, "-lcudart_static", "-lrt",
              "-ldl", "-lpthread"])
    return so


def build_synth(force=False):
    os.makedirs(OBJ, exist_ok=True)
    src = os.path.join(HERE, "synth", "nsp_synth.c")
    so = os.path.join(HERE, "synth", "libnsp_synth.so")
    if force or _stale(so, [src]):
        obj = os.path.join(HERE, "synth", "nsp_synth.o")
        gomp = next((p for p in LIBGOMP_CANDIDATES if os.path.exists(p)), "-lgomp")
        _run(["gcc", "-std=c11", "-O2", "-fPIC", "-fopenmp", "-c", src, "-o", obj])
        _run(["gcc", "-shared", "-o", so, obj, gomp, "-lm"])
    return so


def main(argv):
    force = "--force" in argv
    print(build_synth(force))
    print(build_engine(force))


if __name__ == "__main__":
    main(sys.argv[1:])
