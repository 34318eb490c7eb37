"""Builds libmufflon_core.so in-tree (mufflon_b200/lib/) for sm_100a.

CUDA sources are compiled by nvcc with ``-gencode arch=compute_100a,code=sm_100a``
and ``--fmad=false`` (no implicit FMA contraction; explicit fmaf only), host
sources by the system g++ with ``-ffp-contract=off``. Both settings are what
keeps the renderer bit-identical to the CPU oracle. The CUDA runtime is linked
statically so the library does not depend on which libcudart a process loaded.
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
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libmufflon_core.so")
LOADER_LIB = os.path.join(LIB_DIR, "libmufflon_loader.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

CU_SOURCES = ["lbvh/lbvh.cu", "lbvh/wide.cu", "lbvh/sort_noalloc.cu", "trace/pt.cu", "trace/wavefront.cu",
              "core/light_build.cu", "core/instance_boxes.cu", "trace/lt.cu",
              "trace/bpt.cu", "trace/vcm.cu", "trace/wireframe.cu"]
CPP_SOURCES = ["core/interface.cpp", "core/scene_build.cpp"]
# the scene-file loader: its own library on top of the core's C API
LOADER_SOURCES = ["loader/json.cpp", "loader/mff_binary.cpp", "loader/scene_loader.cpp", "loader/interface.cpp"]
LOADER_HEADERS = ["loader/json.hpp", "loader/mff_binary.hpp", "loader/scene_loader.hpp"]
HEADERS = ["common/fmath.hpp", "common/pfm.hpp", "trace/dmath.cuh", "trace/intersect.cuh", "trace/shading.cuh",
           "trace/scene_types.hpp", "trace/pt_api.hpp", "lbvh/lbvh.hpp", "lbvh/radix_sort.cuh",
           "lbvh/sort_noalloc.hpp", "trace/wavefront.hpp", "trace/wide_traverse.cuh", "lbvh/wide.hpp", "core/world.hpp",
           "core/light_build.hpp", "core/instance_boxes.hpp", "trace/lt_api.hpp",
           "trace/emit.cuh", "trace/accumulate.cuh", "trace/ray_queue.cuh", "trace/bidir.cuh", "trace/aux_targets.cuh"]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false", "-Xptxas", "-v",
              "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr", "-ccbin", CXX]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
             "-Wno-unused-function", f"-I{CUDA_HOME}/include"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src, verbose):
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src.replace("/", "_") + ".o")
    deps = [path] + [os.path.join(CSRC, h) for h in HEADERS + LOADER_HEADERS] + \
        [os.path.join(ROOT, "include", h) for h in ("mufflon_core.h", "mff_interface.h")]
    if not _newer(obj, deps):
        return obj, ""
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", path, "-o", obj]
    else:
        hidden = ["-fvisibility=hidden"] if src.startswith("loader/") else []
        cmd = [CXX] + CXX_FLAGS + hidden + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stdout + r.stderr


def build(verbose: bool = False) -> str:
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), CU_SOURCES + CPP_SOURCES))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log)
    if _newer(LIB, objs):
        cmd = [CXX, "-shared", "-o", LIB] + objs + [f"-L{CUDA_HOME}/lib64", "-lcudart_static", "-ldl", "-lrt",
                                                    "-lpthread", "-Wl,--no-undefined"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        lobjs = [o for o, _ in ex.map(lambda s: _compile(s, verbose), LOADER_SOURCES)]
    if _newer(LOADER_LIB, lobjs + [LIB]):
        cmd = [CXX, "-shared", "-o", LOADER_LIB] + lobjs + [f"-L{LIB_DIR}", "-lmufflon_core", "-lz",
                                                           "-Wl,-rpath,$ORIGIN", "-Wl,--no-undefined"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


def clean():
    shutil.rmtree(BUILD, ignore_errors=True)
    for lib in (LIB, LOADER_LIB):
        if os.path.exists(lib):
            os.remove(lib)


if __name__ == "__main__":
    if "--clean" in sys.argv:
        clean()
    print(build(verbose="-v" in sys.argv))
