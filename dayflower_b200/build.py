"""Builds the native libraries in-tree (no JIT cache):

* ``dayflower_b200/_lib/libdayflower_cuda.so``  - the render path (nvcc, sm_100a)
* ``dayflower_b200/_lib/libdayflower_scene.so`` - the scene-compiler host helper (g++)

Each library is rebuilt only when one of its sources is newer than it.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "_lib")
ROOT = os.path.dirname(HERE)

CUDA_SOURCES = ["dfc_api.cu", "dfc_engine.cu", "dfc_kernels.cu", "dfc_trace.cu", "dfc_shade.cu", "dfc_shade_simple.cu", "dfc_raytrace.cu",
                "dfc_ingest.cpp", "dfc_bvh.cpp", "dfc_devscene.cpp", "dfc_blas.cu"]
CUDA_HEADERS = ["dfc_scene.h", "dfc_device.cuh", "dfc_shapes.cuh", "dfc_kernels.h", "dfc_ingest.h", "dfc_bvh.h", "dfc_devscene.h",
                "dfc_blas.h", "dfc_texture.cuh", "dfc_matderive.h", "dfc_trav.cuh", "dfc_shade.cuh"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s" % (" ".join(cmd), r.stdout))
    return r.stdout


def cuda_lib_path() -> str:
    return os.path.join(LIB, "libdayflower_cuda.so")


def scene_lib_path() -> str:
    return os.path.join(LIB, "libdayflower_scene.so")


def build_cuda(force: bool = False, verbose: bool = False, extra=()) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = cuda_lib_path()
    deps = [os.path.join(CSRC, s) for s in CUDA_SOURCES + CUDA_HEADERS] + [os.path.join(ROOT, "include", "dayflower_cuda.h")]
    if not force and not _stale(out, deps):
        return out
    obj_dir = os.path.join(LIB, "_obj")
    os.makedirs(obj_dir, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in CUDA_HEADERS] + [os.path.join(ROOT, "include", "dayflower_cuda.h")]

    def compile_one(s):
        o = os.path.join(obj_dir, s + ".o")
        if not force and not extra and not _stale(o, [os.path.join(CSRC, s)] + headers):
            return o, ""  # this source and every header are older than its object
        # -fmad=false: every float operation is rounded on its own, as in the
        # reference (Java float arithmetic has no contraction); the traversal's
        # box tests use explicit fmaf where the rounding does not matter.
        cmd = [_nvcc(), "-c", os.path.join(CSRC, s), "-o", o, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
               "-Xptxas", "-O3", "--expt-relaxed-constexpr", "-fmad=false"] + GENCODE + list(extra)
        if verbose and s.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        return o, _run(cmd)

    # the sources compile independently: one nvcc process each
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(CUDA_SOURCES), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, CUDA_SOURCES))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            sys.stdout.write(log)
    _run([_nvcc(), "-shared", "-o", out] + objs + GENCODE + ["-cudart", "static"])
    return out


def build_scene(force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = scene_lib_path()
    src = os.path.join(CSRC, "scene_compiler.cpp")
    if force or _stale(out, [src]):
        _run([shutil.which("g++") or "g++", "-O2", "-std=c++17", "-fPIC", "-shared", src, "-o", out])
    return out


def build_all(force: bool = False, verbose: bool = False):
    return build_scene(force), build_cuda(force, verbose)


if __name__ == "__main__":
    print(build_all(force="--force" in sys.argv, verbose="-v" in sys.argv))
