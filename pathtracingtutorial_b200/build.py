"""Build libpt_b200.so in-tree for sm_100a.

Host C++ (scene I/O, SAH BVH, light tables, C ABI) is compiled by g++ with
-ffp-contract=off so that host-side prep arithmetic is rounded exactly as the
reference's host build rounds it; the CUDA translation unit is compiled by
nvcc for sm_100a only.  Objects go to _build/, the shared library next to this
file (it is what the Python package and the tests load).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build", "pt_b200")
LIB = os.path.join(HERE, "libpt_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

CXX_SOURCES = ["host_prep.cpp", "scene_io.cpp", "image_decode.cpp", "capi.cpp"]
CU_SOURCES = ["integrator.cu", "static_trace.cu", "lbvh.cu"]
HEADERS = ["image_decode.h", "pt_internal.h", "sampler.h", "bsdf.h", "traverse.h", "engine.h", "device_api.h", "batch.cuh", "guide.cuh", "guide_tc.cuh", "guide_host.cuh"]

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-Wall",
            "-Wno-unused-function", f"-I{CUDA_HOME}/include", f"-I{ROOT}/include"]
NVCCFLAGS = GENCODE + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
                       "--expt-relaxed-constexpr", f"-I{ROOT}/include"]


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and os.environ.get("PT_BUILD_VERBOSE"):
        sys.stderr.write(r.stderr)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "pt_b200.h")]
    jobs = []
    objs = []
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            jobs.append(["g++", *CXXFLAGS, "-c", s, "-o", o])
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC, *NVCCFLAGS, *extra, "-c", s, "-o", o])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(_run_verbose if (verbose or ptxas_info) else _run, jobs))
    if jobs or _stale(LIB, objs):
        _run([NVCC, *GENCODE, "-shared", "-o", LIB, *objs, "-cudart", "static", "-lpthread", "-lz"])
    return LIB


def _run_verbose(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}")


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
