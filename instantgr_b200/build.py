"""Builds the native library and command-line tools of instantgr_b200.

Outputs (in-tree, so that they travel with the source tree):
  instantgr_b200/lib/libigr_b200.so   C ABI of include/instantgr_b200.h
  instantgr_b200/bin/igr_route         `-cap/-net/-out` command line
  instantgr_b200/bin/igr_generate      synthetic design generator (stand-alone)
CUDA sources are compiled for sm_100a only; objects are rebuilt when a source
or any header under csrc/ is newer than the object.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib")
BIN = os.path.join(HERE, "bin")
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_INC = "/usr/local/cuda/include"

CU_SOURCES = ["cost.cu", "commit.cu", "ripup.cu", "pattern.cu", "pattern_static.cu", "color.cu", "dag.cu", "plan.cu",
              "seed_nn.cu", "seed_feat.cu", "shapes.cu", "eval.cu", "records.cu", "dagbuild.cu", "launch.cu"]
CPP_SOURCES = ["design_io.cpp", "pins.cpp", "netbuild.cpp", "gen.cpp", "dag_build.cpp", "dag_device.cpp", "router.cpp",
               "capi.cpp", "seed_model.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: the only multiply-add the reference contracts is written as fma() explicitly
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC", "-Xptxas", "-v"] + ARCH
CXX_FLAGS = ["-std=c++17", "-O3", "-fPIC", "-pthread", "-Wall", "-Wno-unused-function", "-I" + CUDA_INC]


def _headers_mtime() -> float:
    m = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".hpp", ".cuh", ".h")):
                m = max(m, os.path.getmtime(os.path.join(d, f)))
    return m


def _stale(src: str, obj: str, hdr: float) -> bool:
    return not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr)


def _run(cmd: list[str], log: list[str]) -> None:
    p = subprocess.run(cmd, capture_output=True, text=True)
    log.append(" ".join(cmd) + "\n" + p.stdout + p.stderr)
    if p.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + p.stdout + p.stderr)


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    hdr = _headers_mtime()
    jobs_list = []
    objs = []
    for s in CU_SOURCES:
        src, obj = os.path.join(CSRC, s), os.path.join(OBJ, s + ".o")
        objs.append(obj)
        if _stale(src, obj, hdr):
            jobs_list.append([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj])
    for s in CPP_SOURCES:
        src, obj = os.path.join(CSRC, s), os.path.join(OBJ, s + ".o")
        objs.append(obj)
        if _stale(src, obj, hdr):
            jobs_list.append(["g++"] + CXX_FLAGS + ["-c", src, "-o", obj])
    log: list[str] = []
    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        list(ex.map(lambda c: _run(c, log), jobs_list))
    so = os.path.join(LIB, "libigr_b200.so")
    if jobs_list or not os.path.exists(so):
        _run([NVCC, "-shared", "-o", so] + objs + ARCH + ["-lpthread", "-ldl"], log)
    exe = os.path.join(BIN, "igr_route")
    main_src = os.path.join(CSRC, "main_route.cpp")
    if _stale(main_src, exe, max(hdr, os.path.getmtime(so))):
        _run(["g++", "-std=c++17", "-O2", main_src, "-o", exe, "-L" + LIB, "-ligr_b200",
              "-Wl,-rpath,$ORIGIN/../lib"], log)
    # the design generator alone, without the router library
    gen = os.path.join(BIN, "igr_generate")
    gen_srcs = [os.path.join(CSRC, "gen_main.cpp"), os.path.join(CSRC, "gen.cpp")]
    if not os.path.exists(gen) or os.path.getmtime(gen) < max(hdr, *(os.path.getmtime(s) for s in gen_srcs)):
        _run(["g++"] + CXX_FLAGS + gen_srcs + ["-o", gen], log)
    if verbose:
        sys.stdout.write("\n".join(log))
    return so


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
