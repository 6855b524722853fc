"""Build the B200 solve-phase library (libxamg_b200.so) and the CPU oracle.

The CUDA sources are compiled for sm_100a only; host C++ is compiled with
-ffp-contract=off so that host-side arithmetic (dense coarse inverse, setup)
keeps its written evaluation order.  Outputs stay in-tree:
  xamg-test_b200/libxamg_b200.so, oracle/liboracle.so
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = os.path.join(HERE, "libxamg_b200.so")
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle.so")

CU_SOURCES = ["kernels.cu", "gs.cu", "gsw.cu", "noalloc.cu", "cnn.cu", "batch.cu"]
CPP_SOURCES = ["host/gen.cpp", "host/amg.cpp", "host/params.cpp", "host/solve.cpp", "host/runs.cpp",
               "host/batch.cpp", "host/dist.cpp", "host/dist_solve.cpp", "host/c_api.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r.stdout + r.stderr


def _newer(src, dst):
    return not os.path.exists(dst) or os.path.getmtime(src) > os.path.getmtime(dst)


def build_library(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in ("kernels.cuh",)] + [
        os.path.join(CSRC, "host", f) for f in os.listdir(os.path.join(CSRC, "host")) if f.endswith(".h")
    ] + [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    hdr_time = max(os.path.getmtime(h) for h in headers)
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(obj)
        if _newer(src, obj) or hdr_time > os.path.getmtime(obj):
            jobs.append([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                         "--expt-relaxed-constexpr", "-Xptxas", "-v" if verbose else "-O3",
                         "-c", "-o", obj, src])
    for s in CPP_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(obj)
        if _newer(src, obj) or hdr_time > os.path.getmtime(obj):
            jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off",
                         "-Wall", "-Wno-unused-variable", "-Wno-sign-compare",
                         "-I" + os.path.join(CUDA, "include"), "-c", "-o", obj, src])
    with ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as ex:
        outs = list(ex.map(_run, jobs))
    if verbose:
        for o in outs:
            sys.stdout.write(o)
    if jobs or not os.path.exists(LIB):
        _run(["g++", "-shared", "-fopenmp", "-o", LIB, *objs, "-L" + os.path.join(CUDA, "lib64"),
              "-lcudart_static", "-lpthread", "-ldl", "-lrt", "-Wl,--no-undefined"])
    return LIB


ORACLE_SOURCES = ["oracle.cpp", "amg_oracle.cpp"]


def build_oracle():
    srcs = [os.path.join(ROOT, "oracle", s) for s in ORACLE_SOURCES]
    if any(_newer(s, ORACLE_LIB) for s in srcs):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-o", ORACLE_LIB,
              *srcs])
    return ORACLE_LIB


if __name__ == "__main__":
    build_library(verbose="-v" in sys.argv)
    build_oracle()
    print("built", LIB, ORACLE_LIB)
