"""Build libpt_b200/lib/libpt_b200.so from csrc/ with nvcc for sm_100a.

    python -m libpt_b200.build [--force] [--verbose]

Objects go to libpt_b200/_build/ (git-ignored); the shared library is built
in-tree so that it travels with the source tree.
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libpt_b200.so")
CLI = os.path.join(LIBDIR, "pt_benchmark")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
HOST_CXX = "/usr/bin/g++"   # the image's $CXX wrapper lacks some runtime specs

SOURCES = ["gemm_dmma.cu", "gemm_tc.cu", "gemm_i8.cu", "epilogue.cu", "prep.cu",
           "exec.cu", "plan.cu", "plan_views.cu", "plan_upload.cu",
           "plan_cases.cu", "plan_emu.cu", "plan_tune.cu", "plan_run.cu",
           "tune.cpp", "api.cpp", "noalloc.cu", "selftest.cu", "server.cpp",
           "producer.cu"]
HEADERS = ["common.cuh", "engine.h", "exec.h", "plan.h", "plan_impl.h",
           "tune.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    hdrs.append(os.path.join(ROOT, "include", "pt.h"))
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            cmd = [NVCC, "-ccbin", HOST_CXX] + ARCH + FLAGS
            if src.endswith(".cpp"):
                cmd += ["-x", "cu"]
            cmd += ["-Xptxas", "-v"] if verbose else []
            cmd += ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _newer(LIB, objs):
        cmd = [NVCC, "-ccbin", HOST_CXX] + ARCH + ["-shared", "-o", LIB] + objs
        cmd += ["-Xcompiler", "-fPIC", "-lcudart_static", "-ldl", "-lrt",
                "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    # the reference's benchmark command line against this library
    cli_src = os.path.join(HERE, "cli", "pt_benchmark.c")
    if force or _newer(CLI, [cli_src, LIB, os.path.join(ROOT, "include", "pt.h")]):
        cmd = ["/usr/bin/gcc", "-O2", "-std=c11", "-Wall",
               "-I" + os.path.join(ROOT, "include"), cli_src, "-o", CLI,
               "-L" + LIBDIR, "-lpt_b200", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    sys.exit(main())
