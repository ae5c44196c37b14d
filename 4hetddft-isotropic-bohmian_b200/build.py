"""Build libhe4b200.so (the C-ABI library) in-tree with nvcc for sm_100a.

Usage: python build.py [--force] [--verbose]
The library lands next to this file so it travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhe4b200.so")
SOURCES = ["abi.cu", "fft.cu", "setup.cu", "field.cu", "impurity.cu", "step.cu", "energy.cu", "diag.cu", "fno.cu", "batch.cu"]
HEADERS = ["common.cuh", "stencil.cuh", "reduce.cuh", "fft_reg.cuh", "fft_passes.cuh", "stream_stencil.cuh", "bulk.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "he4_tddft.h"))
    deps.append(os.path.join(HERE, "..", "include", "he4_fno.h"))
    deps += [os.path.join(HERE, "driver", f) for f in DRIVER_SOURCES + ["he4io.hpp"]]
    if not os.path.exists(DRIVER):
        return True
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [NVCC, *FLAGS, *extra, "-dc" if False else "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if out:
            sys.stdout.write(out.decode())
        if p.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed for " + ", ".join(failed))
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp, "-lcudart",
           "-Xlinker", "--no-undefined"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    build_driver(verbose=verbose)
    return LIB


DRIVER = os.path.join(HERE, "he4run")
DRIVER_SOURCES = ["he4io.cpp", "he4run.cpp"]


def build_driver(verbose=False):
    """The C++ host driver (namelist, readenc mode 2, printoutc, time loop),
    linked against libhe4b200.so next to it."""
    srcs = [os.path.join(HERE, "driver", f) for f in DRIVER_SOURCES]
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-Wall", *srcs, "-o", DRIVER + ".tmp",
           "-L" + HERE, "-lhe4b200", "-Wl,-rpath,$ORIGIN", "-pthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(DRIVER + ".tmp", DRIVER)
    return DRIVER


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)
