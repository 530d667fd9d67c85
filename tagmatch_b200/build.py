"""Build recipe for the native libraries (in-tree, so they travel with the repo).

    python -m tagmatch_b200.build          # everything
    python -m tagmatch_b200.build --quick  # skip up-to-date outputs

Outputs (next to this file):
  libtagmatch_b200.so   engine, CUDA kernels (sm_100a) and the C ABI
  libtm_workload.so     seeded workload generator (CPU)
  tagmatch_facade_test  C++ facade test driver (tagmatch.hh-compatible API)
  tagmatch_serve_bench  serving load generator over the C ABI (tm_submit)
  tagmatch_driver       streaming driver (tagmatch_main.cc flow) and partition file writer
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_SOURCES = ["partition.cu", "match.cu", "noalloc.cu", "sched.cu", "engine.cu", "capi.cu", "facade.cu"]
HEADERS = ["tm_device.cuh", "tm_host.hpp", "scan.cuh", "partition.cuh", "match.cuh", "match_kernels.cuh", "sched.cuh",
           "engine.cuh"]

LIB = os.path.join(HERE, "libtagmatch_b200.so")
WORKLOAD_LIB = os.path.join(HERE, "libtm_workload.so")
FACADE_TEST = os.path.join(HERE, "tagmatch_facade_test")
SERVE_BENCH = os.path.join(HERE, "tagmatch_serve_bench")
DRIVER = os.path.join(HERE, "tagmatch_driver")


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_workload(quick=False):
    src = os.path.join(CSRC, "workload.cc")
    if quick and not _stale(WORKLOAD_LIB, [src]):
        return WORKLOAD_LIB
    _run([CXX, "-O3", "-std=c++17", "-fPIC", "-shared", "-o", WORKLOAD_LIB, src])
    return WORKLOAD_LIB


def build_engine(quick=False, extra=None):
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "tagmatch_b200.h")]
    deps += [os.path.join(INCLUDE, "tagmatch", f) for f in os.listdir(os.path.join(INCLUDE, "tagmatch"))]
    if quick and not _stale(LIB, deps):
        return LIB
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-I" + INCLUDE, "-I" + os.path.join(INCLUDE, "tagmatch"), "-o", LIB, *srcs, "-lpthread"]
    if extra:
        cmd[1:1] = extra
    _run(cmd)
    return LIB


def build_facade_test(quick=False):
    src = os.path.join(CSRC, "facade_test.cc")
    if quick and not _stale(FACADE_TEST, [src, LIB]):
        return FACADE_TEST
    _run([CXX, "-O2", "-std=c++17", "-I" + os.path.join(INCLUDE, "tagmatch"), "-I" + INCLUDE, "-o", FACADE_TEST, src,
          "-L" + HERE, "-ltagmatch_b200", "-Wl,-rpath,$ORIGIN", "-lpthread"])
    return FACADE_TEST


def build_serve_bench(quick=False):
    srcs = [os.path.join(CSRC, "serve_bench.cc"), os.path.join(CSRC, "workload.cc")]
    if quick and not _stale(SERVE_BENCH, srcs + [LIB]):
        return SERVE_BENCH
    _run([CXX, "-O2", "-std=c++17", "-I" + INCLUDE, "-o", SERVE_BENCH, *srcs,
          "-L" + HERE, "-ltagmatch_b200", "-Wl,-rpath,$ORIGIN", "-lpthread"])
    return SERVE_BENCH


def build_driver(quick=False):
    src = os.path.join(CSRC, "tagmatch_driver.cc")
    if quick and not _stale(DRIVER, [src, LIB]):
        return DRIVER
    _run([CXX, "-O2", "-std=c++17", "-I" + os.path.join(INCLUDE, "tagmatch"), "-I" + INCLUDE, "-o", DRIVER, src,
          "-L" + HERE, "-ltagmatch_b200", "-Wl,-rpath,$ORIGIN", "-lpthread"])
    return DRIVER


# Where the reference's sources are read from to build oracle/_ref (the
# reference's own test_matcher and CPU partitioner); TAGMATCH_REF overrides.
REFERENCE_SOURCES = "/root/reference"


def build_oracle():
    cmd = ["make", "-s", "-C", os.path.join(ROOT, "oracle")]
    ref = os.environ.get("TAGMATCH_REF") or (REFERENCE_SOURCES if os.path.isdir(REFERENCE_SOURCES) else "")
    if ref:
        cmd.append("REF=" + ref)
    _run(cmd)


def build_all(quick=False):
    build_workload(quick)
    build_engine(quick)
    build_facade_test(quick)
    build_serve_bench(quick)
    build_driver(quick)


if __name__ == "__main__":
    quick = "--quick" in sys.argv
    build_all(quick)
    if "--no-oracle" not in sys.argv:
        build_oracle()
