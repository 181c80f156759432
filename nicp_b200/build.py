"""Builds the native libraries of nicp_b200 in-tree.

    python -m nicp_b200.build            # both libraries
    python -m nicp_b200.build --force    # rebuild even if up to date

Outputs (next to this file, so they travel with the source tree):
  libnicp_b200.so   the CUDA path (sm_100a), C ABI of include/nicp_gpu.h
  libnicp_synth.so  the synthetic depth renderer, C ABI of include/nicp_synth.h
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")

GPU_LIB = os.path.join(HERE, "libnicp_b200.so")
SYNTH_LIB = os.path.join(HERE, "libnicp_synth.so")

CUDA_SOURCES = ["k_cloud.cu", "k_align.cu", "k_merge.cu", "k_nn.cu", "capi.cu"]
HOST_SOURCES = ["stats_host.cpp", "server.cpp", "cloud_io.cpp"]
HEADERS = ["common.cuh", "kernels.hpp", "host_math.hpp", "abi_guard.hpp"]

NVCC = os.environ.get("NVCC", "nvcc")
# The image may export CXX pointing at a toolchain without libgomp.
CXX = os.environ.get("NICP_CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_FLAGS = ["-O3", "-fPIC", "-std=c++17", "-ffp-contract=off", "-pthread"]


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def build_gpu(force=False, verbose=False):
    deps = [os.path.join(CSRC, f) for f in CUDA_SOURCES + HOST_SOURCES + HEADERS]
    deps += [os.path.join(INCLUDE, "nicp_gpu.h")]
    if not force and _newer(GPU_LIB, deps):
        return GPU_LIB
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for src in CUDA_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-I", INCLUDE, "-I", CSRC,
               "-Xcompiler", "-fPIC,-ffp-contract=off", "-ccbin", CXX, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = _run(cmd)
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    for src in HOST_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        _run([CXX, *HOST_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    tmp = GPU_LIB + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-ccbin", CXX, "-o", tmp, *objs])
    os.replace(tmp, GPU_LIB)
    return GPU_LIB


def build_synth(force=False):
    src = os.path.join(CSRC, "synth.cpp")
    deps = [src, os.path.join(INCLUDE, "nicp_synth.h")]
    if not force and _newer(SYNTH_LIB, deps):
        return SYNTH_LIB
    tmp = SYNTH_LIB + ".tmp"
    _run([CXX, *HOST_FLAGS, "-fopenmp", "-shared", "-I", INCLUDE, src, "-o", tmp])
    os.replace(tmp, SYNTH_LIB)
    return SYNTH_LIB


def build_all(force=False, verbose=False):
    return build_gpu(force, verbose), build_synth(force)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    for p in build_all(a.force, a.verbose):
        print(p)
