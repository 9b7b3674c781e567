"""Builds the B200 dedispersion library in-tree: pirate_b200/libpirate_b200.so (sm_100a), and the
pybind11 module pirate_b200/_pirate_b200_pybind*.so over it (pirate's pybind11 class surface).

Usage: python -m pirate_b200.build [--force] [--verbose]
"""

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpirate_b200.so")

SOURCES = ["plan.cpp", "avar.cpp", "simpulse.cpp", "capi.cpp", "kernels.cu", "dedisperser.cu", "noalloc.cu", "sifter.cu", "batched.cu"]
HEADERS = ["plan.hpp", "avar.hpp", "simpulse.hpp", "yaml_lite.hpp", "kernels.cuh", "dedisperser.hpp", "regtree.cuh", "sifter.hpp", "batched.hpp"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no fused multiply-add contraction, so the kernels perform the same fp32 roundings as
# the reference CPU arithmetic they restate.
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "-Xcudafe", "--diag_suppress=177"]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def build_pybind(force=False):
    """The pybind11 module (pirate_b200/csrc/pybind.cpp over include/pirate_b200.hpp), linked to the
    library with an $ORIGIN rpath."""
    import sysconfig
    import pybind11
    out = os.path.join(HERE, "_pirate_b200_pybind" + sysconfig.get_config_var("EXT_SUFFIX"))
    root = os.path.dirname(HERE)
    deps = [os.path.join(CSRC, "pybind.cpp"), os.path.join(root, "include", "pirate_b200.hpp"),
            os.path.join(root, "include", "pirate_b200.h"), LIB]
    if not force and os.path.exists(out) and os.path.getmtime(out) >= _newest(deps):
        return out
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-shared", "-fPIC", "-std=c++17",
           "-I" + sysconfig.get_paths()["include"], "-I" + pybind11.get_include(),
           os.path.join(CSRC, "pybind.cpp"), "-o", out + ".tmp", "-L" + HERE, "-lpirate_b200", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("pybind11 module build failed:\n%s\n%s" % (r.stdout, r.stderr))
    os.replace(out + ".tmp", out)
    return out


def build(force=False, verbose=False):
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [
        os.path.join(os.path.dirname(HERE), "include", "pirate_b200.h"), os.path.abspath(__file__)]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest(deps):
        return LIB
    os.makedirs(BUILD, exist_ok=True)

    def compile_one(src):
        obj = os.path.join(BUILD, src + ".o")
        cmd = [NVCC] + ARCH + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu") and verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed on %s:\n%s\n%s" % (src, r.stdout, r.stderr))
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    build_pybind(force="--force" in sys.argv)
    print(LIB)
