"""Builds libcaviar_b200.so (the sm_100a kernels + C ABI) in-tree with nvcc.

Usage: python -m caviar_b200.build   (or caviar_b200.build.build())
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libcaviar_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "cvr_abi.cu"), os.path.join(HERE, "csrc", "cvr_noalloc.cu"),
           os.path.join(HERE, "csrc", "cvr_casl.cpp"), os.path.join(HERE, "csrc", "cvr_batch.cu"),
           os.path.join(HERE, "csrc", "cvr_adjoint.cu"), os.path.join(HERE, "csrc", "cvr_peaks.cu")]
CLI = os.path.join(HERE, "caviar_b200_casl")
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in ("cvr_device.cuh", "cvr_build.cuh", "cvr_force.cuh", "cvr_kforce_tc.cuh", "cvr_main.cpp")] + [
    os.path.join(ROOT, "include", "caviar_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-shared",
           "--diag-suppress", "177,550", "-o", LIB + ".tmp", *SOURCES, "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    # command-line front end: caviar_b200_casl script.casl (like `CAVIAR -i script`)
    subprocess.run([nvcc(), *ARCH, "-O2", "-std=c++17", "-o", CLI, os.path.join(HERE, "csrc", "cvr_main.cpp"),
                    "-L" + HERE, "-lcaviar_b200", "-Xlinker", "-rpath,$ORIGIN"], check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
