"""Builds libafqmc_b200.so (sm_100a) in-tree with nvcc, then the driver program.

The library is the product: every CUDA kernel and the C ABI of include/afqmc_b200.h.
It is compiled for sm_100a only (`-gencode arch=compute_100a,code=sm_100a`).  The driver
program `miniafqmc` (app/miniafqmc.cpp, g++) is the miniapp's main over that ABI."""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libafqmc_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
DRIVER_SRC = os.path.join(HERE, "app", "miniafqmc.cpp")
DRIVER = os.path.join(HERE, "miniafqmc")
DRIVER_FLAGS = ["-O2", "-std=c++17", "-Wall"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
    "-shared",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    files = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    files.append(os.path.join(HERE, "..", "include", "afqmc_b200.h"))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if force or not up_to_date():
        cmd = [NVCC, *NVCC_FLAGS, *extra, "-I", os.path.join(HERE, "..", "include"),
               *sources(), "-o", LIB]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
    build_driver(force=force, verbose=verbose)
    return LIB


def driver_command(lib_dir: str, out: str) -> list:
    """g++ line of the driver program linked against libafqmc_b200.so in lib_dir."""
    return ["g++", *DRIVER_FLAGS, "-I", os.path.join(HERE, "..", "include"), DRIVER_SRC,
            "-L", lib_dir, "-lafqmc_b200", f"-Wl,-rpath,{lib_dir}", "-o", out]


def build_driver(force: bool = False, verbose: bool = False) -> str:
    """The miniapp's driver program over the C ABI (`miniafqmc_b200/miniafqmc`)."""
    deps = [DRIVER_SRC, LIB, os.path.join(HERE, "..", "include", "afqmc_b200.h")]
    if (not force and os.path.exists(DRIVER)
            and all(os.path.getmtime(f) <= os.path.getmtime(DRIVER) for f in deps)):
        return DRIVER
    cmd = driver_command("$ORIGIN", DRIVER)
    cmd[cmd.index("-L") + 1] = HERE
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    return DRIVER


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
