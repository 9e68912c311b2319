"""Build the native pieces in-tree.

* pelemp_b200/libpmpspray.so -- the product: C ABI + sm_100a kernels
  (nvcc -gencode arch=compute_100a,code=sm_100a).
* oracle/ (test infrastructure) -- `make -C oracle` builds the CPU oracle and,
  when the PeleMP sources are present, the reference build under oracle/_ref.

Usage: python -m pelemp_b200.build [--verbose-ptxas]
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libpmpspray.so")
SOURCES = ["pmp_spray.cu", "pmp_static.cu"]
HEADERS = ["pmp_device.cuh", "spray_fp64.cuh", "phys/pmp_math.h", "phys/pmp_math_tables.h", "phys/pmp_thermo.h",
           "phys/pmp_thermo_data.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force=False, ptxas_verbose=False):
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "pmp_spray.h"))
    deps.append(os.path.abspath(__file__))
    if not (force or ptxas_verbose or _newer(LIB, deps)):
        return LIB
    # -fmad=false: the FP64 kernel reproduces the oracle's arithmetic exactly
    # (its multiply-adds are explicit fma() calls)
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
           "-shared",
           "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           "-o", LIB + ".tmp"] + [os.path.join(CSRC, s) for s in SOURCES]
    if ptxas_verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


DRIVER = os.path.join(PKG, "pmp_spray_driver")


def build_driver(force=False):
    """The C++ host driver over the C ABI (links libpmpspray.so)."""
    src = os.path.join(CSRC, "host", "spray_driver.cpp")
    deps = [src, os.path.join(CSRC, "host", "SprayParticleContainer.H"),
            os.path.join(ROOT, "include", "pmp_spray.h"), LIB]
    if not (force or _newer(DRIVER, deps)):
        return DRIVER
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(CSRC, "host"), "-o", DRIVER + ".tmp", src,
                    "-L", PKG, "-lpmpspray", "-Wl,-rpath,$ORIGIN"], check=True)
    os.replace(DRIVER + ".tmp", DRIVER)
    return DRIVER


def build_oracle():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def main(argv):
    build_lib(force="--force" in argv, ptxas_verbose="--verbose-ptxas" in argv)
    build_driver(force="--force" in argv)
    if "--no-oracle" not in argv:
        build_oracle()


if __name__ == "__main__":
    main(sys.argv[1:])
