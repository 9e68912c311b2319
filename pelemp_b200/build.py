"""Build the native pieces in-tree.

* pelemp_b200/libpmpspray.so -- the product: C ABI + sm_100a kernels
  (nvcc -gencode arch=compute_100a,code=sm_100a).
* oracle/ (test infrastructure) -- `make -C oracle` builds the CPU oracle and,
  when the PeleMP sources are present, the reference build under oracle/_ref.

Usage: python -m pelemp_b200.build [--force] [--verbose-ptxas] [--define NAME=VALUE ...]
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libpmpspray.so")
# (source, contraction flag): the FP64 kernels reproduce the oracle's
# arithmetic exactly, so their units are compiled without multiply-add
# contraction (their multiply-adds are explicit fma() calls); the mixed and
# learned forms allow it.
SOURCES = [("pmp_spray.cu", "-fmad=false"), ("pmp_static.cu", "-fmad=false"),
           ("pmp_mixed.cu", "-fmad=true"), ("pmp_learn.cu", "-fmad=true"),
           ("pmp_batch.cu", "-fmad=false"), ("batch/pmp_batch_b64.cu", "-fmad=false"),
           ("batch/pmp_batch_b128.cu", "-fmad=false"), ("batch/pmp_batch_b256.cu", "-fmad=false"),
           ("pmp_mesh.cu", "-fmad=false"), ("pmp_peaks.cu", "-fmad=true")]
def _headers():
    """Every header under csrc/ (a change to any of them rebuilds the library)."""
    out = []
    for d, _, files in os.walk(CSRC):
        for f in files:
            if f.endswith((".h", ".cuh", ".H")):
                out.append(os.path.relpath(os.path.join(d, f), CSRC))
    return sorted(out)


HEADERS = _headers()
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
OBJDIR = os.path.join(ROOT, "_build")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


STAMP = LIB + ".flags"  # the extra flags the library was last built with


def build_lib(force=False, ptxas_verbose=False, extra=()):
    deps = [os.path.join(CSRC, s) for s, _ in SOURCES] + [os.path.join(CSRC, h) for h in HEADERS]
    deps.append(os.path.join(ROOT, "include", "pmp_spray.h"))
    deps.append(os.path.abspath(__file__))
    flags = " ".join(extra)
    built_with = open(STAMP).read() if os.path.exists(STAMP) else ""
    if not (force or ptxas_verbose or flags != built_with or _newer(LIB, deps)):
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    procs = []
    objs = []
    for src, fmad in SOURCES:
        obj = os.path.join(OBJDIR, src.replace("/", "_").replace(".cu", ".o"))
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", fmad, "-Xcompiler", "-fPIC",
               "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
               *extra, "-c", "-o", obj, os.path.join(CSRC, src)]
        if ptxas_verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    for p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, "nvcc")
    subprocess.run([NVCC, *ARCH, "-shared", "-o", LIB + ".tmp", *objs], check=True)
    os.replace(LIB + ".tmp", LIB)
    with open(STAMP, "w") as f:
        f.write(flags)
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


# The reference's spray sources, for the reference build under oracle/_ref
# (test infrastructure): PMP_REFERENCE_SRC, else the read-only checkout this
# build recipe compiles them from when it is present.
REFERENCE_SRC = os.environ.get("PMP_REFERENCE_SRC", "/root/reference/Source/PP_Spray")


def build_oracle():
    cmd = ["make", "-s", "-C", os.path.join(ROOT, "oracle")]
    if os.path.exists(os.path.join(REFERENCE_SRC, "Drag.H")):
        cmd.append("REF_DIR=" + REFERENCE_SRC)
    subprocess.run(cmd, check=True)


def main(argv):
    # --define NAME=VALUE (repeatable): a build option of the kernels, e.g.
    # PMP_GATHER_TILE=1, PMP_WARP_AGG_DEPOSITS=1, PMP_FP64_MIN_BLOCKS=4
    defines = ["-D" + argv[i + 1] for i, a in enumerate(argv) if a == "--define" and i + 1 < len(argv)]
    build_lib(force="--force" in argv or bool(defines), ptxas_verbose="--verbose-ptxas" in argv,
              extra=defines)
    build_driver(force="--force" in argv)
    if "--no-oracle" not in argv:
        build_oracle()


if __name__ == "__main__":
    main(sys.argv[1:])
