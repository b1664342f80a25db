"""Build libharmgpu.so in-tree for sm_100a.

nvcc flags: -gencode arch=compute_100a,code=sm_100a, -O3, -lineinfo, and
-fmad=false: no multiply-add is fused, so every FP64 operation is rounded
exactly as in the reference's gcc build and results agree bit for bit.
The step kernels (hg_kernels.cu) are compiled a second time with
-fmad=true -DHG_FMA_BUILD into namespace hg_fma: the HG_PREC_FP64_FMA form,
FP64 with fused multiply-adds (fewer instructions, not bit-identical).
The FP32 kernels of the mixed-precision form (hg_mixed.cu) are not held to
bit parity: they are built with fused multiply-adds, approximate FP32
division and square root and flush-to-zero (FP32_FLAGS), which measured
10% faster with the same accuracy against the FP64 form.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libharmgpu.so")
SOURCES = ["hg_kernels.cu", "hg_api.cu", "hg_geometry.cu", "hg_mixed.cu", "hg_peak.cu"]
# (object name, source, extra flags): the step kernels once more with fused
# multiply-adds, into namespace hg_fma (HG_PREC_FP64_FMA)
EXTRA_OBJECTS = [("hg_kernels_fma.o", "hg_kernels.cu", ["-fmad=true", "-DHG_FMA_BUILD"])]
# FP32 kernels of the mixed-precision form may contract multiply-adds
FMA_SOURCES = {"hg_mixed.cu"}
FP32_FLAGS = ["-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
HEADERS = ["hg_internal.h", "hg_phys.cuh", "hg_fallback.cuh", "hg_common.cuh", "hg_crpow.h", "hg_pow_tables.h"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def flags():
    return ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
            "-Xcompiler", "-fPIC", "-I", os.path.join(REPO, "include"), "-I", CSRC]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(REPO, "include", "harmgpu.h"), __file__]
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force=False, verbose=False, out=None, defines=()):
    lib = out or LIB
    if not force and out is None and up_to_date():
        return LIB
    objs = []
    procs = []
    units = [(s.replace(".cu", ".o"), s, FP32_FLAGS if s in FMA_SOURCES else []) for s in SOURCES] + EXTRA_OBJECTS
    for oname, s, extra in units:
        o = os.path.join(CSRC, oname)
        fl = flags()
        if "-fmad=true" in extra:
            fl = [f for f in fl if f != "-fmad=false"]
        fl = fl + extra
        cmd = [nvcc()] + fl + ["-D" + d for d in defines] + ["-c", os.path.join(CSRC, s), "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((subprocess.Popen(cmd), s))
        objs.append(o)
    for p, s in procs:
        if p.wait() != 0:
            raise RuntimeError("nvcc failed on " + s)
    tmp = lib + ".tmp"
    subprocess.check_call([nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs)
    os.replace(tmp, lib)
    for o in objs:
        os.remove(o)
    return lib


if __name__ == "__main__":
    print(build(force="-f" in sys.argv, verbose="-v" in sys.argv))
