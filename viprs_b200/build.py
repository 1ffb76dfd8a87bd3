"""Build the sm_100a library in-tree: viprs_b200/_lib/libviprs_b200.so.

nvcc compiles the device translation units for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with --fmad=false, so that a
multiply and an add are fused only where the source calls fma(); the host
planning code is compiled with -ffp-contract=off for the same reason.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libviprs_b200.so")
OBJ_DIR = os.path.join(ROOT, "_build", "obj")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

CU_SOURCES = ["resample.cu", "affine.cu", "affine_u8.cu", "affine_u16.cu", "affine_f32.cu", "adjoint.cu", "batch.cu",
              "noalloc.cu"]
CPP_SOURCES = ["plan.cpp", "affine_plan.cpp", "capi.cpp", "batch_plan.cpp", "adjoint_plan.cpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources_present():
    cu = [s for s in CU_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    cpp = [s for s in CPP_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    return cu, cpp


def _deps(obj):
    """Files the compiler recorded as inputs of `obj` (its -MD file), or None."""
    path = obj + ".d"
    if not os.path.exists(path):
        return None
    with open(path) as f:
        text = f.read().replace("\\\n", " ")
    _, _, rest = text.partition(":")
    return [d for d in rest.split() if d]


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    deps = _deps(obj)
    if deps is None:
        return True
    t = os.path.getmtime(obj)
    return any(not os.path.exists(d) or os.path.getmtime(d) > t for d in [src] + deps)


def build(force=False, verbose=False, jobs=8):
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    cu, cpp = _sources_present()
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    cmds = []
    objs = []
    for s in cu:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ_DIR, s + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            cmds.append([NVCC, *ARCH, "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
                         "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", *inc,
                         "-MD", "-MF", obj + ".d", "-c", src, "-o", obj])
    for s in cpp:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ_DIR, s + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            cmds.append(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                         "-Wall", "-Wno-unused-function", *inc, "-I", os.path.join(CUDA_HOME, "include"),
                         "-MD", "-MF", obj + ".d", "-c", src, "-o", obj])
    procs = []
    for c in cmds:
        if verbose:
            print(" ".join(c))
        procs.append(subprocess.Popen(c))
        if len(procs) >= jobs:
            _wait(procs)
            procs = []
    _wait(procs)
    if force or cmds or not os.path.exists(LIB):
        link = [NVCC, *ARCH, "-shared", "-cudart", "shared", "-o", LIB, *objs,
                "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")]
        if verbose:
            print(" ".join(link))
        subprocess.check_call(link)
    return LIB


def _wait(procs):
    bad = [p.args for p in procs if p.wait() != 0]
    if bad:
        raise RuntimeError("compile failed: " + " ".join(bad[0]))


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
