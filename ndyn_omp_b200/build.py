"""Build the sm_100a shared library and the C++ driver in-tree.

    python -m ndyn_omp_b200.build          # -> ndyn_omp_b200/lib/libndyn_gpu.so
                                            #    ndyn_omp_b200/bin/ndyn_gpu

Every CUDA source is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with --fmad=false: the FP64 path
restates the reference's arithmetic operation by operation, and the mixed
kernel requests its FMAs explicitly.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
BINDIR = os.path.join(HERE, "bin")
BUILDDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libndyn_gpu.so")
EXE = os.path.join(BINDIR, "ndyn_gpu")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-ffp-contract=off", "-ccbin", "/usr/bin/g++",
         "-I" + os.path.join(ROOT, "include")]

LIB_SOURCES = ["ndg_kernels.cu", "ndg_context.cu", "ndg_tables.cpp", "ndg_server.cpp",
               "ndg_static.cu"]
EXE_SOURCES = ["ndyn_main.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build failed: " + os.path.basename(cmd[-1]))
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False, force=False):
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BINDIR, exist_ok=True)
    os.makedirs(BUILDDIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    headers.append(os.path.join(ROOT, "include", "ndyn_gpu.h"))
    objs = []
    for src in LIB_SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILDDIR, src + ".o")
        if force or _stale(obj, [path] + headers):
            cmd = [NVCC] + ARCH + FLAGS + ["-Xptxas", "-v"] * verbose + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    exe_src = [os.path.join(CSRC, s) for s in EXE_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if exe_src and (force or _stale(EXE, exe_src + headers + [LIB])):
        _run([NVCC] + ARCH + FLAGS + exe_src + ["-o", EXE, "-L" + LIBDIR, "-lndyn_gpu",
                                                 "-Xlinker", "-rpath=$ORIGIN/../lib"])
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
