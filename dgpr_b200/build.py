"""Builds the in-tree native library dgpr_b200/_lib/libdgb200.so (and the
dgb command-line driver) with nvcc for sm_100a.  No JIT, no torch extension:
the shared object sits in the source tree so it travels with the repository."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "_lib")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr"]
SOURCES = ["host.cpp", "io.cpp", "checkpoint.cpp", "capi.cu", "kernels_fp64.cu", "kernels_fp32.cu",
           "kernels_heat_fp64.cu", "kernels_heat_fp32.cu", "vspace_fp64.cu", "vspace_fp32.cu", "vspace_heat_fp64.cu",
           "vspace_heat_fp32.cu", "vspace_tc.cu", "vspace_visc.cu", "noalloc.cu", "check.cu", "adjoint.cu", "adjoint_heat.cu", "adjoint_gauss.cu",
           "adjoint_gauss_heat.cu", "adjoint_capi.cu", "geometry.cu"]


def _nvcc():
    for c in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), "nvcc"):
        if os.path.sep not in c or os.path.exists(c):
            return c
    return "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def build(verbose=False, jobs=None):
    os.makedirs(LIB, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(LIB, os.path.basename(src) + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(
                os.path.getmtime(src), *[os.path.getmtime(os.path.join(CSRC, h)) for h in os.listdir(CSRC)
                                         if h.endswith((".hpp", ".cuh"))],
                os.path.getmtime(os.path.join(HERE, "..", "include", "dgb200.h"))):
            continue
        cmd = [_nvcc()] + ARCH + FLAGS + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [_nvcc()] + ARCH + FLAGS + ["-x", "cu", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out.decode())
            raise RuntimeError(f"nvcc failed on {src}")
        if verbose and out:
            sys.stdout.write(out.decode())
    so = os.path.join(LIB, "libdgb200.so")
    subprocess.check_call([_nvcc()] + ARCH + ["-shared", "-o", so] + objs + ["-lcudart"])
    main_src = os.path.join(CSRC, "dgb_main.cpp")
    if os.path.exists(main_src):
        exe = os.path.join(LIB, "dgb")
        subprocess.check_call([_nvcc()] + ARCH + FLAGS + ["-x", "cu", main_src, "-o", exe, "-L" + LIB,
                               "-ldgb200", "-Xlinker", "-rpath=$ORIGIN"])
    return so


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
