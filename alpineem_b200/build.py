"""Build the B200 solver library and launcher in-tree.

    python -m alpineem_b200.build        (or: python alpineem_b200/build.py)

Outputs, next to this file under _lib/:
    libalpineem_b200.so   C-ABI library (include/alpineem_b200.h)
    FDTD-B200             drop-in solver executable for master.py
Device code is compiled for sm_100a only.  Kernels are built with
-fmad=false so FP32 expressions round as written (no fused multiply-add
contraction), matching the reference's expression-by-expression rounding.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "_lib")
ROOT = os.path.dirname(HERE)

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.path.dirname(os.path.dirname(os.path.realpath(NVCC)))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: FP32 results round like the reference's expressions;
# -ftz=true: subnormals flush to zero, as in the reference's Intel -O3 builds
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-ftz=true", "-Xcompiler", "-fPIC", "-Xptxas", "-v"] + ARCH
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-pthread", "-I" + os.path.join(CUDA_HOME, "include")]

CU = ["aem_kernels.cu", "aem_yee.cu", "aem_yee4.cu", "aem_aux.cu", "aem_ffbin.cu", "aem_coef.cu", "aem_raster.cu", "aem_dft.cu", "aem_dft_static.cu", "aem_solver.cu", "aem_finalize.cu", "aem_design.cu"]
CPP = ["aem_deck.cpp", "aem_model.cpp", "aem_api.cpp"]
HEADERS = [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".h", ".cuh"))] + [
    os.path.join(ROOT, "include", "alpineem_b200.h")]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    jobs = []
    for f in CU:
        src, obj = os.path.join(SRC, f), os.path.join(OBJ, f + ".o")
        if _stale(obj, [src] + HEADERS):
            jobs.append([NVCC] + NVFLAGS + ["-c", src, "-o", obj])
    for f in CPP:
        src, obj = os.path.join(SRC, f), os.path.join(OBJ, f + ".o")
        if _stale(obj, [src] + HEADERS):
            jobs.append(["g++"] + CXXFLAGS + ["-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        logs = list(ex.map(_run, jobs))
    if verbose:
        for l in logs:
            sys.stdout.write(l)
    objs = [os.path.join(OBJ, f + ".o") for f in CU + CPP]
    so = os.path.join(LIB, "libalpineem_b200.so")
    if _stale(so, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", so] + objs + ["-lcudart", "-Xcompiler", "-pthread"])
    exe = os.path.join(LIB, "FDTD-B200")
    main = os.path.join(SRC, "fdtd_b200_main.cpp")
    if _stale(exe, [main, so]):
        _run(["g++", "-std=c++17", "-O2", main, "-o", exe, "-L" + LIB, "-lalpineem_b200", "-Wl,-rpath,$ORIGIN"])
    kexe = os.path.join(LIB, "FDTD-B200-kmax")
    if not os.path.exists(kexe):
        os.symlink("FDTD-B200", kexe)
    return so


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
