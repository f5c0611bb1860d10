"""Build the CUDA library of the two-phase substep in-tree.

    python parties-vof-ibm_b200/build.py

Compiles csrc/*.cu for sm_100a into pvof/libpvof.so (nvcc, no JIT cache).
FP64 stencils must round like the reference's C, so FMA contraction is off.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "pvof", "libpvof.so")
SOURCES = ["pvof_api.cu", "pvof_kernels.cu", "pvof_cg.cu", "pvof_cgs.cu", "pvof_ibm.cu", "pvof_fft.cu", "pvof_mcl.cu", "pvof_cnn.cu", "pvof_noalloc.cu", "pvof_spec.cu", "pvof_advect.cu", "pvof_3d.cu"]
HEADERS = ["pvof_internal.cuh", "pvof_device.cuh", "pvof_kernels.cuh", "pvof_particles.cuh", "pvof_3d.cuh", "pvof_3d_api.h",
           os.path.join("..", "..", "include", "pvof.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17", "--extended-lambda",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.abspath(__file__)]
    return all(os.path.getmtime(p) <= t for p in deps)


def build(force=False, verbose=False):
    """Compile every source to an object in parallel (objects under
    _build/, git-ignored), then link the shared library."""
    if not force and up_to_date():
        return OUT
    from concurrent.futures import ThreadPoolExecutor
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]

    def one(src):
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc()] + compile_flags + ["-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(one, SOURCES))
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", OUT] + objs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
