"""Build the CUDA library libcup2d.so in-tree for sm_100a.

    python -m cubismup_2d_b200.build [--force] [--trace]

Every translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a`` and, except the FFT-based
Poisson solvers, ``-fmad=false``: the reference's arithmetic is reproduced
operation by operation, and fused multiply-adds would change the rounding of
every stencil.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcup2d.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["context.cu", "fluid.cu", "obstacles.cu", "fish.cu", "poisson.cu", "noalloc.cu", "varrho.cu",
           "adjoint.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-fmad=false", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "--expt-relaxed-constexpr"]


def flags_for(src):
    """poisson.cu contracts multiply-adds: its FFTs need not follow the
    reference's (FFTW's) rounding, and the one value compared exactly, the
    faded RHS, is written with explicit round-to-nearest intrinsics."""
    if src == "poisson.cu":
        return [f if f != "-fmad=false" else "-fmad=true" for f in FLAGS]
    return FLAGS


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


TRACE_LIB = os.path.join(HERE, "libcup2d_trace.so")


def build(force=False, verbose=False, trace=False):
    """Build libcup2d.so, or with trace=True the timeline build
    libcup2d_trace.so (-DCUP2D_TRACE: every kernel stamps %globaltimer at
    entry and exit; read back by cubismup_2d_b200.timeline)."""
    build_dir = os.path.join(BUILD, "trace") if trace else BUILD
    lib = TRACE_LIB if trace else LIB
    extra = ["-DCUP2D_TRACE"] if trace else []
    os.makedirs(build_dir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp"))]
    headers.append(os.path.join(INCLUDE, "cup2d.h"))
    jobs = []
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(build_dir, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s] + headers):
            jobs.append([NVCC] + flags_for(src) + extra + ["-c", s, "-o", o])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr)

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        list(ex.map(run, jobs))
    if force or jobs or _newer(lib, objs):
        run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", lib] + objs + ["-lcudart"])
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, trace="--trace" in sys.argv))
