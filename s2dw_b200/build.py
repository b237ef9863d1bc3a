"""Builds libs2dw_cuda.so in-tree with nvcc for sm_100a.

Usage: python -m s2dw_b200.build [--verbose]
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libs2dw_cuda.so")
SOURCES = ["s2dw_host.cpp", "s2dw_kernels.cu", "s2dw_plan.cu", "s2dw_noalloc.cu", "s2dw_split.cu", "s2dw_stats.cu",
           "s2dw_fileio.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _host_cxx():
    # The system g++ carries libgomp; use it as nvcc's host compiler.
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def build(verbose=False, force=False):
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, "s2dw_internal.h"),
                   os.path.join(HERE, "..", "include", "s2dw_cuda.h")]
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= t for d in deps):
            return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc, cxx = _nvcc(), _host_cxx()
    common = ["-O3", "-std=c++17", "-lineinfo", "-ccbin", cxx,
              "-Xcompiler", "-fPIC,-fopenmp,-O3", "-I", os.path.join(HERE, "..", "include")]
    def compile_one(s):
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = [nvcc, "-c", s, "-o", o] + common + ARCH
        if s.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        return o, cmd, subprocess.run(cmd, capture_output=True, text=True)

    # the translation units are independent: compile them concurrently
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, srcs))
    objs = []
    for s, (o, cmd, r) in zip(srcs, results):
        if verbose:
            print(" ".join(cmd), flush=True)
        if verbose or r.returncode:
            sys.stdout.write(r.stdout)
            sys.stderr.write(r.stderr)
        if r.returncode:
            raise RuntimeError(f"nvcc failed on {s}")
        objs.append(o)
    cmd = [nvcc, "-shared", "-o", OUT] + objs + ["-ccbin", cxx, "-Xcompiler", "-fopenmp",
                                                 "-lgomp", "-lcudart"] + ARCH
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return OUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
