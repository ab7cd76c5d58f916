"""Builds libfilsim_gpu.so in-tree (filsim_b200/_lib/) with nvcc for sm_100a.

Usage: python -m filsim_b200.build [--verbose-ptxas]
"""
import concurrent.futures
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "_lib")
OUT = os.path.join(LIBDIR, "libfilsim_gpu.so")
SOURCES = ["fs_sort.cu", "fs_fcm.cu", "fs_cells.cu", "fs_filament.cu", "fs_capi.cu", "fs_suspension.cu",
           "fs_noalloc.cu", "fs_fft.cu", "fs_mlp.cu", "fs_graph.cu", "fs_tune.cu", "fs_runfiles.cu", "fs_slab.cu",
           "fs_start.cu", "fs_bmem.cu"]
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose_ptxas=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith(".cuh")]
    headers.append(os.path.join(ROOT, "include", "filsim_gpu.h"))
    objs = []
    jobs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s.replace(".cu", ".o"))
        objs.append(obj)
        if force or verbose_ptxas or _newer(obj, [src] + headers):
            cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else []) + ["-c", src, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    failed = False
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        for cmd, r in ex.map(run, jobs):
            if r.returncode != 0 or verbose_ptxas:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                failed = True
                sys.stderr.write("FAILED: %s\n" % " ".join(cmd))
    if failed:
        raise RuntimeError("nvcc compilation failed")
    if force or jobs or _newer(OUT, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + [
            "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcufft",
            "-Xlinker", "-rpath=" + os.path.join(CUDA_HOME, "lib64")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return OUT


if __name__ == "__main__":
    build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv)
    print(OUT)
