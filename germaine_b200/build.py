"""In-tree build of libgermaine_gpu.so (sm_100a) -- the product library --
and of libgermaine_umfpack.so, the UMFPACK-API shim over it (host C++ only,
csrc/umfpack/).

CUDA sources are compiled by nvcc for ``-gencode arch=compute_100a,code=sm_100a``
with ``-lineinfo``; C++ host sources by nvcc's host compiler; the C host
set-up file (host_setup.c) by gcc without -march, so its float/double
roundings are those of the reference's x86-64 build.  Objects go to
germaine_b200/_build/, the library to germaine_b200/libgermaine_gpu.so.
Incremental: a translation unit is rebuilt when it or any header is newer
than its object.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgermaine_gpu.so")
UMF_LIB = os.path.join(HERE, "libgermaine_umfpack.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _cmd(src: str, obj: str) -> list[str]:
    nvcc = _nvcc()
    if src.endswith(".cu"):
        return [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills",
                "-I", INCLUDE, "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "include")
        return ["g++", "-O3", "-std=c++17", "-fPIC", "-Wall", "-I", INCLUDE, "-I", cuda_inc, "-c", src, "-o", obj]
    if src.endswith(".c"):
        return ["gcc", "-O3", "-std=gnu99", "-fPIC", "-Wall", "-I", INCLUDE, "-c", src, "-o", obj]
    raise ValueError(src)


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")) +
                  glob.glob(os.path.join(CSRC, "*.c")))
    hdrs = glob.glob(os.path.join(CSRC, "*.h*")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    hdr_time = max((os.path.getmtime(h) for h in hdrs), default=0.0)
    jobs_todo = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_time):
            jobs_todo.append((s, o))

    def run(so):
        s, o = so
        cmd = _cmd(s, o)
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for msg in ex.map(run, jobs_todo):
            if verbose and msg.strip():
                print(msg)
    if jobs_todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lm"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    _build_umfpack_shim(hdr_time, verbose)
    return LIB


def _build_umfpack_shim(hdr_time: float, verbose: bool) -> None:
    srcs = sorted(glob.glob(os.path.join(CSRC, "umfpack", "*.cpp")))
    newest = max([hdr_time, os.path.getmtime(LIB)] + [os.path.getmtime(s) for s in srcs])
    if os.path.exists(UMF_LIB) and os.path.getmtime(UMF_LIB) >= newest:
        return
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", "-shared", "-I", INCLUDE, *srcs, "-o", UMF_LIB,
           "-L", HERE, "-lgermaine_gpu", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"shim build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
