"""Build libspring_b200.so in-tree for sm_100a (nvcc, no JIT cache).

``python -m spring_b200.build`` compiles every ``csrc/*.cu`` to an object in
``spring_b200/_build`` (parallel, skipping up-to-date objects) and links
``spring_b200/libspring_b200.so``.
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
LIB = os.path.join(HERE, "libspring_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h")) +
            glob.glob(os.path.join(os.path.dirname(CSRC), "host", "*.hpp")))


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + _deps())


# Per-file flags: the point-defect vertex weights cancel catastrophically for near-degenerate
# tetrahedra (as the reference's do), so they are evaluated without contracting a*b + c into one
# rounding, like the host FP64 they are compared with.
FILE_FLAGS = {"k_pdef.cu": ["-fmad=false"]}


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if _stale(obj, src):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *FILE_FLAGS.get(os.path.basename(src), []), "-c", src, "-o", obj]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if verbose_ptxas or "spill" in r.stderr.lower() and "0 bytes spill" not in r.stderr:
            sys.stderr.write(r.stderr)
    return obj


HOST = os.path.join(HERE, "host")
HOST_LIB = os.path.join(HERE, "libspring_host.so")
CLI = os.path.join(HERE, "spring_kappa")
CXX_FLAGS = ["-O2", "-std=c++17", "-Wall"]


def _cxx() -> str:
    for cand in (os.environ.get("CXX"), shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def build_host() -> str:
    """libspring_host.so (the FC / result file formats, no CUDA) and the spring_kappa driver, which
    links libspring_b200.so and libspring_host.so from its own directory."""
    hsrc = [os.path.join(HOST, f) for f in ("h5lite.cpp", "namelist.cpp", "host_api.cpp")]
    deps = hsrc + glob.glob(os.path.join(HOST, "*.hpp")) + [os.path.join(INCLUDE, "spring_host.h")]
    if not os.path.exists(HOST_LIB) or any(os.path.getmtime(d) > os.path.getmtime(HOST_LIB) for d in deps):
        r = subprocess.run([_cxx(), *CXX_FLAGS, "-fPIC", "-shared", *hsrc, "-o", HOST_LIB], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"host library build failed:\n{r.stdout}\n{r.stderr}")
    cli_src = [os.path.join(HOST, "spring_kappa.cpp"), os.path.join(HOST, "namelist.cpp")]
    cdeps = cli_src + [HOST_LIB, LIB, os.path.join(INCLUDE, "spring_gpu.h")]
    if not os.path.exists(CLI) or any(os.path.getmtime(d) > os.path.getmtime(CLI) for d in cdeps):
        r = subprocess.run([_cxx(), *CXX_FLAGS, *cli_src, "-L" + HERE, "-lspring_host", "-lspring_b200",
                            "-Wl,-rpath,$ORIGIN", "-o", CLI], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"spring_kappa build failed:\n{r.stdout}\n{r.stderr}")
    return CLI


def build(verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        tmp = LIB + ".tmp"
        r = subprocess.run([nvcc(), *ARCH, "-shared", "-o", tmp, *objs], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    build_host()
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
