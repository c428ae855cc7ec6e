"""Build the sm_100a solver library ``liblattice_lbm.so`` in-tree.

Every .cu (and host-only .cpp) file under csrc/ is compiled by nvcc for sm_100a
(``-gencode arch=compute_100a,code=sm_100a``) with ``--fmad=false`` and the
default IEEE division / square root, so that single-precision arithmetic
rounds exactly as the C oracle (built with -ffp-contract=off) does; the
objects are then linked into one shared library exporting the C ABI of
include/lattice_lbm.h.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblattice_lbm.so")
TUNNEL = os.path.join(HERE, "lattice_tunnel")
TUNNEL_SRC = os.path.join(HERE, "driver", "lattice_tunnel.c")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-prec-div=true",
         "-prec-sqrt=true", "-ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
         "-I" + os.path.join(HERE, "..", "include")]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cpp")))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
          if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(HERE, "..", "include", "lattice_lbm.h"))
    return max(os.path.getmtime(h) for h in hs)


# the fast-arithmetic translation units (lbm_step_fast_*.cu) contract FMAs
# and use approximate division / square root
FAST_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=true", "-prec-div=false",
              "-prec-sqrt=false", "-ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-I" + os.path.join(HERE, "..", "include")]


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if (os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
            and os.path.getmtime(obj) >= _headers_mtime()):
        return obj
    flags = FAST_FLAGS if os.path.basename(src).startswith("lbm_step_fast") else FLAGS
    cmd = [NVCC, *ARCH, *flags, "-c", src, "-o", obj]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        with open(obj + ".ptxas.txt", "w") as fh:
            fh.write(r.stderr)
    return obj


def build(verbose_ptxas: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if (not os.path.exists(TUNNEL) or os.path.getmtime(TUNNEL) < os.path.getmtime(LIB)
            or os.path.getmtime(TUNNEL) < os.path.getmtime(TUNNEL_SRC)):
        # the headless driver executable, linked against the library beside it
        cmd = ["gcc", "-O2", "-std=gnu11", "-Wall", "-I" + os.path.join(HERE, "..", "include"),
               "-o", TUNNEL, TUNNEL_SRC, "-L" + HERE, "-llattice_lbm",
               "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
