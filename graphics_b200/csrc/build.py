"""Build libsphgpu.so (sm_100a) in-tree.

nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo, one object per
.cu file, linked into graphics_b200/libsphgpu.so next to the package so the
library travels with the source tree.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
OUT = os.path.join(PKG, "libsphgpu.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + os.path.join(PKG, "..", "include")]
SOURCES = ["sph_grid.cu", "sph_dfsph.cu", "sph_wcsph.cu", "sph_pci_ii.cu", "sph_iisph.cu", "sph_batch.cu", "sph_mlp.cu", "sph_engine.cu", "sph_noalloc.cu",
           "sph_rigid.cu", "sph_surface.cu", "sph_vortex.cu"]


def _newer(dst, srcs):
    return os.path.exists(dst) and all(os.path.getmtime(dst) >= os.path.getmtime(s) for s in srcs)


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(PKG, "..", "include", "sphgpu.h"))
    objs, jobs = [], []
    for src in SOURCES:
        s = os.path.join(HERE, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if not _newer(o, [s] + headers):
            jobs.append([NVCC] + ARCH + FLAGS + ["-c", s, "-o", o])

    def run(cmd):
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        for cmd, r in ex.map(run, jobs):
            if r.returncode:
                sys.stderr.write(r.stderr)
                raise RuntimeError("nvcc failed: " + cmd[-3])
    if not _newer(OUT, objs):
        cmd = [NVCC] + ARCH + ["-shared", "--cudart", "static", "-o", OUT] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stderr)
            raise RuntimeError("link failed")
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
