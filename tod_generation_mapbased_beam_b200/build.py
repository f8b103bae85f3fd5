"""Build libtodgpu.so (the C-ABI library with the sm_100a kernels) in-tree.

    python -m tod_generation_mapbased_beam_b200.build [--verbose]

nvcc cross-compiles for B200 without a GPU present.  The library lands in
``tod_generation_mapbased_beam_b200/_lib/libtodgpu.so``; the C-ABI header is
``include/todgpu.h`` at the repository root.

Flags: ``-gencode arch=compute_100a,code=sm_100a`` (B200 only), ``-lineinfo``
for profiling, ``-fmad=false`` so that no multiply-add is contracted (the
pixel decisions reproduce the reference's uncontracted float arithmetic;
kernels that want fused multiply-adds call fma() explicitly), and the CUDA
runtime linked statically so the library has no runtime-version coupling with
the host process.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(OUT_DIR, "libtodgpu.so")

# One translation unit per map element type (they instantiate the gather
# kernels and compile in parallel) plus the C ABI.
SOURCES = ["tod_api.cu", "gather_map_f64.cu", "gather_map_f32.cu", "gather_map_pf32.cu",
           "gather_map_pbf16.cu", "gather_map_pf64.cu", "sky_synth.cu", "tail_mlp.cu", "kmeans.cu"]
HEADERS = ["healpix_ring.cuh", "gather_impl.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2",
              "-cudart", "static", "--expt-relaxed-constexpr"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found (set NVCC or put /usr/local/cuda/bin on PATH)")


def _inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    files.append(os.path.join(INCLUDE, "todgpu.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    nvcc = nvcc_path()
    objs, procs = [], []
    for src in SOURCES:
        obj = os.path.join(OUT_DIR, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [src for src, proc in procs if proc.wait() != 0]
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs, "-lpthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    path = build(force=True, verbose="--verbose" in sys.argv)
    print(path)
