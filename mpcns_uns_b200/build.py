"""Build recipe of the native libraries, in-tree (the built .so files sit beside the package).

    libmhd_mesh.so   host mesh services (csrc/mesh/*.cpp), g++
    libmhd_gpu.so    sm_100a kernels and the C-ABI of include/mhd_gpu.h (csrc/gpu/*.cu), nvcc

`python -m mpcns_uns_b200.build` builds both.  Compilation is skipped when the output is
newer than every source and header it depends on.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")

MESH_SO = os.path.join(LIBDIR, "libmhd_mesh.so")
GPU_SO = os.path.join(LIBDIR, "libmhd_gpu.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build_mesh(force: bool = False) -> str:
    srcs = sorted(glob.glob(os.path.join(PKG, "csrc", "mesh", "*.cpp")))
    deps = srcs + glob.glob(os.path.join(INCLUDE, "*.h"))
    if force or _stale(MESH_SO, deps):
        os.makedirs(LIBDIR, exist_ok=True)
        # -ffp-contract=off keeps the reference's rounding (no fused multiply-add on the host)
        _run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-Wall", "-Wextra",
              "-I" + INCLUDE, "-o", MESH_SO] + srcs + ["-lpthread"])
    return MESH_SO


def _file_flags(src: str) -> list[str]:
    """Extra nvcc flags a source asks for on a line `// nvcc-flags: ...` in its first 5 lines.

    The FP64 kernels that reproduce the reference's rounding ask for -fmad=false (no contraction
    of a*b+c into a fused multiply-add, so every operation rounds as on the host)."""
    with open(src) as fh:
        for _, line in zip(range(5), fh):
            if line.startswith("// nvcc-flags:"):
                return line.split(":", 1)[1].split()
    return []


def build_gpu(force: bool = False, extra: list[str] | None = None) -> str:
    srcs = sorted(glob.glob(os.path.join(PKG, "csrc", "gpu", "*.cu")))
    heads = glob.glob(os.path.join(PKG, "csrc", "gpu", "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    if force or _stale(GPU_SO, srcs + heads):
        objdir = os.path.join(LIBDIR, "_build")
        os.makedirs(objdir, exist_ok=True)
        base = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                "-I" + INCLUDE] + (extra or [])
        objs = []
        for s in srcs:
            o = os.path.join(objdir, os.path.basename(s) + ".o")
            if force or _stale(o, [s] + heads):
                _run(base + _file_flags(s) + ["-c", s, "-o", o])
            objs.append(o)
        _run([NVCC, *ARCH, "-shared", "-o", GPU_SO, *objs])
    return GPU_SO


DROPIN_SO = os.path.join(LIBDIR, "libmhd_dropin.so")
CUDA_LIB = os.environ.get("CUDA_LIB", "/usr/local/cuda/lib64")


def build_dropin(reference_tree: str, force: bool = False) -> str | None:
    """The drop-in library (csrc/dropin/dropin.cpp): the reference's own hot-path signatures over the C-ABI.
    It compiles against the reference's headers, so it is built only where the reference tree is present
    (the built library travels with the package).  MHD_MPI_INCLUDE names the directory of the mpi.h the
    reference is built with; without it, the single-rank header of the checker build (oracle/ref), which is
    what the reference in this repository is compiled against."""
    if not os.path.isdir(os.path.join(reference_tree, "Common")):
        return None
    src = os.path.join(PKG, "csrc", "dropin", "dropin.cpp")
    gpu = build_gpu(force)
    if force or _stale(DROPIN_SO, [src, gpu] + glob.glob(os.path.join(INCLUDE, "*.h"))):
        mpi_inc = os.environ.get("MHD_MPI_INCLUDE", os.path.join(ROOT, "oracle", "ref"))
        inc = ["-I" + INCLUDE, "-I" + mpi_inc, "-I/usr/local/cuda/include"] + [
            "-I" + os.path.join(reference_tree, d) for d in ("include", "src/uns", "Common", "MercuryUns")]
        _run(["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-Wall", "-Wextra", *inc, "-o", DROPIN_SO, src,
              "-L" + LIBDIR, "-lmhd_gpu", "-L" + CUDA_LIB, "-lcudart", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + CUDA_LIB])
    return DROPIN_SO


def build_all(force: bool = False) -> None:
    build_mesh(force)
    build_gpu(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", MESH_SO, GPU_SO)
