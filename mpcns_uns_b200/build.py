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


def build_all(force: bool = False) -> None:
    build_mesh(force)
    build_gpu(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", MESH_SO, GPU_SO)
