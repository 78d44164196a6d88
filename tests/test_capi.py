"""The C-ABI libraries load and export every function their headers declare (CPU, no compute calls)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mhd_gpu_\w+|mhdm_\w+)\s*\(", src)))


def test_gpu_library_exports_header():
    from mpcns_uns_b200 import build
    L = ctypes.CDLL(build.build_gpu())
    names = declared("mhd_gpu.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_mesh_library_exports_header():
    from mpcns_uns_b200 import build
    L = ctypes.CDLL(build.build_mesh())
    names = declared("mhd_mesh.h")
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_codes_without_device():
    """Argument errors are reported as status codes with a message, without touching a device."""
    from mpcns_uns_b200 import build
    L = ctypes.CDLL(build.build_gpu())
    L.mhd_gpu_mesh_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.mhd_gpu_last_error.restype = ctypes.c_char_p
    assert L.mhd_gpu_mesh_create(None, None) == -1
    assert b"null" in L.mhd_gpu_last_error()
