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


def test_noalloc_div_b_size_guard_without_device():
    """The no-allocation div B accepts up to MHD_NOALLOC_DIVB_MAX_BLOCKS x 1024 owned cells and rejects
    one more with MHD_EINVAL and a message (host arithmetic, no device work); the allocation counter
    reads without a device."""
    from mpcns_uns_b200 import build
    L = ctypes.CDLL(build.build_gpu())
    L.mhd_gpu_div_b_noalloc_blocks.argtypes = [ctypes.c_int64, ctypes.c_void_p]
    L.mhd_gpu_alloc_calls.argtypes = [ctypes.c_void_p]
    L.mhd_gpu_last_error.restype = ctypes.c_char_p
    src = open(os.path.join(ROOT, "include", "mhd_gpu.h")).read()
    max_blocks = int(re.search(r"#define MHD_NOALLOC_DIVB_MAX_BLOCKS (\d+)", src).group(1))
    nb = ctypes.c_int64(-1)
    for cells, blocks in ((0, 0), (1, 1), (1024, 1), (1025, 2), (1769472, 1728), (max_blocks * 1024, max_blocks)):
        assert L.mhd_gpu_div_b_noalloc_blocks(cells, ctypes.byref(nb)) == 0
        assert nb.value == blocks, (cells, nb.value)
    nb.value = -7
    assert L.mhd_gpu_div_b_noalloc_blocks(max_blocks * 1024 + 1, ctypes.byref(nb)) == -1
    assert nb.value == -7
    assert b"at most 67108864 owned cells" in L.mhd_gpu_last_error()
    assert L.mhd_gpu_div_b_noalloc_blocks(-1, ctypes.byref(nb)) == -1
    n = ctypes.c_int64(-1)
    assert L.mhd_gpu_alloc_calls(ctypes.byref(n)) == 0 and n.value >= 0
