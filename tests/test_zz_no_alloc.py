"""div B through the entry point that allocates nothing, against the regular one.

mhd_gpu_div_b_noalloc serves callers that must not allocate device memory once they run: a host
application that gives all GPU memory to its own pool at start-up, or a process under a fixed
memory budget.  Its scratch is a static device array of the library.  It is called twice in a row
through the C-ABI, on different fields, and must give what mhd_gpu_div_b gives on each (1e-12
relative, the tolerance of the other parity tests; the worst cell exactly), without a single
cudaMalloc or cudaFree (the library's allocation counter stays put).  The mesh is the 6 x 32 x 32 x
48 x 6 shell (1,769,472 owned cells, 1,728 block partials), so the final reduction folds more
partials than it has threads.  The file name makes pytest collect it after every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _alloc_calls(L):
    n = ctypes.c_int64(-1)
    assert L.mhd_gpu_alloc_calls(ctypes.byref(n)) == 0
    return n.value


def test_div_b_noalloc_matches_div_b_twice():
    from mpcns_uns_b200 import gpu, workloads
    from mpcns_uns_b200.mesh import HostMesh
    L = gpu.lib()
    f = L.mhd_gpu_div_b_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    L.mhd_gpu_alloc_calls.argtypes = [ctypes.c_void_p]
    L.mhd_gpu_alloc_calls.restype = ctypes.c_int
    h = HostMesh.shell(32, 48, 1.0, 6.0, 1.05, tets=True).compute_geometry(device=True)
    h.boundary("outflow", {"inner": "wall", "outer": "farfield"}, (-8.0, 0.0, 0.0))
    assert h.n_cells == 1769472 and (h.n_cells + 1023) // 1024 > 1024
    dm = gpu.DeviceMesh(h)
    rng = np.random.default_rng(31)
    fields = [rng.uniform(-1, 1, h.n_faces),                                        # arbitrary flux
              workloads.d1(h, rng.uniform(-1, 1, h.n_edges)) + 1e-9 * rng.uniform(-1, 1, h.n_faces)]
    extra = rng.uniform(-1, 1, h.n_faces)
    inputs = [(gpu.dev(B), None if ex is None else gpu.dev(ex)) for B in fields for ex in (None, extra)]
    import torch
    torch.cuda.synchronize()
    outs = []
    before = _alloc_calls(L)
    for Bd, exd in inputs:
        out = np.zeros(3)
        dm._enter()
        rc = f(dm.handle, gpu.ptr(Bd), gpu.ptr(exd), out.ctypes.data_as(ctypes.c_void_p))
        assert rc == 0, L.mhd_gpu_last_error().decode()
        outs.append(out)
    assert _alloc_calls(L) == before, "mhd_gpu_div_b_noalloc allocated device memory"
    for k, ((Bd, exd), out) in enumerate(zip(inputs, outs)):
        ref = dm.div_b(Bd, exd)
        assert abs(out[0] - ref["max_abs"]) <= TOL * ref["max_abs"], (k, out, ref)
        assert abs(out[1] - ref["max_rel"]) <= TOL * ref["max_rel"], (k, out, ref)
        assert int(out[2]) == ref["worst_cell"], (k, out, ref)
    assert _alloc_calls(L) > before, "the allocation counter does not see the regular entry point's scratch"
