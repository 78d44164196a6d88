"""div B through the entry point that allocates nothing, against the regular one.

mhd_gpu_div_b_noalloc serves callers that cannot call cudaMalloc (inside a stream capture, under
a memory pool or budget that forbids it): its scratch is a static device array of the library.
It is called twice in a row through the C-ABI, on different fields, and must give what
mhd_gpu_div_b gives on each (1e-12 relative, the tolerance of the other parity tests; the worst
cell exactly).  The file name makes pytest collect it after every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12


def test_div_b_noalloc_matches_div_b_twice():
    from mpcns_uns_b200 import gpu, workloads
    from mpcns_uns_b200.mesh import HostMesh
    L = gpu.lib()
    f = L.mhd_gpu_div_b_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    h = HostMesh.box(12, 12, 12, tets=True, jitter=0.15, seed=2).compute_geometry().boundary("outflow")
    dm = gpu.DeviceMesh(h)
    rng = np.random.default_rng(31)
    fields = [rng.uniform(-1, 1, h.n_faces),                                        # arbitrary flux
              workloads.d1(h, rng.uniform(-1, 1, h.n_edges)) + 1e-9 * rng.uniform(-1, 1, h.n_faces)]
    extra = rng.uniform(-1, 1, h.n_faces)
    for k, B in enumerate(fields):
        for ex in (None, extra):
            Bd = gpu.dev(B)
            exd = None if ex is None else gpu.dev(ex)
            out = np.zeros(3)
            dm._enter()
            rc = f(dm.handle, gpu.ptr(Bd), gpu.ptr(exd), out.ctypes.data_as(ctypes.c_void_p))
            assert rc == 0, L.mhd_gpu_last_error().decode()
            ref = dm.div_b(Bd, exd)
            assert abs(out[0] - ref["max_abs"]) <= TOL * ref["max_abs"], (k, out, ref)
            assert abs(out[1] - ref["max_rel"]) <= TOL * ref["max_rel"], (k, out, ref)
            assert int(out[2]) == ref["worst_cell_gid"], (k, out, ref)
