"""uns::compute_geometry on the device (mhd_gpu_compute_geometry) against the host computation, which
keeps the reference's operation order: every array bit for bit, on tetrahedral, hexahedral, solid-cored
and hanging-node meshes."""
import numpy as np
import pytest

from helpers import BOX_TAGS, host_from_ref
from mpcns_uns_b200.mesh import HostMesh

pytestmark = pytest.mark.gpu

NAMES = ("edge_vec", "edge_mid", "edge_len", "face_area", "face_center", "face_area_mag", "cell_center", "cell_volume",
         "cell_min_tet_volume", "edge_dual_area", "ec_ptr", "ec_cell", "ec_weight", "ef_weight", "ec_misoriented", "star0", "star1",
         "star2", "star3")


def _meshes():
    yield "box_tets", lambda: HostMesh.box(6, 5, 4, tets=True, jitter=0.15, seed=2)
    yield "box_hex", lambda: HostMesh.box(5, 4, 3, tets=False, jitter=0.1, seed=5)
    yield "shell_solid", lambda: HostMesh.shell(4, 4, 0.8, 5.0, 1.2, n_solid=1, tets=True)
    yield "hanging", lambda: host_from_ref(pytest.importorskip("oracle.ref").RefMesh.hanging_box(), BOX_TAGS)


@pytest.mark.parametrize("name,make", list(_meshes()), ids=[n for n, _ in _meshes()])
def test_device_geometry_bit_exact(name, make):
    from mpcns_uns_b200 import gpu
    h = make().compute_geometry()
    want = {k: np.array(h[k]) for k in NAMES}
    got = gpu.compute_geometry(h)
    for k in NAMES:
        a, b = np.asarray(got[k]).ravel(), want[k].ravel()
        assert a.shape == b.shape and np.array_equal(a, b), (name, k)
    # installed in a fresh mesh it gives the same boundary classification and topology
    d = make().compute_geometry(device=True)
    d.boundary("outflow")
    h.boundary("outflow")
    assert np.array_equal(np.asarray(d["face_kind"]), np.asarray(h["face_kind"]))
    assert np.array_equal(np.asarray(d["cell_center"]), want["cell_center"].reshape(-1, 3))
