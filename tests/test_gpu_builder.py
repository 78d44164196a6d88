"""The tetrahedral complex numbered on the device (mhd_gpu_tet_build) against the host library's builder.

The host builder restates uns::ComplexBuilder (its topology hash equals the reference's on every test
mesh, tests/test_mesh.py); the device builder must give the same complex entity for entity: every CSR
table (e2n, f2e, c2f and the upward n2e, e2f, f2c), the cell materials and the face tags, bit for bit.
"""
import numpy as np
import pytest

from mpcns_uns_b200.mesh import HostMesh

pytestmark = pytest.mark.gpu

TABLES = [f"{t}_{p}" for t in ("e2n", "f2e", "c2f", "n2e", "e2f", "f2c") for p in ("ptr", "idx", "sgn")]


@pytest.mark.parametrize("ncube,nr,n_solid,r_in,stretch", [(3, 2, 0, 1.0, 1.0), (4, 5, 0, 1.0, 1.3), (5, 4, 1, 0.8, 1.2),
                                                           (16, 24, 0, 1.0, 1.05)])
def test_device_build_equals_host_build(ncube, nr, n_solid, r_in, stretch):
    h = HostMesh.shell(ncube, nr, r_in, 6.0, stretch, n_solid=n_solid, tets=True)
    d = HostMesh.shell(ncube, nr, r_in, 6.0, stretch, n_solid=n_solid, tets=True, device_build=True)
    assert (d.n_nodes, d.n_edges, d.n_faces, d.n_cells) == (h.n_nodes, h.n_edges, h.n_faces, h.n_cells)
    assert d.topology_hash() == h.topology_hash()
    for k in TABLES + ["cell_material", "face_tag", "x"]:
        assert np.array_equal(np.asarray(d[k]), np.asarray(h[k])), k
    # the device-built complex carries on like the host one: geometry and boundary classification
    d.compute_geometry(device=True).boundary("outflow", {"inner": "wall", "outer": "farfield"}, (-8.0, 0.0, 0.0))
    h.compute_geometry().boundary("outflow", {"inner": "wall", "outer": "farfield"}, (-8.0, 0.0, 0.0))
    for k in ("face_kind", "edge_mode", "cell_volume", "star1"):
        assert np.array_equal(np.asarray(d[k]), np.asarray(h[k])), k
