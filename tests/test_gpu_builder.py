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


def _boundary_pairs():
    from helpers import MIXED_BOX_BC, SHELL_BC
    yield "box_tets_mixed", HostMesh.box(6, 5, 4, tets=True, jitter=0.1, seed=3), MIXED_BOX_BC
    yield "box_hex_farfield", HostMesh.box(5, 4, 6), ("farfield", {}, (0.3, -0.7, 0.2))
    yield "shell_solid", HostMesh.shell(5, 4, 0.8, 6.0, 1.2, n_solid=1, tets=True), SHELL_BC
    yield "shell_default_wall", HostMesh.shell(4, 5, 1.0, 6.0, 1.3, tets=True), ("wall", {"outer": "inflow"}, (0.0, 0.0, 0.0))


@pytest.mark.parametrize("name", ["box_tets_mixed", "box_hex_farfield", "shell_solid", "shell_default_wall"])
def test_device_boundary_equals_host(name):
    """mhd::BoundaryInfo::build on the device (mhd_gpu_boundary) gives the host classification's face kinds and
    edge modes entry for entry: interior, solid-interface walls, skipped faces, tagged walls, inflow and outflow,
    farfield faces split by the side of u_inf, wall edges winning over inflow edges."""
    h, bc = next((m, b) for n, m, b in _boundary_pairs() if n == name)
    d = next(m for n, m, b in _boundary_pairs() if n == name)   # a second, independent copy of the same complex
    assert d.topology_hash() == h.topology_hash()
    h.compute_geometry()
    d.compute_geometry(device=True)
    h.boundary(*bc)
    d.boundary(*bc, device=True)
    for k in ("face_kind", "edge_mode"):
        a, b = np.asarray(d[k]), np.asarray(h[k])
        assert np.array_equal(a, b), (k, np.count_nonzero(a != b))
    assert len(np.unique(np.asarray(h["face_kind"]))) >= 3   # interior and at least two boundary kinds


def test_device_boundary_rejects_unknown_type():
    from mpcns_uns_b200.gpu import MhdError
    h = HostMesh.shell(3, 2, 1.0, 6.0, 1.0, tets=True).compute_geometry()
    with pytest.raises(MhdError, match="unknown boundary type"):
        h.boundary("outflow", {"inner": "bogus"}, device=True)
