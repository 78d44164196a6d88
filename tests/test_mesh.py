"""Native mesh services against the reference's own builder, generators and geometry (CPU).

Topology hash (uns::topology_hash), every CSR table and every geometry array must be identical,
for the reference's hexahedral generators and for the tetrahedral split fed to its builder.
"""
import numpy as np
import pytest

from helpers import BOX_TAGS, SHELL_TAGS, ref_twin
from mpcns_uns_b200.mesh import HostMesh

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("reference checker not built (make -C oracle ref)", allow_module_level=True)

TOP = ["e2n_ptr", "e2n_idx", "e2n_sgn", "f2e_ptr", "f2e_idx", "f2e_sgn", "c2f_ptr", "c2f_idx", "c2f_sgn", "e2f_ptr", "e2f_idx",
       "e2f_sgn", "f2c_ptr", "f2c_idx", "f2c_sgn", "cell_material", "face_tag", "x"]
GEO = ["edge_vec", "edge_mid", "edge_len", "face_area", "face_center", "face_area_mag", "cell_center", "cell_volume",
       "cell_min_tet_volume", "edge_dual_area", "ec_ptr", "ec_cell", "ec_weight", "ef_weight", "ec_misoriented", "star0", "star1",
       "star2", "star3"]


def identical(h, r):
    h.compute_geometry()
    assert h.topology_hash() == r.topology_hash()
    for k in TOP + GEO:
        a, b = np.asarray(h[k]), np.asarray(r[k])
        assert a.shape == b.shape and np.array_equal(a, b), k


def test_box_hex():
    identical(HostMesh.box(5, 4, 3, hi=(5, 4, 3)), ref.RefMesh.box(5, 4, 3, hi=(5, 4, 3)))


@pytest.mark.parametrize("n_solid", [0, 1])
def test_shell_hex(n_solid):
    identical(HostMesh.shell(4, 4, 1.0, 5.0, 1.2, n_solid=n_solid), ref.RefMesh.shell(4, 4, 1.0, 5.0, 1.2, n_solid=n_solid))


def test_box_tets_jittered():
    h = HostMesh.box(4, 4, 4, tets=True, jitter=0.15, seed=0)
    r = ref_twin(h, BOX_TAGS)
    identical(h, r)
    v = r.validate()
    g = r.check_geometry()
    assert v["ok"] and v["euler"] == 1 and v["d1d0"] == 0 and v["d2d1"] == 0
    assert g["ok"] and g["nonpositive_volume"] == 0 and g["misoriented_dual"] == 0


def test_shell_tets():
    h = HostMesh.shell(3, 3, 1.0, 6.0, 1.3, tets=True)
    r = ref_twin(h, SHELL_TAGS)
    identical(h, r)
    v = r.validate()
    assert v["ok"] and v["euler"] == 2 and v["d2d1"] == 0
    assert r.check_geometry()["ok"]


def test_counts_of_the_benchmark_meshes():
    """Entity counts of the 6-tet split: the 16^3-hex unit cube exactly (24,576 tets, 50,688 faces,
    31,024 edges, 4,913 nodes)."""
    h = HostMesh.box(16, 16, 16, tets=True, jitter=0.15, seed=0)
    assert (h.n_nodes, h.n_edges, h.n_faces, h.n_cells) == (4913, 31024, 50688, 24576)
    s = HostMesh.shell(8, 4, 1.0, 6.0, 1.0, tets=True)
    assert s.n_cells == 6 * 8 * 8 * 4 * 6


def test_cell_reordering_round_trip_and_locality():
    """The locality renumbering is explicit and invertible: rebuilding a mesh with its cells permuted and then
    with the inverse permutation restores the original complex exactly (same topology hash, same geometry);
    the Morton order brings face neighbours closer in id than a random order does."""
    import numpy as np
    from mpcns_uns_b200.mesh import HostMesh
    h = HostMesh.shell(6, 6, 1.0, 4.0, 1.1, tets=True).compute_geometry()
    rng = np.random.default_rng(0)
    perm = rng.permutation(h.n_cells).astype(np.int32)
    scrambled = h.reordered(perm).compute_geometry()
    assert scrambled.topology_hash() != h.topology_hash()
    assert np.array_equal(np.asarray(scrambled["cell_volume"]), np.asarray(h["cell_volume"])[perm])
    inv = np.empty_like(perm)
    inv[perm] = np.arange(h.n_cells, dtype=np.int32)
    back = scrambled.reordered(inv).compute_geometry()
    assert back.topology_hash() == h.topology_hash()
    for k in ("face_area", "cell_center", "star1", "ec_weight"):
        assert np.array_equal(np.asarray(back[k]), np.asarray(h[k]))

    def spread(m):
        ptr, idx = np.asarray(m["f2c_ptr"]), np.asarray(m["f2c_idx"])
        two = np.diff(ptr) == 2
        a, b = idx[ptr[:-1][two]], idx[ptr[:-1][two] + 1]
        return float(np.median(np.abs(a - b)))

    local = scrambled.reordered(scrambled.locality_order())
    assert spread(local) < 0.05 * spread(scrambled)


def test_tag_types_resolution():
    """mhdm_tag_types resolves the tag names as mhdm_boundary does: a pair's type, else the default; tag 0 and
    unknown ids take the empty name's type; unknown type names resolve to 0."""
    import ctypes
    from mpcns_uns_b200.mesh import lib
    h = HostMesh.box(2, 2, 2)
    pairs = {"xmin": "inflow", "xmax": "wall", "ymin": "farfield", "zmax": "bogus"}
    tags = (ctypes.c_char_p * len(pairs))(*[k.encode() for k in pairs])
    types = (ctypes.c_char_p * len(pairs))(*[v.encode() for v in pairs.values()])
    tt = np.zeros(64, np.int8)
    tn, nt = ctypes.c_int8(), ctypes.c_int32()
    assert lib().mhdm_tag_types(h._h, b"outflow", len(pairs), ctypes.cast(tags, ctypes.c_void_p), ctypes.cast(types, ctypes.c_void_p),
                                64, tt.ctypes.data, ctypes.byref(tn), ctypes.byref(nt)) == 0
    # box tag ids: 1 xmin, 2 xmax, 3 ymin, 4 ymax, 5 zmin, 6 zmax
    assert nt.value == 7 and tn.value == 3
    assert tt[:7].tolist() == [3, 2, 1, 5, 3, 3, 0]
