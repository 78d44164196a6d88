"""The block-Jacobi ILU(0) pattern of the induction solve (ImplicitInduction::build_precond_pattern,
Common/induction/ImplicitInduction.cpp:209-242) built by the library's host code against the compiled
reference's own pattern (CPU, no GPU needed): same rows, columns and coefficients bit for bit, including
the diagonal, which sums one term per face in the order std::sort leaves them."""
import numpy as np
import pytest

from helpers import BOX_TAGS, MIXED_BOX_BC, SHELL_BC, SHELL_TAGS, host_from_ref, ref_twin
from mpcns_uns_b200.mesh import HostMesh

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("reference checker not built (make -C oracle ref)", allow_module_level=True)


def _mesh(name):
    if name == "box_tets":
        h, bc, tags = HostMesh.box(5, 4, 3, tets=True, jitter=0.1, seed=3), MIXED_BOX_BC, BOX_TAGS
    elif name == "box_hex":
        h, bc, tags = HostMesh.box(4, 3, 3, jitter=0.1, seed=5), MIXED_BOX_BC, BOX_TAGS
    elif name == "shell_solid":
        h, bc, tags = HostMesh.shell(4, 4, 0.8, 5.0, 1.2, n_solid=1, tets=True), SHELL_BC, SHELL_TAGS
    else:
        h, bc, tags = host_from_ref(ref.RefMesh.hanging_box(), BOX_TAGS), MIXED_BOX_BC, BOX_TAGS
    h.compute_geometry().boundary(*bc)
    return h, ref_twin(h, tags).boundary(*bc)


@pytest.mark.parametrize("name", ["box_tets", "box_hex", "shell_solid", "hanging"])
def test_pattern_matches_reference(name):
    from mpcns_uns_b200 import gpu
    h, r = _mesh(name)
    rng = np.random.default_rng(4)
    m_edge = rng.uniform(0.5, 2.0, h.n_edges) / np.asarray(h["star1"])
    ri = ref.RefInduction(r, ilu=True, rtol=1e-8)
    ri.set_m(m_edge)
    csr = lambda k: (np.asarray(h[k + "_ptr"]), np.asarray(h[k + "_idx"]), np.asarray(h[k + "_sgn"]))
    ptr, col, coef = gpu.ilu_pattern(h.n_edges, h.n_edges, h.n_faces, csr("e2f"), csr("f2e"), np.asarray(h["star2"]), m_edge)
    assert np.array_equal(ptr, ri.array("pc_ptr"))
    assert np.array_equal(col, ri.array("pc_col"))
    assert np.array_equal(coef.view(np.int64), ri.array("pc_coef").view(np.int64))
    # every row holds its diagonal; the rows are sorted
    assert all(np.all(np.diff(col[ptr[e]:ptr[e + 1]]) > 0) and e in col[ptr[e]:ptr[e + 1]] for e in range(h.n_edges))


def test_pattern_block_jacobi_drops_other_ranks():
    """With fewer owned edges than edges, couplings into the non-owned edges are dropped (:225).  The
    shorter rows sort their diagonal terms into another order, so the diagonal agrees to rounding."""
    from mpcns_uns_b200 import gpu
    h, _ = _mesh("box_tets")
    m_edge = np.full(h.n_edges, 2.0)
    csr = lambda k: (np.asarray(h[k + "_ptr"]), np.asarray(h[k + "_idx"]), np.asarray(h[k + "_sgn"]))
    no = h.n_edges // 2
    ptr, col, coef = gpu.ilu_pattern(h.n_edges, no, h.n_faces, csr("e2f"), csr("f2e"), np.asarray(h["star2"]), m_edge)
    full = gpu.ilu_pattern(h.n_edges, h.n_edges, h.n_faces, csr("e2f"), csr("f2e"), np.asarray(h["star2"]), m_edge)
    assert len(ptr) == no + 1 and col.max() < no
    for e in range(no):
        a, b = full[0][e], full[0][e + 1]
        keep = full[1][a:b] < no
        assert np.array_equal(col[ptr[e]:ptr[e + 1]], full[1][a:b][keep])
        assert np.allclose(coef[ptr[e]:ptr[e + 1]], full[2][a:b][keep], rtol=1e-14, atol=0)


@pytest.mark.parametrize("name", ["box_tets", "box_hex", "shell_solid", "hanging"])
def test_oracle_ilu_against_reference(name):
    """The oracle's restatement of the ILU(0) (oracle/mhd_oracle.c) against the compiled reference: the pattern's
    columns exactly and its coefficients to rounding (the oracle's column sort keeps ties in gathering order,
    the reference's std::sort in an order of its own: the diagonal sums the same terms in another order), the
    preconditioned vector of factor_precond + apply_precond to 1e-12, with and without Dirichlet edges, and
    the ILU(0)-preconditioned solve to GMRES tolerance with the same iteration count to within two."""
    from oracle import port
    h, r = _mesh(name)
    rng = np.random.default_rng(11)
    m_edge = rng.uniform(0.5, 2.0, h.n_edges) / np.asarray(h["star1"])
    kw = dict(hall=True, hall_coef=0.5, hall_r_min=-100.0, hall_r_max=-99.0, rtol=1e-10, max_it=300, restart=15)
    ri = ref.RefInduction(r, ilu=True, **kw)
    ri.set_m(m_edge)
    oi = port.PortInduction(port.PortMesh(h), m_edge, **kw)
    oi.set_ilu(True, 0.3)
    ptr, col, coef = oi.ilu_pattern()
    assert np.array_equal(ptr, ri.array("pc_ptr")) and np.array_equal(col, ri.array("pc_col"))
    assert np.allclose(coef, ri.array("pc_coef"), rtol=1e-14, atol=0)
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    for d in (np.zeros(h.n_edges, np.int8), dirichlet):
        for dt in (0.05, 3.0):
            v = rng.uniform(-1, 1, h.n_edges)
            zo, zr = oi.precond(dt, d, v), ri.precond(dt, d, v)
            assert np.max(np.abs(zo - zr)) <= 1e-12 * np.max(np.abs(zr)), (dt, int(d.sum()))
    B0 = rng.uniform(-1, 1, 3 * h.n_cells)
    ne = rng.uniform(0.5, 2.0, h.n_cells)
    ri.set_frozen_state(B0, ne)
    oi.set_frozen_state(B0, ne)
    phi = rng.uniform(-1, 1, h.n_faces)
    Ee = rng.uniform(-1, 1, h.n_edges)
    Er, itr, rrr = ri.solve(phi, Ee, dirichlet, 0.05, False)
    Eo, ito, rro = oi.solve(phi, Ee, dirichlet, 0.05, False)
    assert rro <= 1e-10 and rrr <= 1e-10 and abs(ito - itr) <= 2, (ito, itr)
    assert np.max(np.abs(Eo - Er)) <= 1e-8 * np.max(np.abs(Er))
