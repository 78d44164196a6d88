"""Parity of every reference-signature entry point of the C-ABI against the reference's own code.

Each device function runs on the same seeded inputs as the compiled reference
(oracle/_ref) on meshes that cover the boundary kinds (interior, wall, inflow, outflow,
far field, solid interfaces, skipped faces), tetrahedra, hexahedra and hanging-node
polyhedra.  FP64 results must agree to 1e-12 relative to the largest reference value.
"""
import numpy as np
import pytest

from helpers import BOX_TAGS, MIXED_BOX_BC, SHELL_BC, SHELL_TAGS, host_from_ref, random_prims, ref_twin, rel_err
from mpcns_uns_b200.mesh import HostMesh

pytestmark = pytest.mark.gpu
TOL = 1e-12

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("reference checker not built (make -C oracle ref)", allow_module_level=True)


def _mk(name):
    if name == "cfg1":
        h = HostMesh.box(16, 16, 16, tets=True, jitter=0.15, seed=0)
        bc, tags = ("outflow", {}, (1.0, 0.0, 0.0)), BOX_TAGS
    elif name == "box_hex_mixed":
        h = HostMesh.box(4, 3, 5, hi=(2.0, 1.5, 2.5))
        bc, tags = MIXED_BOX_BC, BOX_TAGS
    elif name == "box_tets_mixed":
        h = HostMesh.box(5, 4, 3, tets=True, jitter=0.1, seed=3)
        bc, tags = MIXED_BOX_BC, BOX_TAGS
    elif name == "shell_solid":
        h = HostMesh.shell(4, 4, 0.8, 5.0, 1.2, n_solid=1, tets=True)
        bc, tags = SHELL_BC, SHELL_TAGS
    elif name == "hanging":
        r0 = ref.RefMesh.hanging_box()
        h = host_from_ref(r0, BOX_TAGS)
        bc, tags = MIXED_BOX_BC, BOX_TAGS
    else:
        raise KeyError(name)
    h.compute_geometry().boundary(bc[0], bc[1], bc[2])
    r = ref_twin(h, tags).boundary(bc[0], bc[1], bc[2])
    assert h.topology_hash() == r.topology_hash()
    from mpcns_uns_b200.gpu import DeviceMesh
    return h, r, DeviceMesh(h), bc


MESHES = ["cfg1", "box_hex_mixed", "box_tets_mixed", "shell_solid", "hanging"]
_cache = {}


@pytest.fixture(params=MESHES)
def meshes(request):
    if request.param not in _cache:
        _cache[request.param] = _mk(request.param)
    return _cache[request.param]


def _np(t):
    return t.detach().cpu().numpy()


def test_boundary_classification_bit_exact(meshes):
    h, r, d, bc = meshes
    assert np.array_equal(np.asarray(h["face_kind"]), r["face_kind"])
    assert np.array_equal(np.asarray(h["edge_mode"]), r["edge_mode"])


def test_to_prim(meshes):
    h, r, d, bc = meshes
    rng = np.random.default_rng(11)
    U = rng.uniform(-1, 1, 5 * h.n_cells)
    U[0::5] = rng.uniform(-0.1, 1.0, h.n_cells)  # some below the floor
    W = _np(d.to_prim(U, 5 / 3))
    assert rel_err(W, r.to_prim(U, 5 / 3)) < TOL


@pytest.mark.parametrize("species,limit,rel_limit", [(0, True, 0.0), (1, True, 0.0), (0, False, 0.0), (0, True, 0.5)])
def test_limited_gradients(meshes, species, limit, rel_limit):
    h, r, d, bc = meshes
    rng = np.random.default_rng(100 + species)
    W = random_prims(h.n_cells, rng)
    fs = (1.1, 0.3, -0.2, 0.1, 0.12)
    g = _np(d.limited_gradients(W, species, fs, limit, rel_limit))
    gr = r.limited_gradients(W, species, fs, limit, rel_limit)
    assert rel_err(g, gr) < TOL


@pytest.mark.parametrize("species", [0, 1])
def test_flux_rhs(meshes, species):
    h, r, d, bc = meshes
    rng = np.random.default_rng(200 + species)
    W = random_prims(h.n_cells, rng)
    fs = (1.1, 0.3, -0.2, 0.1, 0.12)
    grad = r.limited_gradients(W, species, fs, True, 0.0)
    rhs = _np(d.fluid_flux_rhs(5 / 3, species, fs, W, grad))
    rr = r.flux_rhs(W, grad, species, fs, 5 / 3)
    assert rel_err(rhs, rr) < TOL


def _wall_table(h, rng):
    walls = np.nonzero(np.asarray(h["face_kind"]) == 1)[0].astype(np.int32)
    faces = walls[::2]   # every other wall face: the rest keep ghost_state
    prims = np.column_stack([rng.uniform(0.2, 2.0, faces.size), rng.uniform(-0.3, 0.3, (faces.size, 3)),
                             rng.uniform(0.05, 0.5, faces.size)])
    return faces, prims


@pytest.mark.parametrize("species", [0, 1])
def test_limited_gradients_and_flux_wall_table(meshes, species):
    """The GhostFn argument of limited_gradients / fluid_flux_rhs as a Dirichlet wall table (the ten-ion
    solver's wall ghost), seeded states on every other wall face, against the reference with the same table."""
    h, r, d, bc = meshes
    rng = np.random.default_rng(300 + species)
    faces, prims = _wall_table(h, rng)
    if faces.size == 0:
        pytest.skip("mesh without wall faces")
    W = random_prims(h.n_cells, rng)
    fs = (1.1, 0.3, -0.2, 0.1, 0.12)
    g = _np(d.limited_gradients(W, species, fs, True, 0.0, wall=(faces, prims)))
    gr = r.limited_gradients_wall(W, species, fs, faces, prims)
    assert rel_err(g, gr) < TOL
    assert not np.array_equal(gr, r.limited_gradients(W, species, fs, True, 0.0))   # the table acts
    rhs = _np(d.fluid_flux_rhs(5 / 3, species, fs, W, gr, wall=(faces, prims)))
    rr = r.flux_rhs_wall(W, gr, species, fs, 5 / 3, faces, prims)
    assert rel_err(rhs, rr) < TOL
    assert not np.array_equal(rr, r.flux_rhs(W, gr, species, fs, 5 / 3))


def test_wall_table_rejects_bad_faces(meshes):
    from mpcns_uns_b200.gpu import MhdError
    h, r, d, bc = meshes
    kind = np.asarray(h["face_kind"])
    W = random_prims(h.n_cells, np.random.default_rng(5))
    fs = (1.0, 0.0, 0.0, 0.0, 0.1)
    other = np.nonzero(kind != 1)[0][:1].astype(np.int32)
    with pytest.raises(MhdError, match="kind wall"):
        d.limited_gradients(W, 0, fs, wall=(other, np.ones((1, 5))))
    walls = np.nonzero(kind == 1)[0].astype(np.int32)
    if walls.size:
        with pytest.raises(MhdError, match="distinct"):
            d.limited_gradients(W, 0, fs, wall=(np.array([walls[0], walls[0]], np.int32), np.ones((2, 5))))


def test_cell_vector(meshes):
    h, r, d, bc = meshes
    rng = np.random.default_rng(300)
    phi = rng.uniform(-1, 1, h.n_faces)
    assert rel_err(_np(d.reconstruct_cell_vector(phi)), r.cell_vector(phi)) < TOL


@pytest.mark.parametrize("cuct", [0.5, 0.0])
def test_ideal_emf(meshes, cuct):
    h, r, d, bc = meshes
    rng = np.random.default_rng(400)
    u = rng.uniform(-1, 1, 3 * h.n_cells)
    Bt = rng.uniform(-1, 1, 3 * h.n_cells)
    Bi = rng.uniform(-1, 1, 3 * h.n_cells)
    pt = rng.uniform(-1, 1, h.n_faces)
    pi = rng.uniform(-1, 1, h.n_faces)
    E0 = rng.uniform(-1, 1, h.n_edges)
    E = _np(d.add_ideal_emf(u, Bt, Bi, pt, pi, cuct, E0))
    Er = r.ideal_emf(u, Bt, Bi, pt, pi, cuct, E0)
    assert rel_err(E, Er) < TOL


def test_edge_modes(meshes):
    h, r, d, bc = meshes
    from mpcns_uns_b200.gpu import dev
    rng = np.random.default_rng(450)
    E0 = rng.uniform(-1, 1, h.n_edges)
    u_inf, B_imf = (0.4, -0.2, 0.3), (0.3, 0.5, -0.2)
    E = dev(E0)
    d.edge_modes(u_inf, B_imf, E)
    d.synchronize()
    Eref = E0.copy()
    mode = np.asarray(h["edge_mode"])
    Einf = -np.cross(u_inf, B_imf)
    Eref[mode == 1] = 0.0
    Eref[mode == 2] = np.asarray(h["edge_vec"])[mode == 2] @ Einf
    assert rel_err(_np(E), Eref) < TOL


def test_faraday_and_div_b(meshes):
    h, r, d, bc = meshes
    rng = np.random.default_rng(500)
    E = rng.uniform(-1, 1, h.n_edges)
    B = rng.uniform(-1, 1, h.n_faces)
    Bn = _np(d.faraday_update(E, B, 0.37))
    Br = r.faraday(E, B, 0.37)
    assert rel_err(Bn, Br) < TOL
    dt_e = rng.uniform(0.1, 1.0, h.n_edges)
    assert rel_err(_np(d.faraday_update_edge_dt(E, dt_e, B)), r.faraday_edge_dt(E, dt_e, B)) < TOL
    extra = rng.uniform(-1, 1, h.n_faces)
    for ex in (None, extra):
        g = d.div_b(B, ex)
        rr = r.div_b(B, ex)
        assert abs(g["max_abs"] - rr["max_abs"]) <= TOL * rr["max_abs"]
        assert abs(g["max_rel"] - rr["max_rel"]) <= TOL * rr["max_rel"]
        assert g["worst_cell_gid"] == rr["worst_cell_gid"]


def test_ct_keeps_div_b(meshes):
    """B = d1 A stays divergence free under any number of CT updates (integer identity d2 d1 = 0)."""
    h, r, d, bc = meshes
    rng = np.random.default_rng(600)
    from mpcns_uns_b200.workloads import d1
    B = d1(h, rng.uniform(-1, 1, h.n_edges))
    from mpcns_uns_b200.gpu import dev
    Bd = dev(B)
    for _ in range(20):
        Bd = d.faraday_update(rng.uniform(-1, 1, h.n_edges), Bd, 0.02)
    assert d.div_b(Bd)["max_rel"] < 1e-13


def test_cell_current(meshes):
    h, r, d, bc = meshes
    rng = np.random.default_rng(700)
    B = rng.uniform(-1, 1, 3 * h.n_cells)
    assert rel_err(_np(d.cell_current(B)), r.cell_current(B)) < TOL


def _two_ion_params(lorentz=True, induce=0.6):
    from mpcns_uns_b200 import gpu
    p = gpu.step_params(2, mass=[1.0, 23.0], lorentz=lorentz, induce_coeff=induce, inver_MA2=0.9, ne_floor=0.02)
    rp = ref.StepParams()
    rp.n_species, rp.second_order, rp.gamma, rp.rho_floor, rp.p_floor = 2, 1, p.gamma, p.rho_floor, p.p_floor
    rp.M_ref, rp.ne_floor = p.M_ref, p.ne_floor
    rp.mass[0], rp.mass[1] = 1.0, 23.0
    rp.lorentz, rp.induce_coeff, rp.inver_MA2 = int(lorentz), induce, p.inver_MA2
    return p, rp


@pytest.mark.parametrize("lorentz", [True, False])
def test_add_sources(meshes, lorentz):
    """mercury::add_sources, J x B part, both ions (the source is zero with the force off)."""
    h, r, d, bc = meshes
    rng = np.random.default_rng(701)
    p, rp = _two_ion_params(lorentz)
    WH, WN = random_prims(h.n_cells, rng), random_prims(h.n_cells, rng, rho=(1e-4, 1e-2))
    B, J = rng.uniform(-2, 2, 3 * h.n_cells), rng.uniform(-1, 1, 3 * h.n_cells)
    for s in (0, 1):
        rhs = rng.uniform(-1, 1, 5 * h.n_cells)
        want = rhs.copy()
        r.add_sources(rp, s, WH, WN, np.zeros(3 * h.n_cells), B, J, 0.02, want)
        assert rel_err(_np(d.add_sources(p, s, WH, WN, B, J, 0.02, rhs)), want) < TOL


def test_ambipolar_and_chemistry_sources(meshes):
    """mercury::electron_pressure_gradient, AmbipolarEMF::add and add_sources with the ambipolar force and the
    chemistry terms of seeded source fields, both ions."""
    from helpers import SOURCE_EXTRA, source_fields
    from mpcns_uns_b200 import gpu
    from oracle import port
    h, r, d, bc = meshes
    rng = np.random.default_rng(703)
    p = gpu.step_params(2, mass=[1.0, 23.0], lorentz=True, induce_coeff=0.6, inver_MA2=0.9, ne_floor=0.02, extra=SOURCE_EXTRA)
    _, rp = _two_ion_params(True)
    keep = port.set_source_terms(rp, SOURCE_EXTRA)
    WH, WN = random_prims(h.n_cells, rng), random_prims(h.n_cells, rng, rho=(1e-4, 1e-2))
    dpe = r.electron_pressure_gradient(WH, WN)
    assert rel_err(_np(d.electron_pressure_gradient(WH, WN)), dpe) < TOL
    E0 = rng.uniform(-1, 1, h.n_edges)
    assert rel_err(_np(d.ambipolar_emf(p, WH, WN, E0)), r.ambipolar_emf(rp, WH, WN, E0)) < TOL
    photo, vst = source_fields(h.n_cells)
    B, J = rng.uniform(-2, 2, 3 * h.n_cells), rng.uniform(-1, 1, 3 * h.n_cells)
    for s in (0, 1):
        rhs = rng.uniform(-1, 1, 5 * h.n_cells)
        want = rhs.copy()
        r.add_sources(rp, s, WH, WN, np.zeros(3 * h.n_cells), B, J, 0.02, want, dpe, photo, vst)
        assert rel_err(_np(d.add_sources(p, s, WH, WN, B, J, 0.02, rhs, dpe, photo, vst)), want) < TOL
    del keep


def test_gyrate(meshes):
    """mercury::gyrate: exact rotation of the relative ion velocity about B."""
    from mpcns_uns_b200 import workloads
    h, r, d, bc = meshes
    rng = np.random.default_rng(702)
    p, rp = _two_ion_params()
    UH = workloads.to_cons(random_prims(h.n_cells, rng), p.gamma).ravel()
    UN = workloads.to_cons(random_prims(h.n_cells, rng, rho=(1e-3, 1e-1)), p.gamma).ravel()
    B = rng.uniform(-2, 2, 3 * h.n_cells)
    UHr, UNr = UH.copy(), UN.copy()
    r.gyrate(rp, B, 0.07, UHr, UNr)
    gH, gN = d.gyrate(p, B, 0.07, UH, UN)
    assert rel_err(_np(gH), UHr) < TOL and rel_err(_np(gN), UNr) < TOL
    assert rel_err(UHr, UH) > 1e-6          # the rotation did something


def _face_keys(m):
    """Sorted node triple/quad of every face, as a tuple per face."""
    e2n = np.asarray(m["e2n_idx"]).reshape(-1, 2)
    fp, fi = np.asarray(m["f2e_ptr"]), np.asarray(m["f2e_idx"])
    return [tuple(sorted(set(e2n[fi[fp[f]:fp[f + 1]]].ravel().tolist()))) for f in range(m.n_faces)]


def test_div_b_worst_cell_after_renumbering():
    """On a renumbered mesh the device reports its local index of the worst cell; mapped through the
    caller's gid table (new cell i = old cell order[i]) it is the cell the reference names on the mesh
    in its original numbering (DivB.cpp:20 returns cx.ent[3].gid[c])."""
    from mpcns_uns_b200.gpu import DeviceMesh
    h0 = HostMesh.box(6, 5, 4, tets=True, jitter=0.1, seed=5)
    order = np.random.default_rng(8).permutation(h0.n_cells).astype(np.int32)
    h0.compute_geometry().boundary("outflow")
    hr = h0.reordered(order).compute_geometry().boundary("outflow")
    r0 = ref_twin(h0, BOX_TAGS).boundary("outflow", {}, (1.0, 0.0, 0.0))
    where = {k: f for f, k in enumerate(_face_keys(h0))}
    fmap = np.array([where[k] for k in _face_keys(hr)])
    rng = np.random.default_rng(9)
    B0 = rng.uniform(-1, 1, h0.n_faces)
    dr = DeviceMesh(hr)
    for ex in (None, rng.uniform(-1, 1, h0.n_faces)):
        rr = r0.div_b(B0, ex)
        g = dr.div_b(B0[fmap], None if ex is None else ex[fmap], gid=order)
        assert abs(g["max_abs"] - rr["max_abs"]) <= TOL * rr["max_abs"]
        assert abs(g["max_rel"] - rr["max_rel"]) <= TOL * rr["max_rel"]
        assert g["worst_cell_gid"] == rr["worst_cell_gid"] and order[g["worst_cell"]] == rr["worst_cell_gid"]
        assert g["worst_cell"] != rr["worst_cell_gid"] or order[g["worst_cell"]] == g["worst_cell"]


def test_empty_mesh_every_entry_point():
    """A rank with no cells (a partition can leave one empty): every entry point accepts the empty mesh and
    returns empty results without launching on empty grids, as the reference's loops run zero times."""
    import torch
    from mpcns_uns_b200 import gpu
    h = HostMesh.from_cells(np.zeros((0, 3)), [])
    h.compute_geometry()
    h.boundary("outflow")
    assert (h.n_cells, h.n_faces, h.n_edges) == (0, 0, 0)
    dm = gpu.DeviceMesh(h)
    e = np.zeros(0)
    fs = (1.0, 0.0, 0.0, 0.0, 1.0)
    W = dm.to_prim(e, 5.0 / 3.0)
    g = dm.limited_gradients(W, 0, fs)
    rhs = dm.fluid_flux_rhs(5.0 / 3.0, 0, fs, W, g)
    B = dm.reconstruct_cell_vector(e)
    E = dm.add_ideal_emf(e, e, e, e, e)
    E = dm.edge_modes((1.0, 0.0, 0.0), (0.0, 0.0, 1.0), E)
    Bn = dm.faraday_update(E, e, 0.1)
    for a in (W, g, rhs, B, E, Bn):
        assert int(torch.as_tensor(a).numel()) == 0
    d = dm.div_b(e)
    assert d["max_abs"] == 0.0
    for precision in ("fp64", "mixed"):
        p = gpu.step_params(1, 5.0 / 3.0, fs=[fs], precision=precision)
        st = gpu.ResidentState(dm, p)
        st.set([e], e, e)
        assert st.step(1e-3) == 1e-3
        assert st.U(0).size == 0 and st.Phi().size == 0
    ind = gpu.DeviceInduction(dm, np.zeros(0), hall=True, hall_coef=1.0, rtol=1e-8)
    ind.set_frozen_state(e, e)
    E2, it, rr = ind.solve(e, e, np.zeros(0, np.int8), 1e-3)
    assert int(E2.numel()) == 0
