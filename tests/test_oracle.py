"""The oracle's C restatement against the reference's own compiled code (CPU, no GPU needed).

Both run on the same seeded inputs and meshes; the restatement keeps the reference's operation
order, so the results must be identical bit for bit.  Skipped where the compiled reference
(oracle/_ref) is absent; tests/test_golden.py pins the restatement to committed vectors instead.
"""
import numpy as np
import pytest

from helpers import BOX_TAGS, MIXED_BOX_BC, SHELL_BC, SHELL_TAGS, host_from_ref, random_prims, ref_twin
from mpcns_uns_b200.mesh import HostMesh
from oracle import port

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("reference checker not built (make -C oracle ref)", allow_module_level=True)

CASES = ["box_tets_mixed", "shell_solid", "hanging"]


def _mk(name):
    if name == "box_tets_mixed":
        h, bc, tags = HostMesh.box(5, 4, 3, tets=True, jitter=0.1, seed=3), MIXED_BOX_BC, BOX_TAGS
    elif name == "shell_solid":
        h, bc, tags = HostMesh.shell(4, 4, 0.8, 5.0, 1.2, n_solid=1, tets=True), SHELL_BC, SHELL_TAGS
    else:
        h, bc, tags = host_from_ref(ref.RefMesh.hanging_box(), BOX_TAGS), MIXED_BOX_BC, BOX_TAGS
    h.compute_geometry().boundary(*bc)
    return h, ref_twin(h, tags).boundary(*bc), port.PortMesh(h)


_cache = {}


@pytest.fixture(params=CASES)
def trio(request):
    if request.param not in _cache:
        _cache[request.param] = _mk(request.param)
    return _cache[request.param]


def same(a, b):
    assert np.array_equal(np.asarray(a), np.asarray(b)), float(np.max(np.abs(np.asarray(a) - np.asarray(b))))


def test_fluid(trio):
    h, r, o = trio
    rng = np.random.default_rng(5)
    W = random_prims(h.n_cells, rng)
    fs = (1.1, 0.3, -0.2, 0.1, 0.12)
    for sp in (0, 1):
        for limit, rel in ((True, 0.0), (False, 0.0), (True, 0.5)):
            g = o.limited_gradients(W, sp == 1, fs, limit, rel)
            same(g, r.limited_gradients(W, sp, fs, limit, rel))
        same(o.flux_rhs(W, g, sp == 1, fs, 5 / 3), r.flux_rhs(W, g, sp, fs, 5 / 3))
    U = rng.uniform(-1, 1, 5 * h.n_cells)
    same(o.to_prim(U, 5 / 3), r.to_prim(U, 5 / 3))


def test_induction_pieces(trio):
    h, r, o = trio
    rng = np.random.default_rng(6)
    phi = rng.uniform(-1, 1, h.n_faces)
    same(o.cell_vector(phi), r.cell_vector(phi))
    args = [rng.uniform(-1, 1, 3 * h.n_cells) for _ in range(3)] + [rng.uniform(-1, 1, h.n_faces) for _ in range(2)]
    E0 = rng.uniform(-1, 1, h.n_edges)
    same(o.ideal_emf(*args, 0.5, E0), r.ideal_emf(*args, 0.5, E0))
    E = rng.uniform(-1, 1, h.n_edges)
    same(o.faraday(E, phi, 0.3), r.faraday(E, phi, 0.3))
    dte = rng.uniform(0.1, 1, h.n_edges)
    same(o.faraday(E, phi, 0.0, dte), r.faraday_edge_dt(E, dte, phi))
    for ex in (None, rng.uniform(-1, 1, h.n_faces)):
        a, b = o.div_b(phi, ex), r.div_b(phi, ex)
        assert a == b
    B = rng.uniform(-1, 1, 3 * h.n_cells)
    same(o.cell_current(B), r.cell_current(B))


def test_cfl_and_step():
    from mpcns_uns_b200 import workloads
    wl = workloads.shell(4, 5)
    h = wl.mesh
    r = ref_twin(h, SHELL_TAGS).boundary(*SHELL_BC)
    o = port.PortMesh(h)
    Badd = r.cell_vector(wl.PhiAdd)
    same(o.cell_vector(wl.PhiAdd), Badd)
    Uo = [np.array(u) for u in wl.U]
    Ur = [np.array(u) for u in wl.U]
    Po, Pr = np.array(wl.Phi), np.array(wl.Phi)
    rp = ref.StepParams()
    rp.n_species, rp.second_order, rp.gamma, rp.rho_floor, rp.p_floor, rp.cuct = 2, 1, wl.gamma, 1e-10, 1e-12, 0.5
    rp.M_ref, rp.ne_floor = 1.0, 0.01
    rp.u_inf[:] = list(wl.u_inf)
    rp.B_imf[:] = list(wl.B_imf)
    for s in range(2):
        rp.mass[s] = wl.mass[s]
        rp.fs[s][:] = list(wl.fs[s])
    for _ in range(3):
        W = [r.to_prim(u, wl.gamma) for u in Ur]
        Bt = r.cell_vector(Pr) + Badd
        dt = r.local_time_step(wl.gamma, 0.4, 1.0, 1e-2, W[0], W[1], Bt)
        assert o.local_time_step([o.to_prim(u, wl.gamma) for u in Uo], o.cell_vector(Po) + Badd, wl.gamma, 0.4) == dt
        o.rk2_step(wl, Uo, Po, Badd, dt)
        r.rk2_step(rp, Ur, Pr, wl.PhiAdd, Badd, dt)
        for a, b in zip(Uo, Ur):
            same(a, b)
        same(Po, Pr)


@pytest.mark.parametrize("hall,resistive", [(True, False), (False, True), (True, True)])
def test_implicit_induction(hall, resistive):
    h = HostMesh.box(6, 5, 4, tets=True, jitter=0.1, seed=8).compute_geometry().boundary(*MIXED_BOX_BC)
    r = ref_twin(h, BOX_TAGS).boundary(*MIXED_BOX_BC)
    o = port.PortMesh(h)
    rng = np.random.default_rng(12)
    m_edge = rng.uniform(0.5, 2.0, h.n_edges) / np.asarray(h["star1"]) if resistive else None
    kw = dict(hall=hall, hall_coef=0.5, hall_r_min=-100.0, hall_r_max=-99.0, rtol=1e-10, max_it=200, restart=15)
    ri = ref.RefInduction(r, **kw)
    if resistive:
        ri.set_m(m_edge)
    oi = port.PortInduction(o, m_edge, **kw)
    B0 = rng.uniform(-1, 1, 3 * h.n_cells)
    ne = rng.uniform(0.5, 2.0, h.n_cells)
    ri.set_frozen_state(B0, ne)
    oi.set_frozen_state(B0, ne)
    phi = rng.uniform(-1, 1, h.n_faces)
    same(oi.apply_F(phi), ri.apply_F(phi))
    x = rng.uniform(-1, 1, h.n_edges)
    same(oi.apply_A(x, 0.05), ri.apply_A(x, 0.05))
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    Ee = rng.uniform(-1, 1, h.n_edges)
    for warm in (False, True):
        Eo, ito, rro = oi.solve(phi, Ee, dirichlet, 0.05, warm)
        Er, itr, rrr = ri.solve(phi, Ee, dirichlet, 0.05, warm)
        assert ito == itr and rro == rrr
        same(Eo, Er)


def _ref_params(wl, lorentz, induce, inver_MA2):
    rp = ref.StepParams()
    rp.n_species, rp.second_order, rp.gamma, rp.rho_floor, rp.p_floor, rp.cuct = 2, 1, wl.gamma, 1e-10, 1e-12, 0.5
    rp.M_ref, rp.ne_floor = 1.0, 0.01
    rp.u_inf[:] = list(wl.u_inf)
    rp.B_imf[:] = list(wl.B_imf)
    for s in range(2):
        rp.mass[s] = wl.mass[s]
        rp.fs[s][:] = list(wl.fs[s])
    rp.lorentz, rp.induce_coeff, rp.inver_MA2 = int(lorentz), induce, inver_MA2
    return rp


def test_lorentz_sources_gyration_and_step():
    """The J x B source (add_sources), the exact gyration and the Strang-split two-ion step, bit for bit."""
    from mpcns_uns_b200 import workloads
    wl = workloads.shell(4, 5)
    h = wl.mesh
    r = ref_twin(h, SHELL_TAGS).boundary(*SHELL_BC)
    o = port.PortMesh(h)
    rng = np.random.default_rng(21)
    rp = _ref_params(wl, True, 0.7, 0.8)
    op = o.step_params(wl, lorentz=True, induce_coeff=0.7, inver_MA2=0.8)
    W = [r.to_prim(u, wl.gamma) for u in wl.U]
    B = rng.uniform(-2, 2, 3 * h.n_cells)
    J = rng.uniform(-1, 1, 3 * h.n_cells)
    for s in range(2):
        ro = rng.uniform(-1, 1, 5 * h.n_cells)
        rr = ro.copy()
        o.add_sources(op, s, W[0], W[1], B, J, 0.03, ro)
        r.add_sources(rp, s, W[0], W[1], np.zeros(3 * h.n_cells), B, J, 0.03, rr)
        same(ro, rr)
    UH, UN = [np.array(u) for u in wl.U]
    UH[1::5] += rng.uniform(-1, 1, h.n_cells)   # relative velocity to rotate
    UHr, UNr = UH.copy(), UN.copy()
    o.gyrate(op, B, 0.05, UH, UN)
    r.gyrate(rp, B, 0.05, UHr, UNr)
    same(UH, UHr)
    same(UN, UNr)
    Badd = r.cell_vector(wl.PhiAdd)
    Uo = [np.array(u) for u in wl.U]
    Ur = [np.array(u) for u in wl.U]
    Po, Pr = np.array(wl.Phi), np.array(wl.Phi)
    for _ in range(3):
        W = [r.to_prim(u, wl.gamma) for u in Ur]
        dt = r.local_time_step(wl.gamma, 0.4, 1.0, 1e-2, W[0], W[1], r.cell_vector(Pr) + Badd)
        o.rk2_step(wl, Uo, Po, Badd, dt, lorentz=True, induce_coeff=0.7, inver_MA2=0.8)
        r.rk2_step(rp, Ur, Pr, wl.PhiAdd, Badd, dt)
        for a, b in zip(Uo, Ur):
            same(a, b)
        same(Po, Pr)
    # the source terms act: one step with them differs from one step without them
    Ua, Ub = [np.array(u) for u in wl.U], [np.array(u) for u in wl.U]
    Pa, Pb = np.array(wl.Phi), np.array(wl.Phi)
    o.rk2_step(wl, Ua, Pa, Badd, dt)
    o.rk2_step(wl, Ub, Pb, Badd, dt, lorentz=True, induce_coeff=0.7, inver_MA2=0.8)
    assert np.linalg.norm(Ua[0] - Ub[0]) > 1e-6 * np.linalg.norm(Ua[0])


def test_resistive_emf_step():
    """The step with the explicit resistive EMF (ImplicitInduction::apply_F, resistive part, per-edge m_e),
    oracle restatement against the compiled reference, bit for bit."""
    from mpcns_uns_b200 import workloads
    wl = workloads.shell(4, 5)
    h = wl.mesh
    r = ref_twin(h, SHELL_TAGS).boundary(*SHELL_BC)
    o = port.PortMesh(h)
    rng = np.random.default_rng(5)
    eta = 10.0 ** rng.uniform(-4, -2, h.n_cells)
    m_res = workloads.edge_resistivity(h, eta)
    assert (m_res > 0).all()
    rp = _ref_params(wl, False, 0.0, 1.0)
    rp.m_res = m_res.ctypes.data
    Badd = r.cell_vector(wl.PhiAdd)
    Uo = [np.array(u) for u in wl.U]
    Ur = [np.array(u) for u in wl.U]
    Po = np.array(wl.Phi) + rng.uniform(-1e-2, 1e-2, h.n_faces)
    Pr = Po.copy()
    for _ in range(3):
        o.rk2_step(wl, Uo, Po, Badd, 2e-3, m_res=m_res)
        r.rk2_step(rp, Ur, Pr, wl.PhiAdd, Badd, 2e-3)
        for a, b in zip(Uo, Ur):
            same(a, b)
        same(Po, Pr)
    # the resistive EMF acts
    Pb = np.array(wl.Phi) + rng.uniform(-1e-2, 1e-2, h.n_faces)
    Pa = Pb.copy()
    Ua, Ub = [np.array(u) for u in wl.U], [np.array(u) for u in wl.U]
    o.rk2_step(wl, Ua, Pa, Badd, 2e-3)
    o.rk2_step(wl, Ub, Pb, Badd, 2e-3, m_res=m_res)
    assert np.abs(Pa - Pb).max() > 1e-9


def test_ambipolar_and_chemistry():
    """The rest of add_sources_n (ambipolar force, chemistry), the electron-pressure gradient, the ambipolar
    edge EMF, and the two-ion step with every source term on: oracle restatement against the compiled
    reference, bit for bit."""
    from helpers import SOURCE_EXTRA, source_fields
    from mpcns_uns_b200 import workloads
    wl = workloads.shell(4, 5)
    h = wl.mesh
    r = ref_twin(h, SHELL_TAGS).boundary(*SHELL_BC)
    o = port.PortMesh(h)
    rng = np.random.default_rng(41)
    photo, vst = source_fields(h.n_cells)
    extra = dict(SOURCE_EXTRA, photo=photo, vst=vst)
    rp = _ref_params(wl, True, 0.7, 0.8)
    keep_r = port.set_source_terms(rp, extra)
    op = o.step_params(wl, lorentz=True, induce_coeff=0.7, inver_MA2=0.8)
    keep_o = port.set_source_terms(op, extra)
    W = [r.to_prim(u, wl.gamma) for u in wl.U]
    W[0][4::5] *= 1 + 0.1 * rng.uniform(-1, 1, h.n_cells)   # pressure structure for grad p_e
    dpe = r.electron_pressure_gradient(W[0], W[1])
    same(o.electron_pressure_gradient(W[0], W[1]), dpe)
    assert np.abs(dpe).max() > 0
    E0 = rng.uniform(-1, 1, h.n_edges)
    Er = r.ambipolar_emf(rp, W[0], W[1], E0)
    same(o.ambipolar_emf(op, W[0], W[1], E0), Er)
    assert np.abs(Er - E0).max() > 0
    B = rng.uniform(-2, 2, 3 * h.n_cells)
    J = rng.uniform(-1, 1, 3 * h.n_cells)
    for s in range(2):
        ro = rng.uniform(-1, 1, 5 * h.n_cells)
        rr = ro.copy()
        o.add_sources(op, s, W[0], W[1], B, J, 0.03, ro, dpe, photo, vst)
        r.add_sources(rp, s, W[0], W[1], np.zeros(3 * h.n_cells), B, J, 0.03, rr, dpe, photo, vst)
        same(ro, rr)
    Badd = r.cell_vector(wl.PhiAdd)
    Uo = [np.array(u) for u in wl.U]
    Ur = [np.array(u) for u in wl.U]
    Po, Pr = np.array(wl.Phi), np.array(wl.Phi)
    for _ in range(3):
        Wr = [r.to_prim(u, wl.gamma) for u in Ur]
        dt = r.local_time_step(wl.gamma, 0.4, 0.8, 1e-2, Wr[0], Wr[1], r.cell_vector(Pr) + Badd)
        o.rk2_step(wl, Uo, Po, Badd, dt, lorentz=True, induce_coeff=0.7, inver_MA2=0.8, extra=extra)
        r.rk2_step(rp, Ur, Pr, wl.PhiAdd, Badd, dt)
        for a, b in zip(Uo, Ur):
            same(a, b)
        same(Po, Pr)
    # the terms act
    Ua = [np.array(u) for u in wl.U]
    Pa = np.array(wl.Phi)
    o.rk2_step(wl, Ua, Pa, Badd, dt, lorentz=True, induce_coeff=0.7, inver_MA2=0.8)
    Ub = [np.array(u) for u in wl.U]
    Pb = np.array(wl.Phi)
    o.rk2_step(wl, Ub, Pb, Badd, dt, lorentz=True, induce_coeff=0.7, inver_MA2=0.8, extra=extra)
    assert np.abs(Ua[1] - Ub[1]).max() > 0 and np.abs(Pa - Pb).max() > 0
    del keep_r, keep_o


@pytest.mark.parametrize("ncube,nr,n_solid", [(8, 6, 0), (5, 4, 1)])
def test_reference_built_shell_is_the_workload_shell(ncube, nr, n_solid):
    """The bench's reference arm builds its shell with the reference's code alone (make_cubed_sphere_shell,
    the tetrahedral split through ComplexBuilder, compute_geometry, BoundaryInfo::build) and its state with
    workloads.shell_state: the same complex (topology hash), metric, boundary classification and state as the
    workload of this library's own generator, bit for bit."""
    from mpcns_uns_b200 import workloads
    st = workloads.shell_stretch(ncube, nr)
    h = HostMesh.shell(ncube, nr, 1.0, 6.0, st, n_solid=n_solid, tets=True).compute_geometry().boundary(*SHELL_BC)
    r = ref.RefMesh.shell_tets(ncube, nr, 1.0, 6.0, st, n_solid=n_solid).boundary(*SHELL_BC)
    assert h.topology_hash() == r.topology_hash()
    for k in ("x", "cell_material", "face_tag", "face_kind", "edge_mode", "cell_center", "cell_volume", "face_area",
              "face_center", "edge_vec", "edge_mid", "star1", "star2", "ec_cell", "ec_weight", "ef_weight"):
        a, b = np.asarray(h[k]).ravel(), np.asarray(r[k]).ravel()
        assert a.shape == b.shape and np.array_equal(a, b), k
    wh = workloads.shell_state(h, "h", 1.0, st, sources=True)
    wr = workloads.shell_state(r, "r", 1.0, st, sources=True)
    assert all(np.array_equal(a, b) for a, b in zip(wh.U, wr.U)) and np.array_equal(wh.PhiAdd, wr.PhiAdd)


def test_semi_implicit_step():
    """Solver::step_first_order (time_order = 1): forward Euler of both ions with the J x B force and the Strang-split
    gyration, the EMF from the Hall + resistive ImplicitInduction::solve (warm start across steps), CT with it,
    bit for bit against the reference's sequence; the solve's iterations and residual equal."""
    from mpcns_uns_b200 import workloads
    wl = workloads.shell(4, 5)
    h = wl.mesh
    r = ref_twin(h, SHELL_TAGS).boundary(*SHELL_BC)
    o = port.PortMesh(h)
    rp = _ref_params(wl, True, 1.0, 1.0)
    r_e = np.linalg.norm(np.asarray(h["edge_mid"]), axis=1)
    m_edge = np.where(r_e < 1.5, 1e-2, 1e-4) / np.asarray(h["star1"])
    kw = dict(hall=True, hall_coef=0.5, hall_r_min=1.0, hall_r_max=1.6, rtol=1e-10, max_it=300, restart=30)
    ri = ref.RefInduction(r, **kw)
    ri.set_m(m_edge)
    oi = port.PortInduction(o, m_edge, **kw)
    Badd = r.cell_vector(wl.PhiAdd)
    Uo = [np.array(u) for u in wl.U]
    Ur = [np.array(u) for u in wl.U]
    Po, Pr = np.array(wl.Phi), np.array(wl.Phi)
    for _ in range(3):
        W = [r.to_prim(u, wl.gamma) for u in Ur]
        dt = r.local_time_step(wl.gamma, 0.4, 1.0, 1e-2, W[0], W[1], r.cell_vector(Pr) + Badd)
        ito, rro = o.first_order_step(wl, oi, Uo, Po, Badd, dt, lorentz=True, induce_coeff=1.0, inver_MA2=1.0)
        itr, rrr = r.first_order_step(rp, ri, Ur, Pr, wl.PhiAdd, Badd, dt)
        assert ito == itr and rro == rrr and rrr <= 1e-10
        for a, b in zip(Uo, Ur):
            same(a, b)
        same(Po, Pr)


@pytest.mark.parametrize("case", ["box", "shell"])
def test_induction_steady_mode_forms(case):
    """The implicit ideal part of F (Config::implicit_ideal: set_ideal_state, ideal_linear, apply_F, apply_A)
    and the per-edge pseudo-time step of solve (dt_edge), alone and together, bit for bit against the
    reference: operator outputs, iterations, residuals and E."""
    if case == "box":
        h = HostMesh.box(6, 5, 4, tets=True, jitter=0.1, seed=8).compute_geometry().boundary(*MIXED_BOX_BC)
        r = ref_twin(h, BOX_TAGS).boundary(*MIXED_BOX_BC)
        taper = dict(hall_r_min=-100.0, hall_r_max=-99.0)
    else:
        h = HostMesh.shell(4, 4, 0.8, 5.0, 1.2, n_solid=1, tets=True).compute_geometry().boundary(*SHELL_BC)
        r = ref_twin(h, SHELL_TAGS).boundary(*SHELL_BC)
        taper = dict(hall_r_min=1.0, hall_r_max=1.6)
    o = port.PortMesh(h)
    rng = np.random.default_rng(17)
    m_edge = rng.uniform(0.5, 2.0, h.n_edges) / np.asarray(h["star1"])
    kw = dict(hall=True, hall_coef=0.5, rtol=1e-10, max_it=300, restart=15, **taper)
    B0 = rng.uniform(-1, 1, 3 * h.n_cells)
    ne = rng.uniform(0.5, 2.0, h.n_cells)
    u = rng.uniform(-1, 1, 3 * h.n_cells)
    mask = (np.asarray(h["edge_mode"]) == 0).astype(np.int8)
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    phi = rng.uniform(-1, 1, h.n_faces)
    x = rng.uniform(-1, 1, h.n_edges)
    Ee = rng.uniform(-1, 1, h.n_edges)
    dte = rng.uniform(0.005, 0.05, h.n_edges)
    for ideal in (False, True):
        ri = ref.RefInduction(r, implicit_ideal=ideal, cuct=0.5, **kw)
        ri.set_m(m_edge)
        oi = port.PortInduction(o, m_edge, **kw)
        ri.set_frozen_state(B0, ne)
        oi.set_frozen_state(B0, ne)
        if ideal:
            ri.set_ideal_state(u, mask)
            oi.set_ideal_state(u, mask, 0.5)
            same(oi.ideal_linear(phi), ri.ideal_linear(phi))
        same(oi.apply_F(phi), ri.apply_F(phi))
        same(oi.apply_A(x, 0.05), ri.apply_A(x, 0.05))
        for warm in (False, True):
            Eo, ito, rro = oi.solve_dt_edge(phi, Ee, dirichlet, dte, warm)
            Er, itr, rrr = ri.solve_dt_edge(phi, Ee, dirichlet, dte, warm)
            assert ito == itr and rro == rrr and rrr <= 1e-10
            same(Eo, Er)
        if ideal:
            Eo, ito, rro = oi.solve(phi, Ee, dirichlet, 0.02, False)
            Er, itr, rrr = ri.solve(phi, Ee, dirichlet, 0.02, False)
            assert ito == itr and rro == rrr and rrr <= 1e-10
            same(Eo, Er)
