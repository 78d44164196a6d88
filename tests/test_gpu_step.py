"""The fused SSP-RK2 step on the device against the reference's step sequence.

The reference side is mercury::Solver::step restricted to the hot path (prepare, limited
gradients, fluxes, ideal EMF with the boundary edge values, advance with floors, SSP-RK2
average), composed from the reference's own functions in oracle/ref/ref_shim.cpp.  The
CFL step is mercury::local_time_step.  FP64 agreement 1e-12 relative after several steps.
"""
import numpy as np
import pytest

from helpers import BOX_TAGS, MIXED_BOX_BC, SHELL_BC, SHELL_TAGS, ref_twin, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("reference checker not built (make -C oracle ref)", allow_module_level=True)


def ref_params(p):
    rp = ref.StepParams()
    rp.n_species, rp.second_order = p.n_species, p.second_order
    rp.gamma, rp.rho_floor, rp.p_floor, rp.cuct = p.gamma, p.rho_floor, p.p_floor, p.cuct
    rp.M_ref, rp.ne_floor, rp.rel_limit = p.M_ref, p.ne_floor, p.rel_limit
    rp.u_inf[:] = list(p.u_inf)
    rp.B_imf[:] = list(p.B_imf)
    for s in range(p.n_species):
        rp.mass[s] = p.mass[s]
        f = p.fs[s]
        rp.fs[s][:] = [f.rho, f.u, f.v, f.w, f.p]
    rp.lorentz, rp.induce_coeff, rp.inver_MA2 = p.lorentz, p.induce_coeff, p.inver_MA2
    rp.ambipolar, rp.chemistry = p.ambipolar, p.chemistry
    for n in ("pressure_coef", "a1_Na", "a4", "a5", "a6", "state_coeff_H", "state_coeff_Na", "T_ref", "Tn0"):
        setattr(rp, n, getattr(p, n))
    return rp


def run_pair(wl, tags, bc, nsteps, params_kw=None, use_cfl=True, fields=None, wall=None, ref_mesh=None):
    from mpcns_uns_b200 import gpu
    h = wl.mesh
    r = (ref_mesh if ref_mesh is not None else ref_twin(h, tags)).boundary(*bc)
    assert r.topology_hash() == h.topology_hash()
    dm = gpu.DeviceMesh(h)
    p = gpu.step_params(wl.n_species, wl.gamma, fs=wl.fs, mass=wl.mass, u_inf=wl.u_inf, B_imf=wl.B_imf,
                        **(params_kw or {}))
    st = gpu.ResidentState(dm, p)
    st.set(wl.U, wl.Phi, wl.PhiAdd)
    Badd = r.cell_vector(wl.PhiAdd)
    assert rel_err(st.download(gpu.FIELD_BADD), Badd) < TOL
    U = [np.array(u, np.float64) for u in wl.U]
    Phi = np.array(wl.Phi, np.float64)
    rp = ref_params(p)
    if fields is not None:   # the chemistry's source fields (photo, vst) on both sides
        st.set_source_fields(*fields)
        keep = [np.ascontiguousarray(x, np.float64) for x in fields]
        rp.photo, rp.vst = keep[0].ctypes.data, keep[1].ctypes.data
    if wall is not None:     # the Dirichlet wall table (faces, prims n_species x n_wall x 5) on both sides
        st.set_wall_ghosts(*wall)
        wkeep = (np.ascontiguousarray(wall[0], np.int32), np.ascontiguousarray(wall[1], np.float64))
        rp.n_wall, rp.wall_faces, rp.wall_prims = wkeep[0].size, wkeep[0].ctypes.data, wkeep[1].ctypes.data
    for k in range(nsteps):
        if use_cfl and wl.n_species <= 2:
            # mercury::local_time_step is the two-ion form; one ion is the same step with an empty second species
            # (its sound speed is zero and its velocity term vanishes, so the first species sets every cell's step)
            W = [r.to_prim(u, wl.gamma) for u in U]
            if wl.n_species == 1:
                W.append(np.zeros_like(W[0]))
            Btot = r.cell_vector(Phi) + Badd
            dt_ref = r.local_time_step(wl.gamma, p.cfl, p.inver_MA2, p.rho_floor_dt, W[0], W[1], Btot)
            dt_gpu = st.cfl_dt()
            assert dt_gpu == dt_ref or abs(dt_gpu - dt_ref) <= 1e-14 * dt_ref
            dt = dt_ref
        else:
            dt = 0.2 * float(np.min(np.asarray(h["edge_len"])))
        used = st.step(dt)
        assert used == dt
        r.rk2_step(rp, U, Phi, wl.PhiAdd, Badd, dt)
        for s in range(wl.n_species):
            e = rel_err(st.U(s), U[s])
            assert e < TOL, (k, s, e)
        assert rel_err(st.Phi(), Phi) < TOL
    dmesh_div = dm.div_b(st.Phi())["max_rel"]
    return dmesh_div


def test_step_box_single_ion():
    from mpcns_uns_b200 import workloads
    wl = workloads.box(8)
    div = run_pair(wl, BOX_TAGS, ("outflow", {}, (1.0, 0.0, 0.0)), 4)
    assert div < 1e-12


def test_step_shell_two_ions_cfl():
    from mpcns_uns_b200 import workloads
    wl = workloads.shell(4, 5, r_in=1.0, r_out=6.0)
    div = run_pair(wl, SHELL_TAGS, SHELL_BC, 4)
    assert div < 1e-12


def test_step_box_three_species_mixed_bc():
    from mpcns_uns_b200 import workloads
    from mpcns_uns_b200.mesh import HostMesh
    wl = workloads.box(5)
    h = HostMesh.box(5, 5, 5, tets=True, jitter=0.1, seed=4).compute_geometry().boundary(*MIXED_BOX_BC)
    rng = np.random.default_rng(9)
    U = []
    for s in range(3):
        W = np.zeros((h.n_cells, 5))
        W[:, 0] = rng.uniform(0.5, 1.5, h.n_cells) * 10.0 ** (-s)
        W[:, 1:4] = np.asarray(MIXED_BOX_BC[2]) + rng.uniform(-0.1, 0.1, (h.n_cells, 3))
        W[:, 4] = 0.1 * W[:, 0]
        U.append(workloads.to_cons(W, wl.gamma).ravel())
    wl.mesh, wl.U, wl.n_species = h, U, 3
    wl.Phi = workloads.d1(h, workloads.fourier_potential(h, 5))
    wl.PhiAdd = np.asarray(h["face_area"]) @ np.array([0.05, -0.1, 0.2])
    wl.fs = [(1.0, 0.5, 0.2, -0.3, 0.1), (0.1, 0.5, 0.2, -0.3, 0.01), (0.01, 0.5, 0.2, -0.3, 0.001)]
    wl.mass = [1.0, 16.0, 32.0]
    wl.u_inf, wl.B_imf = MIXED_BOX_BC[2], (0.05, -0.1, 0.2)
    div = run_pair(wl, BOX_TAGS, MIXED_BOX_BC, 3, use_cfl=False)
    assert div < 1e-12


@pytest.mark.parametrize("induce", [0.0, 0.8])
def test_step_shell_two_ions_lorentz(induce):
    """The two-ion step with the J x B force (and, induce > 0, the Strang-split exact gyration)."""
    from mpcns_uns_b200 import workloads
    wl = workloads.shell(4, 5, r_in=1.0, r_out=6.0)
    div = run_pair(wl, SHELL_TAGS, SHELL_BC, 4, params_kw=dict(lorentz=True, induce_coeff=induce, inver_MA2=0.7))
    assert div < 1e-12


@pytest.mark.parametrize("induce", [0.0, 0.8])
def test_step_shell_two_ions_all_sources(induce):
    """The two-ion step with every model term of the hot path on: J x B, the ambipolar force and edge EMF,
    the chemistry terms of seeded source fields (and, induce > 0, the Strang-split gyration)."""
    from helpers import SOURCE_EXTRA, source_fields
    from mpcns_uns_b200 import workloads
    wl = workloads.shell(4, 5, r_in=1.0, r_out=6.0)
    div = run_pair(wl, SHELL_TAGS, SHELL_BC, 4, params_kw=dict(lorentz=True, induce_coeff=induce, inver_MA2=0.7, extra=SOURCE_EXTRA),
                   fields=source_fields(wl.mesh.n_cells))
    assert div < 1e-12


def test_step_shell_ten_ions():
    """The ten-ion shell (masses 1..44, log-uniform upstream densities, crustal background field): five
    species groups per stage."""
    from mpcns_uns_b200 import workloads
    wl = workloads.ten_ion(4, 5)
    div = run_pair(wl, SHELL_TAGS, SHELL_BC, 3, use_cfl=False)
    assert div < 1e-12


def test_step_shell_two_ions_wall_table():
    """The two-ion step with the Dirichlet wall table of the ten-ion solver's GhostFn on every wall face."""
    from mpcns_uns_b200 import workloads
    wl = workloads.shell(4, 5, r_in=1.0, r_out=6.0)
    wall = workloads.wall_states(wl.mesh, [f[0] for f in wl.fs], wl.mass, seed=3)
    assert wall[0].size > 0
    div = run_pair(wl, SHELL_TAGS, SHELL_BC, 4, params_kw=dict(lorentz=True, induce_coeff=0.8, inver_MA2=0.7), wall=wall)
    assert div < 1e-12


def test_step_shell_ten_ions_wall_table():
    """Ten ions (five species groups per stage) with the wall table: each group reads its own species' states."""
    from mpcns_uns_b200 import workloads
    wl = workloads.ten_ion(4, 5)
    wall = workloads.wall_states(wl.mesh, [f[0] for f in wl.fs], wl.mass, seed=4)
    div = run_pair(wl, SHELL_TAGS, SHELL_BC, 3, use_cfl=False, wall=wall)
    assert div < 1e-12


def test_config1_box_twenty_cfl_steps():
    """Config 1 itself: the unit cube of 16^3 hexahedra x 6 tetrahedra (24,576 cells), interior nodes jittered
    +-0.15 h with seed 0, rho = 1, p = 0.1, u = (1, 0, 0) with 1% seeded noise, gamma = 5/3, B = d1 of 8 seeded
    Fourier modes of amplitude 0.05 plus B0 = (0.1, 0.2, 0), outflow everywhere; the reference's limited
    least-squares gradients with the Barth-Jespersen limiter (the only limiter the reference has), Rusanov
    fluxes, UCT EMF and CT; 20 steps at CFL 0.4 (device CFL step equal to the reference's).  Every step agrees
    to 1e-12 and div B stays at round-off."""
    from mpcns_uns_b200 import workloads
    wl = workloads.box(16)
    assert wl.mesh.n_cells == 24576 and wl.cfl == 0.4 and wl.steps == 20
    div = run_pair(wl, BOX_TAGS, ("outflow", {}, wl.u_inf), wl.steps, params_kw=dict(cfl=wl.cfl))
    assert div < 1e-12


def test_shell_two_ions_config2_construction_221k_cells():
    """The config-2 construction at 6 x 16 x 16 x 24 x 6 (221,184 cells): two ions (H+, Na+ of mass 23 with the
    seeded exosphere profile), inflow u = (-8, 0, 0), IMF and the offset dipole in the background flux, wall at
    r = 1, the J x B force and the Strang-split exact gyration; 5 steps at the device's CFL 0.4 step.  The
    reference side's mesh is built by the reference's own generator (the cubed sphere cut into tetrahedra by
    its ComplexBuilder), which must be this mesh entity for entity (same topology hash)."""
    from mpcns_uns_b200 import workloads
    wl = workloads.shell(16, 24, r_in=1.0, r_out=6.0, sources=True)
    assert wl.mesh.n_cells == 221184
    rm = ref.RefMesh.shell_tets(16, 24, 1.0, 6.0, wl.extra["stretch"])
    div = run_pair(wl, SHELL_TAGS, SHELL_BC, 5, ref_mesh=rm,
                   params_kw=dict(cfl=wl.cfl, lorentz=wl.lorentz, induce_coeff=wl.induce_coeff, inver_MA2=wl.inver_MA2))
    assert div < 1e-12


def test_semi_implicit_step_matches_reference():
    """mercury::Solver::step_first_order (time_order = 1, MercuryUns/driver/Solver.cpp:228-277) on the device: the
    opening half-step gyration, forward Euler of both ions with the J x B force, the EMF from the Hall + resistive
    ImplicitInduction::solve (frozen total field and n_e,eff of the step, inflow edges Dirichlet, warm start), CT
    with it and the closing gyration, against the same sequence of the reference's functions.  The first step's
    fluid update precedes the solve and is bit-for-bit the reference's; after it, the states agree to the
    solve's tolerance (the EMF is a GMRES iterate)."""
    from mpcns_uns_b200 import gpu, workloads
    wl = workloads.shell(4, 5, r_in=1.0, r_out=6.0)
    h = wl.mesh
    r = ref_twin(h, SHELL_TAGS).boundary(*SHELL_BC)
    dm = gpu.DeviceMesh(h)
    p = gpu.step_params(2, wl.gamma, fs=wl.fs, mass=wl.mass, u_inf=wl.u_inf, B_imf=wl.B_imf, lorentz=1, induce_coeff=1.0,
                        inver_MA2=1.0)
    st = gpu.ResidentState(dm, p)
    st.set(wl.U, wl.Phi, wl.PhiAdd)
    r_e = np.linalg.norm(np.asarray(h["edge_mid"]), axis=1)
    m_edge = np.where(r_e < 1.5, 1e-2, 1e-4) / np.asarray(h["star1"])
    kw = dict(hall=True, hall_coef=0.5, hall_r_min=1.0, hall_r_max=1.6, rtol=1e-10, max_it=300, restart=30)
    di = gpu.DeviceInduction(dm, m_edge, **kw)
    ri = ref.RefInduction(r, **kw)
    ri.set_m(m_edge)
    rp = ref_params(p)
    U = [np.array(u, np.float64) for u in wl.U]
    Phi = np.array(wl.Phi, np.float64)
    Badd = r.cell_vector(wl.PhiAdd)
    for k in range(4):
        W = [r.to_prim(u, wl.gamma) for u in U]
        Btot = r.cell_vector(Phi) + Badd
        dt = r.local_time_step(wl.gamma, p.cfl, p.inver_MA2, p.rho_floor_dt, W[0], W[1], Btot)
        assert abs(st.cfl_dt() - dt) <= 1e-12 * dt
        used, itd, rrd = st.step_semi_implicit(di, dt=dt)
        itr, rrr = r.first_order_step(rp, ri, U, Phi, wl.PhiAdd, Badd, dt)
        assert used == dt
        assert rrd <= 1e-10 and rrr <= 1e-10, (k, rrd, rrr)
        assert abs(itd - itr) <= 2, (k, itd, itr)
        tol = TOL if k == 0 else 1e-8
        for s in range(2):
            # the first step's fluid update precedes the solve; the closing gyration uses the step's own field
            assert rel_err(st.U(s), U[s]) < tol, (k, s, rel_err(st.U(s), U[s]))
        assert rel_err(st.Phi(), Phi) < 1e-8, (k, rel_err(st.Phi(), Phi))
    assert dm.div_b(st.Phi())["max_rel"] < 1e-12


def test_semi_implicit_step_rejects_other_states():
    from mpcns_uns_b200 import gpu, workloads
    wl = workloads.shell(3, 4, r_in=1.0, r_out=6.0)
    dm = gpu.DeviceMesh(wl.mesh)
    di = gpu.DeviceInduction(dm, None, hall=True, hall_coef=0.5)
    for kw, match in ((dict(precision="mixed"), "FP64"), (dict(), None)):
        p = gpu.step_params(2, wl.gamma, fs=wl.fs, mass=wl.mass, u_inf=wl.u_inf, B_imf=wl.B_imf, **kw)
        st = gpu.ResidentState(dm, p)
        st.set(wl.U, wl.Phi, wl.PhiAdd)
        if match:
            with pytest.raises(gpu.MhdError, match=match):
                st.step_semi_implicit(di, dt_max=1.0)
    other = gpu.DeviceMesh(wl.mesh)
    di2 = gpu.DeviceInduction(other, None, hall=True, hall_coef=0.5)
    with pytest.raises(gpu.MhdError, match="another mesh"):
        st.step_semi_implicit(di2, dt_max=1.0)
