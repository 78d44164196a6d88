"""The differentiated explicit run on the device: forward, tangent-linear and adjoint.

The reference has no adjoint, so the gradient is pinned by
  * the forward map itself: the FP64 step with the explicit resistive EMF against the compiled
    reference (ImplicitInduction::apply_F's resistive part added to the edge EMF), bit for bit;
  * the tangent-linear model's values against the forward run, bit for bit;
  * dot-product tests of the hand-written adjoint against the tangent-linear model, for one stage
    (every state and parameter direction) and for the whole run (the parameter directions);
  * central finite differences of J computed with the compiled reference's own step on the CPU.
"""
import numpy as np
import pytest

from helpers import SHELL_BC, SHELL_TAGS, ref_twin

pytestmark = pytest.mark.gpu

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("reference checker not built (make -C oracle ref)", allow_module_level=True)

DOT_TOL = 1e-10      # dot-product identities (round-off of sums over the whole mesh)
FD_TOL = 1e-6        # adjoint against central differences of the reference


def _case(n_steps=4, checkpoint_every=2):
    from mpcns_uns_b200 import workloads
    case = workloads.adjoint_case(ncube=4, nr=5, n_steps=n_steps, checkpoint_every=checkpoint_every, r_lo=1.0, r_hi=2.5)
    assert case.mask.sum() > 10
    return case


def _state(case):
    from mpcns_uns_b200 import gpu
    wl = case.wl
    dm = gpu.DeviceMesh(wl.mesh)
    p = gpu.step_params(wl.n_species, wl.gamma, fs=wl.fs, mass=wl.mass, u_inf=wl.u_inf, B_imf=wl.B_imf)
    st = gpu.ResidentState(dm, p)
    st.set(wl.U, wl.Phi, wl.PhiAdd)
    return dm, st


def _soa(U_list, nc):
    return np.concatenate([np.asarray(u).reshape(nc, 5).T.ravel() for u in U_list])


def _ref_params(wl, u_inf, m_res):
    rp = ref.StepParams()
    rp.n_species, rp.second_order, rp.gamma, rp.rho_floor, rp.p_floor, rp.cuct = wl.n_species, 1, wl.gamma, 1e-10, 1e-12, 0.5
    rp.M_ref, rp.ne_floor = 1.0, 0.01
    rp.u_inf[:] = list(u_inf)
    rp.B_imf[:] = list(wl.B_imf)
    for s in range(wl.n_species):
        rp.mass[s] = wl.mass[s]
        f = list(wl.fs[s])
        f[1:4] = list(u_inf)
        rp.fs[s][:] = f
    rp.lorentz, rp.induce_coeff, rp.inver_MA2 = 0, 0.0, 1.0
    rp.m_res = m_res.ctypes.data
    return rp


def _initial(wl, r, u_inf):
    """The run's initial state: the workload's flow shifted by u_inf - wl.u_inf (uniform_flow)."""
    from mpcns_uns_b200 import workloads
    sh = np.asarray(u_inf, np.float64) - np.asarray(wl.u_inf, np.float64)
    U = []
    for u in wl.U:
        W = r.to_prim(u, wl.gamma).reshape(-1, 5).copy()
        W[:, 1:4] = W[:, 1:4] + sh
        U.append(workloads.to_cons(W, wl.gamma).ravel())
    return U


def _ref_J(case, r, eta, u_inf, dt):
    """J of the run with the compiled reference's step (CPU)."""
    from mpcns_uns_b200 import workloads
    wl = case.wl
    m_res = workloads.edge_resistivity(wl.mesh, eta)
    rp = _ref_params(wl, u_inf, m_res)
    Badd = r.cell_vector(wl.PhiAdd)
    U = _initial(wl, r, u_inf)
    Phi = np.array(wl.Phi, np.float64)
    for _ in range(case.n_steps):
        r.rk2_step(rp, U, Phi, wl.PhiAdd, Badd, dt)
    B = (r.cell_vector(Phi) + Badd).reshape(-1, 3)
    V = np.asarray(wl.mesh["cell_volume"])
    return float(np.sum(case.mask * (B * B).sum(1) * V)), U, Phi


def test_resistive_step_matches_reference():
    """The FP64 step with the explicit resistive EMF, device against the compiled reference, bit for bit."""
    from mpcns_uns_b200 import gpu, workloads
    case = _case()
    wl = case.wl
    r = ref_twin(wl.mesh, SHELL_TAGS).boundary(*SHELL_BC)
    dm, st = _state(case)
    m_res = workloads.edge_resistivity(wl.mesh, case.eta)
    st.set_resistivity(m_res)
    dt = st.cfl_dt()
    rp = _ref_params(wl, wl.u_inf, m_res)
    Badd = r.cell_vector(wl.PhiAdd)
    U = [np.array(u, np.float64) for u in wl.U]
    Phi = np.array(wl.Phi, np.float64)
    for _ in range(3):
        st.step(dt)
        r.rk2_step(rp, U, Phi, wl.PhiAdd, Badd, dt)
    for s in range(2):
        assert np.array_equal(st.U(s), U[s])
    assert np.array_equal(st.Phi(), Phi)
    assert np.abs(Phi).max() > 0


def test_forward_and_tangent_values():
    """J of the forward run equals the compiled reference's J bit for bit, and the tangent-linear run's
    values (J and the final state) equal the forward run's."""
    from mpcns_uns_b200 import gpu
    case = _case()
    wl = case.wl
    r = ref_twin(wl.mesh, SHELL_TAGS).boundary(*SHELL_BC)
    dm, st = _state(case)
    dt = 0.8 * st.cfl_dt()
    fn = gpu.DeviceFunction(st, case.eta, case.mask, case.n_steps, case.checkpoint_every, dt)
    J = fn.forward()
    Jr, Ur, Pr = _ref_J(case, r, case.eta, wl.u_inf, dt)
    assert abs(J - Jr) <= 1e-13 * abs(Jr)   # the device sums J in another order
    assert np.array_equal(st.Phi(), Pr)
    for s in range(2):
        assert np.array_equal(st.U(s), Ur[s])
    Jt, dJ = fn.tangent(np.ones(wl.mesh.n_cells) * 1e-3, (0.1, 0.2, -0.3))
    assert Jt == J
    assert np.array_equal(st.Phi(), Pr)
    for s in range(2):
        assert np.array_equal(st.U(s), Ur[s])
    assert np.isfinite(dJ) and dJ != 0.0


def test_stage_dot_product():
    """<lUt, dUt> + <lE, dE> = <lU, dU> + <lPhi, dPhi> + <l_eta, d_eta> + <l_u, d_u> for one stage, every
    direction at once, at a state two steps into the run."""
    from mpcns_uns_b200 import gpu
    case = _case()
    wl = case.wl
    nc, nf, ne = wl.mesh.n_cells, wl.mesh.n_faces, wl.mesh.n_edges
    dm, st = _state(case)
    dt = 0.8 * st.cfl_dt()
    fn = gpu.DeviceFunction(st, case.eta, case.mask, 2, 1, dt)
    fn.forward()   # two steps: a state with structure in both ions and the field
    U = _soa([st.U(s) for s in range(2)], nc)
    Phi = st.Phi()
    rng = np.random.default_rng(3)
    dU = rng.standard_normal(U.size) * (np.abs(U) + 1e-3)
    dPhi = rng.standard_normal(nf) * (np.abs(Phi).mean() + 1e-3)
    d_eta = rng.standard_normal(nc) * case.eta
    d_u = rng.standard_normal(3)
    dUt, dE = fn.stage_tangent(U, Phi, dU, dPhi, d_eta, d_u)
    lUt = rng.standard_normal(U.size)
    lE = rng.standard_normal(ne)
    lU, lP, le, lu = fn.stage_adjoint(U, Phi, lUt, lE)
    terms_out = np.concatenate([lUt * dUt, lE * dE])
    terms_in = np.concatenate([lU * dU, lP * dPhi, le * d_eta, lu * d_u])
    lhs, rhs = terms_out.sum(), terms_in.sum()
    scale = np.abs(terms_out).sum() + np.abs(terms_in).sum()
    assert abs(lhs - rhs) <= DOT_TOL * scale, (lhs, rhs, scale)
    # each parameter block on its own
    for kw, lam in ((dict(d_eta=d_eta), le @ d_eta), (dict(d_u=d_u), lu @ d_u)):
        z = np.zeros_like
        dUt2, dE2 = fn.stage_tangent(U, Phi, z(U), z(Phi), **kw)
        l2 = lUt @ dUt2 + lE @ dE2
        assert abs(l2 - lam) <= DOT_TOL * (np.abs(lUt * dUt2).sum() + np.abs(lE * dE2).sum() + 1e-300), (kw.keys(), l2, lam)


def test_run_dot_product_and_checkpointing():
    """The adjoint gradient of the whole run against the tangent-linear run along random parameter
    directions; the same gradient for every checkpoint spacing."""
    from mpcns_uns_b200 import gpu
    case = _case(n_steps=5)
    wl = case.wl
    nc = wl.mesh.n_cells
    dm, st = _state(case)
    dt = 0.8 * st.cfl_dt()
    rng = np.random.default_rng(11)
    grads = []
    for K in (1, 2, 5):
        st.set(wl.U, wl.Phi)
        fn = gpu.DeviceFunction(st, case.eta, case.mask, case.n_steps, K, dt)
        fn.forward()
        grads.append(fn.backward())
        again = fn.backward()   # the recorded segments are gone: recomputed from the checkpoints
        # (atomic accumulation: equal up to the order of the additions)
        assert np.allclose(again[0], grads[-1][0], rtol=1e-12, atol=1e-13 * np.abs(grads[-1][0]).max())
        assert np.allclose(again[1], grads[-1][1], rtol=1e-12, atol=1e-13 * np.abs(grads[-1][1]).max())
    ge, gu = grads[0]
    for g2e, g2u in grads[1:]:
        assert np.allclose(g2e, ge, rtol=1e-12, atol=1e-13 * np.abs(ge).max())
        assert np.allclose(g2u, gu, rtol=1e-12, atol=1e-13 * np.abs(gu).max())
    assert np.abs(ge).max() > 0 and np.abs(gu).max() > 0
    for _ in range(3):
        d_eta = rng.standard_normal(nc) * case.eta
        d_u = rng.standard_normal(3)
        J, dJ = fn.tangent(d_eta, d_u)
        adj = ge @ d_eta + gu @ d_u
        assert abs(adj - dJ) <= DOT_TOL * (np.abs(ge * d_eta).sum() + np.abs(gu * d_u).sum()), (adj, dJ)


def test_gradient_against_reference_finite_differences():
    """Central differences of J computed by the compiled reference's step on the CPU, along seeded directions,
    against the device adjoint.  J is smooth in eta (the resistive EMF is linear in it): h = 1e-4 relative,
    where the differences are not yet limited by round-off.  In u_inf the scheme is only piecewise smooth
    (limiter and upwind switches): h = 1e-7 relative stays clear of the switches near this state (at 1e-6 a
    few directions cross one and differ by a few 1e-6)."""
    from mpcns_uns_b200 import gpu
    case = _case(n_steps=4)
    wl = case.wl
    nc = wl.mesh.n_cells
    r = ref_twin(wl.mesh, SHELL_TAGS).boundary(*SHELL_BC)
    dm, st = _state(case)
    dt = 0.8 * st.cfl_dt()
    fn = gpu.DeviceFunction(st, case.eta, case.mask, case.n_steps, 2, dt)
    fn.forward()
    ge, gu = fn.backward()
    rng = np.random.default_rng(17)
    u0 = np.asarray(wl.u_inf, np.float64)
    for k in range(6):
        d_eta = rng.standard_normal(nc) * case.eta
        d_u = rng.standard_normal(3) * np.linalg.norm(u0)
        if k < 2:
            d_u, h = 0 * d_u, 1e-4        # resistivity alone
        elif k < 4:
            d_eta, h = 0 * d_eta, 1e-7    # inflow velocity alone
        else:
            h = 1e-7
        Jp = _ref_J(case, r, case.eta + h * d_eta, u0 + h * d_u, dt)[0]
        Jm = _ref_J(case, r, case.eta - h * d_eta, u0 - h * d_u, dt)[0]
        fd = (Jp - Jm) / (2 * h)
        adj = ge @ d_eta + gu @ d_u
        assert abs(adj - fd) <= FD_TOL * abs(fd), (k, adj, fd)


def _switch_fd(fn, ge, gu, eta, u0, d_eta, d_u, h):
    """Central difference of the device forward run along (d_eta, d_u) from the double-double J, its
    relative distance from the adjoint, and the entities whose discrete choices differ between the runs."""
    fn.set_params(eta=eta + h * d_eta, u_inf=u0 + h * d_u)
    fn.forward()
    Jp, sp = fn.last_J(), fn.switches()
    fn.set_params(eta=eta - h * d_eta, u_inf=u0 - h * d_u)
    fn.forward()
    Jm, sm = fn.last_J(), fn.switches()
    fd = fn.central_difference(Jp, Jm, h)
    adj = float(ge @ d_eta + gu @ d_u)
    return abs(adj - fd) / abs(fd), fn.switch_flips(sp, sm)


def test_switch_log_is_silent_and_repeatable():
    """The switch log changes nothing that the forward run computes (J bit for bit with and without it),
    two runs with the same parameters make the same choices everywhere, and a run whose inflow velocity
    moves by 1e-3 crosses limiter, wave-speed and upwind switches that the log sees."""
    from mpcns_uns_b200 import gpu
    case = _case(n_steps=4)
    dm, st = _state(case)
    fn = gpu.DeviceFunction(st, case.eta, case.mask, case.n_steps, 2, 0.8 * st.cfl_dt())
    J0 = fn.forward()
    hi0 = fn.last_J()
    fn.switch_log(True)
    J1 = fn.forward()
    a = fn.switches()
    J2 = fn.forward()
    b = fn.switches()
    assert J0 == J1 == J2 and fn.last_J() == hi0
    assert hi0[0] == J0 and abs(hi0[1]) <= 0.5 * np.spacing(J0)
    assert fn.switch_flips(a, b) == {"limiter": 0, "flux": 0, "edge": 0, "floor": 0, "face_emf": 0}
    assert all(int(np.count_nonzero(v)) > 0 for k, v in a.items() if k != "floor")
    u0 = np.asarray(case.wl.u_inf, np.float64)
    fn.set_params(u_inf=u0 * (1 + 1e-3))
    fn.forward()
    c = fn.switches()
    flips = fn.switch_flips(a, c)
    assert flips["limiter"] > 0 and flips["flux"] > 0 and flips["edge"] > 0 and flips["face_emf"] > 0, flips
    fn.switch_log(False)
    with pytest.raises(gpu.MhdError, match="switch log is off"):
        fn.switches()


def test_finite_differences_at_h_1e6_split_by_switches():
    """Central differences at h = 1e-6 (relative to the seeded directions) on a 36,864-cell shell, 8 steps,
    split by the switch log: every direction along which the J(p + h d) and J(p - h d) runs made the same
    discrete choices everywhere agrees with the adjoint to 1e-6.  The resistivity directions are switch-free
    by construction (without model sources the fluid does not see B, and the induction is linear in eta);
    directions with an inflow-velocity part cross limiter and upwind switches at this h on this mesh, and
    their differences are reported, not bounded (J is only piecewise smooth there)."""
    from mpcns_uns_b200 import gpu, workloads
    case = workloads.adjoint_case(ncube=8, nr=16, n_steps=8, checkpoint_every=4)
    wl = case.wl
    nc = wl.mesh.n_cells
    assert nc == 36864
    dm, st = _state(case)
    fn = gpu.DeviceFunction(st, case.eta, case.mask, case.n_steps, case.checkpoint_every, st.cfl_dt())
    fn.forward()
    ge, gu = fn.backward()
    fn.switch_log(True)
    rng = np.random.default_rng(23)
    u0 = np.asarray(wl.u_inf, np.float64)
    free, crossing = [], []
    for k in range(10):
        d_eta = rng.standard_normal(nc) * case.eta
        d_u = rng.standard_normal(3) * np.linalg.norm(u0)
        if k < 6:
            d_u = 0 * d_u
        err, flips = _switch_fd(fn, ge, gu, case.eta, u0, d_eta, d_u, 1e-6)
        (free if sum(flips.values()) == 0 else crossing).append((k, err, flips))
    assert len(free) >= 6, (free, crossing)
    for k, err, flips in free:
        assert err <= FD_TOL, (k, err)
    for k, err, flips in crossing:
        assert k >= 6 and flips["limiter"] + flips["edge"] > 0, (k, err, flips)
