"""The ten-ion (Mars) source pieces and step on the device against mars::MarsSolver itself.

The reference side is the compiled MarsSolver (oracle/ref/ref_shim.cpp: RefMars) on the same mesh, each
phase of its step run alone: prepare, local_dt_, fluid_and_sources_ (gradients and fluxes through its
wall GhostFn, J x B and ambipolar force), emf_, implicit_sources_, floors_, and the step without the
photochemistry.  The device side is mpcns_uns_b200.mars.MarsStep over the C-ABI passes.  FP64 agreement
1e-12 relative per ion and per array after several steps.
"""
import numpy as np
import pytest

from helpers import SHELL_TAGS, ref_twin, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("reference checker not built (make -C oracle ref)", allow_module_level=True)

NS = 10


def _setup(second_order=1, ambipolar=1, seed=0, hall=0, induction=None):
    from mpcns_uns_b200 import gpu, workloads
    from mpcns_uns_b200.mars import MarsStep
    from mpcns_uns_b200.mesh import HostMesh
    h = HostMesh.shell(4, 5, 1.04, 3.0, tets=True).compute_geometry()
    r = ref_twin(h, SHELL_TAGS)
    m = ref.RefMars(r, [f"is_Hall_Efield={hall}", f"second_order={second_order}", "CFL=0.4", f"is_Ambipolar_Efield={ambipolar}"])
    P = m.params
    u_inf = (P["sw_ux"], P["sw_uy"], P["sw_uz"])
    B_imf = (P["sw_Bx"], P["sw_By"], P["sw_Bz"])
    h.boundary("outflow", {"inner": "wall", "outer": "farfield"}, u_inf)
    fk, em = m.boundary()
    assert np.array_equal(np.asarray(h["face_kind"]), fk) and np.array_equal(np.asarray(h["edge_mode"]), em)
    dm = gpu.DeviceMesh(h)
    # the solver's initial state (solar-wind H+, the other ions at the floor) with seeded H+ density
    # perturbations of 10 % and trace heavy ions (1e-6..1e-4) moving with the H+; an induced field of a few
    # Fourier modes.  (States far from this, e.g. dense heavy ions next to the floor-density wall ghosts, drive
    # densities negative, which the reference's floors turn into unbounded velocities.)
    rng = np.random.default_rng(seed)
    U = m.get("U").reshape(NS, -1, 5)
    U[4] *= (1.0 + 0.1 * rng.uniform(-1.0, 1.0, U.shape[1]))[:, None]
    for s in range(NS):
        if s != 4:
            rho = 10.0 ** rng.uniform(-6, -4, U.shape[1])
            U[s, :, 0] = rho
            U[s, :, 1:4] = rho[:, None] * U[4, :, 1:4] / U[4, :, 0:1]
            U[s, :, 4] = U[4, :, 4] / U[4, :, 0] * rho
    U = U.ravel()
    Phi = 0.05 * workloads.d1(h, workloads.fourier_potential(h, seed + 1, amp=0.2, B0=(0.0, 0.0, 0.0)))
    m.set("U", U)
    m.set("Phi", Phi)
    scales = dict(P, u_inf=u_inf, B_imf=B_imf)
    if induction:
        m.set_induction(induction["rtol"], induction["max_it"], induction["restart"])
    st = MarsStep(dm, scales, m.freestream, m.wall_table(), m.get("neutral"), m.get("PhiAdd"), induction=induction)
    st.set(U, Phi)
    return h, m, st


def _np(t):
    return t.detach().cpu().numpy()


def _per_ion(a, b, tol=TOL):
    a, b = np.asarray(a).reshape(NS, -1), np.asarray(b).reshape(NS, -1)
    for s in range(NS):
        e = rel_err(a[s], b[s])
        assert e < tol, (s, e)


@pytest.fixture(scope="module")
def case():
    return _setup()


def test_mars_prepare(case):
    h, m, st = case
    m.prepare()
    q = st.prepare()
    _per_ion(_np(q["W"]), m.get("W"))
    for k in ("Bind", "Btot", "ne", "ne_eff", "pe", "uplus", "PhiTot", "J", "dpe"):
        assert rel_err(_np(q[k]), m.get(k)) < TOL, k


def test_mars_time_step(case):
    h, m, st = case
    m.prepare()
    q = st.prepare()
    d = st.dm.mars_time_step(st.mp, st.sc["cfl"], st.U, q["W"], q["Btot"], q["uplus"])
    d_ref = m.local_dt()
    assert d == d_ref or abs(d - d_ref) <= 1e-14 * d_ref


@pytest.mark.parametrize("second_order,ambipolar", [(1, 1), (0, 1), (1, 0)])
def test_mars_rhs_and_emf(second_order, ambipolar):
    """fluid_and_sources_ (fluxes through the wall GhostFn + J x B + ambipolar force) and emf_."""
    h, m, st = _setup(second_order, ambipolar, seed=2)
    m.prepare()
    q = st.prepare()
    m.fluid_and_sources(1e-3)
    _per_ion(_np(st.rhs(q)), m.get("rhs"))
    assert rel_err(_np(st.emf(q)), m.emf()) < TOL


@pytest.mark.parametrize("dt", [1e-3, 0.5])
def test_mars_implicit_sources(dt):
    """The point-implicit gyration, drag and thermal relaxation, also at a step far above the explicit limits."""
    h, m, st = _setup(seed=3)
    U0 = m.get("U")
    m.prepare()
    q = st.prepare()
    m.implicit_sources(dt)
    st.dm.mars_implicit_sources(st.mp, q["Btot"], st.neutral, dt, st.U)
    _per_ion(_np(st.U), m.get("U"))
    assert rel_err(m.get("U"), U0) > 1e-6   # the sources act


def test_mars_floors():
    h, m, st = _setup(seed=4)
    rng = np.random.default_rng(44)
    U = m.get("U").reshape(NS, -1, 5)
    pick = rng.random(U.shape[:2]) < 0.05
    U[pick, 0] = rng.uniform(-1e-9, 1e-11, int(pick.sum()))     # below the floor, some negative
    low = rng.random(U.shape[:2]) < 0.05
    U[low, 4] = 0.5 * (U[low, 1] ** 2 + U[low, 2] ** 2 + U[low, 3] ** 2) / np.maximum(U[low, 0], 1e-10) * 0.9
    m.set("U", U.ravel())
    st.set(U.ravel(), st.Phi)
    m.floors()
    st.dm.mars_floors(st.mp, st.U)
    _per_ion(_np(st.U), m.get("U"))


def test_mars_step():
    """Three steps of MarsSolver::step without the photochemistry: U of every ion and Phi, div B."""
    h, m, st = _setup(seed=5)
    for k in range(3):
        dt_ref = m.step_nochem()
        dt = st.step()
        assert dt == dt_ref or abs(dt - dt_ref) <= 1e-14 * dt_ref
        _per_ion(_np(st.U), m.get("U"))
        assert rel_err(_np(st.Phi), m.get("Phi")) < TOL
    assert st.dm.div_b(st.Phi)["max_rel"] < 1e-12


def test_mars_step_with_hall_solve():
    """MarsSolver::step with the Hall term on (is_Hall_Efield=1): the implicit edge EMF of the semi-implicit
    induction solve (ImplicitInduction with the solver's hall_scale, no taper, wall and inflow edges fixed,
    warm start across steps) between the explicit update and Faraday.  Both sides run GMRES(20) to 1e-10:
    the dot products round differently (block reductions against sequential sums), so the solve agrees to
    its tolerance, not bit for bit; U and Phi after three steps to 1e-8, iterations within 2."""
    ind = dict(rtol=1e-10, max_it=400, restart=20)
    h, m, st = _setup(seed=5, hall=1, induction=ind)
    assert m.params["hall"] == 1.0 and m.params["hall_scale"] > 0 and st.ind is not None
    for k in range(3):
        dt_ref = m.step_nochem()
        dt = st.step()
        assert abs(dt - dt_ref) <= 1e-12 * dt_ref
        it_ref, rr_ref = m.last_solve()
        it, rr = st.last_solve
        assert rr <= 1e-10 and rr_ref <= 1e-10, (rr, rr_ref)
        assert abs(it - it_ref) <= 2, (k, it, it_ref)
        _per_ion(_np(st.U), m.get("U"), 1e-8)
        assert rel_err(_np(st.Phi), m.get("Phi")) < 1e-8
    assert st.dm.div_b(st.Phi)["max_rel"] < 1e-12


def test_mars_step_hall_default_settings():
    """The same step at the reference's own GMRES settings (rtol 1e-4, 100 iterations, restart 20): both
    sides stop at the tolerance after the same number of iterations within 2, and the states agree to the
    solve's tolerance."""
    h, m, st = _setup(seed=6, hall=1)
    for k in range(2):
        m.step_nochem()
        st.step()
        it_ref, rr_ref = m.last_solve()
        it, rr = st.last_solve
        assert rr <= 1e-4 and rr_ref <= 1e-4 and abs(it - it_ref) <= 2, (it, it_ref, rr, rr_ref)
        assert rel_err(_np(st.Phi), m.get("Phi")) < 1e-4
