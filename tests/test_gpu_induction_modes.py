"""The two off-by-default forms of mhd::ImplicitInduction on the device against the compiled reference
(Common/induction/ImplicitInduction.cpp): the per-edge pseudo-time step of solve (dt_edge, the steady mode's
local time stepping) and the implicit ideal part of F (Config::implicit_ideal, set_ideal_state / ideal_linear).

The operator keeps the reference's summation order, so apply_F, apply_A and ideal_linear agree to 1e-13
relative (FP64); solves agree as the other solve tests do: the true residual at most rtol, E within a small
multiple of rtol, iterations within two.
"""
import numpy as np
import pytest

from helpers import BOX_TAGS, MIXED_BOX_BC, SHELL_BC, SHELL_TAGS, rel_err, ref_twin
from mpcns_uns_b200.mesh import HostMesh

pytestmark = pytest.mark.gpu
OP_TOL = 1e-13

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("reference checker not built (make -C oracle ref)", allow_module_level=True)


def _np(t):
    return t.detach().cpu().numpy()


_cache = {}


def _mesh(name):
    if name not in _cache:
        from mpcns_uns_b200.gpu import DeviceMesh
        if name == "box":
            h, bc, tags = HostMesh.box(6, 5, 4, tets=True, jitter=0.1, seed=8), MIXED_BOX_BC, BOX_TAGS
        elif name == "box_hex":
            h, bc, tags = HostMesh.box(5, 4, 4, jitter=0.1, seed=5), MIXED_BOX_BC, BOX_TAGS
        else:
            h, bc, tags = HostMesh.shell(5, 6, 0.8, 4.0, 1.3, n_solid=1, tets=True), SHELL_BC, SHELL_TAGS
        h.compute_geometry().boundary(*bc)
        _cache[name] = (h, ref_twin(h, tags).boundary(*bc), DeviceMesh(h))
    return _cache[name]


def _pair(name, hall=True, resistive=True, ideal=False, seed=21, precision="fp64", **kw):
    from mpcns_uns_b200.gpu import DeviceInduction
    h, r, dm = _mesh(name)
    rng = np.random.default_rng(seed)
    m_edge = rng.uniform(0.5, 2.0, h.n_edges) / np.asarray(h["star1"]) if resistive else None
    taper = dict(hall_r_min=1.0, hall_r_max=1.6) if name == "shell" else dict(hall_r_min=-100.0, hall_r_max=-99.0)
    args = dict(hall=hall, hall_coef=0.5, rtol=1e-10, max_it=300, restart=15, **taper)
    args.update(kw)
    ri = ref.RefInduction(r, implicit_ideal=ideal, cuct=0.5, **args)
    if resistive:
        ri.set_m(m_edge)
    di = DeviceInduction(dm, m_edge, precision=precision, **args)
    B0 = rng.uniform(-1, 1, 3 * h.n_cells)
    ne = rng.uniform(0.5, 2.0, h.n_cells)
    ri.set_frozen_state(B0, ne)
    di.set_frozen_state(B0, ne)
    if ideal:
        u = rng.uniform(-1, 1, 3 * h.n_cells)
        mask = (np.asarray(h["edge_mode"]) == 0).astype(np.int8)
        ri.set_ideal_state(u, mask)
        di.set_ideal_state(u, mask, 0.5)
    return h, ri, di, rng


def _check_solve(h, got, want, Ee, dirichlet, rtol=1e-10):
    (Ed, itd, rrd), (Er, itr, rrr) = got, want
    Ed = _np(Ed)
    assert rrd <= rtol and rrr <= rtol, (rrd, rrr)
    assert abs(itd - itr) <= 2, (itd, itr)
    assert rel_err(Ed, Er) <= 1e-8
    assert np.array_equal(Ed[dirichlet != 0], Ee[dirichlet != 0])


@pytest.mark.parametrize("name,hall,resistive", [("box", True, True), ("box", False, True), ("shell", True, True),
                                                 ("box_hex", True, False)])
def test_solve_dt_edge_matches_reference(name, hall, resistive):
    """solve(..., dt_edge): A x = x + F(d1 diag(dt_e) x), Jacobi 1 / (1 + dt_e m d2); cold and warm."""
    h, ri, di, rng = _pair(name, hall, resistive)
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    phi = rng.uniform(-1, 1, h.n_faces)
    Ee = rng.uniform(-1, 1, h.n_edges)
    dte = rng.uniform(0.005, 0.05, h.n_edges)
    for warm in (False, True):
        _check_solve(h, di.solve_dt_edge(phi, Ee, dirichlet, dte, warm), ri.solve_dt_edge(phi, Ee, dirichlet, dte, warm), Ee,
                     dirichlet)


def test_solve_dt_edge_ignores_ilu_and_returns_to_scalar_dt():
    """The reference builds ILU(0) for a scalar dt only (:317): with ILU on, a dt_edge solve is still the
    Jacobi one; the scalar solves before and after it keep their own iterates."""
    h, ri, di, rng = _pair("box")
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    phi = rng.uniform(-1, 1, h.n_faces)
    Ee = rng.uniform(-1, 1, h.n_edges)
    dte = rng.uniform(0.005, 0.05, h.n_edges)
    di.set_ilu(True, 0.3)
    E1, it1, _ = di.solve(phi, Ee, dirichlet, 0.05, False)
    _check_solve(h, di.solve_dt_edge(phi, Ee, dirichlet, dte, False), ri.solve_dt_edge(phi, Ee, dirichlet, dte, False), Ee,
                 dirichlet)
    E2, it2, _ = di.solve(phi, Ee, dirichlet, 0.05, False)
    assert it2 == it1 and np.array_equal(_np(E2), _np(E1))


@pytest.mark.parametrize("name", ["box", "shell", "box_hex"])
def test_ideal_part_of_the_operator_matches_reference(name):
    h, ri, di, rng = _pair(name, ideal=True)
    for _ in range(2):
        phi = rng.uniform(-1, 1, h.n_faces)
        assert rel_err(_np(di.ideal_linear(phi)), ri.ideal_linear(phi)) <= OP_TOL
        assert rel_err(_np(di.apply_F(phi)), ri.apply_F(phi)) <= OP_TOL
        x = rng.uniform(-1, 1, h.n_edges)
        for dt in (0.05, 3.0):
            assert rel_err(_np(di.apply_A(x, dt)), ri.apply_A(x, dt)) <= OP_TOL
    # the part off again: F is the Hall + resistive operator alone
    di.set_ideal_state(None, None)
    ri_plain = _pair(name, ideal=False)[1]
    phi = rng.uniform(-1, 1, h.n_faces)
    assert rel_err(_np(di.apply_F(phi)), ri_plain.apply_F(phi)) <= OP_TOL


@pytest.mark.parametrize("name,precision", [("box", "fp64"), ("shell", "fp64"), ("box", "mixed")])
def test_solve_with_ideal_part_matches_reference(name, precision):
    h, ri, di, rng = _pair(name, ideal=True, precision=precision)
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    phi = rng.uniform(-1, 1, h.n_faces)
    Ee = rng.uniform(-1, 1, h.n_edges)
    for warm in (False, True):
        _check_solve(h, di.solve(phi, Ee, dirichlet, 0.02, warm), ri.solve(phi, Ee, dirichlet, 0.02, warm), Ee, dirichlet)


def test_ideal_part_with_dt_edge():
    """The steady mode's combination: implicit ideal part and per-edge pseudo-time step (Solver.cpp:428-463)."""
    h, ri, di, rng = _pair("box", ideal=True)
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    phi = rng.uniform(-1, 1, h.n_faces)
    Ee = rng.uniform(-1, 1, h.n_edges)
    dte = np.full(h.n_edges, 0.03)
    _check_solve(h, di.solve_dt_edge(phi, Ee, dirichlet, dte, False), ri.solve_dt_edge(phi, Ee, dirichlet, dte, False), Ee,
                 dirichlet)
