"""Block-Jacobi ILU(0) preconditioner of the induction solve on the device (Config::ind_ilu; mhd::ImplicitInduction,
Common/induction/ImplicitInduction.cpp:209-297) against the compiled reference.

The pattern, the factors of factor_precond and the result of apply_precond keep the reference's
arithmetic row by row, so they must agree bit for bit.  Solves are compared as in test_gpu_induction.py
(the Gram-Schmidt dots round differently): true residual at most rtol, E within a small multiple of
rtol, iterations within two.  The reference's own test of the preconditioners (tests/test_implicit_induction.cpp
block (4)) is repeated on the device.
"""
import numpy as np
import pytest

from helpers import BOX_TAGS, MIXED_BOX_BC, SHELL_BC, SHELL_TAGS, rel_err, ref_twin
from mpcns_uns_b200.mesh import HostMesh

pytestmark = pytest.mark.gpu

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


def _pair(name, hall, seed=12, precision="fp64", **kw):
    from mpcns_uns_b200.gpu import DeviceInduction
    h, r, dm = _mesh(name)
    rng = np.random.default_rng(seed)
    m_edge = rng.uniform(0.5, 2.0, h.n_edges) / np.asarray(h["star1"])
    taper = dict(hall_r_min=1.0, hall_r_max=1.6) if name == "shell" else dict(hall_r_min=-100.0, hall_r_max=-99.0)
    args = dict(hall=hall, hall_coef=0.5, rtol=1e-10, max_it=300, restart=15, **taper)
    args.update(kw)
    ri = ref.RefInduction(r, ilu=True, **args)
    ri.set_m(m_edge)
    di = DeviceInduction(dm, m_edge, precision=precision, **args)
    di.set_ilu(True, 0.3)
    B0 = rng.uniform(-1, 1, 3 * h.n_cells)
    ne = rng.uniform(0.5, 2.0, h.n_cells)
    ri.set_frozen_state(B0, ne)
    di.set_frozen_state(B0, ne)
    return h, ri, di, rng


def _bits(a):
    return np.asarray(a, np.float64).view(np.int64)


@pytest.mark.parametrize("name", ["box", "box_hex", "shell"])
def test_factors_and_apply_bit_exact(name):
    h, ri, di, rng = _pair(name, True)
    arr = di.ilu_arrays()
    assert np.array_equal(arr["pc_ptr"], ri.array("pc_ptr"))
    assert np.array_equal(arr["pc_col"], ri.array("pc_col"))
    assert np.array_equal(arr["pc_diag"], ri.array("pc_diag"))
    assert np.array_equal(_bits(arr["pc_coef"]), _bits(ri.array("pc_coef")))
    dir_bc = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    assert dir_bc.any()
    for dirichlet in (np.zeros(h.n_edges, np.int8), dir_bc):
        for dt in (0.05, 3.0):
            v = rng.uniform(-1, 1, h.n_edges)
            z_ref = ri.precond(dt, dirichlet, v)
            di.ilu_factor(dt, dirichlet)
            z = _np(di.ilu_apply(v, dirichlet))
            assert np.array_equal(_bits(di.ilu_arrays()["pc_val"]), _bits(ri.array("pc_val"))), (dt, int(dirichlet.sum()))
            assert np.array_equal(_bits(z), _bits(z_ref)), (dt, int(dirichlet.sum()))
            assert np.all(z[dirichlet != 0] == 0.0)


def test_factor_repeats_and_shift():
    """Factoring again (another dt, the same handle) and a zero shift both stay bit-exact."""
    h, ri, di, rng = _pair("box", False)
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    v = rng.uniform(-1, 1, h.n_edges)
    for dt in (0.5, 0.01, 0.5):
        di.ilu_factor(dt, dirichlet)
        assert np.array_equal(_bits(_np(di.ilu_apply(v, dirichlet))), _bits(ri.precond(dt, dirichlet, v)))
    r2 = ref.RefInduction(_mesh("box")[1], ilu=True, ilu_shift=0.0, rtol=1e-8)
    r2.set_m(np.asarray(ri.array("m")))
    di.set_ilu(True, 0.0)
    di.ilu_factor(0.2, dirichlet)
    assert np.array_equal(_bits(_np(di.ilu_apply(v, dirichlet))), _bits(r2.precond(0.2, dirichlet, v)))


def _true_rel_res(di, phi, Ee, E, dirichlet, dt):
    b = Ee + _np(di.apply_F(phi))
    r = b - _np(di.apply_A(E, dt))
    r[dirichlet != 0] = 0.0
    return np.linalg.norm(r) / np.linalg.norm(b)


@pytest.mark.parametrize("name,hall", [("box", False), ("box", True), ("shell", True), ("box_hex", True)])
def test_solve_with_ilu_matches_reference(name, hall):
    h, ri, di, rng = _pair(name, hall)
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    phi = rng.uniform(-1, 1, h.n_faces)
    Ee = rng.uniform(-1, 1, h.n_edges)
    dt = 0.05
    for warm in (False, True):
        Er, itr, rrr = ri.solve(phi, Ee, dirichlet, dt, warm)
        Ed, itd, rrd = di.solve(phi, Ee, dirichlet, dt, warm)
        Ed = _np(Ed)
        assert rrd <= 1e-10 and rrr <= 1e-10, (rrd, rrr)
        assert abs(itd - itr) <= 2, (warm, itd, itr)
        assert rel_err(Ed, Er) <= 1e-8
        assert _true_rel_res(di, phi, Ee, Ed, dirichlet, dt) <= 2e-10
        assert np.array_equal(Ed[dirichlet != 0], Ee[dirichlet != 0])


def test_mixed_precision_with_ilu_refines_to_fp64():
    h, ri, di, rng = _pair("shell", True, precision="mixed")
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    phi = rng.uniform(-1, 1, h.n_faces)
    Ee = rng.uniform(-1, 1, h.n_edges)
    Er, itr, _ = ri.solve(phi, Ee, dirichlet, 0.05, False)
    Ed, itd, rrd = di.solve(phi, Ee, dirichlet, 0.05, False)
    Ed = _np(Ed)
    assert rrd <= 1e-10
    assert _true_rel_res(di, phi, Ee, Ed, dirichlet, 0.05) <= 2e-10
    assert rel_err(Ed, Er) <= 1e-8
    assert itd <= 2 * itr + 15


def test_reference_preconditioner_test_on_device():
    """tests/test_implicit_induction.cpp block (4) of the reference on the device: the 12^3 box on [-1, 1]^3,
    resistive with inver_Rem = 10 everywhere (eta window -100 .. 100), dt 0.02, rtol 1e-10, GMRES(30), Phi = d1
    of A = sin(7x + 3y) cos(5z) at the edge midpoints, E_expl = 0, no Dirichlet edges: ILU(0) takes at most twice
    Jacobi's iterations, a warm-started repeat at most 2, and the two solutions agree to 1e-7."""
    from mpcns_uns_b200.gpu import DeviceInduction, DeviceMesh
    h = HostMesh.box(12, 12, 12, lo=(-1, -1, -1), hi=(1, 1, 1)).compute_geometry().boundary("outflow")
    r = ref_twin(h, BOX_TAGS).boundary("outflow")
    ri = ref.RefInduction(r, resistive=True, inver_Rem=10.0, eta_r_inner=-100.0, eta_r_outer=100.0, eta_width=1.0, ilu=True,
                          rtol=1e-10, max_it=400, restart=30)
    m_edge = ri.array("m")
    mid = np.asarray(h["edge_mid"])
    A = np.sin(7.0 * mid[:, 0] + 3.0 * mid[:, 1]) * np.cos(5.0 * mid[:, 2])
    fp, fi, fs = np.asarray(h["f2e_ptr"]), np.asarray(h["f2e_idx"]), np.asarray(h["f2e_sgn"])
    Phi = np.array([sum(fs[k] * A[fi[k]] for k in range(fp[f], fp[f + 1])) for f in range(h.n_faces)])
    E0 = np.zeros(h.n_edges)
    dirichlet = np.zeros(h.n_edges, np.int8)
    dm = DeviceMesh(h)
    sols, its = {}, {}
    for ilu in (False, True):
        di = DeviceInduction(dm, m_edge, rtol=1e-10, max_it=400, restart=30)
        if ilu:
            di.set_ilu(True, 0.3)
        E, its[ilu], rr = di.solve(Phi, E0, dirichlet, 0.02, False)
        assert rr <= 1e-10
        sols[ilu] = _np(E)
        if ilu:
            _, itw, _ = di.solve(Phi, E0, dirichlet, 0.02, True)
            assert itw <= 2
    assert its[True] <= 2 * its[False], its
    sc = max(np.max(np.abs(sols[False])), 1.0)
    assert np.max(np.abs(sols[True] - sols[False])) < 1e-7 * sc
    # and the reference's own ILU(0) solve of the same system takes the same iterations to within 2
    _, itr, _ = ri.solve(Phi, E0, dirichlet, 0.02, False)
    assert abs(itr - its[True]) <= 2, (itr, its[True])


def test_switching_ilu_off_restores_jacobi():
    """Turning ILU(0) off again gives the Jacobi solve's iterates (the captured restart cycle is rebuilt)."""
    from mpcns_uns_b200.gpu import DeviceInduction
    h, ri, di, rng = _pair("box", True)
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    phi = rng.uniform(-1, 1, h.n_faces)
    Ee = rng.uniform(-1, 1, h.n_edges)
    plain = DeviceInduction(_mesh("box")[2], ri.array("m"), hall=True, hall_coef=0.5, hall_r_min=-100.0, hall_r_max=-99.0,
                            rtol=1e-10, max_it=300, restart=15)
    plain.set_frozen_state(*_frozen(h, 12))
    di.set_frozen_state(*_frozen(h, 12))
    Ej, itj, _ = plain.solve(phi, Ee, dirichlet, 0.05, False)
    Ei, iti, _ = di.solve(phi, Ee, dirichlet, 0.05, False)
    di.set_ilu(False)
    Eo, ito, _ = di.solve(phi, Ee, dirichlet, 0.05, False)
    assert ito == itj
    assert np.array_equal(_bits(_np(Eo)), _bits(_np(Ej)))
    di.set_ilu(True)
    Ei2, iti2, _ = di.solve(phi, Ee, dirichlet, 0.05, False)
    assert iti2 == iti and np.array_equal(_bits(_np(Ei2)), _bits(_np(Ei)))


def _frozen(h, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, 3 * h.n_cells), rng.uniform(0.5, 2.0, h.n_cells)


def test_bounded_wait_gives_up_and_recovers():
    """A row that never raises its flag (test hook): the rows that read it give up after the wait limit, the
    call returns MHD_ECUDA, and the handle factors and applies correctly afterwards."""
    from mpcns_uns_b200.gpu import MhdError
    h, ri, di, rng = _pair("box", True)
    dirichlet = np.zeros(h.n_edges, np.int8)
    v = rng.uniform(-1, 1, h.n_edges)
    di.ilu_debug(0.05, 0)
    with pytest.raises(MhdError, match="timed out"):
        di.ilu_factor(0.05, dirichlet)
    di.ilu_debug(2.0, -1)
    di.ilu_factor(0.05, dirichlet)
    assert np.array_equal(_bits(_np(di.ilu_apply(v, dirichlet))), _bits(ri.precond(0.05, dirichlet, v)))
