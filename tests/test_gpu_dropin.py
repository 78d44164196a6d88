"""The drop-in library: the reference's own C++ signatures with device bodies (mpcns_uns_b200/lib/libmhd_dropin.so).

A test driver (oracle/ref/dropin_driver.cpp, linked against the drop-in and not against the reference) calls
mhd::fluid_flux_rhs, mhd::Stencil::limited_gradients, uns::reconstruct_cell_vector, mhd::add_ideal_emf,
mhd::faraday_update(_edge_dt), mhd::div_b and mhd::ImplicitInduction::solve on the reference's own objects
(LocalMesh, Geometry, BoundaryInfo, Config, Stencil, ImplicitInduction built by the compiled reference), so
every call lands on the device through the reference's declarations.  The reference's CPU bodies run on the
same objects and inputs: 1e-12 relative (FP64; the solve to GMRES tolerance, as the other solve tests).
"""
import ctypes
import os

import numpy as np
import pytest

from helpers import BOX_TAGS, MIXED_BOX_BC, SHELL_BC, random_prims, ref_twin, rel_err
from mpcns_uns_b200.mesh import HostMesh

pytestmark = pytest.mark.gpu
TOL = 1e-12
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "libdropin_driver.so")

ref = pytest.importorskip("oracle.ref")
if not ref.available() or not os.path.exists(DRIVER):
    pytest.skip("reference checker or drop-in driver not built (make -C oracle ref dropin)", allow_module_level=True)

vp, dbl, i32 = ctypes.c_void_p, ctypes.c_double, ctypes.c_int32
_drv = None


def drv():
    global _drv
    if _drv is None:
        from mpcns_uns_b200 import gpu
        gpu.lib()    # the device library first (its context and stream set-up), then the driver on top of it
        L = ctypes.CDLL(DRIVER)
        L.drv_last_error.restype = ctypes.c_char_p
        for name, args in {"drv_attach": [vp] * 3, "drv_detach": [vp],
                           "drv_flux_rhs": [vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, vp],
                           "drv_limited_gradients": [vp, vp, vp, vp, vp, ctypes.c_int, vp, ctypes.c_int, dbl, vp],
                           "drv_cell_vector": [vp, vp, vp, i32, vp], "drv_ideal_emf": [vp, vp, vp, vp, vp, vp, vp, dbl, vp],
                           "drv_faraday": [vp, vp, vp, dbl], "drv_faraday_edge_dt": [vp, vp, vp, vp],
                           "drv_div_b": [vp, vp, vp, vp],
                           "drv_ind_solve": [vp, vp, vp, vp, ctypes.c_int64, dbl, vp, ctypes.POINTER(i32), ctypes.POINTER(dbl)],
                           "drv_ind_solve_dte": [vp, vp, vp, vp, ctypes.c_int64, vp, vp, ctypes.POINTER(i32),
                                                 ctypes.POINTER(dbl)]}.items():
            getattr(L, name).argtypes = args
            getattr(L, name).restype = ctypes.c_int
        _drv = L
    return _drv


def call(fn, *args):
    rc = fn(*args)
    assert rc == 0, drv().drv_last_error().decode()


def _p(a):
    return None if a is None else a.ctypes.data_as(vp)


def _mk(name):
    if name == "box_tets_mixed":
        h = HostMesh.box(5, 4, 3, tets=True, jitter=0.1, seed=3)
        bc, tags = MIXED_BOX_BC, BOX_TAGS
        h.compute_geometry().boundary(*bc)
        r = ref_twin(h, tags).boundary(*bc)
    elif name == "box_hex":
        r = ref.RefMesh.box(4, 3, 5, hi=(2.0, 1.5, 2.5)).boundary(*MIXED_BOX_BC)
    else:
        r = ref.RefMesh.shell_tets(4, 5, 1.0, 6.0, 1.3).boundary(*SHELL_BC)
    return r


MESHES = ["box_tets_mixed", "box_hex", "shell_tets"]
_cache = {}


@pytest.fixture(params=MESHES)
def mesh(request):
    if request.param not in _cache:
        r = _mk(request.param)
        objs = r.objects()
        call(drv().drv_attach, objs[0], objs[1], objs[2])
        _cache[request.param] = (r, objs)
    return _cache[request.param]


def test_fluid_signatures(mesh):
    r, (lm, geo, bc, cfg, st) = mesh
    rng = np.random.default_rng(71)
    nc = r.n_cells
    for s, fs in ((0, (1.0, 0.5, 0.2, -0.3, 0.1)), (1, (0.1, 0.5, 0.2, -0.3, 0.01))):
        W = random_prims(nc, rng)
        fsa = np.asarray(fs, np.float64)
        for rel in (0.0, 0.3):
            g_ref = r.limited_gradients(W, s, fs, True, rel)
            g = np.zeros(15 * nc)
            call(drv().drv_limited_gradients, st, lm, geo, bc, _p(W), s, _p(fsa), 1, rel, _p(g))
            assert rel_err(g, g_ref) < TOL, (s, rel)
        rhs_ref = r.flux_rhs(W, g_ref, s, fs, 5.0 / 3.0)       # also sets the Config's gamma the driver passes on
        rhs = np.zeros(5 * nc)
        call(drv().drv_flux_rhs, lm, geo, bc, cfg, s, _p(fsa), _p(W), _p(g_ref), _p(rhs))
        assert rel_err(rhs, rhs_ref) < TOL, s


def test_induction_signatures(mesh):
    r, (lm, geo, bc, cfg, st) = mesh
    rng = np.random.default_rng(72)
    nc, nf, ne = r.n_cells, r.n_faces, r.n_edges
    phi = rng.uniform(-1, 1, nf)
    b = np.zeros(3 * nc)
    call(drv().drv_cell_vector, lm, geo, _p(phi), nc, _p(b))
    assert rel_err(b, r.cell_vector(phi)) < TOL
    u, Bt, Bi = (rng.uniform(-1, 1, 3 * nc) for _ in range(3))
    pt, pi = rng.uniform(-1, 1, nf), rng.uniform(-1, 1, nf)
    E0 = rng.uniform(-1, 1, ne)
    E = E0.copy()
    call(drv().drv_ideal_emf, lm, geo, _p(u), _p(Bt), _p(Bi), _p(pt), _p(pi), 0.5, _p(E))
    assert rel_err(E, r.ideal_emf(u, Bt, Bi, pt, pi, 0.5, E0.copy())) < TOL
    B = rng.uniform(-1, 1, nf)
    Bn = B.copy()
    call(drv().drv_faraday, lm, _p(E0), _p(Bn), 0.37)
    assert rel_err(Bn, r.faraday(E0, B, 0.37)) < TOL
    dte = rng.uniform(0.1, 1.0, ne)
    Bn = B.copy()
    call(drv().drv_faraday_edge_dt, lm, _p(E0), _p(dte), _p(Bn))
    assert rel_err(Bn, r.faraday_edge_dt(E0, dte, B)) < TOL
    for ex in (None, rng.uniform(-1, 1, nf)):
        o = np.zeros(3)
        call(drv().drv_div_b, lm, _p(B), _p(ex), _p(o))
        rr = r.div_b(B, ex)
        assert abs(o[0] - rr["max_abs"]) <= TOL * rr["max_abs"] and abs(o[1] - rr["max_rel"]) <= TOL * rr["max_rel"]
        assert int(o[2]) == rr["worst_cell_gid"]


@pytest.mark.parametrize("variant", ["jacobi", "ilu", "dt_edge", "ideal"])
def test_implicit_induction_solve_signature(mesh, variant):
    """ImplicitInduction::solve on the reference's object: the drop-in hands the object's resistivity, Hall
    coefficient per cell (alpha_ = taper hall_coef / n_e,eff) and frozen field to the device solve, with the
    object's preconditioner (Jacobi, or block ILU(0) when its Config asked for it), its per-edge pseudo-time
    step when the call passes one, and its implicit ideal part (Config::implicit_ideal, set_ideal_state)."""
    r, (lm, geo, bc, cfg, st) = mesh
    rng = np.random.default_rng(73)
    nc, nf, ne = r.n_cells, r.n_faces, r.n_edges
    ri = ref.RefInduction(r, hall=True, hall_coef=0.5, hall_r_min=-100.0, hall_r_max=-99.0, rtol=1e-10, max_it=200, restart=15,
                          ilu=variant == "ilu", implicit_ideal=variant == "ideal", cuct=0.5)
    ri.set_m(rng.uniform(0.5, 2.0, ne) / np.asarray(r["star1"]))
    ri.set_frozen_state(rng.uniform(-1, 1, 3 * nc), rng.uniform(0.5, 2.0, nc))
    phi = rng.uniform(-1, 1, nf)
    Ee = rng.uniform(-1, 1, ne)
    dirichlet = (np.asarray(r["edge_mode"]) == 2).astype(np.int8)
    if variant == "ideal":
        ri.set_ideal_state(rng.uniform(-1, 1, 3 * nc), (np.asarray(r["edge_mode"]) == 0).astype(np.int8))
    E = np.zeros(ne)
    it, rr = i32(), dbl()
    if variant == "dt_edge":
        dte = rng.uniform(0.02, 0.08, ne)
        E_ref, it_ref, rr_ref = ri.solve_dt_edge(phi, Ee, dirichlet, dte, False)
        call(drv().drv_ind_solve_dte, ri.object(), _p(phi), _p(Ee), _p(dirichlet), ne, _p(dte), _p(E), ctypes.byref(it),
             ctypes.byref(rr))
    else:
        E_ref, it_ref, rr_ref = ri.solve(phi, Ee, dirichlet, 0.05, False)
        call(drv().drv_ind_solve, ri.object(), _p(phi), _p(Ee), _p(dirichlet), ne, 0.05, _p(E), ctypes.byref(it), ctypes.byref(rr))
    assert rr.value <= 1e-10 and rr_ref <= 1e-10
    # the upwind ideal part makes the operator strongly non-normal: the rounding differences of the two
    # Gram-Schmidt variants move the iteration where the residual crosses rtol by a few more steps
    spread = max(2, it_ref // 10) if variant == "ideal" else 2
    assert abs(it.value - it_ref) <= spread, (it.value, it_ref)
    assert rel_err(E, E_ref) <= 1e-8
    assert np.array_equal(E[dirichlet != 0], Ee[dirichlet != 0])
