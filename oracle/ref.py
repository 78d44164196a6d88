"""ctypes binding of oracle/_ref/libmhdref.so: the reference's own hot-path C++ compiled in place.

TEST INFRASTRUCTURE ONLY.  Used by tests/, tests/golden/make_golden.py and bench.py's CPU
baseline; never by the shipped library.  Build it with `make -C oracle ref` (needs the
reference tree; the built .so then runs anywhere this image runs).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_ref", "libmhdref.so")

_lib = None
vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double


def available() -> bool:
    return os.path.exists(SO)


class IndParams(ctypes.Structure):
    _fields_ = [("resistive", i32), ("hall", i32), ("max_it", i32), ("restart", i32), ("ilu", i32), ("implicit_ideal", i32),
                ("inver_Rem", dbl), ("eta_r_inner", dbl), ("eta_r_outer", dbl), ("eta_width", dbl),
                ("hall_coef", dbl), ("hall_r_min", dbl), ("hall_r_max", dbl), ("rtol", dbl), ("ilu_shift", dbl), ("cuct", dbl)]


class StepParams(ctypes.Structure):
    _fields_ = [("n_species", i32), ("second_order", i32), ("gamma", dbl), ("rho_floor", dbl), ("p_floor", dbl),
                ("cuct", dbl), ("M_ref", dbl), ("ne_floor", dbl), ("rel_limit", dbl), ("u_inf", dbl * 3),
                ("B_imf", dbl * 3), ("mass", dbl * 16), ("fs", (dbl * 5) * 16), ("lorentz", i32), ("pad", i32),
                ("induce_coeff", dbl), ("inver_MA2", dbl), ("m_res", ctypes.c_void_p), ("ambipolar", i32), ("chemistry", i32),
                ("pressure_coef", dbl), ("a1_Na", dbl), ("a4", dbl), ("a5", dbl), ("a6", dbl), ("state_coeff_H", dbl),
                ("state_coeff_Na", dbl), ("T_ref", dbl), ("Tn0", dbl), ("photo", ctypes.c_void_p), ("vst", ctypes.c_void_p),
                ("n_wall", i32), ("pad2", i32), ("wall_faces", ctypes.c_void_p), ("wall_prims", ctypes.c_void_p),
                ("first_order", i32), ("ind_iterations", i32), ("ind", ctypes.c_void_p), ("ind_rel_res", dbl)]


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("reference checker not built: make -C oracle ref")
        L = ctypes.CDLL(SO)
        L.ref_last_error.restype = ctypes.c_char_p
        for name, args, res in [
            ("ref_mesh_from_cells", [i32, vp, i32, vp, vp, vp, vp, i32, vp, vp, vp, i32, vp], vp),
            ("ref_mesh_box", [i32, i32, i32, vp, vp], vp),
            ("ref_mesh_shell", [i32, i32, i32, dbl, dbl, dbl], vp),
            ("ref_mesh_shell_tets", [i32, i32, i32, dbl, dbl, dbl], vp),
            ("ref_mesh_objects", [vp, vp], ctypes.c_int),
            ("ref_ind_object", [vp], vp),
            ("ref_mesh_hanging_box", [i32, i32, i32, vp, vp, i32], vp),
            ("ref_mesh_free", [vp], None),
            ("ref_mesh_counts", [vp, vp], None),
            ("ref_topology_hash", [vp], ctypes.c_uint64),
            ("ref_validate", [vp, vp], None),
            ("ref_check_geometry", [vp, vp], None),
            ("ref_array", [vp, ctypes.c_char_p, vp], i64),
            ("ref_boundary_build", [vp, ctypes.c_char_p, i32, vp, vp, vp], ctypes.c_int),
            ("ref_to_prim", [vp, i64, dbl, dbl, dbl, vp], None),
            ("ref_limited_gradients", [vp, vp, i32, vp, i32, dbl, vp], ctypes.c_int),
            ("ref_flux_rhs", [vp, dbl, i32, vp, vp, vp, vp], ctypes.c_int),
            ("ref_mars_create", [vp, i32, vp], vp),
            ("ref_mars_free", [vp], None),
            ("ref_mars_params", [vp, vp], None),
            ("ref_mars_freestream", [vp, vp], None),
            ("ref_mars_size", [vp, ctypes.c_char_p], ctypes.c_int64),
            ("ref_mars_get", [vp, ctypes.c_char_p, vp], ctypes.c_int),
            ("ref_mars_set", [vp, ctypes.c_char_p, vp], ctypes.c_int),
            ("ref_mars_prepare", [vp], ctypes.c_int),
            ("ref_mars_local_dt", [vp, vp], ctypes.c_int),
            ("ref_mars_fluid_and_sources", [vp, dbl], ctypes.c_int),
            ("ref_mars_ambipolar_emf", [vp, vp], ctypes.c_int),
            ("ref_mars_implicit_sources", [vp, dbl], ctypes.c_int),
            ("ref_mars_floors", [vp], ctypes.c_int),
            ("ref_mars_emf", [vp, vp], ctypes.c_int),
            ("ref_mars_step_nochem", [vp, dbl, vp], ctypes.c_int),
            ("ref_mars_set_induction", [vp, dbl, i32, i32], ctypes.c_int),
            ("ref_mars_last_solve", [vp, vp, vp], None),
            ("ref_mars_wall_table", [vp, vp, vp], i32),
            ("ref_mars_boundary", [vp, vp, vp], None),
            ("ref_limited_gradients_wall", [vp, vp, i32, vp, i32, dbl, i32, vp, vp, vp], ctypes.c_int),
            ("ref_flux_rhs_wall", [vp, dbl, i32, vp, vp, vp, i32, vp, vp, vp], ctypes.c_int),
            ("ref_cell_vector", [vp, vp, vp], None),
            ("ref_ideal_emf", [vp, vp, vp, vp, vp, vp, dbl, vp], None),
            ("ref_faraday", [vp, vp, vp, dbl], None),
            ("ref_faraday_edge_dt", [vp, vp, vp, vp], None),
            ("ref_div_b", [vp, vp, vp, vp], None),
            ("ref_cell_current", [vp, vp, vp], None),
            ("ref_local_time_step", [vp, dbl, dbl, dbl, dbl, vp, vp, vp], dbl),
            ("ref_ind_create", [vp, ctypes.POINTER(IndParams)], vp),
            ("ref_ind_free", [vp], None),
            ("ref_ind_set_m", [vp, vp], None),
            ("ref_ind_array", [vp, ctypes.c_char_p, vp], i64),
            ("ref_ind_set_frozen", [vp, vp, vp], None),
            ("ref_ind_apply_F", [vp, vp, vp], None),
            ("ref_ind_apply_A", [vp, vp, dbl, vp], None),
            ("ref_ind_solve", [vp, vp, vp, vp, dbl, i32, vp, vp], i32),
            ("ref_ind_precond", [vp, dbl, vp, vp, vp], i32),
            ("ref_ind_set_ideal", [vp, vp, vp], None),
            ("ref_ind_ideal_linear", [vp, vp, vp], None),
            ("ref_ind_solve_dte", [vp, vp, vp, vp, vp, i32, vp, vp], i32),
            ("ref_rk2_step", [vp, ctypes.POINTER(StepParams), vp, vp, vp, vp, dbl], ctypes.c_int),
            ("ref_add_sources", [vp, ctypes.POINTER(StepParams), i32, vp, vp, vp, vp, vp, vp, vp, vp, dbl, vp], None),
            ("ref_electron_pressure_gradient", [vp, vp, vp, vp], None),
            ("ref_write_fields", [ctypes.c_char_p, ctypes.c_uint64, i32, vp, vp, vp, vp, vp], ctypes.c_int),
            ("ref_read_fields", [ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64)], i32),
            ("ref_fields_get", [i32, ctypes.c_char_p, i32, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i64), vp], None),
            ("ref_ambipolar_emf", [vp, ctypes.POINTER(StepParams), vp, vp, vp], None),
            ("ref_gyrate", [vp, ctypes.POINTER(StepParams), vp, dbl, vp, vp], None),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().ref_last_error().decode())


_INT = {"cell_material": np.int32, "face_tag": np.int32, "face_kind": np.int8, "edge_mode": np.int8,
        "ec_ptr": np.int64, "ec_cell": np.int32, "ec_misoriented": np.int32}
_VEC3 = {"x", "edge_vec", "edge_mid", "face_area", "face_center", "cell_center", "edge_dual_area"}


class RefMesh:
    """A reference LocalMesh (one rank) with its Geometry, BoundaryInfo and Stencil."""

    def __init__(self, h):
        if not h:
            raise RuntimeError(lib().ref_last_error().decode())
        self._h = ctypes.c_void_p(h)
        c = np.zeros(4, np.int32)
        lib().ref_mesh_counts(self._h, _p(c))
        self.n_nodes, self.n_edges, self.n_faces, self.n_cells = (int(v) for v in c)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ref_mesh_free(self._h)

    @classmethod
    def box(cls, nx, ny, nz, lo=(0, 0, 0), hi=(1, 1, 1)):
        lo_ = np.asarray(lo, np.float64)
        hi_ = np.asarray(hi, np.float64)
        return cls(lib().ref_mesh_box(nx, ny, nz, _p(lo_), _p(hi_)))

    @classmethod
    def shell(cls, ncube, nr, r_in=1.0, r_out=10.0, r_stretch=1.0, n_solid=0):
        return cls(lib().ref_mesh_shell(ncube, nr, n_solid, r_in, r_out, r_stretch))

    @classmethod
    def shell_tets(cls, ncube, nr, r_in=1.0, r_out=10.0, r_stretch=1.0, n_solid=0):
        """The reference's cubed-sphere shell with every hexahedron cut into 6 tetrahedra, built by the
        reference's ComplexBuilder alone (ref_mesh_shell_tets): the benchmark's shell without this
        library's mesh services."""
        return cls(lib().ref_mesh_shell_tets(ncube, nr, n_solid, r_in, r_out, r_stretch))

    @classmethod
    def hanging_box(cls, nx=5, ny=4, nz=4, hi=(5, 4, 4), sphere=(2.2, 1.8, 2.1, 1.3), level=2):
        hi_ = np.asarray(hi, np.float64)
        sp = np.asarray(sphere, np.float64)
        return cls(lib().ref_mesh_hanging_box(nx, ny, nz, _p(hi_), _p(sp), level))

    @classmethod
    def from_cells(cls, x, cells, material=None, tagged=(), tag_names=("",)):
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        cell_ptr, loop_ptr, nodes = [0], [0], []
        for cell in cells:
            for loop in cell:
                nodes.extend(int(v) for v in loop)
                loop_ptr.append(len(nodes))
            cell_ptr.append(len(loop_ptr) - 1)
        cell_ptr = np.asarray(cell_ptr, np.int64)
        loop_ptr = np.asarray(loop_ptr, np.int64)
        nodes = np.asarray(nodes, np.int32)
        mat = None if material is None else np.ascontiguousarray(material, np.int32)
        tptr, tnodes, tid = [0], [], []
        for t_nodes, t in tagged:
            tnodes.extend(int(v) for v in t_nodes)
            tptr.append(len(tnodes))
            tid.append(int(t))
        tptr = np.asarray(tptr, np.int64)
        tnodes = np.asarray(tnodes, np.int32)
        tid = np.asarray(tid, np.int32)
        names = (ctypes.c_char_p * len(tag_names))(*[n.encode() for n in tag_names])
        return cls(lib().ref_mesh_from_cells(len(x), _p(x), len(cells), _p(cell_ptr), _p(loop_ptr), _p(nodes), _p(mat),
                                             len(tid), _p(tptr), _p(tnodes), _p(tid), len(tag_names),
                                             ctypes.cast(names, ctypes.c_void_p)))

    @classmethod
    def from_flat(cls, x, cell_ptr, loop_ptr, loop_nodes, material, tagged=(), tag_names=("",)):
        """Generic polyhedra from flat builder arrays (see HostMesh.cell_loops_flat)."""
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        cell_ptr = np.ascontiguousarray(cell_ptr, np.int64)
        loop_ptr = np.ascontiguousarray(loop_ptr, np.int64)
        loop_nodes = np.ascontiguousarray(loop_nodes, np.int32)
        mat = np.ascontiguousarray(material, np.int32)
        tptr, tnodes, tid = [0], [], []
        for t_nodes, t in tagged:
            tnodes.extend(int(v) for v in t_nodes)
            tptr.append(len(tnodes))
            tid.append(int(t))
        tptr = np.asarray(tptr, np.int64)
        tnodes = np.asarray(tnodes, np.int32)
        tid = np.asarray(tid, np.int32)
        names = (ctypes.c_char_p * len(tag_names))(*[n.encode() for n in tag_names])
        return cls(lib().ref_mesh_from_cells(len(x), _p(x), len(cell_ptr) - 1, _p(cell_ptr), _p(loop_ptr), _p(loop_nodes),
                                             _p(mat), len(tid), _p(tptr), _p(tnodes), _p(tid), len(tag_names),
                                             ctypes.cast(names, ctypes.c_void_p)))

    def topology_hash(self):
        return int(lib().ref_topology_hash(self._h))

    def objects(self):
        """Addresses of the reference objects (LocalMesh, Geometry, BoundaryInfo, Config, Stencil) of this mesh."""
        out = (ctypes.c_void_p * 5)()
        _check(lib().ref_mesh_objects(self._h, out))
        return [out[i] for i in range(5)]

    def validate(self):
        o = np.zeros(5, np.int64)
        lib().ref_validate(self._h, _p(o))
        return dict(ok=bool(o[0]), euler=int(o[1]), d1d0=int(o[2]), d2d1=int(o[3]), boundary_faces=int(o[4]))

    def check_geometry(self):
        o = np.zeros(8)
        lib().ref_check_geometry(self._h, _p(o))
        return dict(ok=bool(o[0]), min_volume=o[1], max_volume=o[2], min_tet=o[3], max_closure=o[4],
                    nonpositive_volume=int(o[5]), nonpositive_star=int(o[6]), misoriented_dual=int(o[7]))

    def __getitem__(self, name):
        n = lib().ref_array(self._h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        if name.endswith("_ptr"):
            dt = np.int64
        elif name.endswith("_idx"):
            dt = np.int32
        elif name.endswith("_sgn"):
            dt = np.int8
        else:
            dt = _INT.get(name, np.float64)
        a = np.zeros(n, dt)
        lib().ref_array(self._h, name.encode(), _p(a))
        return a.reshape(-1, 3) if name in _VEC3 else a

    def boundary(self, bc_default="outflow", by_tag=None, u_inf=(0, 0, 0)):
        by_tag = dict(by_tag or {})
        tags = (ctypes.c_char_p * max(1, len(by_tag)))(*[k.encode() for k in by_tag])
        types = (ctypes.c_char_p * max(1, len(by_tag)))(*[v.encode() for v in by_tag.values()])
        u = np.asarray(u_inf, np.float64)
        _check(lib().ref_boundary_build(self._h, bc_default.encode(), len(by_tag), ctypes.cast(tags, ctypes.c_void_p),
                                        ctypes.cast(types, ctypes.c_void_p), _p(u)))
        return self

    # ------------------------------------------------------------- hot path
    def to_prim(self, U, gamma, rho_floor=1e-10, p_floor=1e-12):
        U = np.ascontiguousarray(U, np.float64)
        W = np.zeros_like(U)
        lib().ref_to_prim(_p(U), U.size // 5, gamma, rho_floor, p_floor, _p(W))
        return W

    def limited_gradients(self, W, species, fs, limit=True, rel_limit=0.0):
        W = np.ascontiguousarray(W, np.float64)
        fs_ = np.asarray(fs, np.float64)
        g = np.zeros(15 * self.n_cells)
        _check(lib().ref_limited_gradients(self._h, _p(W), species, _p(fs_), int(limit), rel_limit, _p(g)))
        return g

    def limited_gradients_wall(self, W, species, fs, faces, prims, limit=True, rel_limit=0.0):
        """limited_gradients with the Dirichlet wall table (prims: n_wall x 5 of this species)."""
        W = np.ascontiguousarray(W, np.float64)
        fs_ = np.asarray(fs, np.float64)
        fc = np.ascontiguousarray(faces, np.int32)
        pr = np.ascontiguousarray(prims, np.float64)
        g = np.zeros(15 * self.n_cells)
        _check(lib().ref_limited_gradients_wall(self._h, _p(W), species, _p(fs_), int(limit), rel_limit, fc.size, _p(fc), _p(pr), _p(g)))
        return g

    def flux_rhs_wall(self, W, grad, species, fs, gamma, faces, prims):
        """fluid_flux_rhs with the Dirichlet wall table (prims: n_wall x 5 of this species)."""
        W = np.ascontiguousarray(W, np.float64)
        grad = np.ascontiguousarray(grad, np.float64)
        fs_ = np.asarray(fs, np.float64)
        fc = np.ascontiguousarray(faces, np.int32)
        pr = np.ascontiguousarray(prims, np.float64)
        r = np.zeros(5 * self.n_cells)
        _check(lib().ref_flux_rhs_wall(self._h, gamma, species, _p(fs_), _p(W), _p(grad), fc.size, _p(fc), _p(pr), _p(r)))
        return r

    def flux_rhs(self, W, grad, species, fs, gamma):
        W = np.ascontiguousarray(W, np.float64)
        grad = np.ascontiguousarray(grad, np.float64)
        fs_ = np.asarray(fs, np.float64)
        r = np.zeros(5 * self.n_cells)
        _check(lib().ref_flux_rhs(self._h, gamma, species, _p(fs_), _p(W), _p(grad), _p(r)))
        return r

    def cell_vector(self, phi):
        phi = np.ascontiguousarray(phi, np.float64)
        o = np.zeros(3 * self.n_cells)
        lib().ref_cell_vector(self._h, _p(phi), _p(o))
        return o

    def ideal_emf(self, u, Btot, Bind, phitot, phiind, cuct=0.5, E=None):
        E = np.zeros(self.n_edges) if E is None else np.array(E, np.float64)
        arrs = [np.ascontiguousarray(a, np.float64) for a in (u, Btot, Bind, phitot, phiind)]
        lib().ref_ideal_emf(self._h, *[_p(a) for a in arrs], cuct, _p(E))
        return E

    def faraday(self, E, B, dt):
        E = np.ascontiguousarray(E, np.float64)
        B = np.array(B, np.float64)
        lib().ref_faraday(self._h, _p(E), _p(B), dt)
        return B

    def faraday_edge_dt(self, E, dt_edge, B):
        E = np.ascontiguousarray(E, np.float64)
        d = np.ascontiguousarray(dt_edge, np.float64)
        B = np.array(B, np.float64)
        lib().ref_faraday_edge_dt(self._h, _p(E), _p(d), _p(B))
        return B

    def div_b(self, B, extra=None):
        B = np.ascontiguousarray(B, np.float64)
        ex = None if extra is None else np.ascontiguousarray(extra, np.float64)
        o = np.zeros(3)
        lib().ref_div_b(self._h, _p(B), _p(ex), _p(o))
        return dict(max_abs=o[0], max_rel=o[1], worst_cell_gid=int(o[2]))

    def cell_current(self, B):
        B = np.ascontiguousarray(B, np.float64)
        J = np.zeros(3 * self.n_cells)
        lib().ref_cell_current(self._h, _p(B), _p(J))
        return J

    def local_time_step(self, gamma, cfl, inver_MA2, rho_floor_dt, WH, WNa, B):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (WH, WNa, B)]
        return lib().ref_local_time_step(self._h, gamma, cfl, inver_MA2, rho_floor_dt, *[_p(a) for a in arrs])

    def add_sources(self, params: StepParams, species, WH, WNa, up, B, J, dt, rhs, dpe=None, photo=None, vst=None):
        """mercury::add_sources (MercuryUns/fluid/MercurySources.cpp:13-63); rhs in place."""
        a = [None if x is None else np.ascontiguousarray(x, np.float64) for x in (WH, WNa, up, B, J, dpe, photo, vst)]
        lib().ref_add_sources(self._h, ctypes.byref(params), species, *[_p(x) for x in a], dt, _p(rhs))

    def electron_pressure_gradient(self, WH, WNa):
        """mercury::electron_pressure_gradient (MercuryUns/physics/Ambipolar.cpp:10-31)."""
        WH, WNa = (np.ascontiguousarray(x, np.float64) for x in (WH, WNa))
        out = np.zeros(3 * (WH.size // 5))
        lib().ref_electron_pressure_gradient(self._h, _p(WH), _p(WNa), _p(out))
        return out

    def ambipolar_emf(self, params: StepParams, WH, WNa, E):
        """mercury::AmbipolarEMF::add (Ambipolar.cpp:52-88): E minus the ambipolar EMF (a new array)."""
        E = np.array(E, np.float64)
        WH, WNa = (np.ascontiguousarray(x, np.float64) for x in (WH, WNa))
        lib().ref_ambipolar_emf(self._h, ctypes.byref(params), _p(WH), _p(WNa), _p(E))
        return E

    def gyrate(self, params: StepParams, B, dt, UH, UNa):
        """mercury::gyrate (MercuryUns/physics/Gyration.cpp); UH, UNa in place."""
        B = np.ascontiguousarray(B, np.float64)
        lib().ref_gyrate(self._h, ctypes.byref(params), _p(B), dt, _p(UH), _p(UNa))

    def rk2_step(self, params: StepParams, U_list, Phi, PhiAdd, BaddCell, dt):
        """One SSP-RK2 step of the hot path (Solver::step; with params.lorentz the J x B source and the
        Strang-split gyration of the two-ion model; with params.m_res the explicit resistive EMF
        E += ImplicitInduction::apply_F(Phi), resistive part, per-edge m_e); U_list and Phi in place."""
        arr = (ctypes.c_void_p * len(U_list))(*[a.ctypes.data for a in U_list])
        PhiAdd = np.ascontiguousarray(PhiAdd, np.float64)
        BaddCell = np.ascontiguousarray(BaddCell, np.float64)
        _check(lib().ref_rk2_step(self._h, ctypes.byref(params), ctypes.cast(arr, ctypes.c_void_p), _p(Phi), _p(PhiAdd),
                                  _p(BaddCell), dt))

    def first_order_step(self, params: StepParams, ind, U_list, Phi, PhiAdd, BaddCell, dt):
        """One semi-implicit step (Solver::step_first_order, MercuryUns/driver/Solver.cpp:228-277): forward
        Euler of the fluid, then the EMF from ind's ImplicitInduction::solve (frozen total field and n_e,eff of
        the step's prepare, inflow edges Dirichlet, the rhs's EMF as E_expl), CT with it, and with
        params.lorentz the Strang-split gyration; U_list and Phi in place -> (iterations, rel_res)."""
        params.first_order = 1
        params.ind = ind._h
        self.rk2_step(params, U_list, Phi, PhiAdd, BaddCell, dt)
        params.first_order = 0
        params.ind = None
        return params.ind_iterations, params.ind_rel_res


class RefInduction:
    """mhd::ImplicitInduction on a RefMesh (Common/induction/ImplicitInduction.cpp)."""

    def __init__(self, mesh: RefMesh, **kw):
        p = IndParams()
        p.resistive = int(kw.get("resistive", False))
        p.hall = int(kw.get("hall", False))
        p.max_it = int(kw.get("max_it", 100))
        p.restart = int(kw.get("restart", 20))
        p.ilu = int(kw.get("ilu", False))
        p.inver_Rem = kw.get("inver_Rem", 0.0)
        p.eta_r_inner = kw.get("eta_r_inner", 0.84)
        p.eta_r_outer = kw.get("eta_r_outer", 1.04)
        p.eta_width = kw.get("eta_width", 0.02)
        p.hall_coef = kw.get("hall_coef", 0.0)
        p.hall_r_min = kw.get("hall_r_min", 1.0)
        p.hall_r_max = kw.get("hall_r_max", 1.012)
        p.rtol = kw.get("rtol", 1e-4)
        p.ilu_shift = kw.get("ilu_shift", 0.3)
        p.implicit_ideal = int(kw.get("implicit_ideal", False))
        p.cuct = kw.get("cuct", 0.5)
        self.mesh = mesh
        h = lib().ref_ind_create(mesh._h, ctypes.byref(p))
        if not h:
            raise RuntimeError(lib().ref_last_error().decode())
        self._h = ctypes.c_void_p(h)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ref_ind_free(self._h)

    def set_m(self, m):
        m = np.ascontiguousarray(m, np.float64)
        lib().ref_ind_set_m(self._h, _p(m))

    def object(self):
        """Address of the reference's mhd::ImplicitInduction object."""
        return lib().ref_ind_object(self._h)

    def array(self, name):
        n = lib().ref_ind_array(self._h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        dt = np.int64 if name in ("ce_ptr", "pc_ptr", "pc_diag") else np.int32 if name in ("ce_edge", "pc_col") else np.float64
        a = np.zeros(n, dt)
        lib().ref_ind_array(self._h, name.encode(), _p(a))
        return a

    def set_ideal_state(self, u_cell, mask):
        """ImplicitInduction::set_ideal_state (:112-116): u 3 per cell, mask 1 per edge."""
        u = np.ascontiguousarray(u_cell, np.float64)
        m = np.ascontiguousarray(mask, np.int8)
        lib().ref_ind_set_ideal(self._h, _p(u), _p(m))

    def ideal_linear(self, phi):
        """ImplicitInduction::ideal_linear (:118-124)."""
        phi = np.ascontiguousarray(phi, np.float64)
        o = np.zeros(self.mesh.n_edges)
        lib().ref_ind_ideal_linear(self._h, _p(phi), _p(o))
        return o

    def solve_dt_edge(self, Phi, E_expl, dirichlet, dt_edge, warm=True):
        """ImplicitInduction::solve with the per-edge step dt_edge (:299-390)."""
        Phi = np.ascontiguousarray(Phi, np.float64)
        Ee = np.ascontiguousarray(E_expl, np.float64)
        d = np.ascontiguousarray(dirichlet, np.int8)
        dte = np.ascontiguousarray(dt_edge, np.float64)
        E = np.zeros(self.mesh.n_edges)
        rr = ctypes.c_double()
        it = lib().ref_ind_solve_dte(self._h, _p(Phi), _p(Ee), _p(d), _p(dte), int(warm), _p(E), ctypes.byref(rr))
        return E, int(it), rr.value

    def precond(self, dt, dirichlet, v):
        """factor_precond(dt, dir) then apply_precond(v) (ImplicitInduction.cpp:247-297) -> z."""
        d = np.ascontiguousarray(dirichlet, np.int8)
        v = np.ascontiguousarray(v, np.float64)
        z = np.zeros(self.mesh.n_edges)
        _check(lib().ref_ind_precond(self._h, float(dt), _p(d), _p(v), _p(z)))
        return z

    def set_frozen_state(self, B0, ne):
        B0 = np.ascontiguousarray(B0, np.float64)
        ne = np.ascontiguousarray(ne, np.float64)
        lib().ref_ind_set_frozen(self._h, _p(B0), _p(ne))

    def apply_F(self, phi):
        phi = np.ascontiguousarray(phi, np.float64)
        o = np.zeros(self.mesh.n_edges)
        lib().ref_ind_apply_F(self._h, _p(phi), _p(o))
        return o

    def apply_A(self, x, dt):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.mesh.n_edges)
        lib().ref_ind_apply_A(self._h, _p(x), dt, _p(y))
        return y

    def solve(self, Phi, E_expl, dirichlet, dt, warm=True):
        Phi = np.ascontiguousarray(Phi, np.float64)
        Ee = np.ascontiguousarray(E_expl, np.float64)
        d = np.ascontiguousarray(dirichlet, np.int8)
        E = np.zeros(self.mesh.n_edges)
        rr = ctypes.c_double()
        it = lib().ref_ind_solve(self._h, _p(Phi), _p(Ee), _p(d), dt, int(warm), _p(E), ctypes.byref(rr))
        return E, int(it), rr.value


def write_fields(path, topology_hash, records):
    """uns::io::write_fields (src/uns/io/MeshIO.cpp:117-130); records: (name, dim, ncomp, values)."""
    recs = list(records)
    vals = [np.ascontiguousarray(v, np.float64).ravel() for _, _, _, v in recs]
    names = (ctypes.c_char_p * max(1, len(recs)))(*[r[0].encode() for r in recs])
    dims = np.array([r[1] for r in recs] or [0], np.int32)
    ncomps = np.array([r[2] for r in recs] or [1], np.int32)
    counts = np.array([v.size for v in vals] or [0], np.int64)
    ptrs = (ctypes.c_void_p * max(1, len(recs)))(*[v.ctypes.data for v in vals])
    _check(lib().ref_write_fields(path.encode(), topology_hash, len(recs), ctypes.cast(names, ctypes.c_void_p), _p(dims), _p(ncomps),
                                  _p(counts), ctypes.cast(ptrs, ctypes.c_void_p)))


def read_fields(path):
    """uns::io::read_fields (MeshIO.cpp:132-150): ([(name, dim, ncomp, values)], hash)."""
    h = ctypes.c_uint64()
    n = lib().ref_read_fields(path.encode(), ctypes.byref(h))
    if n < 0:
        raise RuntimeError(lib().ref_last_error().decode())
    out = []
    name = ctypes.create_string_buffer(4096)
    for i in range(n):
        d, c, k = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        lib().ref_fields_get(i, name, 4096, ctypes.byref(d), ctypes.byref(c), ctypes.byref(k), None)
        v = np.empty(k.value)
        lib().ref_fields_get(i, name, 4096, ctypes.byref(d), ctypes.byref(c), ctypes.byref(k), _p(v))
        out.append((name.value.decode(), d.value, c.value, v))
    return out, h.value


MARS_PARAM_NAMES = ("rho_ref", "n_ref", "p_ref", "time_ref", "kB", "L", "U", "q", "B", "mag_scale", "pressure_scale", "ne_floor",
                    "rho_floor", "p_floor", "gamma", "cfl", "sw_ux", "sw_uy", "sw_uz", "sw_Bx", "sw_By", "sw_Bz", "ambipolar", "hall",
                    "second_order", "cuct", "rel_limit", "hall_scale")


class RefMars:
    """mars::MarsSolver on a reference mesh (the mesh must outlive it), initialised, with each phase of its step
    callable alone.  Ion arrays are species-major, 5 values per cell."""

    NS = 10

    def __init__(self, mesh: RefMesh, overrides=()):
        self.mesh = mesh
        enc = [o.encode() for o in overrides]
        arr = (ctypes.c_char_p * max(1, len(enc)))(*enc)
        h = lib().ref_mars_create(mesh._h, len(enc), ctypes.cast(arr, ctypes.c_void_p))
        if not h:
            raise RuntimeError(lib().ref_last_error().decode())
        self._h = ctypes.c_void_p(h)
        v = np.zeros(len(MARS_PARAM_NAMES))
        lib().ref_mars_params(self._h, _p(v))
        self.params = dict(zip(MARS_PARAM_NAMES, v.tolist()))
        fs = np.zeros(5 * self.NS)
        lib().ref_mars_freestream(self._h, _p(fs))
        self.freestream = fs.reshape(self.NS, 5)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ref_mars_free(self._h)

    def get(self, name):
        n = lib().ref_mars_size(self._h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        _check(lib().ref_mars_get(self._h, name.encode(), _p(out)))
        return out

    def set(self, name, values):
        v = np.ascontiguousarray(values, np.float64)
        if v.size != lib().ref_mars_size(self._h, name.encode()):
            raise ValueError(f"{name}: size mismatch")
        _check(lib().ref_mars_set(self._h, name.encode(), _p(v)))

    def prepare(self):
        _check(lib().ref_mars_prepare(self._h))

    def local_dt(self):
        d = np.zeros(1)
        _check(lib().ref_mars_local_dt(self._h, _p(d)))
        return float(d[0])

    def fluid_and_sources(self, dt):
        _check(lib().ref_mars_fluid_and_sources(self._h, dt))

    def ambipolar_emf(self, E):
        E = np.array(E, np.float64)
        _check(lib().ref_mars_ambipolar_emf(self._h, _p(E)))
        return E

    def emf(self):
        E = np.zeros(self.mesh.n_edges)
        _check(lib().ref_mars_emf(self._h, _p(E)))
        return E

    def implicit_sources(self, dt):
        _check(lib().ref_mars_implicit_sources(self._h, dt))

    def floors(self):
        _check(lib().ref_mars_floors(self._h))

    def set_induction(self, rtol, max_it, restart):
        """The Hall solve's GMRES settings (rtol, iteration limit, restart)."""
        _check(lib().ref_mars_set_induction(self._h, float(rtol), int(max_it), int(restart)))

    def last_solve(self):
        """(GMRES iterations, relative residual) of the last step's Hall solve."""
        it, res = ctypes.c_int32(), ctypes.c_double()
        lib().ref_mars_last_solve(self._h, ctypes.byref(it), ctypes.byref(res))
        return it.value, res.value

    def step_nochem(self, dt_max=1e300):
        d = np.zeros(1)
        _check(lib().ref_mars_step_nochem(self._h, dt_max, _p(d)))
        return float(d[0])

    def wall_table(self):
        n = lib().ref_mars_wall_table(self._h, None, None)
        faces = np.zeros(n, np.int32)
        prims = np.zeros((self.NS, n, 5))
        lib().ref_mars_wall_table(self._h, _p(faces), _p(prims))
        return faces, prims

    def boundary(self):
        fk = np.zeros(self.mesh.n_faces, np.int8)
        em = np.zeros(self.mesh.n_edges, np.int8)
        lib().ref_mars_boundary(self._h, _p(fk), _p(em))
        return fk, em
