"""ctypes binding of the oracle's C restatement (oracle/mhd_oracle.c -> oracle/_build/libmhd_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker of the parity tests and, where the compiled reference is
absent, of smoke() and bench.py's CPU baseline.  It is pinned against the reference itself by
tests/test_oracle.py (bit for bit on the same inputs) and against tests/golden/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_build", "libmhd_oracle.so")
vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
_lib = None


class OrMesh(ctypes.Structure):
    _fields_ = [(n, i32) for n in ("n_nodes", "n_edges", "n_faces", "n_cells", "n_owned_cells", "n_owned_edges")] + \
               [(n, vp) for n in ("c2f_ptr", "c2f_idx", "c2f_sgn", "f2e_ptr", "f2e_idx", "f2e_sgn", "e2f_ptr", "e2f_idx",
                                  "e2f_sgn", "f2c_ptr", "f2c_idx", "f2c_sgn", "cell_material", "edge_vec", "edge_mid",
                                  "edge_len", "face_area", "face_center", "face_area_mag", "cell_center", "cell_volume",
                                  "ec_ptr", "ec_cell", "ec_weight", "ef_weight", "star1", "star2", "face_kind", "edge_mode",
                                  "edge_nodes")]


class OrPrim(ctypes.Structure):
    _fields_ = [("rho", dbl), ("u", dbl), ("v", dbl), ("w", dbl), ("p", dbl)]


# Scales / Config::chem constants of the ambipolar and chemistry terms, in the order of the C structs
SOURCE_CONSTANTS = ("pressure_coef", "a1_Na", "a4", "a5", "a6", "state_coeff_H", "state_coeff_Na", "T_ref", "Tn0")


def set_source_terms(p, extra):
    """Fill the ambipolar / chemistry fields of a step-parameter struct from a dict (switches, constants, and
    the source fields photo / vst as arrays); returns the arrays the struct points to (keep them alive)."""
    keep = []
    if not extra:
        return keep
    p.ambipolar = int(bool(extra.get("ambipolar", False)))
    p.chemistry = int(bool(extra.get("chemistry", False)))
    for n in SOURCE_CONSTANTS:
        setattr(p, n, float(extra.get(n, 1.0 if n.startswith("state_coeff") or n == "T_ref" else 0.0)))
    for n in ("photo", "vst"):
        a = extra.get(n)
        if a is not None:
            a = np.ascontiguousarray(a, np.float64)
            keep.append(a)
            setattr(p, n, a.ctypes.data)
    return keep


class OrStepParams(ctypes.Structure):
    _fields_ = [("n_species", i32), ("second_order", i32), ("gamma", dbl), ("rho_floor", dbl), ("p_floor", dbl), ("cuct", dbl),
                ("M_ref", dbl), ("ne_floor", dbl), ("rel_limit", dbl), ("u_inf", dbl * 3), ("B_imf", dbl * 3),
                ("mass", dbl * 16), ("fs", OrPrim * 16), ("absorb", ctypes.c_int8 * 16), ("lorentz", i32),
                ("induce_coeff", dbl), ("inver_MA2", dbl), ("m_res", ctypes.c_void_p), ("ambipolar", i32), ("chemistry", i32)] + \
               [(n, dbl) for n in SOURCE_CONSTANTS] + [("photo", ctypes.c_void_p), ("vst", ctypes.c_void_p)]


class OrIndParams(ctypes.Structure):
    _fields_ = [("hall", i32), ("max_it", i32), ("restart", i32), ("hall_coef", dbl), ("hall_r_min", dbl), ("hall_r_max", dbl),
                ("rtol", dbl)]


def available() -> bool:
    return os.path.exists(SO)


def lib():
    global _lib
    if _lib is None:
        if not available():
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = ctypes.CDLL(SO)
        P = ctypes.POINTER
        for name, args, res in [
            ("or_to_prim", [vp, i64, dbl, dbl, dbl, vp], None),
            ("or_limited_gradients", [P(OrMesh), vp, i32, P(OrPrim), i32, dbl, vp], None),
            ("or_flux_rhs", [P(OrMesh), dbl, i32, P(OrPrim), vp, vp, vp], None),
            ("or_cell_vector", [P(OrMesh), vp, i32, vp], None),
            ("or_ideal_emf", [P(OrMesh), vp, vp, vp, vp, vp, dbl, vp], None),
            ("or_edge_modes", [P(OrMesh), vp, vp, vp], None),
            ("or_faraday", [P(OrMesh), vp, vp, dbl, vp], None),
            ("or_div_b", [P(OrMesh), vp, vp, vp], None),
            ("or_cell_current", [P(OrMesh), vp, vp], None),
            ("or_local_time_step", [P(OrMesh), i32, vp, vp, dbl, dbl, dbl, dbl], dbl),
            ("or_rk2_step", [P(OrMesh), P(OrStepParams), vp, vp, vp, vp, dbl], ctypes.c_int),
            ("or_first_order_step", [P(OrMesh), P(OrStepParams), vp, vp, vp, vp, vp, dbl, P(i32), P(dbl)], ctypes.c_int),
            ("or_add_sources", [P(OrMesh), P(OrStepParams), i32, vp, vp, vp, vp, vp, vp, vp, dbl, vp], None),
            ("or_electron_pressure_gradient", [P(OrMesh), vp, vp, vp], None),
            ("or_ambipolar_emf", [P(OrMesh), P(OrStepParams), vp, vp, vp], None),
            ("or_gyrate", [P(OrMesh), P(OrStepParams), vp, dbl, vp, vp], None),
            ("or_ind_create", [P(OrMesh), P(OrIndParams), vp], vp),
            ("or_ind_free", [vp], None),
            ("or_ind_set_frozen", [vp, vp, vp], None),
            ("or_ind_apply_F", [vp, vp, vp], None),
            ("or_ind_apply_A", [vp, vp, dbl, vp], None),
            ("or_ind_solve", [vp, vp, vp, vp, dbl, i32, vp, vp], i32),
            ("or_ind_set_ilu", [vp, i32, dbl], None),
            ("or_ind_solve_dte", [vp, vp, vp, vp, vp, i32, vp, vp], i32),
            ("or_ind_set_ideal", [vp, vp, vp, dbl], None),
            ("or_ind_ideal_linear", [vp, vp, vp], None),
            ("or_ind_ilu_pattern", [vp, vp, vp, vp], i64),
            ("or_ind_ilu_precond", [vp, dbl, vp, vp, vp], None),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _f(a):
    return np.ascontiguousarray(a, np.float64)


class PortMesh:
    """The oracle's view of a mesh given as arrays (a HostMesh, or anything indexable by the same names)."""

    _T = {"_ptr": np.int64, "_idx": np.int32, "_sgn": np.int8}

    def __init__(self, h):
        self._keep = {}
        d = OrMesh()
        d.n_nodes, d.n_edges, d.n_faces, d.n_cells = h.n_nodes, h.n_edges, h.n_faces, h.n_cells
        d.n_owned_cells, d.n_owned_edges = h.n_cells, h.n_edges
        for name, _ in OrMesh._fields_[6:]:
            if name == "edge_nodes":
                a = np.ascontiguousarray(np.asarray(h["e2n_idx"]).ravel(), np.int32)
                self._keep[name] = a
                d.edge_nodes = ctypes.c_void_p(a.ctypes.data)
                continue
            if name in ("cell_material",):
                dt = np.int32
            elif name in ("face_kind", "edge_mode"):
                dt = np.int8
            elif name == "ec_ptr":
                dt = np.int64
            elif name == "ec_cell":
                dt = np.int32
            else:
                dt = next((t for suf, t in self._T.items() if name.endswith(suf)), np.float64)
            a = np.ascontiguousarray(np.asarray(h[name]).ravel(), dt)
            self._keep[name] = a
            setattr(d, name, ctypes.c_void_p(a.ctypes.data))
        self.d = d
        self.n_cells, self.n_faces, self.n_edges = h.n_cells, h.n_faces, h.n_edges

    @property
    def ref(self):
        return ctypes.byref(self.d)

    def to_prim(self, U, gamma, rho_floor=1e-10, p_floor=1e-12):
        U = _f(U)
        W = np.zeros_like(U)
        lib().or_to_prim(_p(U), U.size // 5, gamma, rho_floor, p_floor, _p(W))
        return W

    def limited_gradients(self, W, absorb, fs, limit=True, rel_limit=0.0):
        W = _f(W)
        g = np.zeros(15 * self.n_cells)
        pr = OrPrim(*[float(v) for v in fs])
        lib().or_limited_gradients(self.ref, _p(W), int(absorb), ctypes.byref(pr), int(limit), rel_limit, _p(g))
        return g

    def flux_rhs(self, W, grad, absorb, fs, gamma):
        W, grad = _f(W), _f(grad)
        r = np.zeros(5 * self.n_cells)
        pr = OrPrim(*[float(v) for v in fs])
        lib().or_flux_rhs(self.ref, gamma, int(absorb), ctypes.byref(pr), _p(W), _p(grad), _p(r))
        return r

    def cell_vector(self, phi):
        phi = _f(phi)
        o = np.zeros(3 * self.n_cells)
        lib().or_cell_vector(self.ref, _p(phi), self.n_cells, _p(o))
        return o

    def ideal_emf(self, u, Bt, Bi, pt, pi, cuct=0.5, E=None):
        E = np.zeros(self.n_edges) if E is None else np.array(E, np.float64)
        a = [_f(x) for x in (u, Bt, Bi, pt, pi)]
        lib().or_ideal_emf(self.ref, *[_p(x) for x in a], cuct, _p(E))
        return E

    def edge_modes(self, u_inf, B_imf, E):
        E = np.array(E, np.float64)
        lib().or_edge_modes(self.ref, _p(_f(u_inf)), _p(_f(B_imf)), _p(E))
        return E

    def faraday(self, E, B, dt, dt_edge=None):
        E = _f(E)
        B = np.array(B, np.float64)
        lib().or_faraday(self.ref, _p(E), _p(None if dt_edge is None else _f(dt_edge)), dt, _p(B))
        return B

    def div_b(self, B, extra=None):
        o = np.zeros(3)
        lib().or_div_b(self.ref, _p(_f(B)), _p(None if extra is None else _f(extra)), _p(o))
        return dict(max_abs=o[0], max_rel=o[1], worst_cell_gid=int(o[2]))

    def cell_current(self, B):
        J = np.zeros(3 * self.n_cells)
        lib().or_cell_current(self.ref, _p(_f(B)), _p(J))
        return J

    def local_time_step(self, W_list, B, gamma, cfl, inver_MA2=1.0, rho_floor_dt=1e-2):
        Ws = [_f(w) for w in W_list]
        arr = (ctypes.c_void_p * len(Ws))(*[w.ctypes.data for w in Ws])
        return lib().or_local_time_step(self.ref, len(Ws), ctypes.cast(arr, ctypes.c_void_p), _p(_f(B)), gamma, cfl, inver_MA2,
                                        rho_floor_dt)

    @staticmethod
    def step_params(wl, absorb=None, lorentz=False, induce_coeff=0.0, inver_MA2=1.0):
        """OrStepParams of a Workload (the reference's Config defaults for the rest)."""
        p = OrStepParams()
        p.n_species, p.second_order = wl.n_species, 1
        p.gamma, p.rho_floor, p.p_floor, p.cuct, p.M_ref, p.ne_floor, p.rel_limit = wl.gamma, 1e-10, 1e-12, 0.5, 1.0, 0.01, 0.0
        p.u_inf[:] = list(wl.u_inf)
        p.B_imf[:] = list(wl.B_imf)
        for s in range(wl.n_species):
            p.mass[s] = wl.mass[s]
            p.fs[s] = OrPrim(*[float(v) for v in wl.fs[s]])
            p.absorb[s] = int(s == 1) if absorb is None else int(absorb[s])
        p.lorentz, p.induce_coeff, p.inver_MA2 = int(bool(lorentz)), float(induce_coeff), float(inver_MA2)
        return p

    def add_sources(self, p, species, WH, WNa, B, J, dt, rhs, dpe=None, photo=None, vst=None):
        """mercury::add_sources (oracle restatement); rhs in place."""
        opt = [None if x is None else _f(x) for x in (B, J, dpe, photo, vst)]
        lib().or_add_sources(self.ref, ctypes.byref(p), species, _p(_f(WH)), _p(_f(WNa)), *[_p(x) for x in opt], dt, _p(rhs))

    def electron_pressure_gradient(self, WH, WNa):
        out = np.zeros(3 * self.n_cells)
        lib().or_electron_pressure_gradient(self.ref, _p(_f(WH)), _p(_f(WNa)), _p(out))
        return out

    def ambipolar_emf(self, p, WH, WNa, E):
        """E minus the ambipolar EMF (a new array)."""
        E = np.array(E, np.float64)
        lib().or_ambipolar_emf(self.ref, ctypes.byref(p), _p(_f(WH)), _p(_f(WNa)), _p(E))
        return E

    def gyrate(self, p, B, dt, UH, UNa):
        """mercury::gyrate (oracle restatement); UH, UNa in place."""
        lib().or_gyrate(self.ref, ctypes.byref(p), _p(_f(B)), dt, _p(UH), _p(UNa))

    def rk2_step(self, wl, U_list, Phi, Badd, dt, absorb=None, lorentz=False, induce_coeff=0.0, inver_MA2=1.0, m_res=None,
                 extra=None):
        """One SSP-RK2 step of the hot path for a Workload's parameters; U_list and Phi updated in place.
        With lorentz: the J x B source and (induce_coeff > 0) the Strang-split gyration of the two-ion model;
        with m_res (per edge): the explicit resistive EMF E_e += m_e (d1^T star2 Phi)_e; extra: the ambipolar
        and chemistry terms (set_source_terms)."""
        p = self.step_params(wl, absorb, lorentz, induce_coeff, inver_MA2)
        keep = set_source_terms(p, extra)
        mr = None if m_res is None else _f(m_res)
        p.m_res = None if mr is None else mr.ctypes.data
        arr = (ctypes.c_void_p * len(U_list))(*[u.ctypes.data for u in U_list])
        rc = lib().or_rk2_step(self.ref, ctypes.byref(p), ctypes.cast(arr, ctypes.c_void_p), _p(Phi), _p(_f(wl.PhiAdd)), _p(_f(Badd)), dt)
        if rc != 0:
            raise RuntimeError("oracle rk2 step failed")

    def first_order_step(self, wl, ind, U_list, Phi, Badd, dt, lorentz=False, induce_coeff=0.0, inver_MA2=1.0):
        """One semi-implicit step (Solver::step_first_order) with the EMF of ind's solve (a PortInduction of this
        mesh); U_list and Phi updated in place -> (iterations, rel_res)."""
        p = self.step_params(wl, None, lorentz, induce_coeff, inver_MA2)
        arr = (ctypes.c_void_p * len(U_list))(*[u.ctypes.data for u in U_list])
        it, rr = i32(), dbl()
        rc = lib().or_first_order_step(self.ref, ctypes.byref(p), ind._h, ctypes.cast(arr, ctypes.c_void_p), _p(Phi), _p(_f(wl.PhiAdd)),
                                       _p(_f(Badd)), dt, ctypes.byref(it), ctypes.byref(rr))
        if rc != 0:
            raise RuntimeError("oracle first-order step failed")
        return it.value, rr.value


class PortInduction:
    """The oracle's mhd::ImplicitInduction (restarted GMRES, Jacobi or block ILU(0) preconditioner)."""

    def __init__(self, pm: PortMesh, m_edge=None, hall=False, hall_coef=0.0, hall_r_min=1.0, hall_r_max=1.012, rtol=1e-4,
                 max_it=100, restart=20):
        p = OrIndParams(int(hall), int(max_it), int(restart), hall_coef, hall_r_min, hall_r_max, rtol)
        self.pm = pm
        self._m = None if m_edge is None else _f(m_edge)
        self._h = ctypes.c_void_p(lib().or_ind_create(pm.ref, ctypes.byref(p), _p(self._m)))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.or_ind_free(self._h)

    def set_frozen_state(self, B0, ne):
        lib().or_ind_set_frozen(self._h, _p(_f(B0)), _p(_f(ne)))

    def apply_F(self, phi):
        o = np.zeros(self.pm.n_edges)
        lib().or_ind_apply_F(self._h, _p(_f(phi)), _p(o))
        return o

    def apply_A(self, x, dt):
        o = np.zeros(self.pm.n_edges)
        lib().or_ind_apply_A(self._h, _p(_f(x)), dt, _p(o))
        return o

    def solve_dt_edge(self, Phi, E_expl, dirichlet, dt_edge, warm=True):
        """solve with the per-edge pseudo-time step dt_edge -> (E, iterations, rel_res)."""
        E = np.zeros(self.pm.n_edges)
        rr = ctypes.c_double()
        d = np.ascontiguousarray(dirichlet, np.int8)
        it = lib().or_ind_solve_dte(self._h, _p(_f(Phi)), _p(_f(E_expl)), _p(d), _p(_f(dt_edge)), int(warm), _p(E), ctypes.byref(rr))
        return E, int(it), rr.value

    def set_ideal_state(self, u_cell, mask, cuct=0.5):
        """Config::implicit_ideal with set_ideal_state: u 3 per cell, mask 1 per edge (None: the part off)."""
        if u_cell is None:
            lib().or_ind_set_ideal(self._h, None, None, float(cuct))
            return
        self._u = _f(u_cell)
        self._mask = np.ascontiguousarray(mask, np.int8)
        lib().or_ind_set_ideal(self._h, _p(self._u), _p(self._mask), float(cuct))

    def ideal_linear(self, phi):
        o = np.zeros(self.pm.n_edges)
        lib().or_ind_ideal_linear(self._h, _p(_f(phi)), _p(o))
        return o

    def set_ilu(self, enable=True, shift=0.3):
        """Config::ind_ilu / ind_ilu_shift: block-Jacobi ILU(0) in place of the Jacobi scaling."""
        lib().or_ind_set_ilu(self._h, int(bool(enable)), float(shift))

    def ilu_pattern(self):
        """(pc_ptr, pc_col, pc_coef) of the owned rows."""
        nnz = lib().or_ind_ilu_pattern(self._h, None, None, None)
        if nnz < 0:
            raise RuntimeError("no ILU(0) pattern")
        ptr = np.zeros(self.pm.n_edges + 1, np.int64)
        col, coef = np.zeros(nnz, np.int32), np.zeros(nnz)
        lib().or_ind_ilu_pattern(self._h, _p(ptr), _p(col), _p(coef))
        return ptr, col, coef

    def precond(self, dt, dirichlet, v):
        """factor_precond(dt, dir) then apply_precond(v) -> z."""
        z = np.zeros(self.pm.n_edges)
        d = np.ascontiguousarray(dirichlet, np.int8)
        lib().or_ind_ilu_precond(self._h, dt, _p(d), _p(_f(v)), _p(z))
        return z

    def solve(self, Phi, E_expl, dirichlet, dt, warm=True):
        E = np.zeros(self.pm.n_edges)
        rr = ctypes.c_double()
        d = np.ascontiguousarray(dirichlet, np.int8)
        it = lib().or_ind_solve(self._h, _p(_f(Phi)), _p(_f(E_expl)), _p(d), dt, int(warm), _p(E), ctypes.byref(rr))
        return E, int(it), rr.value


def rk2_step_box(wl, dt):
    """One step of a single-ion box workload from its initial state (used by smoke() without the reference)."""
    pm = PortMesh(wl.mesh)
    U = [np.array(u, np.float64) for u in wl.U]
    Phi = np.array(wl.Phi, np.float64)
    pm.rk2_step(wl, U, Phi, pm.cell_vector(wl.PhiAdd), dt)
    return U[0], Phi
