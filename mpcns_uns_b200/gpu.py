"""Python mirror of the reference's hot-path interface, dispatching to libmhd_gpu.so (include/mhd_gpu.h).

The names, argument meaning and layouts follow the reference functions they replace (AoS
arrays: value(i, comp) = a[i * ncomp + comp]); torch CUDA tensors carry the device memory.
There is no CPU fallback: without the built library or a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import build as _build

_lib = None
vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double

MHD_OK, MHD_EINVAL, MHD_ECUDA, MHD_ESTATE, MHD_ENOCONV = 0, -1, -2, -3, -4


class MhdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class MeshDesc(ctypes.Structure):
    _fields_ = [("n_nodes", i32), ("n_edges", i32), ("n_faces", i32), ("n_cells", i32),
                ("n_owned_cells", i32), ("n_owned_edges", i32)] + \
               [(n, vp) for n in ("c2f_ptr", "c2f_idx", "c2f_sgn", "f2e_ptr", "f2e_idx", "f2e_sgn",
                                  "e2f_ptr", "e2f_idx", "e2f_sgn", "f2c_ptr", "f2c_idx", "f2c_sgn", "cell_material",
                                  "edge_vec", "edge_mid", "edge_len", "face_area", "face_center", "face_area_mag",
                                  "cell_center", "cell_volume", "ec_ptr", "ec_cell", "ec_weight", "ef_weight",
                                  "star1", "star2", "face_kind", "edge_mode", "edge_nodes")]


class Prim(ctypes.Structure):
    """mhd::Prim (Common/physics/Euler.h:7-10)."""
    _fields_ = [("rho", dbl), ("u", dbl), ("v", dbl), ("w", dbl), ("p", dbl)]


class StepParams(ctypes.Structure):
    """MhdStepParams of include/mhd_gpu.h (the Config / Scales fields the explicit step reads)."""
    _fields_ = [("n_species", i32), ("second_order", i32), ("gamma", dbl), ("rho_floor", dbl), ("p_floor", dbl),
                ("cuct", dbl), ("M_ref", dbl), ("ne_floor", dbl), ("rel_limit", dbl), ("cfl", dbl), ("inver_MA2", dbl),
                ("rho_floor_dt", dbl), ("u_inf", dbl * 3), ("B_imf", dbl * 3), ("mass", dbl * 16), ("fs", Prim * 16),
                ("absorb", ctypes.c_int8 * 16), ("precision", i32), ("lorentz", i32), ("induce_coeff", dbl),
                ("ambipolar", i32), ("chemistry", i32), ("pressure_coef", dbl), ("a1_Na", dbl), ("a4", dbl), ("a5", dbl),
                ("a6", dbl), ("state_coeff_H", dbl), ("state_coeff_Na", dbl), ("T_ref", dbl), ("Tn0", dbl)]


class InductionParams(ctypes.Structure):
    """MhdInductionParams of include/mhd_gpu.h (the Config fields mhd::ImplicitInduction reads)."""
    _fields_ = [("hall", i32), ("max_it", i32), ("restart", i32), ("precision", i32), ("hall_coef", dbl),
                ("hall_r_min", dbl), ("hall_r_max", dbl), ("rtol", dbl)]


FIELD_U, FIELD_PHI, FIELD_PHIADD, FIELD_BADD = 0, 1, 2, 3
PREC_FP64, PREC_MIXED = 0, 1

_SIGS = {
    "mhd_gpu_last_error": ([], ctypes.c_char_p),
    "mhd_gpu_state_create": ([vp, ctypes.POINTER(StepParams), ctypes.POINTER(vp)], ctypes.c_int),
    "mhd_gpu_state_destroy": ([vp], ctypes.c_int),
    "mhd_gpu_state_upload": ([vp, i32, i32, vp], ctypes.c_int),
    "mhd_gpu_state_download": ([vp, i32, i32, vp], ctypes.c_int),
    "mhd_gpu_state_device_ptr": ([vp, i32, ctypes.POINTER(vp)], ctypes.c_int),
    "mhd_gpu_cfl_dt": ([vp, dbl, ctypes.POINTER(dbl)], ctypes.c_int),
    "mhd_gpu_step_rk2": ([vp, dbl, dbl, ctypes.POINTER(dbl)], ctypes.c_int),
    "mhd_gpu_step_semi_implicit": ([vp, vp, dbl, dbl, ctypes.POINTER(dbl), ctypes.POINTER(i32), ctypes.POINTER(dbl)], ctypes.c_int),
    "mhd_gpu_state_profile": ([vp, i32], ctypes.c_int),
    "mhd_gpu_state_profile_read": ([vp, i32, vp, vp, vp, ctypes.POINTER(i32)], ctypes.c_int),
    "mhd_gpu_state_launches": ([vp, ctypes.POINTER(i64)], ctypes.c_int),
    "mhd_gpu_device_info": ([ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "mhd_gpu_mesh_create": ([ctypes.POINTER(MeshDesc), ctypes.POINTER(vp)], ctypes.c_int),
    "mhd_gpu_mesh_destroy": ([vp], ctypes.c_int),
    "mhd_gpu_mesh_stream": ([vp], vp),
    "mhd_gpu_mesh_set_stream": ([vp, vp], ctypes.c_int),
    "mhd_gpu_synchronize": ([vp], ctypes.c_int),
    "mhd_gpu_to_prim": ([vp, vp, i32, dbl, dbl, dbl, vp], ctypes.c_int),
    "mhd_gpu_limited_gradients": ([vp, vp, i32, ctypes.POINTER(Prim), i32, dbl, vp], ctypes.c_int),
    "mhd_gpu_flux_rhs": ([vp, dbl, i32, ctypes.POINTER(Prim), vp, vp, vp], ctypes.c_int),
    "mhd_gpu_limited_gradients_wall": ([vp, vp, i32, ctypes.POINTER(Prim), i32, dbl, i32, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_flux_rhs_wall": ([vp, dbl, i32, ctypes.POINTER(Prim), vp, vp, i32, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_state_set_wall_ghosts": ([vp, i32, vp, vp], ctypes.c_int),
    "mhd_gpu_mars_plasma": ([vp, vp, vp, vp, vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_pressure_gradient": ([vp, vp, vp], ctypes.c_int),
    "mhd_gpu_mars_explicit_sources": ([vp, vp, vp, vp, vp, vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_mars_ambipolar_emf": ([vp, vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_mars_time_step": ([vp, vp, dbl, vp, vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_mars_implicit_sources": ([vp, vp, vp, vp, dbl, vp], ctypes.c_int),
    "mhd_gpu_mars_advance": ([vp, i32, vp, dbl, vp], ctypes.c_int),
    "mhd_gpu_mars_floors": ([vp, vp, vp], ctypes.c_int),
    "mhd_gpu_cell_vector": ([vp, vp, i32, vp], ctypes.c_int),
    "mhd_gpu_ideal_emf": ([vp, vp, vp, vp, vp, vp, dbl, vp], ctypes.c_int),
    "mhd_gpu_edge_modes": ([vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_faraday": ([vp, vp, vp, dbl], ctypes.c_int),
    "mhd_gpu_faraday_edge_dt": ([vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_div_b": ([vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_cell_current": ([vp, vp, vp], ctypes.c_int),
    "mhd_gpu_add_sources": ([vp, ctypes.POINTER(StepParams), i32, vp, vp, vp, vp, vp, vp, vp, dbl, vp], ctypes.c_int),
    "mhd_gpu_electron_pressure_gradient": ([vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_ambipolar_emf": ([vp, ctypes.POINTER(StepParams), vp, vp, vp], ctypes.c_int),
    "mhd_gpu_state_set_source_fields": ([vp, vp, vp], ctypes.c_int),
    "mhd_gpu_gyrate": ([vp, ctypes.POINTER(StepParams), vp, dbl, vp, vp], ctypes.c_int),
    "mhd_gpu_induction_create": ([vp, ctypes.POINTER(InductionParams), vp, ctypes.POINTER(vp)], ctypes.c_int),
    "mhd_gpu_induction_destroy": ([vp], ctypes.c_int),
    "mhd_gpu_induction_set_frozen": ([vp, vp, vp], ctypes.c_int),
    "mhd_gpu_induction_apply_F": ([vp, vp, vp], ctypes.c_int),
    "mhd_gpu_induction_apply_A": ([vp, vp, dbl, vp], ctypes.c_int),
    "mhd_gpu_induction_solve": ([vp, vp, vp, vp, dbl, i32, vp, ctypes.POINTER(i32), ctypes.POINTER(dbl)], ctypes.c_int),
    "mhd_gpu_induction_profile": ([vp, i32], ctypes.c_int),
    "mhd_gpu_induction_profile_read": ([vp, i32, vp, vp, vp, ctypes.POINTER(i32)], ctypes.c_int),
    "mhd_gpu_induction_launches": ([vp, ctypes.POINTER(i64)], ctypes.c_int),
    "mhd_gpu_induction_last_solve_stats": ([vp, ctypes.POINTER(i32)], ctypes.c_int),
    "mhd_gpu_induction_set_ilu": ([vp, i32, dbl], ctypes.c_int),
    "mhd_gpu_induction_solve_dt_edge": ([vp, vp, vp, vp, vp, i32, vp, ctypes.POINTER(i32), ctypes.POINTER(dbl)], ctypes.c_int),
    "mhd_gpu_induction_set_ideal": ([vp, vp, vp, dbl], ctypes.c_int),
    "mhd_gpu_induction_ideal_linear": ([vp, vp, vp], ctypes.c_int),
    "mhd_gpu_induction_ilu_factor": ([vp, dbl, vp], ctypes.c_int),
    "mhd_gpu_induction_ilu_apply": ([vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_induction_ilu_debug": ([vp, dbl, i32], ctypes.c_int),
    "mhd_gpu_induction_ilu_tune": ([vp, i32, i32, i32], ctypes.c_int),
    "mhd_gpu_induction_ilu_arrays": ([vp, ctypes.POINTER(i32), ctypes.POINTER(i64), vp, vp, vp, vp, vp], ctypes.c_int),
    "mhd_ilu_pattern": ([i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_tet_build": ([i32, i64, vp, vp, i32, vp, vp, ctypes.POINTER(vp)], ctypes.c_int),
    "mhd_gpu_tet_build_counts": ([vp, vp], ctypes.c_int),
    "mhd_gpu_tet_build_copy": ([vp, vp], ctypes.c_int),
    "mhd_gpu_tet_build_free": ([vp], ctypes.c_int),
    "mhd_gpu_state_set_resistivity": ([vp, vp], ctypes.c_int),
    "mhd_gpu_compute_geometry": ([vp], ctypes.c_int),
    "mhd_gpu_boundary": ([vp], ctypes.c_int),
    "mhd_gpu_fn_create": ([vp, vp, vp, vp, ctypes.POINTER(vp)], ctypes.c_int),
    "mhd_gpu_fn_destroy": ([vp], ctypes.c_int),
    "mhd_gpu_fn_set_params": ([vp, vp, vp], ctypes.c_int),
    "mhd_gpu_fn_reset": ([vp], ctypes.c_int),
    "mhd_gpu_fn_forward": ([vp, ctypes.POINTER(dbl)], ctypes.c_int),
    "mhd_gpu_fn_backward": ([vp, vp, vp], ctypes.c_int),
    "mhd_gpu_fn_tangent": ([vp, vp, vp, ctypes.POINTER(dbl), ctypes.POINTER(dbl)], ctypes.c_int),
    "mhd_gpu_fn_stage_tangent": ([vp, vp, vp, vp, vp, vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_fn_stage_adjoint": ([vp, vp, vp, vp, vp, vp, vp, vp, vp], ctypes.c_int),
    "mhd_gpu_fn_profile": ([vp, i32], ctypes.c_int),
    "mhd_gpu_fn_switch_log": ([vp, i32], ctypes.c_int),
    "mhd_gpu_fn_last_J": ([vp, vp], ctypes.c_int),
    "mhd_gpu_fn_switch_read": ([vp, i32, vp, ctypes.c_int64], ctypes.c_int),
    "mhd_gpu_fn_profile_read": ([vp, i32, vp, vp, vp, ctypes.POINTER(i32)], ctypes.c_int),
}


def lib():
    """The loaded C-ABI library (built in-tree on first use if missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_build.GPU_SO):
            _build.build_gpu()
        L = ctypes.CDLL(_build.GPU_SO)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def register(name, args, res=ctypes.c_int):
    """Declare a further C-ABI symbol (used by the modules that extend this one)."""
    _SIGS[name] = (args, res)
    if _lib is not None:
        f = getattr(_lib, name)
        f.argtypes = args
        f.restype = res


def check(rc):
    if rc != MHD_OK:
        raise MhdError(rc, lib().mhd_gpu_last_error().decode())


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("mpcns_uns_b200.gpu needs a CUDA device (no CPU fallback)")
    return torch


def dev(a, dtype=None):
    """numpy array / tensor -> contiguous CUDA tensor (float64 unless an integer dtype is given)."""
    torch = _torch()
    if isinstance(a, torch.Tensor):
        t = a if dtype is None else a.to(dtype)
        return t.contiguous().cuda()
    a = np.ascontiguousarray(a)
    t = torch.from_numpy(a)
    if dtype is not None:
        t = t.to(dtype)
    elif t.dtype == torch.float32:
        t = t.double()
    return t.cuda()


def ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class DeviceMesh:
    """A device copy of one rank's mesh (MhdMesh handle)."""

    def __init__(self, host_mesh):
        torch = _torch()
        hm = host_mesh
        keep = {}

        def arr(name, dtype):
            a = np.ascontiguousarray(hm[name], dtype)
            keep[name] = a
            return ctypes.c_void_p(a.ctypes.data)

        d = MeshDesc()
        d.n_nodes, d.n_edges, d.n_faces, d.n_cells = hm.n_nodes, hm.n_edges, hm.n_faces, hm.n_cells
        d.n_owned_cells, d.n_owned_edges = hm.n_cells, hm.n_edges
        for t in ("c2f", "f2e", "e2f", "f2c"):
            setattr(d, t + "_ptr", arr(t + "_ptr", np.int64))
            setattr(d, t + "_idx", arr(t + "_idx", np.int32))
            setattr(d, t + "_sgn", arr(t + "_sgn", np.int8))
        d.cell_material = arr("cell_material", np.int32)
        for n in ("edge_vec", "edge_mid", "edge_len", "face_area", "face_center", "face_area_mag", "cell_center",
                  "cell_volume", "ec_weight", "ef_weight", "star1", "star2"):
            setattr(d, n, arr(n, np.float64))
        d.ec_ptr = arr("ec_ptr", np.int64)
        d.ec_cell = arr("ec_cell", np.int32)
        d.face_kind = arr("face_kind", np.int8)
        d.edge_mode = arr("edge_mode", np.int8)
        d.edge_nodes = arr("e2n_idx", np.int32)   # start, end per edge: the ambipolar EMF's node lists
        h = vp()
        torch.cuda.init()
        check(lib().mhd_gpu_mesh_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        self.host = hm
        self.n_nodes, self.n_edges, self.n_faces, self.n_cells = hm.n_nodes, hm.n_edges, hm.n_faces, hm.n_cells
        self._stream = torch.cuda.ExternalStream(lib().mhd_gpu_mesh_stream(self._h))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.mhd_gpu_mesh_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @property
    def stream(self):
        """torch view of the handle's CUDA stream."""
        return self._stream

    def synchronize(self):
        check(lib().mhd_gpu_synchronize(self._h))

    def _enter(self):
        # the handle's stream must see every tensor that torch's current stream produced
        self._stream.wait_stream(_torch().cuda.current_stream())

    def _leave(self):
        _torch().cuda.current_stream().wait_stream(self._stream)

    # ------------------------------------------------------------- reference functions
    def to_prim(self, U, gamma, rho_floor=1e-10, p_floor=1e-12):
        """mhd::to_prim (Common/physics/Euler.h:13-21) for every cell."""
        torch = _torch()
        U = dev(U)
        W = torch.empty_like(U)
        self._enter()
        check(lib().mhd_gpu_to_prim(self._h, ptr(U), U.numel() // 5, gamma, rho_floor, p_floor, ptr(W)))
        self._leave()
        return W

    def limited_gradients(self, W, species, freestream, limit=True, rel_limit=0.0, wall=None):
        """Stencil::limited_gradients (Common/fluid/Reconstruction.cpp:80-142): 15 per cell.  wall: (faces,
        prims n_wall x 5 of this species), the Dirichlet wall table of the GhostFn argument."""
        torch = _torch()
        W = dev(W)
        g = torch.empty(15 * self.n_cells, dtype=torch.float64, device="cuda")
        fs = Prim(*[float(v) for v in freestream])
        self._enter()
        if wall is None:
            check(lib().mhd_gpu_limited_gradients(self._h, ptr(W), int(species), ctypes.byref(fs), int(bool(limit)),
                                                  float(rel_limit), ptr(g)))
        else:
            fc, pr = _wall_dev(wall)
            check(lib().mhd_gpu_limited_gradients_wall(self._h, ptr(W), int(species), ctypes.byref(fs), int(bool(limit)),
                                                       float(rel_limit), fc.numel(), ptr(fc), ptr(pr), ptr(g)))
        self._leave()
        return g

    def fluid_flux_rhs(self, gamma, species, freestream, W, grad, wall=None):
        """mhd::fluid_flux_rhs (Common/fluid/FluxRHS.cpp:30-74): 5 per cell.  wall: as limited_gradients."""
        torch = _torch()
        W, grad = dev(W), dev(grad)
        r = torch.empty(5 * self.n_cells, dtype=torch.float64, device="cuda")
        fs = Prim(*[float(v) for v in freestream])
        self._enter()
        if wall is None:
            check(lib().mhd_gpu_flux_rhs(self._h, float(gamma), int(species), ctypes.byref(fs), ptr(W), ptr(grad), ptr(r)))
        else:
            fc, pr = _wall_dev(wall)
            check(lib().mhd_gpu_flux_rhs_wall(self._h, float(gamma), int(species), ctypes.byref(fs), ptr(W), ptr(grad), fc.numel(),
                                              ptr(fc), ptr(pr), ptr(r)))
        self._leave()
        return r

    def reconstruct_cell_vector(self, flux, ncells=None):
        """uns::reconstruct_cell_vector (src/uns/geometry/Reconstruct.cpp:8-46): 3 per cell."""
        torch = _torch()
        flux = dev(flux)
        n = self.n_cells if ncells is None else int(ncells)
        out = torch.empty(3 * n, dtype=torch.float64, device="cuda")
        self._enter()
        check(lib().mhd_gpu_cell_vector(self._h, ptr(flux), n, ptr(out)))
        self._leave()
        return out

    def add_ideal_emf(self, u_cell, B_cell_tot, B_cell_ind, phi_tot, phi_ind, cuct=0.5, E=None):
        """mhd::add_ideal_emf (Common/induction/IdealEMF.cpp:25-129): adds into E (zeros if None)."""
        torch = _torch()
        args = [dev(a) for a in (u_cell, B_cell_tot, B_cell_ind, phi_tot, phi_ind)]
        E = torch.zeros(self.n_edges, dtype=torch.float64, device="cuda") if E is None else dev(E).clone()
        self._enter()
        check(lib().mhd_gpu_ideal_emf(self._h, *[ptr(a) for a in args], float(cuct), ptr(E)))
        self._leave()
        return E

    def edge_modes(self, u_inf, B_imf, E):
        """Boundary edge values of Solver::rhs (MercuryUns/driver/Solver.cpp:162-167), in place."""
        u = np.asarray(u_inf, np.float64)
        b = np.asarray(B_imf, np.float64)
        self._enter()
        check(lib().mhd_gpu_edge_modes(self._h, u.ctypes.data_as(vp), b.ctypes.data_as(vp), ptr(E)))
        self._leave()
        return E

    def faraday_update(self, E, B, dt):
        """mhd::faraday_update (Common/induction/Faraday.cpp:15-24); returns the updated copy of B."""
        E = dev(E)
        B = dev(B).clone()
        self._enter()
        check(lib().mhd_gpu_faraday(self._h, ptr(E), ptr(B), float(dt)))
        self._leave()
        return B

    def faraday_update_edge_dt(self, E, dt_edge, B):
        """mhd::faraday_update_edge_dt (Common/induction/Faraday.cpp:27-36)."""
        E, d = dev(E), dev(dt_edge)
        B = dev(B).clone()
        self._enter()
        check(lib().mhd_gpu_faraday_edge_dt(self._h, ptr(E), ptr(d), ptr(B)))
        self._leave()
        return B

    def div_b(self, B, extra=None, gid=None):
        """mhd::div_b (Common/diagnostics/DivB.cpp:8-24) -> dict(max_abs, max_rel, worst_cell, worst_cell_gid).

        worst_cell is the handle's local index of the worst owned cell (-1: none).  The reference
        reports its global id cx.ent[3].gid[c] (DivB.cpp:20): worst_cell_gid = gid[worst_cell] with the
        caller's gid table, or the local index when gid is None (one rank built by ComplexBuilder,
        whose gid is the identity)."""
        B = dev(B)
        ex = None if extra is None else dev(extra)
        out = np.zeros(3)
        self._enter()
        check(lib().mhd_gpu_div_b(self._h, ptr(B), ptr(ex), out.ctypes.data_as(vp)))
        c = int(out[2])
        g = c if (gid is None or c < 0) else int(np.asarray(gid)[c])
        return dict(max_abs=float(out[0]), max_rel=float(out[1]), worst_cell=c, worst_cell_gid=g)

    def add_sources(self, params, species, WH, WNa, B, J, dt, rhs, dpe=None, photo=None, vst=None):
        """mercury::add_sources (MercuryUns/fluid/MercurySources.cpp:13-63); returns rhs + source."""
        WH, WNa = dev(WH), dev(WNa)
        B, J, dpe, photo, vst = (None if x is None else dev(x) for x in (B, J, dpe, photo, vst))
        rhs = dev(rhs).clone()
        self._enter()
        check(lib().mhd_gpu_add_sources(self._h, ctypes.byref(params), int(species), ptr(WH), ptr(WNa), ptr(B), ptr(J), ptr(dpe),
                                         ptr(photo), ptr(vst), float(dt), ptr(rhs)))
        self._leave()
        return rhs

    def electron_pressure_gradient(self, WH, WNa):
        """mercury::electron_pressure_gradient (MercuryUns/physics/Ambipolar.cpp:10-31): 3 per cell."""
        torch = _torch()
        WH, WNa = dev(WH), dev(WNa)
        out = torch.empty(3 * self.n_cells, dtype=torch.float64, device="cuda")
        self._enter()
        check(lib().mhd_gpu_electron_pressure_gradient(self._h, ptr(WH), ptr(WNa), ptr(out)))
        self._leave()
        return out

    def ambipolar_emf(self, params, WH, WNa, E):
        """mercury::AmbipolarEMF::add (Ambipolar.cpp:52-88): returns E minus the ambipolar EMF."""
        WH, WNa = dev(WH), dev(WNa)
        E = dev(E).clone()
        self._enter()
        check(lib().mhd_gpu_ambipolar_emf(self._h, ctypes.byref(params), ptr(WH), ptr(WNa), ptr(E)))
        self._leave()
        return E

    def gyrate(self, params, B, dt, UH, UNa):
        """mercury::gyrate (MercuryUns/physics/Gyration.cpp); returns the updated copies of UH, UNa."""
        B = dev(B)
        UH, UNa = dev(UH).clone(), dev(UNa).clone()
        self._enter()
        check(lib().mhd_gpu_gyrate(self._h, ctypes.byref(params), ptr(B), float(dt), ptr(UH), ptr(UNa)))
        self._leave()
        return UH, UNa

    def cell_current(self, B):
        """mhd::cell_current (Common/induction/Current.cpp:9-31): 3 per cell."""
        torch = _torch()
        B = dev(B)
        J = torch.empty(3 * self.n_cells, dtype=torch.float64, device="cuda")
        self._enter()
        check(lib().mhd_gpu_cell_current(self._h, ptr(B), ptr(J)))
        self._leave()
        return J

    # ------------------------------------------------------------- the ten-ion (Mars) source pieces
    # ion arrays species-major, 5 values per cell; mp: MarsParams
    def mars_plasma(self, mp, U, W):
        """MarsSolver::prepare (MarsUns/driver/MarsSolver.cpp:287-303): (n_e, n_e,eff, p_e, u+)."""
        torch = _torch()
        U, W = dev(U), dev(W)
        ne, nee, pe = (torch.empty(self.n_cells, dtype=torch.float64, device="cuda") for _ in range(3))
        up = torch.empty(3 * self.n_cells, dtype=torch.float64, device="cuda")
        self._enter()
        check(lib().mhd_gpu_mars_plasma(self._h, ctypes.byref(mp), ptr(U), ptr(W), ptr(ne), ptr(nee), ptr(pe), ptr(up)))
        self._leave()
        return ne, nee, pe, up

    def pressure_gradient(self, pe):
        """grad p by Gauss' theorem with the face-averaged p (MarsSolver.cpp:305-325): 3 per cell."""
        torch = _torch()
        pe = dev(pe)
        d = torch.empty(3 * self.n_cells, dtype=torch.float64, device="cuda")
        self._enter()
        check(lib().mhd_gpu_pressure_gradient(self._h, ptr(pe), ptr(d)))
        self._leave()
        return d

    def mars_explicit_sources(self, mp, U, W, Btot, J, dpe, ne_eff, rhs):
        """The explicit J x B and ambipolar force of MarsSolver::fluid_and_sources_ (:400-418), added to rhs in place."""
        args = [dev(a) for a in (U, W, Btot, J, dpe, ne_eff)]
        self._enter()
        check(lib().mhd_gpu_mars_explicit_sources(self._h, ctypes.byref(mp), *[ptr(a) for a in args], ptr(rhs)))
        self._leave()
        return rhs

    def mars_ambipolar_emf(self, mp, pe, ne, E):
        """MarsSolver::ambipolar_emf_ (:529-562), E in place."""
        pe, ne = dev(pe), dev(ne)
        self._enter()
        check(lib().mhd_gpu_mars_ambipolar_emf(self._h, ctypes.byref(mp), ptr(pe), ptr(ne), ptr(E)))
        self._leave()
        return E

    def mars_time_step(self, mp, cfl, U, W, Btot, uplus):
        """MarsSolver::local_dt_ (:330-376)."""
        args = [dev(a) for a in (U, W, Btot, uplus)]
        out = ctypes.c_double()
        self._enter()
        check(lib().mhd_gpu_mars_time_step(self._h, ctypes.byref(mp), float(cfl), *[ptr(a) for a in args], ctypes.byref(out)))
        return out.value

    def mars_implicit_sources(self, mp, Btot, neutral, dt, U):
        """MarsSolver::implicit_sources_ (:420-520), U in place."""
        Btot, neutral = dev(Btot), dev(neutral)
        self._enter()
        check(lib().mhd_gpu_mars_implicit_sources(self._h, ctypes.byref(mp), ptr(Btot), ptr(neutral), float(dt), ptr(U)))
        self._leave()
        return U

    def mars_advance(self, n_species, rhs, dt, U):
        """U += dt rhs on the owned non-solid cells (MarsSolver::step :719-726), in place."""
        rhs = dev(rhs)
        self._enter()
        check(lib().mhd_gpu_mars_advance(self._h, int(n_species), ptr(rhs), float(dt), ptr(U)))
        self._leave()
        return U

    def mars_floors(self, mp, U):
        """MarsSolver::floors_ (:686-702), U in place."""
        self._enter()
        check(lib().mhd_gpu_mars_floors(self._h, ctypes.byref(mp), ptr(U)))
        self._leave()
        return U


class MarsParams(ctypes.Structure):
    """MhdMarsParams of include/mhd_gpu.h (the scales of MarsParams::from_params, MarsSolver.cpp:40-110)."""
    _fields_ = [("n_species", i32), ("n_neutral", i32), ("neutral_stride", i32), ("ambipolar", i32), ("mass", dbl * 16)] + \
               [(n, dbl) for n in ("rho_ref", "n_ref", "p_ref", "time_ref", "kB", "L", "U", "q", "B", "mag_scale", "pressure_scale",
                                   "ne_floor", "rho_floor", "p_floor", "gamma")]


def step_params(n_species, gamma=5.0 / 3.0, fs=None, mass=None, u_inf=(0.0, 0.0, 0.0), B_imf=(0.0, 0.0, 0.0), cuct=0.5,
                second_order=True, rho_floor=1e-10, p_floor=1e-12, rel_limit=0.0, cfl=0.4, inver_MA2=1.0, rho_floor_dt=1e-2,
                M_ref=1.0, ne_floor=0.01, absorb=None, precision="fp64", lorentz=False, induce_coeff=0.0, extra=None):
    """MhdStepParams with the reference's Config / Scales defaults (Common/config/Config.h:19-96); extra: the
    ambipolar and chemistry switches and constants (keys ambipolar, chemistry, pressure_coef, a1_Na, a4, a5, a6,
    state_coeff_H, state_coeff_Na, T_ref, Tn0)."""
    p = StepParams()
    p.state_coeff_H = p.state_coeff_Na = p.T_ref = 1.0
    for k, v in (extra or {}).items():
        if k in ("photo", "vst"):
            continue
        setattr(p, k, int(bool(v)) if k in ("ambipolar", "chemistry") else float(v))
    p.precision = PREC_MIXED if precision == "mixed" else PREC_FP64
    p.lorentz, p.induce_coeff = int(bool(lorentz)), float(induce_coeff)
    p.n_species, p.second_order = int(n_species), int(bool(second_order))
    p.gamma, p.rho_floor, p.p_floor, p.cuct = gamma, rho_floor, p_floor, cuct
    p.M_ref, p.ne_floor, p.rel_limit = M_ref, ne_floor, rel_limit
    p.cfl, p.inver_MA2, p.rho_floor_dt = cfl, inver_MA2, rho_floor_dt
    p.u_inf[:] = [float(v) for v in u_inf]
    p.B_imf[:] = [float(v) for v in B_imf]
    mass = mass or [1.0] * n_species
    fs = fs or [(1.0, 0.0, 0.0, 0.0, 1.0)] * n_species
    for s in range(n_species):
        p.mass[s] = float(mass[s])
        p.fs[s] = Prim(*[float(v) for v in fs[s]])
        # reference ghost_state: species 1 is absorbed at walls (Common/fluid/Reconstruction.cpp:15)
        p.absorb[s] = int(s == 1) if absorb is None else int(bool(absorb[s]))
    return p


class ResidentState:
    """Device-resident state of the fused explicit step (MhdState of include/mhd_gpu.h)."""

    def __init__(self, dmesh: DeviceMesh, params: StepParams):
        self.mesh = dmesh
        self.params = params
        self.n_species = params.n_species
        h = vp()
        check(lib().mhd_gpu_state_create(dmesh.handle, ctypes.byref(params), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.mhd_gpu_state_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def upload(self, field, data, species=0):
        a = np.ascontiguousarray(data, np.float64)
        check(lib().mhd_gpu_state_upload(self._h, field, species, a.ctypes.data_as(vp)))

    def download(self, field, species=0, out=None):
        """Copy a field to host memory: a new array, or `out` (contiguous float64 of the field's size,
        e.g. a view of pinned memory, which the device then writes directly)."""
        n = {FIELD_U: 5 * self.mesh.n_cells, FIELD_PHI: self.mesh.n_faces, FIELD_PHIADD: self.mesh.n_faces,
             FIELD_BADD: 3 * self.mesh.n_cells}[field]
        if out is None:
            out = np.empty(n)
        elif out.dtype != np.float64 or out.size != n or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"out must be a contiguous float64 array of {n} values")
        check(lib().mhd_gpu_state_download(self._h, field, species, out.ctypes.data_as(vp)))
        return out

    def set(self, U_list, Phi, PhiAdd=None):
        for s, U in enumerate(U_list):
            self.upload(FIELD_U, U, s)
        self.upload(FIELD_PHI, Phi)
        if PhiAdd is not None:
            self.upload(FIELD_PHIADD, PhiAdd)

    def U(self, species):
        return self.download(FIELD_U, species)

    def Phi(self):
        return self.download(FIELD_PHI)

    def device_ptr(self, field):
        p = vp()
        check(lib().mhd_gpu_state_device_ptr(self._h, field, ctypes.byref(p)))
        return p.value

    def cfl_dt(self, dt_max=1e300):
        d = dbl()
        check(lib().mhd_gpu_cfl_dt(self._h, float(dt_max), ctypes.byref(d)))
        return d.value

    def step(self, dt=0.0, dt_max=1e300, sync=True):
        """One SSP-RK2 step (Solver::step of the hot path); returns the dt used when sync."""
        d = dbl()
        check(lib().mhd_gpu_step_rk2(self._h, float(dt), float(dt_max), ctypes.byref(d) if sync else None))
        return d.value if sync else None

    def step_semi_implicit(self, induction, dt=0.0, dt_max=1e300):
        """One semi-implicit step (Solver::step_first_order, time_order = 1): forward Euler of the fluid and the
        EMF of ImplicitInduction::solve on `induction` (a DeviceInduction of the same mesh) -> (dt, iterations,
        rel_res).  Like the reference, a solve stopped at max_it above rtol does not raise."""
        d, it, rr = dbl(), i32(), dbl()
        rc = lib().mhd_gpu_step_semi_implicit(self._h, induction._h, float(dt), float(dt_max), ctypes.byref(d), ctypes.byref(it),
                                              ctypes.byref(rr))
        if rc != MHD_ENOCONV:
            check(rc)
        return d.value, it.value, rr.value

    def profile(self, enable=True):
        check(lib().mhd_gpu_state_profile(self._h, int(bool(enable))))

    def profile_read(self):
        """{kernel class: (summed ms, launches)} since the last read (synchronises)."""
        return _read_profile(lib().mhd_gpu_state_profile_read, self._h)

    def launches(self):
        v = i64()
        check(lib().mhd_gpu_state_launches(self._h, ctypes.byref(v)))
        return v.value

    def set_source_fields(self, photo=None, vst=None):
        """The chemistry terms' source fields (one value per cell; None: absent)."""
        a = [None if x is None else np.ascontiguousarray(x, np.float64) for x in (photo, vst)]
        check(lib().mhd_gpu_state_set_source_fields(self._h, *[None if x is None else x.ctypes.data_as(vp) for x in a]))

    def set_wall_ghosts(self, faces=None, prims=None):
        """The step's Dirichlet wall table: faces (distinct faces of kind wall) and prims (n_species x n_wall x 5);
        None removes it."""
        if faces is None or len(faces) == 0:
            check(lib().mhd_gpu_state_set_wall_ghosts(self._h, 0, None, None))
            return
        fc = np.ascontiguousarray(faces, np.int32)
        pr = np.ascontiguousarray(prims, np.float64)
        if pr.size != self.params.n_species * fc.size * 5:
            raise ValueError("prims must hold n_species x n_wall x 5 values")
        check(lib().mhd_gpu_state_set_wall_ghosts(self._h, fc.size, fc.ctypes.data_as(vp), pr.ctypes.data_as(vp)))

    def set_resistivity(self, m_edge):
        """Explicit resistive EMF m_e (d1^T star2 Phi)_e per stage (m_edge per edge; None: off)."""
        if m_edge is None:
            check(lib().mhd_gpu_state_set_resistivity(self._h, None))
            return
        a = np.ascontiguousarray(m_edge, np.float64)
        check(lib().mhd_gpu_state_set_resistivity(self._h, a.ctypes.data_as(vp)))


def _wall_dev(wall):
    torch = _torch()
    faces, prims = wall
    fc = torch.as_tensor(np.ascontiguousarray(faces, np.int32)).to("cuda")
    pr = dev(np.ascontiguousarray(prims, np.float64).ravel())
    return fc, pr


class GeometryArgs(ctypes.Structure):
    """MhdGeometryArgs of include/mhd_gpu.h."""
    _fields_ = [("n_nodes", i32), ("n_edges", i32), ("n_faces", i32), ("n_cells", i32)] + \
               [(n, vp) for n in ("x", "edge_nodes", "f2e_ptr", "f2e_idx", "f2e_sgn", "c2f_ptr", "c2f_idx", "c2f_sgn", "e2f_ptr",
                                  "e2f_idx", "f2c_ptr", "f2c_idx", "edge_vec", "edge_mid", "edge_len", "face_area", "face_center",
                                  "face_area_mag", "cell_center", "cell_volume", "cell_min_tet_volume", "star0", "star1", "star2",
                                  "star3", "edge_dual_area", "ec_misoriented", "ef_weight", "ec_ptr", "ec_cell", "ec_weight")] + \
               [("ec_capacity", i64)]


_GEO_OUT = {"edge_vec": 3, "edge_mid": 3, "edge_len": 1, "face_area": 3, "face_center": 3, "face_area_mag": 1, "cell_center": 3,
            "cell_volume": 1, "cell_min_tet_volume": 1, "star0": 1, "star1": 1, "star2": 1, "star3": 1, "edge_dual_area": 3}
_GEO_ENT = {"edge_vec": "e", "edge_mid": "e", "edge_len": "e", "face_area": "f", "face_center": "f", "face_area_mag": "f",
            "cell_center": "c", "cell_volume": "c", "cell_min_tet_volume": "c", "star0": "n", "star1": "e", "star2": "f", "star3": "c",
            "edge_dual_area": "e"}


def compute_geometry(host_mesh):
    """uns::compute_geometry on the device for a host mesh's topology and coordinates: a dict of every
    geometry array (bit-identical to the host computation)."""
    h = host_mesh
    keep = {}

    def inp(name, dtype, src=None):
        a = np.ascontiguousarray(np.asarray(h[src or name]).ravel(), dtype)
        keep[name] = a
        return ctypes.c_void_p(a.ctypes.data)

    g = GeometryArgs()
    g.n_nodes, g.n_edges, g.n_faces, g.n_cells = h.n_nodes, h.n_edges, h.n_faces, h.n_cells
    g.x = inp("x", np.float64)
    g.edge_nodes = inp("edge_nodes", np.int32, "e2n_idx")
    for t in ("f2e", "c2f", "e2f", "f2c"):
        setattr(g, t + "_ptr", inp(t + "_ptr", np.int64))
        setattr(g, t + "_idx", inp(t + "_idx", np.int32))
    g.f2e_sgn = inp("f2e_sgn", np.int8)
    g.c2f_sgn = inp("c2f_sgn", np.int8)
    n = {"n": h.n_nodes, "e": h.n_edges, "f": h.n_faces, "c": h.n_cells}
    out = {k: np.empty(n[_GEO_ENT[k]] * w) for k, w in _GEO_OUT.items()}
    out["ec_misoriented"] = np.empty(h.n_edges, np.int32)
    out["ef_weight"] = np.empty(int(np.asarray(h["e2f_ptr"])[-1]))
    out["ec_ptr"] = np.empty(h.n_edges + 1, np.int64)
    cap = 2 * out["ef_weight"].size
    out["ec_cell"] = np.empty(cap, np.int32)
    out["ec_weight"] = np.empty(cap)
    for k, a in out.items():
        setattr(g, k, ctypes.c_void_p(a.ctypes.data))
    g.ec_capacity = cap
    check(lib().mhd_gpu_compute_geometry(ctypes.byref(g)))
    m = int(out["ec_ptr"][-1])
    out["ec_cell"], out["ec_weight"] = out["ec_cell"][:m].copy(), out["ec_weight"][:m].copy()
    return out


class BoundaryArgs(ctypes.Structure):
    _fields_ = [("n_edges", i32), ("n_faces", i32), ("n_cells", i32), ("n_tags", i32)] + \
               [(k, vp) for k in ("f2c_ptr", "f2c_idx", "f2c_sgn", "e2f_ptr", "e2f_idx", "cell_material", "face_tag", "face_area",
                                  "face_area_mag", "tag_type")] + \
               [("type_none", ctypes.c_int8), ("pad", ctypes.c_int8 * 7), ("u_inf", dbl * 3), ("face_kind", vp), ("edge_mode", vp)]


def boundary(host_mesh, tag_type, type_none, u_inf):
    """mhd::BoundaryInfo::build on the device (mhd_gpu_boundary) for a host mesh with geometry and the per-tag-id
    boundary types (HostMesh.boundary(device=True) resolves them): (face_kind int8, edge_mode int8)."""
    h = host_mesh
    keep = []

    def inp(name, dtype, a=None):
        a = np.ascontiguousarray(np.asarray(h[name] if a is None else a).ravel(), dtype)
        keep.append(a)
        return ctypes.c_void_p(a.ctypes.data)

    b = BoundaryArgs()
    b.n_edges, b.n_faces, b.n_cells = h.n_edges, h.n_faces, h.n_cells
    tt = np.ascontiguousarray(tag_type, np.int8)
    b.n_tags = tt.size
    b.f2c_ptr, b.f2c_idx, b.f2c_sgn = inp("f2c_ptr", np.int64), inp("f2c_idx", np.int32), inp("f2c_sgn", np.int8)
    b.e2f_ptr, b.e2f_idx = inp("e2f_ptr", np.int64), inp("e2f_idx", np.int32)
    b.cell_material, b.face_tag = inp("cell_material", np.int32), inp("face_tag", np.int32)
    b.face_area, b.face_area_mag = inp("face_area", np.float64), inp("face_area_mag", np.float64)
    b.tag_type = inp(None, np.int8, tt)
    b.type_none = int(type_none)
    b.u_inf[:] = [float(x) for x in u_inf]
    fk = np.empty(h.n_faces, np.int8)
    em = np.empty(h.n_edges, np.int8)
    b.face_kind, b.edge_mode = ctypes.c_void_p(fk.ctypes.data), ctypes.c_void_p(em.ctypes.data)
    check(lib().mhd_gpu_boundary(ctypes.byref(b)))
    return fk, em


class FnParams(ctypes.Structure):
    _fields_ = [("n_steps", i32), ("checkpoint_every", i32), ("dt", dbl), ("uniform_flow", i32), ("pad", i32)]


def _vp(a):
    return None if a is None else a.ctypes.data_as(vp)


class DeviceFunction:
    """Differentiated explicit run (MhdFn of include/mhd_gpu.h): J = sum over `mask` of |B_tot|^2 V after
    n_steps FP64 steps at the fixed dt, with its adjoint gradient with respect to the per-cell resistivity
    and the inflow velocity, and its tangent-linear derivative.  Starts from the state's current U, Phi."""

    def __init__(self, state: ResidentState, eta, mask, n_steps, checkpoint_every, dt, uniform_flow=True):
        self.state = state
        self.n_cells = state.mesh.n_cells
        self.n_faces = state.mesh.n_faces
        self.n_edges = state.mesh.n_edges
        self.n_species = state.n_species
        p = FnParams(int(n_steps), int(checkpoint_every), float(dt), int(bool(uniform_flow)), 0)
        e = np.ascontiguousarray(eta, np.float64)
        mk = np.ascontiguousarray(mask, np.int8)
        h = vp()
        check(lib().mhd_gpu_fn_create(state.handle, ctypes.byref(p), _vp(e), _vp(mk), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.mhd_gpu_fn_destroy(self._h)
            self._h = None

    def set_params(self, eta=None, u_inf=None):
        e = None if eta is None else np.ascontiguousarray(eta, np.float64)
        u = None if u_inf is None else np.ascontiguousarray(u_inf, np.float64)
        check(lib().mhd_gpu_fn_set_params(self._h, _vp(e), _vp(u)))

    def reset(self):
        check(lib().mhd_gpu_fn_reset(self._h))

    def forward(self):
        J = dbl()
        check(lib().mhd_gpu_fn_forward(self._h, ctypes.byref(J)))
        return J.value

    def last_J(self):
        """(hi, lo): the last run's J as a double-double, for differences finer than J's ulp."""
        a = np.empty(2)
        check(lib().mhd_gpu_fn_last_J(self._h, _vp(a)))
        return float(a[0]), float(a[1])

    @staticmethod
    def central_difference(Jp, Jm, h):
        """(J(p + h d) - J(p - h d)) / 2h from two last_J() pairs."""
        return ((Jp[0] - Jm[0]) + (Jp[1] - Jm[1])) / (2 * h)

    def backward(self):
        """(dJ/deta per cell, dJ/du_inf (3,)) of the last forward run."""
        ge = np.empty(self.n_cells)
        gu = np.empty(3)
        check(lib().mhd_gpu_fn_backward(self._h, _vp(ge), _vp(gu)))
        return ge, gu

    def tangent(self, d_eta=None, d_u=None):
        """(J, dJ) of a tangent-linear run along (d_eta, d_u)."""
        de = None if d_eta is None else np.ascontiguousarray(d_eta, np.float64)
        du = None if d_u is None else np.ascontiguousarray(d_u, np.float64)
        J, dJ = dbl(), dbl()
        check(lib().mhd_gpu_fn_tangent(self._h, _vp(de), _vp(du), ctypes.byref(J), ctypes.byref(dJ)))
        return J.value, dJ.value

    def stage_tangent(self, U, Phi, dU, dPhi, d_eta=None, d_u=None):
        """Derivatives of one stage's U~ and E along (dU, dPhi, d_eta, d_u); U in the device layout."""
        a = [np.ascontiguousarray(x, np.float64) for x in (U, Phi, dU, dPhi)]
        de = None if d_eta is None else np.ascontiguousarray(d_eta, np.float64)
        du = None if d_u is None else np.ascontiguousarray(d_u, np.float64)
        dUt = np.empty(5 * self.n_species * self.n_cells)
        dE = np.empty(self.n_edges)
        check(lib().mhd_gpu_fn_stage_tangent(self._h, *[_vp(x) for x in a], _vp(de), _vp(du), _vp(dUt), _vp(dE)))
        return dUt, dE

    def profile(self, enable=True):
        check(lib().mhd_gpu_fn_profile(self._h, int(bool(enable))))

    def profile_read(self):
        """{kernel class: (summed ms, launches)} since the last read (synchronises)."""
        return _read_profile(lib().mhd_gpu_fn_profile_read, self._h)

    SWITCH_KINDS = ("limiter", "flux", "edge", "floor", "face_emf")

    def switch_log(self, enable=True):
        """While enabled, each forward run leaves per entity a hash of the discrete choices it made
        (mhd_gpu_fn_switch_log)."""
        check(lib().mhd_gpu_fn_switch_log(self._h, int(bool(enable))))

    def switches(self):
        """{kind: uint32 hashes} of the last forward run (kinds: limiter, flux, edge, floor, face_emf)."""
        ns, nc, nf, ne = self.n_species, self.n_cells, self.n_faces, self.n_edges
        out = {}
        for k, (name, n) in enumerate(zip(self.SWITCH_KINDS, (ns * 5 * nc, ns * nf, ne, ns * nc, nf))):
            a = np.empty(n, np.uint32)
            check(lib().mhd_gpu_fn_switch_read(self._h, k, _vp(a), n))
            out[name] = a
        return out

    @staticmethod
    def switch_flips(a, b):
        """{kind: entities whose choices differ} between two switches() results."""
        return {k: int(np.count_nonzero(a[k] != b[k])) for k in a}

    def stage_adjoint(self, U, Phi, lUt, lE):
        """Adjoints of one stage's inputs (U, Phi, eta, u_inf) from those of its U~ and E."""
        a = [np.ascontiguousarray(x, np.float64) for x in (U, Phi, lUt, lE)]
        lU = np.empty(5 * self.n_species * self.n_cells)
        lP = np.empty(self.n_faces)
        le = np.empty(self.n_cells)
        lu = np.empty(3)
        check(lib().mhd_gpu_fn_stage_adjoint(self._h, *[_vp(x) for x in a], _vp(lU), _vp(lP), _vp(le), _vp(lu)))
        return lU, lP, le, lu


class DeviceInduction:
    """mhd::ImplicitInduction on the device (Common/induction/ImplicitInduction.cpp; MhdInduction of include/mhd_gpu.h).

    ``m_edge`` is the per-edge resistive coefficient m_e (the reference's ``m_``, ctor :16-22), ``None`` for
    a Hall-only solve.  ``precision="mixed"`` runs the Arnoldi matvecs with the FP32 operator and keeps the
    Krylov basis, Hessenberg, Givens and the true residual of every restart in FP64.  Vectors may be numpy
    arrays or CUDA tensors; results are CUDA float64 tensors.  Like the reference, ``solve`` does not raise
    when GMRES stops at ``max_it`` above ``rtol``: it returns the iterations and the relative residual.
    """

    def __init__(self, dmesh: DeviceMesh, m_edge=None, hall=False, hall_coef=0.0, hall_r_min=1.0, hall_r_max=1.012,
                 rtol=1e-4, max_it=100, restart=20, precision="fp64"):
        self.mesh = dmesh
        p = InductionParams(int(bool(hall)), int(max_it), int(restart), PREC_MIXED if precision == "mixed" else PREC_FP64,
                            float(hall_coef), float(hall_r_min), float(hall_r_max), float(rtol))
        self.params = p
        m = None if m_edge is None else np.ascontiguousarray(m_edge, np.float64)
        h = vp()
        check(lib().mhd_gpu_induction_create(dmesh.handle, ctypes.byref(p), None if m is None else m.ctypes.data_as(vp),
                                             ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.mhd_gpu_induction_destroy(self._h)
            self._h = None

    def set_frozen_state(self, B0, ne_eff):
        B0, ne = dev(B0), dev(ne_eff)
        self.mesh._enter()
        check(lib().mhd_gpu_induction_set_frozen(self._h, ptr(B0), ptr(ne)))
        self.mesh._leave()

    def apply_F(self, phi):
        torch = _torch()
        phi = dev(phi)
        out = torch.empty(self.mesh.n_edges, dtype=torch.float64, device="cuda")
        self.mesh._enter()
        check(lib().mhd_gpu_induction_apply_F(self._h, ptr(phi), ptr(out)))
        self.mesh._leave()
        return out

    def apply_A(self, x, dt):
        torch = _torch()
        x = dev(x)
        y = torch.empty(self.mesh.n_edges, dtype=torch.float64, device="cuda")
        self.mesh._enter()
        check(lib().mhd_gpu_induction_apply_A(self._h, ptr(x), float(dt), ptr(y)))
        self.mesh._leave()
        return y

    def solve(self, Phi, E_expl, dirichlet, dt, warm=True, E=None):
        """ImplicitInduction::solve (:299-390) -> (E, iterations, rel_res)."""
        torch = _torch()
        Phi, Ee = dev(Phi), dev(E_expl)
        d = dev(np.ascontiguousarray(dirichlet, np.int8)) if not isinstance(dirichlet, torch.Tensor) else dirichlet.to(
            torch.int8).contiguous().cuda()
        if E is None:
            E = torch.empty(self.mesh.n_edges, dtype=torch.float64, device="cuda")
        it, rr = i32(), dbl()
        self.mesh._enter()
        rc = lib().mhd_gpu_induction_solve(self._h, ptr(Phi), ptr(Ee), ptr(d), float(dt), int(bool(warm)), ptr(E),
                                           ctypes.byref(it), ctypes.byref(rr))
        self.mesh._leave()
        if rc != MHD_ENOCONV:
            check(rc)
        return E, it.value, rr.value

    def solve_dt_edge(self, Phi, E_expl, dirichlet, dt_edge, warm=True, E=None):
        """ImplicitInduction::solve with the per-edge pseudo-time step dt_edge (:299-390) -> (E, iterations, rel_res)."""
        torch = _torch()
        Phi, Ee, dte = dev(Phi), dev(E_expl), dev(dt_edge)
        d = self._dir(dirichlet)
        if E is None:
            E = torch.empty(self.mesh.n_edges, dtype=torch.float64, device="cuda")
        it, rr = i32(), dbl()
        self.mesh._enter()
        rc = lib().mhd_gpu_induction_solve_dt_edge(self._h, ptr(Phi), ptr(Ee), ptr(d), ptr(dte), int(bool(warm)), ptr(E),
                                                   ctypes.byref(it), ctypes.byref(rr))
        self.mesh._leave()
        if rc != MHD_ENOCONV:
            check(rc)
        return E, it.value, rr.value

    def set_ideal_state(self, u_cell, mask, cuct=0.5):
        """ImplicitInduction::set_ideal_state (:112-116) with Config::implicit_ideal: u 3 per cell, mask 1 per edge
        (None: the ideal part off)."""
        if u_cell is None:
            check(lib().mhd_gpu_induction_set_ideal(self._h, None, None, float(cuct)))
            return
        u, m = dev(u_cell), self._dir(mask)
        self.mesh._enter()
        check(lib().mhd_gpu_induction_set_ideal(self._h, ptr(u), ptr(m), float(cuct)))
        self.mesh._leave()

    def ideal_linear(self, phi):
        """ImplicitInduction::ideal_linear (:118-124): the implicit ideal part alone."""
        torch = _torch()
        phi = dev(phi)
        out = torch.empty(self.mesh.n_edges, dtype=torch.float64, device="cuda")
        self.mesh._enter()
        check(lib().mhd_gpu_induction_ideal_linear(self._h, ptr(phi), ptr(out)))
        self.mesh._leave()
        return out

    def profile(self, enable=True):
        check(lib().mhd_gpu_induction_profile(self._h, int(bool(enable))))

    def profile_read(self):
        """{kernel class: (summed ms, launches)} since the last read (synchronises)."""
        return _read_profile(lib().mhd_gpu_induction_profile_read, self._h)

    def launches(self):
        v = i64()
        check(lib().mhd_gpu_induction_launches(self._h, ctypes.byref(v)))
        return v.value

    def reorth_passes(self):
        """Gram-Schmidt second passes (re-orthogonalisations) of the last solve."""
        v = i32()
        check(lib().mhd_gpu_induction_last_solve_stats(self._h, ctypes.byref(v)))
        return v.value

    def set_ilu(self, enable=True, shift=0.3):
        """Config::ind_ilu / ind_ilu_shift: block-Jacobi ILU(0) in place of the Jacobi preconditioner
        (ImplicitInduction.cpp:209-297); builds the pattern on the first call."""
        self.mesh._enter()
        check(lib().mhd_gpu_induction_set_ilu(self._h, int(bool(enable)), float(shift)))
        self.mesh._leave()

    def _dir(self, dirichlet):
        torch = _torch()
        if dirichlet is None:
            return None
        if isinstance(dirichlet, torch.Tensor):
            return dirichlet.to(torch.int8).contiguous().cuda()
        return dev(np.ascontiguousarray(dirichlet, np.int8))

    def ilu_factor(self, dt, dirichlet=None):
        """factor_precond (:247-275) for dt and the Dirichlet flags."""
        d = self._dir(dirichlet)
        self.mesh._enter()
        check(lib().mhd_gpu_induction_ilu_factor(self._h, float(dt), None if d is None else ptr(d)))
        self.mesh._leave()

    def ilu_apply(self, v, dirichlet=None):
        """apply_precond (:277-297) with the current factors -> z (CUDA float64)."""
        torch = _torch()
        v, d = dev(v), self._dir(dirichlet)
        z = torch.empty(self.mesh.n_edges, dtype=torch.float64, device="cuda")
        self.mesh._enter()
        check(lib().mhd_gpu_induction_ilu_apply(self._h, None if d is None else ptr(d), ptr(v), ptr(z)))
        self.mesh._leave()
        return z

    def ilu_debug(self, wait_s=2.0, unpublished_row=-1):
        """Test hook of the ILU(0) passes' bounded waits (mhd_gpu_induction_ilu_debug)."""
        check(lib().mhd_gpu_induction_ilu_debug(self._h, float(wait_s), int(unpublished_row)))

    def ilu_tune(self, window_levels=8, max_backoff_ns=128, spin_polls=0):
        """Launch shape of the ILU(0) passes (mhd_gpu_induction_ilu_tune)."""
        check(lib().mhd_gpu_induction_ilu_tune(self._h, int(window_levels), int(max_backoff_ns), int(spin_polls)))

    def ilu_arrays(self):
        """{pc_ptr, pc_col, pc_coef, pc_val, pc_diag} of the pattern and the current factors (host)."""
        no, nnz = i32(), i64()
        check(lib().mhd_gpu_induction_ilu_arrays(self._h, ctypes.byref(no), ctypes.byref(nnz), None, None, None, None, None))
        out = dict(pc_ptr=np.zeros(no.value + 1, np.int64), pc_col=np.zeros(nnz.value, np.int32), pc_coef=np.zeros(nnz.value),
                   pc_val=np.zeros(nnz.value), pc_diag=np.zeros(no.value, np.int64))
        check(lib().mhd_gpu_induction_ilu_arrays(self._h, ctypes.byref(no), ctypes.byref(nnz),
                                                 *[out[k].ctypes.data_as(vp) for k in ("pc_ptr", "pc_col", "pc_coef", "pc_val",
                                                                                         "pc_diag")]))
        return out


def ilu_pattern(n_edges, n_owned, n_faces, e2f, f2e, star2, m_edge):
    """ImplicitInduction::build_precond_pattern (Common/induction/ImplicitInduction.cpp:209-242) on host arrays
    (no GPU work): e2f and f2e as (ptr int64, idx int32, sgn int8) -> (pc_ptr, pc_col, pc_coef)."""
    a = [np.ascontiguousarray(e2f[0], np.int64), np.ascontiguousarray(e2f[1], np.int32), np.ascontiguousarray(e2f[2], np.int8),
         np.ascontiguousarray(f2e[0], np.int64), np.ascontiguousarray(f2e[1], np.int32), np.ascontiguousarray(f2e[2], np.int8),
         np.ascontiguousarray(star2, np.float64), np.ascontiguousarray(m_edge, np.float64)]
    pp = np.zeros(n_owned + 1, np.int64)
    args = [int(n_edges), int(n_owned), int(n_faces)] + [x.ctypes.data_as(vp) for x in a]
    check(lib().mhd_ilu_pattern(*args, pp.ctypes.data_as(vp), None, None))
    col, coef = np.zeros(int(pp[-1]), np.int32), np.zeros(int(pp[-1]))
    check(lib().mhd_ilu_pattern(*args, pp.ctypes.data_as(vp), col.ctypes.data_as(vp), coef.ctypes.data_as(vp)))
    return pp, col, coef


class ComplexOut(ctypes.Structure):
    """MhdComplexOut of include/mhd_gpu.h: host outputs of the device tetrahedral builder."""
    _fields_ = [("ptr", vp * 6), ("idx", vp * 6), ("sgn", vp * 6), ("cell_material", vp), ("face_tag", vp)]


def build_tets(m):
    """The tetrahedral complex of a HostMesh that holds a hexahedral list (mhdm_shell_hexes), numbered on the
    device (mhd_gpu_tet_build) and installed in m: the complex of uns::ComplexBuilder fed the Kuhn tetrahedra."""
    from . import mesh as _mesh
    L = lib()
    hexes = np.ascontiguousarray(m["hex"], np.int32)
    mat = np.ascontiguousarray(m["hex_material"], np.int32)
    tri = np.ascontiguousarray(m["tag_tri"], np.int32)
    tid = np.ascontiguousarray(m["tag_tri_id"], np.int32)
    b = vp()
    check(L.mhd_gpu_tet_build(int(m.n_nodes), hexes.size // 8, hexes.ctypes.data_as(vp), mat.ctypes.data_as(vp), tid.size,
                              tri.ctypes.data_as(vp), tid.ctypes.data_as(vp), ctypes.byref(b)))
    try:
        counts = np.zeros(4, np.int64)
        check(L.mhd_gpu_tet_build_counts(b, counts.ctypes.data_as(vp)))
        del hexes, mat, tri, tid
        m._cache.clear()
        ML = _mesh.lib()
        _mesh._check(ML.mhdm_reserve_complex(m._h, int(counts[1]), int(counts[2]), int(counts[3]), 4, 3))
        out = ComplexOut()

        def arr(name):
            n = i64()
            return ML.mhdm_array_mut(m._h, name.encode(), ctypes.byref(n))
        for k, t in enumerate(("e2n", "f2e", "c2f", "n2e", "e2f", "f2c")):
            out.ptr[k], out.idx[k], out.sgn[k] = arr(t + "_ptr"), arr(t + "_idx"), arr(t + "_sgn")
        out.cell_material, out.face_tag = arr("cell_material"), arr("face_tag")
        check(L.mhd_gpu_tet_build_copy(b, ctypes.byref(out)))
    finally:
        L.mhd_gpu_tet_build_free(b)
    m._recount()
    return m


def _read_profile(fn, h):
    names = ctypes.create_string_buffer(32 * 16)
    ms = np.zeros(16)
    cnt = np.zeros(16, np.int64)
    n = i32()
    check(fn(h, 16, names, ms.ctypes.data_as(vp), cnt.ctypes.data_as(vp), ctypes.byref(n)))
    raw = names.raw
    return {raw[32 * k:32 * k + 32].split(b"\0")[0].decode(): (float(ms[k]), int(cnt[k])) for k in range(n.value)}
