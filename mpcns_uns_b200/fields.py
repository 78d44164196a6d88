"""UNSBIN field files and the Mercury solver's restart semantics.

write_fields / read_fields are uns::io::write_fields / read_fields (src/uns/io/MeshIO.cpp:117-150) over
the UNSBIN container (src/uns/io/BinContainer.cpp), implemented in the host library (libmhd_mesh).
write_global_fields and read_init_fields follow mercury::Solver::write_global_fields
(MercuryUns/driver/Solver.cpp:720-744) and the init_fields branch of the initial state
(MercuryUns/initial/Initial.cpp:38-63), with the derived fields computed on the device.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import mesh as _mesh

DIM_NODE, DIM_EDGE, DIM_FACE, DIM_CELL = 0, 1, 2, 3   # uns::Dim


@dataclass
class FieldRecord:
    """uns::io::FieldRecord: `values` holds count(dim) * ncomp doubles in entity order."""
    name: str
    dim: int
    ncomp: int
    values: np.ndarray


def _lib():
    L = _mesh.lib()
    if not hasattr(L, "_fields_bound"):
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        L.mhdm_write_fields.argtypes = [ctypes.c_char_p, ctypes.c_uint64, i32, vp, vp, vp, vp, vp]
        L.mhdm_read_fields.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp)]
        L.mhdm_fields_free.argtypes = [vp]
        L.mhdm_fields_count.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
        L.mhdm_fields_count.restype = i32
        L.mhdm_field.argtypes = [vp, i32, ctypes.c_char_p, i32, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i64), vp]
        L._fields_bound = True
    return L


def _check(rc):
    if rc != 0:
        raise RuntimeError(_mesh.lib().mhdm_last_error().decode())


def write_fields(path: str, topology_hash: int, records) -> None:
    """uns::io::write_fields: a "hash" record, per field "f.<name>.info" (dim, ncomp) and "f.<name>"
    (ncomp columns), then the "index" of the names."""
    recs = list(records)
    vals = [np.ascontiguousarray(r.values, np.float64).ravel() for r in recs]
    names = (ctypes.c_char_p * max(1, len(recs)))(*[r.name.encode() for r in recs])
    dims = np.array([r.dim for r in recs] or [0], np.int32)
    ncomps = np.array([r.ncomp for r in recs] or [1], np.int32)
    counts = np.array([v.size for v in vals] or [0], np.int64)
    ptrs = (ctypes.c_void_p * max(1, len(recs)))(*[v.ctypes.data for v in vals])
    _check(_lib().mhdm_write_fields(path.encode(), ctypes.c_uint64(topology_hash & (2 ** 64 - 1)), len(recs),
                                    ctypes.cast(names, ctypes.c_void_p), dims.ctypes.data, ncomps.ctypes.data,
                                    counts.ctypes.data, ctypes.cast(ptrs, ctypes.c_void_p)))


def read_fields(path: str):
    """uns::io::read_fields: (records in the order of the file's index, topology hash)."""
    L = _lib()
    h = ctypes.c_void_p()
    _check(L.mhdm_read_fields(path.encode(), ctypes.byref(h)))
    try:
        hv = ctypes.c_uint64()
        n = L.mhdm_fields_count(h, ctypes.byref(hv))
        out = []
        name = ctypes.create_string_buffer(4096)
        for i in range(n):
            dim, ncomp, count = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
            _check(L.mhdm_field(h, i, name, 4096, ctypes.byref(dim), ctypes.byref(ncomp), ctypes.byref(count), None))
            v = np.empty(count.value)
            _check(L.mhdm_field(h, i, name, 4096, ctypes.byref(dim), ctypes.byref(ncomp), ctypes.byref(count), v.ctypes.data))
            out.append(FieldRecord(name.value.decode(), dim.value, ncomp.value, v))
        return out, hv.value
    finally:
        L.mhdm_fields_free(h)


def global_fields(state, time=0.0):
    """The records of mercury::Solver::write_global_fields for a resident two-ion state: U_H, U_Na (cell, 5),
    B (face, 1), rho and p (cell, 1: the sums over the ions), B_cell (cell, 3: the total field), J_cell
    (cell, 3: the current of the induced field) and _time (node, 1).  The derived fields are those of
    Solver::prepare, computed on the device."""
    from . import gpu
    if state.n_species != 2:
        raise ValueError("write_global_fields is the two-ion solver's output")
    dm, p = state.mesh, state.params
    U = [state.U(s) for s in range(2)]
    Phi = state.Phi()
    W = [dm.to_prim(u, p.gamma, p.rho_floor, p.p_floor).cpu().numpy().reshape(-1, 5) for u in U]
    Bind = dm.reconstruct_cell_vector(Phi)
    Btot = (Bind + gpu.dev(state.download(gpu.FIELD_BADD))).cpu().numpy()
    J = dm.cell_current(Bind).cpu().numpy()
    return [FieldRecord("U_H", DIM_CELL, 5, U[0]), FieldRecord("U_Na", DIM_CELL, 5, U[1]), FieldRecord("B", DIM_FACE, 1, Phi),
            FieldRecord("rho", DIM_CELL, 1, W[0][:, 0] + W[1][:, 0]), FieldRecord("p", DIM_CELL, 1, W[0][:, 4] + W[1][:, 4]),
            FieldRecord("B_cell", DIM_CELL, 3, Btot), FieldRecord("J_cell", DIM_CELL, 3, J),
            FieldRecord("_time", DIM_NODE, 1, np.array([float(time)]))]


def write_global_fields(state, path: str, time=0.0) -> None:
    """mercury::Solver::write_global_fields (Solver.cpp:720-744): the records of global_fields with the
    topology hash 0, as the reference writes it."""
    write_fields(path, 0, global_fields(state, time))


def read_init_fields(path: str):
    """The init_fields branch of the initial state (Initial.cpp:38-63): U_H and U_Na (cell, 5 per cell), B
    (face) and _time; raises when U_H, U_Na or B is missing."""
    recs, _ = read_fields(path)
    got = {}
    time = None
    for r in recs:
        if r.name in ("U_H", "U_Na") and r.dim == DIM_CELL and r.ncomp == 5:
            got[r.name] = r.values
        elif r.name == "_time" and r.values.size:
            time = float(r.values[0])
        elif r.name == "B" and r.dim == DIM_FACE:
            got["B"] = r.values
    if not all(k in got for k in ("U_H", "U_Na", "B")):
        raise RuntimeError(f"init_fields '{path}' lacks U_H, U_Na or B")
    return got["U_H"], got["U_Na"], got["B"], time


def restart(state, path: str):
    """Load a field file into a resident two-ion state (U of both ions and the induced face flux); returns
    the stored time (None if absent)."""
    from . import gpu
    UH, UNa, B, time = read_init_fields(path)
    state.upload(gpu.FIELD_U, UH, 0)
    state.upload(gpu.FIELD_U, UNa, 1)
    state.upload(gpu.FIELD_PHI, B)
    return time
