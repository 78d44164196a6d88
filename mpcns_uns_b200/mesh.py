"""Host-side signed cell complex, metric and boundary classification (ctypes over libmhd_mesh.so).

`HostMesh` carries the reference's data model as numpy arrays: the signed CSR incidence
tables of uns::CellComplex (include/uns/complex/CellComplex.h:29-53), the metric of
uns::Geometry (include/uns/geometry/Geometry.h:25-43) and the face kinds / edge modes of
mhd::BoundaryInfo (Common/boundary/BoundaryInfo.h:21-29).  It is what the device mesh of
`mpcns_uns_b200.gpu` is created from.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

_lib = None

# face kinds of mhd::FaceKind (Common/boundary/BoundaryInfo.h:21)
INTERIOR, WALL, INFLOW, OUTFLOW, SKIP = 0, 1, 2, 3, 4

_DT = {
    "x": np.float64, "cell_material": np.int32, "face_tag": np.int32, "hex": np.int32, "hex_material": np.int32,
    "tag_tri": np.int32, "tag_tri_id": np.int32,
    "face_kind": np.int8, "edge_mode": np.int8, "ec_ptr": np.int64, "ec_cell": np.int32,
    "ec_misoriented": np.int32,
}
_VEC3 = {"x", "edge_vec", "edge_mid", "face_area", "face_center", "cell_center", "edge_dual_area"}


class _GeometryArrays(ctypes.Structure):
    """MhdGeometryArrays of include/mhd_mesh.h."""
    _fields_ = [(n, ctypes.c_void_p) for n in ("edge_vec", "edge_mid", "edge_len", "face_area", "face_center", "face_area_mag",
                                               "cell_center", "cell_volume", "cell_min_tet_volume", "edge_dual_area", "ec_weight",
                                               "ef_weight", "star0", "star1", "star2", "star3", "ec_ptr", "ec_cell",
                                               "ec_misoriented")]


def lib():
    global _lib
    if _lib is None:
        path = _build.MESH_SO
        if not os.path.exists(path):
            _build.build_mesh()
        L = ctypes.CDLL(path)
        vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        L.mhdm_last_error.restype = ctypes.c_char_p
        L.mhdm_box.argtypes = [i32, i32, i32, vp, vp, i32, dbl, ctypes.c_uint64, ctypes.POINTER(vp)]
        L.mhdm_shell.argtypes = [i32, i32, i32, dbl, dbl, dbl, i32, ctypes.POINTER(vp)]
        L.mhdm_shell_hexes.argtypes = [i32, i32, i32, dbl, dbl, dbl, ctypes.POINTER(vp)]
        L.mhdm_reserve_complex.argtypes = [vp, i64, i64, i64, i32, i32]
        L.mhdm_array_mut.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(i64)]
        L.mhdm_array_mut.restype = vp
        L.mhdm_from_cells.argtypes = [i32, vp, i32, vp, vp, vp, vp, i32, vp, vp, vp, i32, vp, ctypes.POINTER(vp)]
        L.mhdm_free.argtypes = [vp]
        L.mhdm_counts.argtypes = [vp, vp]
        L.mhdm_topology_hash.argtypes = [vp]
        L.mhdm_topology_hash.restype = ctypes.c_uint64
        L.mhdm_compute_geometry.argtypes = [vp]
        L.mhdm_set_geometry.argtypes = [vp, vp]
        L.mhdm_reorder_cells.argtypes = [vp, vp, ctypes.POINTER(vp)]
        L.mhdm_boundary.argtypes = [vp, ctypes.c_char_p, i32, vp, vp, vp]
        L.mhdm_tag_types.argtypes = [vp, ctypes.c_char_p, i32, vp, vp, i32, vp, vp, vp]
        L.mhdm_set_boundary.argtypes = [vp, vp, vp]
        L.mhdm_array.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(i64)]
        L.mhdm_array.restype = vp
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(lib().mhdm_last_error().decode())


def _dptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class HostMesh:
    """A cell complex with its geometry; arrays are read-only views owned by the native handle."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)
        c = np.zeros(4, np.int32)
        lib().mhdm_counts(self._h, c.ctypes.data)
        self.n_nodes, self.n_edges, self.n_faces, self.n_cells = (int(v) for v in c)
        self._cache = {}

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.mhdm_free(self._h)
            self._h = None

    # ------------------------------------------------------------- constructors
    @classmethod
    def box(cls, nx, ny, nz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), tets=False, jitter=0.0, seed=0):
        """uns::make_box (src/uns/generate/BoxMesh.cpp:5-33); tets=True cuts each hexahedron into 6."""
        out = ctypes.c_void_p()
        lo_ = np.asarray(lo, np.float64)
        hi_ = np.asarray(hi, np.float64)
        _check(lib().mhdm_box(nx, ny, nz, lo_.ctypes.data, hi_.ctypes.data, int(tets), float(jitter), int(seed),
                              ctypes.byref(out)))
        return cls(out.value)

    @classmethod
    def shell(cls, ncube, nr, r_in=1.0, r_out=10.0, r_stretch=1.0, n_solid=0, tets=False, device_build=False):
        """uns::make_cubed_sphere_shell (src/uns/generate/CubedSphereMesh.cpp:12-83).  device_build (with tets):
        the hexahedral list on the host, the tetrahedral complex numbered on the GPU (mhd_gpu_tet_build: the same
        complex, same topology hash, in a fraction of the time for large shells)."""
        out = ctypes.c_void_p()
        if device_build:
            if not tets:
                raise ValueError("device_build builds the tetrahedral split")
            _check(lib().mhdm_shell_hexes(ncube, nr, n_solid, float(r_in), float(r_out), float(r_stretch), ctypes.byref(out)))
            m = cls(out.value)
            from . import gpu
            gpu.build_tets(m)
            return m
        _check(lib().mhdm_shell(ncube, nr, n_solid, float(r_in), float(r_out), float(r_stretch), int(tets), ctypes.byref(out)))
        return cls(out.value)

    def _recount(self):
        c = np.zeros(4, np.int32)
        lib().mhdm_counts(self._h, c.ctypes.data)
        self.n_nodes, self.n_edges, self.n_faces, self.n_cells = (int(v) for v in c)
        self._cache.clear()

    @classmethod
    def from_cells(cls, x, cells, material=None, tagged=(), tag_names=("",)):
        """Generic polyhedra: `cells` is a list of cells, each a list of outward node loops."""
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
        out = ctypes.c_void_p()
        _check(lib().mhdm_from_cells(len(x), _dptr(x), len(cells), _dptr(cell_ptr), _dptr(loop_ptr), _dptr(nodes),
                                     _dptr(mat), len(tid), _dptr(tptr), _dptr(tnodes), _dptr(tid), len(tag_names),
                                     ctypes.cast(names, ctypes.c_void_p), ctypes.byref(out)))
        return cls(out.value)

    # ------------------------------------------------------------- services
    def topology_hash(self) -> int:
        return int(lib().mhdm_topology_hash(self._h))

    def reordered(self, order) -> "HostMesh":
        """The same complex rebuilt with its cells in `order` (new cell i = old cell order[i]); faces and edges
        are renumbered by the builder in the new creation order.  No geometry yet."""
        o = np.ascontiguousarray(order, np.int32)
        if o.size != self.n_cells:
            raise ValueError("order must list every cell once")
        out = ctypes.c_void_p()
        _check(lib().mhdm_reorder_cells(self._h, o.ctypes.data, ctypes.byref(out)))
        return HostMesh(out.value)

    def locality_order(self):
        """Morton (Z-order) permutation of the cell centres, 21 bits per axis: cells close in space get close ids."""
        cc = np.asarray(self["cell_center"], np.float64).reshape(-1, 3)
        span = max(float((cc.max(0) - cc.min(0)).max()), 1e-300)
        q = ((cc - cc.min(0)) / span * (2 ** 21 - 1)).astype(np.uint64)

        def spread(v):
            v = v & np.uint64(0x1FFFFF)
            for sh, mask in ((32, 0x1F00000000FFFF), (16, 0x1F0000FF0000FF), (8, 0x100F00F00F00F00F), (4, 0x10C30C30C30C30C3),
                             (2, 0x1249249249249249)):
                v = (v | (v << np.uint64(sh))) & np.uint64(mask)
            return v

        key = spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1)) | (spread(q[:, 2]) << np.uint64(2))
        return np.argsort(key, kind="stable").astype(np.int32)

    def compute_geometry(self, device=False) -> "HostMesh":
        """uns::compute_geometry (src/uns/geometry/Geometry.cpp:17-169) on the host, or with device=True on the
        GPU (mhd_gpu_compute_geometry, bit-identical) and installed in this mesh."""
        if device:
            from . import gpu
            g = gpu.compute_geometry(self)
            names = ("edge_vec", "edge_mid", "edge_len", "face_area", "face_center", "face_area_mag", "cell_center", "cell_volume",
                     "cell_min_tet_volume", "edge_dual_area", "ec_weight", "ef_weight", "star0", "star1", "star2", "star3")
            arr = _GeometryArrays(*[ctypes.c_void_p(g[k].ctypes.data) for k in names],
                                  ctypes.c_void_p(g["ec_ptr"].ctypes.data), ctypes.c_void_p(g["ec_cell"].ctypes.data),
                                  ctypes.c_void_p(g["ec_misoriented"].ctypes.data))
            _check(lib().mhdm_set_geometry(self._h, ctypes.byref(arr)))
        else:
            _check(lib().mhdm_compute_geometry(self._h))
        self._cache.clear()
        return self

    def boundary(self, bc_default="outflow", by_tag=None, u_inf=(0.0, 0.0, 0.0), device=False) -> "HostMesh":
        """mhd::BoundaryInfo::build (Common/boundary/BoundaryInfo.cpp:9-49) on the host, or with device=True on the
        GPU (mhd_gpu_boundary: the same face kinds and edge modes) and installed in this mesh."""
        by_tag = dict(by_tag or {})
        tags = (ctypes.c_char_p * max(1, len(by_tag)))(*[k.encode() for k in by_tag])
        types = (ctypes.c_char_p * max(1, len(by_tag)))(*[v.encode() for v in by_tag.values()])
        u = np.asarray(u_inf, np.float64)
        if device:
            from . import gpu
            try:
                self["face_area"]
            except KeyError:
                self.compute_geometry()
            cap = 4096
            tt = np.zeros(cap, np.int8)
            tn, nt = ctypes.c_int8(), ctypes.c_int32()
            _check(lib().mhdm_tag_types(self._h, bc_default.encode(), len(by_tag), ctypes.cast(tags, ctypes.c_void_p),
                                        ctypes.cast(types, ctypes.c_void_p), cap, tt.ctypes.data, ctypes.byref(tn), ctypes.byref(nt)))
            fk, em = gpu.boundary(self, tt[:nt.value], tn.value, u)
            _check(lib().mhdm_set_boundary(self._h, fk.ctypes.data, em.ctypes.data))
        else:
            _check(lib().mhdm_boundary(self._h, bc_default.encode(), len(by_tag), ctypes.cast(tags, ctypes.c_void_p),
                                       ctypes.cast(types, ctypes.c_void_p), u.ctypes.data))
        self._cache.clear()
        return self

    def __getitem__(self, name: str) -> np.ndarray:
        if name in self._cache:
            return self._cache[name]
        n = ctypes.c_int64()
        p = lib().mhdm_array(self._h, name.encode(), ctypes.byref(n))
        if n.value < 0 or (not p and n.value > 0):
            raise KeyError(name)
        if name.endswith("_ptr"):
            dt = np.int64
        elif name.endswith("_idx"):
            dt = np.int32
        elif name.endswith("_sgn"):
            dt = np.int8
        else:
            dt = _DT.get(name, np.float64)
        buf = (ctypes.c_char * (n.value * np.dtype(dt).itemsize)).from_address(p) if n.value else b""
        a = np.frombuffer(buf, dtype=dt, count=n.value) if n.value else np.zeros(0, dt)
        if name in _VEC3:
            a = a.reshape(-1, 3)
        a.flags.writeable = False
        self._cache[name] = a
        return a

    def cell_loops_flat(self):
        """Builder input of this complex as flat arrays (cell_ptr, loop_ptr, loop_nodes): per cell its
        face loops oriented outward, in c2f order."""
        e2n = np.asarray(self["e2n_idx"]).reshape(-1, 2)
        f2e_ptr, f2e_idx, f2e_sgn = (np.asarray(self[k]) for k in ("f2e_ptr", "f2e_idx", "f2e_sgn"))
        c2f_ptr, c2f_idx, c2f_sgn = (np.asarray(self[k]) for k in ("c2f_ptr", "c2f_idx", "c2f_sgn"))
        # node at which each f2e entry enters its edge: start if traversed forward, else end
        enter = np.where(f2e_sgn > 0, e2n[f2e_idx, 0], e2n[f2e_idx, 1]).astype(np.int32)
        lens = (f2e_ptr[c2f_idx + 1] - f2e_ptr[c2f_idx]).astype(np.int64)
        loop_ptr = np.zeros(len(c2f_idx) + 1, np.int64)
        np.cumsum(lens, out=loop_ptr[1:])
        pos = np.arange(loop_ptr[-1], dtype=np.int64) - np.repeat(loop_ptr[:-1], lens)   # position inside the loop
        start = np.repeat(f2e_ptr[c2f_idx], lens)
        L = np.repeat(lens, lens)
        rev = np.repeat(c2f_sgn < 0, lens)
        src = np.where(rev, start + (L - 1 - pos), start + pos)
        return np.asarray(c2f_ptr, np.int64), loop_ptr, enter[src]

    def outward_loops(self):
        """Per cell, its face loops oriented outward (c2f order): the builder input that reproduces this complex."""
        e2n_idx = self["e2n_idx"].reshape(-1, 2)
        f2e_ptr, f2e_idx, f2e_sgn = self["f2e_ptr"], self["f2e_idx"], self["f2e_sgn"]
        c2f_ptr, c2f_idx, c2f_sgn = self["c2f_ptr"], self["c2f_idx"], self["c2f_sgn"]
        cells = []
        for c in range(self.n_cells):
            loops = []
            for k in range(c2f_ptr[c], c2f_ptr[c + 1]):
                f = c2f_idx[k]
                es = f2e_idx[f2e_ptr[f]:f2e_ptr[f + 1]]
                ss = f2e_sgn[f2e_ptr[f]:f2e_ptr[f + 1]]
                loop = [int(e2n_idx[e, 0] if s > 0 else e2n_idx[e, 1]) for e, s in zip(es, ss)]
                if c2f_sgn[k] < 0:
                    loop = loop[::-1]
                loops.append(loop)
            cells.append(loops)
        return cells
