"""Shared helpers of the parity tests: test meshes in both worlds and comparison utilities."""
from __future__ import annotations

import numpy as np

from mpcns_uns_b200.mesh import HostMesh

BOX_TAGS = ("", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax")
SHELL_TAGS = ("", "inner", "outer")

# boundary set-ups exercised by the tests: (bc_default, per-tag types, u_inf)
MIXED_BOX_BC = ("outflow", {"xmin": "inflow", "xmax": "outflow", "ymin": "wall", "ymax": "wall",
                            "zmin": "farfield", "zmax": "farfield"}, (0.5, 0.2, -0.3))
SHELL_BC = ("outflow", {"inner": "wall", "outer": "farfield"}, (-8.0, 0.0, 0.0))


def tagged_faces(m: HostMesh):
    """(node loop, tag) of every tagged face of a built mesh."""
    ft = np.asarray(m["face_tag"])
    e2n = np.asarray(m["e2n_idx"]).reshape(-1, 2)
    fp, fi, fs = m["f2e_ptr"], m["f2e_idx"], m["f2e_sgn"]
    out = []
    for f in np.nonzero(ft)[0]:
        nodes = [int(e2n[e, 0] if s > 0 else e2n[e, 1]) for e, s in zip(fi[fp[f]:fp[f + 1]], fs[fp[f]:fp[f + 1]])]
        out.append((nodes, int(ft[f])))
    return out


def ref_twin(m: HostMesh, tag_names):
    """The same complex built by the reference's ComplexBuilder from this mesh's cells."""
    from oracle.ref import RefMesh
    cp, lp, ln = m.cell_loops_flat()
    return RefMesh.from_flat(np.asarray(m["x"]), cp, lp, ln, np.asarray(m["cell_material"]), tagged_faces(m), tag_names)


def host_from_ref(r, tag_names):
    """A HostMesh built natively from the cells of a reference mesh (e.g. its refined polyhedra)."""
    x = r["x"]
    e2n = r["e2n_idx"].reshape(-1, 2)
    fp, fi, fs = r["f2e_ptr"], r["f2e_idx"], r["f2e_sgn"]
    cp, ci, cs = r["c2f_ptr"], r["c2f_idx"], r["c2f_sgn"]
    loops_of_face = []
    for f in range(r.n_faces):
        loops_of_face.append([int(e2n[e, 0] if s > 0 else e2n[e, 1]) for e, s in zip(fi[fp[f]:fp[f + 1]], fs[fp[f]:fp[f + 1]])])
    cells = []
    for c in range(r.n_cells):
        cells.append([loops_of_face[ci[k]] if cs[k] > 0 else loops_of_face[ci[k]][::-1] for k in range(cp[c], cp[c + 1])])
    ft = r["face_tag"]
    tagged = [(loops_of_face[f], int(ft[f])) for f in np.nonzero(ft)[0]]
    return HostMesh.from_cells(x, cells, r["cell_material"], tagged, tag_names)


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-300)
    return float(np.max(np.abs(a - b))) / scale if a.size else 0.0


def random_prims(n, rng, rho=(0.5, 1.5), p=(0.05, 0.15), u=1.0):
    W = np.zeros((n, 5))
    W[:, 0] = rng.uniform(*rho, n)
    W[:, 1:4] = rng.uniform(-u, u, (n, 3))
    W[:, 4] = rng.uniform(*p, n)
    return W.ravel()


# Switches and constants of the ambipolar and chemistry terms used by the parity tests (the sizes of the
# terms are moderate against the fluxes of the shell workload; the source fields are seeded per test)
SOURCE_EXTRA = dict(ambipolar=True, chemistry=True, pressure_coef=0.3, a1_Na=0.5, a4=0.2, a5=1e-6, a6=1e-7,
                    state_coeff_H=1.0, state_coeff_Na=1.0 / 23.0, T_ref=1e4, Tn0=600.0)


def source_fields(n_cells, seed=31):
    """Seeded photo (Na+ production) and vst (drag frequency) fields of the chemistry terms."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 1e-3, n_cells), rng.uniform(0.0, 2e-2, n_cells)


def exosphere_source_fields(mesh, r_in=1.0, scale_height=0.5):
    """Smooth photo and vst fields of an exosphere-like profile: both fall off as exp(-(r - r_in) / H) with the
    radius of the cell centre, photo-ionisation stronger on the sunward (+x) side."""
    import numpy as np
    cc = np.asarray(mesh["cell_center"], np.float64).reshape(-1, 3)
    r = np.linalg.norm(cc, axis=1)
    prof = np.exp(-(r - r_in) / scale_height)
    return 1e-3 * prof * 0.5 * (1.0 + cc[:, 0] / r), 2e-2 * prof
