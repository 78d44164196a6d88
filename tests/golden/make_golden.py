"""Generates the golden vectors of tests/golden/ from the reference's own compiled code.

    make -C oracle ref && python tests/golden/make_golden.py

Needs oracle/_ref/libmhdref.so (the reference compiled in place); the vectors it writes are what
tests/test_golden.py (CPU: native mesh services and the oracle restatement) and
tests/test_gpu_golden.py (the device path) check against, without the reference tree.

Meshes are built by the reference's ComplexBuilder from the cells of the native generators (the
tetrahedral split has no reference generator); inputs come from numpy's PCG64 with the seeds
below and are stored with the outputs.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from helpers import BOX_TAGS, MIXED_BOX_BC, SHELL_BC, SHELL_TAGS, random_prims, ref_twin  # noqa: E402
from mpcns_uns_b200 import workloads  # noqa: E402
from mpcns_uns_b200.mesh import HostMesh  # noqa: E402
from oracle import ref  # noqa: E402

GEOM = ["edge_vec", "edge_mid", "edge_len", "face_area", "face_center", "face_area_mag", "cell_center", "cell_volume",
        "ec_weight", "ef_weight", "star1", "star2"]


def mesh_case(name):
    if name == "box_tets_mixed":
        return HostMesh.box(4, 3, 3, tets=True, jitter=0.15, seed=0), BOX_TAGS, MIXED_BOX_BC
    if name == "shell_solid":
        return HostMesh.shell(3, 4, 0.8, 5.0, 1.2, n_solid=1, tets=True), SHELL_TAGS, SHELL_BC
    if name == "box_hex_mixed":
        return HostMesh.box(3, 2, 2, hi=(1.5, 1.0, 1.0)), BOX_TAGS, MIXED_BOX_BC
    raise KeyError(name)


def kernels(name):
    h, tags, bc = mesh_case(name)
    r = ref_twin(h, tags).boundary(*bc)
    out = {"topology_hash": np.uint64(r.topology_hash()), "face_kind": r["face_kind"], "edge_mode": r["edge_mode"]}
    for g in GEOM:
        out["geom_" + g] = r[g]
    rng = np.random.default_rng(2024)
    W = random_prims(h.n_cells, rng)
    fs = np.array([1.1, 0.3, -0.2, 0.1, 0.12])
    out["in_W"] = W
    out["in_fs"] = fs
    for sp in (0, 1):
        g = r.limited_gradients(W, sp, fs, True, 0.0)
        out[f"grad_sp{sp}"] = g
        out[f"rhs_sp{sp}"] = r.flux_rhs(W, g, sp, fs, 5.0 / 3.0)
    out["grad_rel05"] = r.limited_gradients(W, 0, fs, True, 0.5)
    phi = rng.uniform(-1, 1, h.n_faces)
    out["in_phi"] = phi
    out["cell_vector"] = r.cell_vector(phi)
    u, Bt, Bi = (rng.uniform(-1, 1, 3 * h.n_cells) for _ in range(3))
    pt, pi = rng.uniform(-1, 1, h.n_faces), rng.uniform(-1, 1, h.n_faces)
    E0 = rng.uniform(-1, 1, h.n_edges)
    out.update(in_u=u, in_Bt=Bt, in_Bi=Bi, in_pt=pt, in_pi=pi, in_E0=E0)
    out["ideal_emf"] = r.ideal_emf(u, Bt, Bi, pt, pi, 0.5, E0)
    out["faraday"] = r.faraday(E0, phi, 0.37)
    d = r.div_b(phi, pt)
    out["div_b"] = np.array([d["max_abs"], d["max_rel"], d["worst_cell_gid"]])
    out["cell_current"] = r.cell_current(Bt)
    return out


def step_case():
    """Three SSP-RK2 steps of a small two-ion shell, CFL step from the reference."""
    wl = workloads.shell(3, 4)
    h = wl.mesh
    r = ref_twin(h, SHELL_TAGS).boundary(*SHELL_BC)
    Badd = r.cell_vector(wl.PhiAdd)
    p = ref.StepParams()
    p.n_species, p.second_order, p.gamma, p.rho_floor, p.p_floor, p.cuct, p.M_ref, p.ne_floor = 2, 1, wl.gamma, 1e-10, 1e-12, 0.5, 1.0, 0.01
    p.u_inf[:] = list(wl.u_inf)
    p.B_imf[:] = list(wl.B_imf)
    for s in range(2):
        p.mass[s] = wl.mass[s]
        p.fs[s][:] = list(wl.fs[s])
    U = [np.array(u) for u in wl.U]
    Phi = np.array(wl.Phi)
    out = {"topology_hash": np.uint64(r.topology_hash()), "in_U0": wl.U[0], "in_U1": wl.U[1], "in_Phi": wl.Phi,
           "in_PhiAdd": wl.PhiAdd, "Badd": Badd}
    dts = []
    for _ in range(3):
        W = [r.to_prim(x, wl.gamma) for x in U]
        dt = r.local_time_step(wl.gamma, 0.4, 1.0, 1e-2, W[0], W[1], r.cell_vector(Phi) + Badd)
        r.rk2_step(p, U, Phi, wl.PhiAdd, Badd, dt)
        dts.append(dt)
    out.update(dts=np.array(dts), U0=U[0], U1=U[1], Phi=Phi)
    return out


def induction_case():
    """ImplicitInduction::solve, Hall + resistive, Jacobi GMRES(15), cold then warm start."""
    h = HostMesh.box(6, 5, 4, tets=True, jitter=0.1, seed=8).compute_geometry().boundary(*MIXED_BOX_BC)
    r = ref_twin(h, BOX_TAGS).boundary(*MIXED_BOX_BC)
    rng = np.random.default_rng(12)
    m_edge = rng.uniform(0.5, 2.0, h.n_edges) / np.asarray(h["star1"])
    ri = ref.RefInduction(r, hall=True, hall_coef=0.5, hall_r_min=-100.0, hall_r_max=-99.0, rtol=1e-10, max_it=200, restart=15)
    ri.set_m(m_edge)
    B0 = rng.uniform(-1, 1, 3 * h.n_cells)
    ne = rng.uniform(0.5, 2.0, h.n_cells)
    ri.set_frozen_state(B0, ne)
    phi = rng.uniform(-1, 1, h.n_faces)
    x = rng.uniform(-1, 1, h.n_edges)
    Ee = rng.uniform(-1, 1, h.n_edges)
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    out = {"topology_hash": np.uint64(r.topology_hash()), "in_m": m_edge, "in_B0": B0, "in_ne": ne, "in_phi": phi, "in_x": x,
           "in_Ee": Ee, "apply_F": ri.apply_F(phi), "apply_A": ri.apply_A(x, 0.05)}
    for warm in (0, 1):
        E, it, rr = ri.solve(phi, Ee, dirichlet, 0.05, bool(warm))
        out[f"solve{warm}_E"], out[f"solve{warm}_it"], out[f"solve{warm}_rel_res"] = E, np.array(it), np.array(rr)
    return out


def config1_checksums():
    """The 24,576-cell box of the benchmark's first configuration: topology hash and geometry checksums."""
    wl = workloads.box(16)
    r = ref_twin(wl.mesh, BOX_TAGS)
    out = {"topology_hash": np.uint64(r.topology_hash()), "counts": np.array([r.n_nodes, r.n_edges, r.n_faces, r.n_cells])}
    for g in GEOM:
        a = np.asarray(r[g]).ravel()
        w = np.random.default_rng(99).uniform(-1, 1, a.size)
        out["sum_" + g] = np.array([a.sum(), (a * w).sum(), np.abs(a).max()])
    return out


def main():
    if not ref.available():
        sys.exit("oracle/_ref/libmhdref.so missing: make -C oracle ref")
    for name in ("box_tets_mixed", "shell_solid", "box_hex_mixed"):
        np.savez_compressed(os.path.join(HERE, f"kernels_{name}.npz"), **kernels(name))
    np.savez_compressed(os.path.join(HERE, "step_shell.npz"), **step_case())
    np.savez_compressed(os.path.join(HERE, "induction_box.npz"), **induction_case())
    np.savez_compressed(os.path.join(HERE, "config1_checksums.npz"), **config1_checksums())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
