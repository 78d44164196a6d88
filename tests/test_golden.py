"""Golden vectors generated by the reference's own code (tests/golden/make_golden.py), checked on CPU.

* The native mesh services rebuild every golden mesh with the reference's topology hash, boundary
  classification and geometry, bit for bit.
* The oracle's C restatement reproduces every golden output bit for bit (kernels, three SSP-RK2
  steps with the CFL step, the GMRES solve), so it is a pinned checker wherever the compiled
  reference is absent.
"""
import os

import numpy as np
import pytest

from golden.make_golden import GEOM, mesh_case
from mpcns_uns_b200 import workloads
from mpcns_uns_b200.mesh import HostMesh
from oracle import port

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KCASES = ["box_tets_mixed", "shell_solid", "box_hex_mixed"]


def load(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape and np.array_equal(a, b), float(np.max(np.abs(a - b))) if a.shape == b.shape else (a.shape, b.shape)


@pytest.mark.parametrize("name", KCASES)
def test_mesh_services_match_golden(name):
    g = load("kernels_" + name)
    h, tags, bc = mesh_case(name)
    h.compute_geometry().boundary(*bc)
    assert np.uint64(h.topology_hash()) == g["topology_hash"]
    same(h["face_kind"], g["face_kind"])
    same(h["edge_mode"], g["edge_mode"])
    for k in GEOM:
        same(np.asarray(h[k]).ravel(), np.asarray(g["geom_" + k]).ravel())


@pytest.mark.parametrize("name", KCASES)
def test_oracle_kernels_match_golden(name):
    g = load("kernels_" + name)
    h, tags, bc = mesh_case(name)
    h.compute_geometry().boundary(*bc)
    o = port.PortMesh(h)
    W, fs = g["in_W"], g["in_fs"]
    for sp in (0, 1):
        gr = o.limited_gradients(W, sp == 1, fs)
        same(gr, g[f"grad_sp{sp}"])
        same(o.flux_rhs(W, gr, sp == 1, fs, 5 / 3), g[f"rhs_sp{sp}"])
    same(o.limited_gradients(W, False, fs, True, 0.5), g["grad_rel05"])
    same(o.cell_vector(g["in_phi"]), g["cell_vector"])
    same(o.ideal_emf(g["in_u"], g["in_Bt"], g["in_Bi"], g["in_pt"], g["in_pi"], 0.5, g["in_E0"]), g["ideal_emf"])
    same(o.faraday(g["in_E0"], g["in_phi"], 0.37), g["faraday"])
    d = o.div_b(g["in_phi"], g["in_pt"])
    same(np.array([d["max_abs"], d["max_rel"], d["worst_cell_gid"]]), g["div_b"])
    same(o.cell_current(g["in_Bt"]), g["cell_current"])


def test_oracle_steps_match_golden():
    g = load("step_shell")
    wl = workloads.shell(3, 4)
    assert np.uint64(wl.mesh.topology_hash()) == g["topology_hash"]
    same(wl.U[0], g["in_U0"])
    same(wl.PhiAdd, g["in_PhiAdd"])
    o = port.PortMesh(wl.mesh)
    Badd = o.cell_vector(wl.PhiAdd)
    same(Badd, g["Badd"])
    U = [np.array(u) for u in wl.U]
    Phi = np.array(wl.Phi)
    for k in range(3):
        W = [o.to_prim(u, wl.gamma) for u in U]
        dt = o.local_time_step(W, o.cell_vector(Phi) + Badd, wl.gamma, 0.4)
        assert dt == g["dts"][k]
        o.rk2_step(wl, U, Phi, Badd, dt)
    same(U[0], g["U0"])
    same(U[1], g["U1"])
    same(Phi, g["Phi"])


def test_oracle_induction_matches_golden():
    from helpers import MIXED_BOX_BC
    g = load("induction_box")
    h = HostMesh.box(6, 5, 4, tets=True, jitter=0.1, seed=8).compute_geometry().boundary(*MIXED_BOX_BC)
    assert np.uint64(h.topology_hash()) == g["topology_hash"]
    o = port.PortMesh(h)
    oi = port.PortInduction(o, g["in_m"], hall=True, hall_coef=0.5, hall_r_min=-100.0, hall_r_max=-99.0, rtol=1e-10, max_it=200,
                            restart=15)
    oi.set_frozen_state(g["in_B0"], g["in_ne"])
    same(oi.apply_F(g["in_phi"]), g["apply_F"])
    same(oi.apply_A(g["in_x"], 0.05), g["apply_A"])
    dirichlet = (np.asarray(h["edge_mode"]) == 2).astype(np.int8)
    for warm in (0, 1):
        E, it, rr = oi.solve(g["in_phi"], g["in_Ee"], dirichlet, 0.05, bool(warm))
        assert it == int(g[f"solve{warm}_it"]) and rr == float(g[f"solve{warm}_rel_res"])
        same(E, g[f"solve{warm}_E"])


def test_config1_mesh_checksums():
    g = load("config1_checksums")
    wl = workloads.box(16)
    h = wl.mesh
    assert np.uint64(h.topology_hash()) == g["topology_hash"]
    same(np.array([h.n_nodes, h.n_edges, h.n_faces, h.n_cells]), g["counts"])
    for k in GEOM:
        a = np.asarray(h[k]).ravel()
        w = np.random.default_rng(99).uniform(-1, 1, a.size)
        same(np.array([a.sum(), (a * w).sum(), np.abs(a).max()]), g["sum_" + k])
