"""The device path against the golden vectors of the reference (needs no reference tree).

Every entry point, three fused SSP-RK2 steps with the on-device CFL step, on the meshes of
tests/golden/.  FP64 agreement 1e-12 relative to the largest golden value.
"""
import os

import numpy as np
import pytest

from golden.make_golden import mesh_case
from helpers import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("name", ["box_tets_mixed", "shell_solid", "box_hex_mixed"])
def test_kernels_golden(name):
    from mpcns_uns_b200 import gpu
    g = load("kernels_" + name)
    h, tags, bc = mesh_case(name)
    h.compute_geometry().boundary(*bc)
    d = gpu.DeviceMesh(h)
    W, fs = g["in_W"], g["in_fs"]
    for sp in (0, 1):
        gr = _np(d.limited_gradients(W, sp, fs))
        assert rel_err(gr, g[f"grad_sp{sp}"]) < TOL
        assert rel_err(_np(d.fluid_flux_rhs(5 / 3, sp, fs, W, g[f"grad_sp{sp}"])), g[f"rhs_sp{sp}"]) < TOL
    assert rel_err(_np(d.limited_gradients(W, 0, fs, True, 0.5)), g["grad_rel05"]) < TOL
    assert rel_err(_np(d.reconstruct_cell_vector(g["in_phi"])), g["cell_vector"]) < TOL
    E = _np(d.add_ideal_emf(g["in_u"], g["in_Bt"], g["in_Bi"], g["in_pt"], g["in_pi"], 0.5, g["in_E0"]))
    assert rel_err(E, g["ideal_emf"]) < TOL
    assert rel_err(_np(d.faraday_update(g["in_E0"], g["in_phi"], 0.37)), g["faraday"]) < TOL
    db = d.div_b(g["in_phi"], g["in_pt"])
    assert rel_err([db["max_abs"], db["max_rel"]], g["div_b"][:2]) < TOL and db["worst_cell_gid"] == int(g["div_b"][2])
    assert rel_err(_np(d.cell_current(g["in_Bt"])), g["cell_current"]) < TOL


def test_fused_steps_golden():
    from mpcns_uns_b200 import gpu, workloads
    g = load("step_shell")
    wl = workloads.shell(3, 4)
    dm = gpu.DeviceMesh(wl.mesh)
    st = gpu.ResidentState(dm, gpu.step_params(2, wl.gamma, fs=wl.fs, mass=wl.mass, u_inf=wl.u_inf, B_imf=wl.B_imf))
    st.set(wl.U, wl.Phi, wl.PhiAdd)
    assert rel_err(st.download(gpu.FIELD_BADD), g["Badd"]) < TOL
    for k in range(3):
        dt = st.step(0.0)
        assert abs(dt - g["dts"][k]) <= 1e-14 * g["dts"][k]
    assert rel_err(st.U(0), g["U0"]) < TOL
    assert rel_err(st.U(1), g["U1"]) < TOL
    assert rel_err(st.Phi(), g["Phi"]) < TOL
