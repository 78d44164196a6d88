"""The Mercury solver's field output and restart from a resident device state: the records of
Solver::write_global_fields, read back by the reference's own uns::io::read_fields, against the
reference's prepare-time fields; and a restart through the file continues the run bit for bit."""
import os

import numpy as np
import pytest

from helpers import SHELL_BC, SHELL_TAGS, ref_twin

pytestmark = pytest.mark.gpu

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("reference checker not built (make -C oracle ref)", allow_module_level=True)


def _state(wl, dm):
    from mpcns_uns_b200 import gpu
    p = gpu.step_params(wl.n_species, wl.gamma, fs=wl.fs, mass=wl.mass, u_inf=wl.u_inf, B_imf=wl.B_imf, lorentz=True,
                        induce_coeff=0.8, inver_MA2=0.7)
    st = gpu.ResidentState(dm, p)
    st.set(wl.U, wl.Phi, wl.PhiAdd)
    return st


def test_global_fields_and_restart(tmp_path):
    from mpcns_uns_b200 import fields, gpu, workloads
    wl = workloads.shell(4, 5)
    h = wl.mesh
    r = ref_twin(h, SHELL_TAGS).boundary(*SHELL_BC)
    dm = gpu.DeviceMesh(h)
    st = _state(wl, dm)
    dt = 0.8 * st.cfl_dt()
    for _ in range(2):
        st.step(dt)
    path = os.path.join(tmp_path, "fields_final.unsb")
    fields.write_global_fields(st, path, time=2 * dt)
    recs, hsh = ref.read_fields(path)
    got = {n: (d, c, v) for n, d, c, v in recs}
    assert hsh == 0 and [n for n, *_ in recs] == ["U_H", "U_Na", "B", "rho", "p", "B_cell", "J_cell", "_time"]
    UH, UN, Phi = st.U(0), st.U(1), st.Phi()
    assert np.array_equal(got["U_H"][2], UH) and np.array_equal(got["U_Na"][2], UN) and np.array_equal(got["B"][2], Phi)
    WH, WN = r.to_prim(UH, wl.gamma), r.to_prim(UN, wl.gamma)
    assert np.array_equal(got["rho"][2], WH[0::5] + WN[0::5]) and np.array_equal(got["p"][2], WH[4::5] + WN[4::5])
    Bind = r.cell_vector(Phi)
    assert np.array_equal(got["B_cell"][2], Bind + r.cell_vector(wl.PhiAdd))
    assert np.array_equal(got["J_cell"][2], r.cell_current(Bind))
    assert got["_time"][2][0] == 2 * dt and got["B"][0] == fields.DIM_FACE and got["U_H"][1] == 5
    # restart from the file into a fresh state: the continued runs agree bit for bit
    st2 = _state(wl, dm)
    assert fields.restart(st2, path) == 2 * dt
    for _ in range(2):
        st.step(dt)
        st2.step(dt)
    for s in range(2):
        assert np.array_equal(st.U(s), st2.U(s))
    assert np.array_equal(st.Phi(), st2.Phi())
