"""Host side of the ten-ion pieces (CPU): the wall table generator, the parameter block, argument errors of
the new entry points without a device, and the compiled reference's ten-ion solver as the checker runs it."""
import ctypes

import numpy as np
import pytest

from helpers import SHELL_TAGS, ref_twin


def test_wall_states_cover_the_wall_faces():
    from mpcns_uns_b200 import workloads
    wl = workloads.shell(4, 5, r_in=1.0, r_out=6.0)
    faces, prims = workloads.wall_states(wl.mesh, [f[0] for f in wl.fs], wl.mass, seed=3)
    kind = np.asarray(wl.mesh["face_kind"])
    assert np.array_equal(np.sort(faces), np.nonzero(kind == 1)[0])
    assert prims.shape == (wl.n_species, faces.size, 5)
    assert np.all(prims[:, :, 0] > 0) and np.all(prims[:, :, 4] > 0) and np.all(prims[:, :, 1:4] == 0)
    again = workloads.wall_states(wl.mesh, [f[0] for f in wl.fs], wl.mass, seed=3)
    assert np.array_equal(again[1], prims)


def test_mars_params_block():
    from mpcns_uns_b200 import gpu
    from mpcns_uns_b200.mars import PARTICLE_MASS, mars_params
    sc = dict(rho_ref=6.6e-21, n_ref=4e6, p_ref=7.1e-12, time_ref=103.9, kB=1.38e-23, L=3.396e6, U=3.27e4, q=1.6e-19, B=3e-9,
              mag_scale=1.0, pressure_scale=0.033, ne_floor=0.01, rho_floor=1e-10, p_floor=1e-10, gamma=1.4, ambipolar=0)
    mp = mars_params(sc)
    assert isinstance(mp, gpu.MarsParams)
    assert (mp.n_species, mp.n_neutral, mp.neutral_stride, mp.ambipolar) == (10, 10, 12, 0)
    assert list(mp.mass[:10]) == list(PARTICLE_MASS) and mp.gamma == 1.4


def test_new_entry_points_reject_null_arguments():
    from mpcns_uns_b200 import build
    L = ctypes.CDLL(build.build_gpu())
    L.mhd_gpu_last_error.restype = ctypes.c_char_p
    vp = ctypes.c_void_p
    for name, nargs in (("mhd_gpu_mars_plasma", 8), ("mhd_gpu_mars_explicit_sources", 9), ("mhd_gpu_mars_ambipolar_emf", 5),
                        ("mhd_gpu_mars_floors", 3), ("mhd_gpu_pressure_gradient", 3)):
        f = getattr(L, name)
        f.argtypes = [vp] * nargs
        assert f(*([None] * nargs)) == -1, name
        assert b"null" in L.mhd_gpu_last_error()
    L.mhd_gpu_state_set_wall_ghosts.argtypes = [vp, ctypes.c_int32, vp, vp]
    assert L.mhd_gpu_state_set_wall_ghosts(None, 0, None, None) == -1
    assert b"null state" in L.mhd_gpu_last_error()


ref = pytest.importorskip("oracle.ref")


@pytest.mark.skipif(not ref.available(), reason="reference checker not built (make -C oracle ref)")
def test_reference_ten_ion_solver_as_checker():
    """The compiled MarsSolver on a checker mesh: its boundary classification is the host library's, its wall
    table covers the wall faces, and its step without the photochemistry keeps a finite state."""
    from mpcns_uns_b200.mesh import HostMesh
    h = HostMesh.shell(4, 4, 1.04, 3.0, tets=True).compute_geometry()
    r = ref_twin(h, SHELL_TAGS)
    m = ref.RefMars(r, ["is_Hall_Efield=0", "second_order=1", "CFL=0.4"])
    P = m.params
    h.boundary("outflow", {"inner": "wall", "outer": "farfield"}, (P["sw_ux"], P["sw_uy"], P["sw_uz"]))
    fk, em = m.boundary()
    assert np.array_equal(np.asarray(h["face_kind"]), fk) and np.array_equal(np.asarray(h["edge_mode"]), em)
    faces, prims = m.wall_table()
    assert np.array_equal(faces, np.nonzero(fk == 1)[0]) and prims.shape == (10, faces.size, 5)
    assert m.get("neutral").size == 12 * h.n_cells
    U0 = m.get("U")
    for _ in range(2):
        assert m.step_nochem() > 0
    U = m.get("U")
    assert np.all(np.isfinite(U)) and not np.array_equal(U, U0)
