"""The ten-ion (Mars) step on the device: mars::MarsSolver::step (MarsUns/driver/MarsSolver.cpp:705-744) composed
from the device passes of the C-ABI, with the state resident on the device.

One step: prepare (primitives of every ion, B_ind / B_tot, n_e, n_e,eff, p_e, u+, J, grad p_e), the CFL step,
per ion the limited gradients and Rusanov fluxes with the Dirichlet wall table (the solver's GhostFn), the
explicit J x B and ambipolar force, the EMF (ideal UCT + ambipolar + boundary edge values), the forward-Euler
update, the CT update of Phi, the point-implicit gyration / drag / thermal relaxation and the floors.

Not part of it: the photochemistry (chemistry_, the network of MarsUns/physics/MarsChemistry.cpp) and the
atmosphere model that supplies the neutral densities and the wall states (the caller passes both), and the
Hall term (the implicit induction solve, mhd_gpu_induction_*, takes the frozen B_tot and n_e,eff of prepare).
"""
from __future__ import annotations

import numpy as np

from . import gpu

# MARS::ParticleMass (MarsUns/physics/MarsSpecies.h): Ar CO2 CO C H N2 N NO O O2 [kg]; neutral n of the drag
# has the mass of species n
PARTICLE_MASS = (6.645e-26, 7.309e-26, 4.651e-26, 1.993e-26, 1.673e-27, 4.651e-26, 2.326e-26, 4.983e-26, 2.658e-26, 5.316e-26)
NUM_NEUTRAL, NUM_REACTIVE = 12, 10


def mars_params(scales: dict, masses=PARTICLE_MASS, n_neutral=NUM_REACTIVE, neutral_stride=NUM_NEUTRAL) -> gpu.MarsParams:
    """MhdMarsParams from the scales of MarsParams::from_params (keys rho_ref n_ref p_ref time_ref kB L U q B
    mag_scale pressure_scale ne_floor rho_floor p_floor gamma ambipolar)."""
    mp = gpu.MarsParams()
    mp.n_species, mp.n_neutral, mp.neutral_stride = len(masses), n_neutral, neutral_stride
    mp.ambipolar = int(bool(scales.get("ambipolar", 1)))
    for i, m in enumerate(masses):
        mp.mass[i] = m
    for k in ("rho_ref", "n_ref", "p_ref", "time_ref", "kB", "L", "U", "q", "B", "mag_scale", "pressure_scale", "ne_floor",
              "rho_floor", "p_floor", "gamma"):
        setattr(mp, k, float(scales[k]))
    return mp


class MarsStep:
    """A resident ten-ion state on one device mesh.  U: species-major, 5 per cell; Phi: induced face flux.

    scales: as mars_params, plus cfl, cuct, rel_limit, second_order, u_inf (3), B_imf (3).  freestream: the
    inflow ghost state of each ion (n_species x 5).  wall: (faces, prims n_species x n_wall x 5), the wall
    ghost table.  neutral: neutral_stride densities per cell [cm^-3].  PhiAdd: the background face flux."""

    def __init__(self, dmesh: gpu.DeviceMesh, scales: dict, freestream, wall, neutral, PhiAdd, masses=PARTICLE_MASS,
                 induction=None):
        """induction: the Hall solve's GMRES settings (rtol, max_it, restart, precision; the reference's Config
        defaults 1e-4, 100, 20, FP64 otherwise).  The solve runs when scales["hall"] is on and
        scales["hall_scale"] > 0, as MarsSolver builds its ImplicitInduction: Hall only, no radial taper."""
        torch = gpu._torch()
        self.dm = dmesh
        self.sc = dict(scales)
        self.mp = mars_params(scales, masses)
        self.nsp = len(masses)
        self.fs = [tuple(float(v) for v in f) for f in np.asarray(freestream, np.float64).reshape(self.nsp, 5)]
        faces, prims = wall
        self.wall_faces = np.ascontiguousarray(faces, np.int32)
        self.wall_prims = np.ascontiguousarray(prims, np.float64).reshape(self.nsp, -1, 5)
        self.neutral = gpu.dev(np.ascontiguousarray(neutral, np.float64))
        self.PhiAdd = gpu.dev(PhiAdd)
        self.Badd = dmesh.reconstruct_cell_vector(self.PhiAdd)
        nc = dmesh.n_cells
        self.U = torch.zeros(self.nsp * 5 * nc, dtype=torch.float64, device="cuda")
        self.Phi = torch.zeros(dmesh.n_faces, dtype=torch.float64, device="cuda")
        self.ind, self.last_solve = None, None
        if self.sc.get("hall", 0) and self.sc.get("hall_scale", 0.0) > 0:
            k = {"rtol": 1e-4, "max_it": 100, "restart": 20, "precision": "fp64", **(induction or {})}
            self.ind = gpu.DeviceInduction(dmesh, None, hall=True, hall_coef=self.sc["hall_scale"], hall_r_min=0.0, hall_r_max=0.0,
                                           rtol=k["rtol"], max_it=k["max_it"], restart=k["restart"], precision=k["precision"])
            self.fluid = gpu.dev(np.asarray(dmesh.host["cell_material"]) == 0)
            self.dirichlet = gpu.dev((np.asarray(dmesh.host["edge_mode"]) != 0).astype(np.int8))

    def set(self, U, Phi):
        self.U.copy_(gpu.dev(U).reshape(-1))
        self.Phi.copy_(gpu.dev(Phi).reshape(-1))

    def prepare(self):
        """MarsSolver::prepare (:271-326) -> dict of W, Bind, Btot, ne, ne_eff, pe, uplus, PhiTot, J, dpe."""
        dm, sc, nc = self.dm, self.sc, self.dm.n_cells
        torch = gpu._torch()
        W = torch.cat([dm.to_prim(self.U[5 * nc * s:5 * nc * (s + 1)], sc["gamma"], sc["rho_floor"], sc["p_floor"])
                       for s in range(self.nsp)])
        Bind = dm.reconstruct_cell_vector(self.Phi)
        Btot = Bind + self.Badd
        ne, ne_eff, pe, up = dm.mars_plasma(self.mp, self.U, W)
        J = dm.cell_current(Bind)
        dpe = dm.pressure_gradient(pe)
        return dict(W=W, Bind=Bind, Btot=Btot, ne=ne, ne_eff=ne_eff, pe=pe, uplus=up, PhiTot=self.Phi + self.PhiAdd, J=J, dpe=dpe)

    def rhs(self, q):
        """fluid_and_sources_ (:386-419): per ion gradients and fluxes with the wall table, then the explicit sources."""
        dm, sc, nc = self.dm, self.sc, self.dm.n_cells
        torch = gpu._torch()
        out = []
        for s in range(self.nsp):
            Ws = q["W"][5 * nc * s:5 * nc * (s + 1)]
            wall = (self.wall_faces, self.wall_prims[s])
            if sc.get("second_order", 0):
                g = dm.limited_gradients(Ws, s, self.fs[s], True, sc.get("rel_limit", 0.0), wall=wall)
            else:
                g = torch.zeros(15 * nc, dtype=torch.float64, device="cuda")
            out.append(dm.fluid_flux_rhs(sc["gamma"], s, self.fs[s], Ws, g, wall=wall))
        rhs = torch.cat(out)
        dm.mars_explicit_sources(self.mp, self.U, q["W"], q["Btot"], q["J"], q["dpe"], q["ne_eff"], rhs)
        return rhs

    def emf(self, q):
        """emf_ (:564-580): the ideal UCT EMF, the ambipolar EMF, the boundary edge values."""
        dm, sc = self.dm, self.sc
        E = dm.add_ideal_emf(q["uplus"], q["Btot"], q["Bind"], q["PhiTot"], self.Phi, sc.get("cuct", 0.5))
        if self.mp.ambipolar:
            dm.mars_ambipolar_emf(self.mp, q["pe"], q["ne"], E)
        return dm.edge_modes(sc["u_inf"], sc["B_imf"], E)

    def step(self, dt_max=1e300):
        """MarsSolver::step (:705-744) without the photochemistry; returns the step size.  With the Hall term on,
        the edge EMF is the implicit one of the semi-implicit induction solve (:723-735): the frozen total field
        and n_e,eff of the fluid cells, wall and inflow edges held at their prescribed values, GMRES warm-started
        from the previous step's correction; last_solve holds its (iterations, relative residual)."""
        torch = gpu._torch()
        dm, sc = self.dm, self.sc
        q = self.prepare()
        dt = min(dm.mars_time_step(self.mp, sc["cfl"], self.U, q["W"], q["Btot"], q["uplus"]), dt_max)
        if not (np.isfinite(dt) and dt > 0):
            raise gpu.MhdError(-3, "invalid time step")
        rhs = self.rhs(q)
        E = self.emf(q)
        dm.mars_advance(self.nsp, rhs, dt, self.U)
        if self.ind is not None:
            ne = torch.where(self.fluid, q["ne_eff"], torch.zeros_like(q["ne_eff"]))
            self.ind.set_frozen_state(q["Btot"], ne)
            E, it, rr = self.ind.solve(self.Phi, E, self.dirichlet, dt, warm=True)
            self.last_solve = (it, rr)
        self.Phi = dm.faraday_update(E, self.Phi, dt)
        dm.mars_implicit_sources(self.mp, q["Btot"], self.neutral, dt, self.U)
        dm.mars_floors(self.mp, self.U)
        return dt
