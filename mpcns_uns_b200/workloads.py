"""Seeded synthetic workloads: the meshes and initial states of the benchmark configurations.

No public dataset is involved; every input is generated here from documented seeds.
Random numbers come from numpy's PCG64 (`np.random.default_rng(seed)`); the node jitter of the
box comes from the splitmix64 stream of the native mesh builder.

  box(n)     unit cube, n^3 hexahedra x 6 tetrahedra, interior nodes jittered +-0.15 h (seed 0),
             rho = 1, p = 0.1, u = (1, 0, 0) with 1% uniform noise, gamma = 5/3, B = d1(A)
             with A = 8 Fourier modes of amplitude 0.05 plus the uniform B0 = (0.1, 0.2, 0)
             (B0 enters the evolved flux, so d2 B = 0 holds as an integer identity), outflow
             on every boundary.  n = 16 is the 24,576-cell configuration.
  shell(...) cubed-sphere shells, 6 tetrahedra per hexahedron, geometric radial layers:
             two ions (H+, Na+ of mass 23) upstream u = (-8, 0, 0), p = 0.05; Na+ density
             1e-3 * lognormal(0, 0.5) * exp(-(r - 1)/0.2); IMF (0, 0, -0.5) and a dipole of
             moment 1 at (0, 0, 0.2) in the static background flux; wall at the inner surface,
             far field outside.  sources=True adds the two-ion J x B force and the exact gyration
             (inver_MA2 = 1, induce_coeff = 1 in these units).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mesh import HostMesh

GAMMA = 5.0 / 3.0


def to_cons(W, gamma):
    """mhd::to_cons (Common/physics/Euler.h:22-26) on an (n, 5) array of primitives."""
    W = np.asarray(W, np.float64).reshape(-1, 5)
    U = np.empty_like(W)
    U[:, 0] = W[:, 0]
    U[:, 1:4] = W[:, :1] * W[:, 1:4]
    U[:, 4] = W[:, 4] / (gamma - 1.0) + 0.5 * W[:, 0] * (W[:, 1:4] ** 2).sum(1)
    return U


def prims(U, gamma):
    """Primitives (n, 5) of conservative AoS values (no floors: the inverse of to_cons)."""
    U = np.asarray(U, np.float64).reshape(-1, 5)
    W = np.empty_like(U)
    W[:, 0] = U[:, 0]
    W[:, 1:4] = U[:, 1:4] / U[:, :1]
    W[:, 4] = (gamma - 1.0) * (U[:, 4] - 0.5 * W[:, 0] * (W[:, 1:4] ** 2).sum(1))
    return W


def d1(mesh: HostMesh, A):
    """(d1 A)_f = sum_e f2e[f,e] A_e, each row summed in f2e order."""
    ptr, idx, sgn = np.asarray(mesh["f2e_ptr"]), np.asarray(mesh["f2e_idx"]), np.asarray(mesh["f2e_sgn"])
    rows = np.repeat(np.arange(mesh.n_faces), np.diff(ptr))
    return np.bincount(rows, weights=sgn * np.asarray(A)[idx], minlength=mesh.n_faces)


def fourier_potential(mesh: HostMesh, seed, modes=8, amp=0.05, B0=(0.1, 0.2, 0.0)):
    """Edge vector potential A_e = (a(x_mid) + 1/2 B0 x x_mid) . t_e, a = sum of seeded Fourier modes."""
    rng = np.random.default_rng(seed)
    x = np.asarray(mesh["edge_mid"])
    t = np.asarray(mesh["edge_vec"])
    a = np.zeros_like(x)
    for _ in range(modes):
        k = rng.integers(-2, 3, size=3)
        while not k.any():
            k = rng.integers(-2, 3, size=3)
        d = rng.normal(size=3)
        d *= amp / np.linalg.norm(d)
        ph = rng.uniform(0, 2 * np.pi)
        a += np.cos(2 * np.pi * x @ k + ph)[:, None] * d
    a += 0.5 * np.cross(np.asarray(B0, np.float64), x)
    return (a * t).sum(1)


@dataclass
class Workload:
    name: str
    mesh: HostMesh
    n_species: int
    gamma: float
    U: list                     # per species (n_cells*5,) conservative AoS
    Phi: np.ndarray             # induced face flux
    PhiAdd: np.ndarray          # static background face flux
    fs: list                    # free-stream primitives per species
    mass: list
    u_inf: tuple
    B_imf: tuple
    cfl: float = 0.4
    steps: int = 20
    extra: dict = field(default_factory=dict)
    lorentz: bool = False          # two-ion J x B force (mercury::add_sources_n)
    induce_coeff: float = 0.0      # > 0: exact gyration, Strang-split around the step (mercury::gyrate)
    inver_MA2: float = 1.0


def box(n=16, seed=0, jitter=0.15, tets=True):
    m = HostMesh.box(n, n, n, tets=tets, jitter=jitter, seed=seed).compute_geometry().boundary("outflow")
    rng = np.random.default_rng(seed + 1)
    nc = m.n_cells
    W = np.zeros((nc, 5))
    W[:, 0] = 1.0 * (1 + 0.01 * rng.uniform(-1, 1, nc))
    W[:, 1] = 1.0 * (1 + 0.01 * rng.uniform(-1, 1, nc))
    W[:, 2] = 0.01 * rng.uniform(-1, 1, nc)
    W[:, 3] = 0.01 * rng.uniform(-1, 1, nc)
    W[:, 4] = 0.1 * (1 + 0.01 * rng.uniform(-1, 1, nc))
    Phi = d1(m, fourier_potential(m, seed + 2))
    return Workload(name=f"box{n}^3x6", mesh=m, n_species=1, gamma=GAMMA, U=[to_cons(W, GAMMA).ravel()], Phi=Phi,
                    PhiAdd=np.zeros(m.n_faces), fs=[(1.0, 1.0, 0.0, 0.0, 0.1)], mass=[1.0], u_inf=(1.0, 0.0, 0.0),
                    B_imf=(0.0, 0.0, 0.0), cfl=0.4, steps=20)


def background(mesh: HostMesh, B_imf, dipole_m, dipole_c, soft=1e-3):
    """Static background flux of mercury::set_background (MercuryUns/initial/Initial.cpp:66-84)."""
    PhiAdd = np.asarray(mesh["face_area"]).reshape(-1, 3) @ np.asarray(B_imf, np.float64)
    r = np.asarray(mesh["edge_mid"]).reshape(-1, 3) - np.asarray(dipole_c, np.float64)
    d2 = (r * r).sum(1) + soft * soft
    a = np.cross(np.asarray(dipole_m, np.float64), r) / (d2 * np.sqrt(d2))[:, None]
    A = (a * np.asarray(mesh["edge_vec"]).reshape(-1, 3)).sum(1)
    return PhiAdd + d1(mesh, A)


def geometric_stretch(nr, r_in, r_out, first):
    """Ratio q of nr geometric layers between r_in and r_out with first layer thickness `first`."""
    lo, hi = 1.0, 2.0
    f = lambda q: first * (q ** nr - 1) / (q - 1) - (r_out - r_in)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid) > 0:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


def shell_stretch(ncube, nr, r_in=1.0, r_out=6.0):
    """Radial stretch of the shell workloads: the first layer as thick as the angular spacing at r_in."""
    return geometric_stretch(nr, r_in, r_out, r_in * (np.pi / 2) / ncube)


def shell_mesh(ncube, nr, r_in=1.0, r_out=6.0, stretch=None, u_inf=(-8.0, 0.0, 0.0), device_geometry=False):
    """The shell workloads' mesh: cubed sphere, 6 tetrahedra per hexahedron, wall inside, far field outside.
    device_geometry: number the complex, compute the metric and classify the boundary on the GPU (bit-identical,
    much faster for large shells)."""
    if stretch is None:
        stretch = shell_stretch(ncube, nr, r_in, r_out)
    m = HostMesh.shell(ncube, nr, r_in, r_out, stretch, tets=True, device_build=device_geometry).compute_geometry(device=device_geometry)
    m.boundary("outflow", {"inner": "wall", "outer": "farfield"}, u_inf, device=device_geometry)
    return m, stretch


def shell(ncube, nr, r_in=1.0, r_out=6.0, stretch=None, seed=0, n_species=2, masses=None, u_inf=(-8.0, 0.0, 0.0), sources=False,
          device_geometry=False):
    """device_geometry: build the complex and compute the metric on the GPU (bit-identical, faster for large shells)."""
    m, stretch = shell_mesh(ncube, nr, r_in, r_out, stretch, u_inf, device_geometry)
    return shell_state(m, f"shell6x{ncube}x{ncube}x{nr}x6", r_in, stretch, seed, n_species, masses, u_inf, sources)


def shell_state(m, name, r_in=1.0, stretch=1.0, seed=0, n_species=2, masses=None, u_inf=(-8.0, 0.0, 0.0), sources=False):
    """The shell workload's seeded state on a built shell mesh `m` (any object with n_cells, n_faces and the
    reference's named arrays: cell_center, face_area, edge_mid, edge_vec, f2e_*), numpy only."""
    rng = np.random.default_rng(seed)
    nc = m.n_cells
    r = np.linalg.norm(np.asarray(m["cell_center"]).reshape(-1, 3), axis=1)
    masses = masses or ([1.0, 23.0] if n_species == 2 else [1.0] * n_species)
    U, fs = [], []
    for s in range(n_species):
        W = np.zeros((nc, 5))
        W[:, 1:4] = np.asarray(u_inf)
        if s == 0:
            W[:, 0] = 1.0
            W[:, 4] = 0.05
            fs.append((1.0, *u_inf, 0.05))
        else:
            rho0 = 1e-3 if n_species == 2 else 10 ** rng.uniform(-4, 0)
            W[:, 0] = rho0 * rng.lognormal(0.0, 0.5, nc) * np.exp(-(r - r_in) / 0.2) + 1e-3 * rho0
            W[:, 4] = 0.05 * W[:, 0]
            fs.append((rho0 * 1e-3, *u_inf, 0.05 * rho0 * 1e-3))
        U.append(to_cons(W, GAMMA).ravel())
    B_imf = (0.0, 0.0, -0.5)
    PhiAdd = background(m, B_imf, (0.0, 0.0, 1.0), (0.0, 0.0, 0.2))
    two = n_species == 2
    return Workload(name=name, mesh=m, n_species=n_species, gamma=GAMMA, U=U,
                    Phi=np.zeros(m.n_faces), PhiAdd=PhiAdd, fs=fs, mass=masses, u_inf=tuple(u_inf), B_imf=B_imf,
                    cfl=0.4, steps=100, extra=dict(stretch=stretch), lorentz=two and sources,
                    induce_coeff=1.0 if two and sources else 0.0)


def dipole_field(x, m=(0.0, 0.0, 1.0), c=(0.0, 0.0, 0.2), B_imf=(0.0, 0.0, -0.5)):
    """Point-dipole field (3 (m.r^) r^ - m) / |r|^3 about c plus a uniform IMF, at the points x (n, 3)."""
    r = np.asarray(x, np.float64) - np.asarray(c, np.float64)
    d = np.linalg.norm(r, axis=1)
    rh = r / d[:, None]
    mv = np.asarray(m, np.float64)
    return (3.0 * (rh @ mv)[:, None] * rh - mv) / (d ** 3)[:, None] + np.asarray(B_imf, np.float64)


def whistler_dt(mesh: HostMesh, B0, ne, hall_coef, hall_r_min):
    """Explicit Hall (whistler) time-step limit of mercury::Solver::collect (MercuryUns/driver/Solver.cpp:588-601):
    min over fluid cells with r >= hall_r_min of h^2 n_e / (9.8696 hall_coef |B|), h = 6 V / sum_f |A_f|."""
    ptr = np.asarray(mesh["c2f_ptr"])
    area = np.add.reduceat(np.asarray(mesh["face_area_mag"])[np.asarray(mesh["c2f_idx"])], ptr[:-1])
    h = 6.0 * np.asarray(mesh["cell_volume"]) / area
    r = np.linalg.norm(np.asarray(mesh["cell_center"]), axis=1)
    B = np.linalg.norm(np.asarray(B0).reshape(-1, 3), axis=1)
    ok = (np.asarray(mesh["cell_material"]) != 1) & (r >= hall_r_min)
    return float(np.min(h[ok] ** 2 * np.asarray(ne)[ok] / (9.8696 * hall_coef * np.maximum(B[ok], 1e-30))))


@dataclass
class InductionCase:
    """Inputs of one semi-implicit induction solve (mhd::ImplicitInduction::solve)."""
    name: str
    mesh: HostMesh
    m_edge: np.ndarray      # per-edge resistive coefficient m_e = eta(r_e) / star1_e
    B0: np.ndarray          # frozen total field per cell (3 per cell)
    ne: np.ndarray          # frozen effective electron density per cell
    Phi: np.ndarray         # induced face flux Phi^n
    E_expl: np.ndarray      # explicit EMF per edge
    dirichlet: np.ndarray   # int8 per edge: edge_mode == 2 (far-field inflow edges keep E_expl)
    dt: float
    dt_whistler: float
    hall_coef: float
    hall_r_min: float
    hall_r_max: float


def induction_case(ncube=48, nr=96, r_in=0.8, r_out=6.0, eta_inner=1.0, eta_outer=1e-3, r_eta=1.0, hall_coef=1.0,
                   hall_r_min=1.0, hall_r_max=1.012, dt_factor=20.0, seed=0, u_inf=(-8.0, 0.0, 0.0), device_geometry=False):
    """The semi-implicit Hall + resistive solve on a cubed-sphere shell r in [r_in, r_out] (6 tetrahedra per hexahedron,
    nr geometric layers): eta = eta_inner below r_eta and eta_outer above it, set per edge as m_e = eta / star1_e; Hall
    on with the reference's radial taper; B0 = dipole of moment 1 at (0, 0, 0.2) plus the IMF (0, 0, -0.5) at the cell
    centres; n_e = 1 + U(0, 0.5) (seeded); Phi^n = d1 of 8 seeded Fourier modes of amplitude 0.05; E_expl = (-u x B0) . t
    at the edge midpoints; dt = dt_factor x the explicit whistler limit.  ncube = 48, nr = 96 is the 7.96M-cell case."""
    m, _ = shell_mesh(ncube, nr, r_in, r_out, None, u_inf, device_geometry)
    rng = np.random.default_rng(seed)
    r_e = np.linalg.norm(np.asarray(m["edge_mid"]), axis=1)
    m_edge = np.where(r_e < r_eta, eta_inner, eta_outer) / np.asarray(m["star1"])
    B0 = dipole_field(np.asarray(m["cell_center"])).ravel()
    ne = 1.0 + 0.5 * rng.uniform(0.0, 1.0, m.n_cells)
    Phi = d1(m, fourier_potential(m, seed + 2, B0=(0.0, 0.0, 0.0)))
    Bm = dipole_field(np.asarray(m["edge_mid"]))
    E_expl = (-np.cross(np.asarray(u_inf, np.float64), Bm) * np.asarray(m["edge_vec"])).sum(1)
    dirichlet = (np.asarray(m["edge_mode"]) == 2).astype(np.int8)
    dtw = whistler_dt(m, B0, ne, hall_coef, hall_r_min)
    return InductionCase(name=f"shell6x{ncube}x{ncube}x{nr}x6_r{r_in:g}-{r_out:g}", mesh=m, m_edge=m_edge, B0=B0, ne=ne, Phi=Phi,
                         E_expl=E_expl, dirichlet=dirichlet, dt=dt_factor * dtw, dt_whistler=dtw, hall_coef=hall_coef,
                         hall_r_min=hall_r_min, hall_r_max=hall_r_max)


def edge_resistivity(mesh: HostMesh, eta_cell):
    """Per-edge coefficient m_e = eta_e / star1_e of the explicit resistive EMF, eta_e the mean of the per-cell
    resistivity over the cells around edge e (summed in the edge's cell-list order, then divided by the count)."""
    ptr, cells = np.asarray(mesh["ec_ptr"]), np.asarray(mesh["ec_cell"])
    eta = np.asarray(eta_cell, np.float64)
    out = np.zeros(mesh.n_edges)
    for e in range(mesh.n_edges):
        a, b = int(ptr[e]), int(ptr[e + 1])
        acc = 0.0
        for k in range(a, b):
            acc += eta[cells[k]]
        out[e] = (acc / (b - a)) / mesh["star1"][e] if b > a else 0.0
    return out


@dataclass
class AdjointCase:
    """Inputs of the gradient of J = sum |B_tot|^2 V over the dayside cells with r in [r_lo, r_hi] after n_steps
    explicit steps at a fixed dt, with respect to the per-cell resistivity and the inflow velocity."""
    wl: Workload
    eta: np.ndarray          # per-cell resistivity, log-uniform in [eta_lo, eta_hi] (seeded)
    mask: np.ndarray         # int8 per cell: the cells of the functional
    n_steps: int
    checkpoint_every: int


def adjoint_case(ncube=32, nr=64, r_in=1.0, r_out=6.0, n_steps=40, checkpoint_every=8, eta_lo=1e-4, eta_hi=1e-2, r_lo=1.2,
                 r_hi=1.6, induced_amp=0.05, noise=0.01, seed=0, device_geometry=False):
    """The two-ion shell of the explicit step (no model sources) with a seeded per-cell resistivity; ncube = 32,
    nr = 64 is the 2.36M-cell case.  Dayside: x > 0 (the inflow comes from +x).  The induced flux starts as d1
    of 8 seeded Fourier modes of amplitude induced_amp (the box's potential without B0), so that the resistive
    EMF acts from the first step; the dipole and the IMF stay in the background flux.  Every species' density
    and pressure carry seeded uniform noise of relative size `noise` and its velocity noise of size
    noise * |u_inf| per component (as the box's state does): without it the free stream's exactly equal
    neighbour values put every limiter and wave-speed max / min on a tie, where J has no derivative."""
    wl = shell(ncube, nr, r_in, r_out, seed=seed, device_geometry=device_geometry)
    if induced_amp:
        wl.Phi = d1(wl.mesh, fourier_potential(wl.mesh, seed + 2, amp=induced_amp, B0=(0.0, 0.0, 0.0)))
    if noise:
        rng_n = np.random.default_rng(seed + 11)
        nc = wl.mesh.n_cells
        U = []
        for u in wl.U:
            W = prims(u, wl.gamma)
            W[:, 0] *= 1 + noise * rng_n.uniform(-1, 1, nc)
            W[:, 4] *= 1 + noise * rng_n.uniform(-1, 1, nc)
            W[:, 1:4] += noise * np.linalg.norm(wl.u_inf) * rng_n.uniform(-1, 1, (nc, 3))
            U.append(to_cons(W, wl.gamma).ravel())
        wl.U = U
    rng = np.random.default_rng(seed + 7)
    eta = 10.0 ** rng.uniform(np.log10(eta_lo), np.log10(eta_hi), wl.mesh.n_cells)
    x = np.asarray(wl.mesh["cell_center"])
    r = np.linalg.norm(x, axis=1)
    mask = ((r >= r_lo) & (r <= r_hi) & (x[:, 0] > 0)).astype(np.int8)
    return AdjointCase(wl=wl, eta=eta, mask=mask, n_steps=n_steps, checkpoint_every=checkpoint_every)


def wall_states(mesh: HostMesh, rho_up, masses, T_wall=0.05, seed=0):
    """A Dirichlet wall table in the form of the ten-ion solver's wall ghost (MarsUns/driver/MarsSolver.cpp:147-165:
    a photochemical-equilibrium ion density at the wall face centre, at rest, p = n k T_wall), with a seeded stand-in
    for the atmosphere model: per wall face and species rho = rho_up[s] 10^U(0, 1) (1 + 0.5 x/r) (dayside-enhanced),
    u = 0, p = rho / m_s * T_wall.  Returns (faces int32, prims n_species x n_wall x 5)."""
    kind = np.asarray(mesh["face_kind"])
    faces = np.nonzero(kind == 1)[0].astype(np.int32)
    fc = np.asarray(mesh["face_center"], np.float64).reshape(-1, 3)[faces]
    r = np.linalg.norm(fc, axis=1)
    rng = np.random.default_rng(seed)
    prims = np.zeros((len(rho_up), faces.size, 5))
    for s, (rho0, m) in enumerate(zip(rho_up, masses)):
        rho = rho0 * 10.0 ** rng.uniform(0.0, 1.0, faces.size) * (1.0 + 0.5 * fc[:, 0] / r)
        prims[s, :, 0] = rho
        prims[s, :, 4] = rho / m * T_wall
    return faces, prims


TEN_ION_MASSES = [1.0, 2.0, 4.0, 12.0, 14.0, 16.0, 28.0, 30.0, 32.0, 44.0]


def crustal_background(mesh: HostMesh, seed=0, n_dipoles=16, r_src=0.95, moment=0.05, global_moment=0.01, B_imf=(0.0, 0.0, -0.5),
                       soft=1e-3):
    """Static background flux of a crustal field: n_dipoles seeded point dipoles at radius r_src (uniform seeded
    directions, seeded orientations, strengths uniform in [0.5, 1] x moment) plus a weak global dipole of moment
    global_moment along z and the IMF, each as d1 of its edge vector potential (the set_background form)."""
    rng = np.random.default_rng(seed)
    x = np.asarray(mesh["edge_mid"])
    t = np.asarray(mesh["edge_vec"])
    sources = [((0.0, 0.0, 0.0), (0.0, 0.0, global_moment))]
    for _ in range(n_dipoles):
        d = rng.normal(size=3)
        pos = r_src * d / np.linalg.norm(d)
        m = rng.normal(size=3)
        m *= moment * rng.uniform(0.5, 1.0) / np.linalg.norm(m)
        sources.append((tuple(pos), tuple(m)))
    return np.asarray(mesh["face_area"]) @ np.asarray(B_imf, np.float64) + d1(mesh, _dipole_potential(x, t, sources, soft))


def _dipole_potential(x, t, sources, soft):
    """A_e = (sum over the point dipoles (c, m) of m x r / |r|_soft^3, r = x_e - c) . t_e, one elementwise
    operation at a time in a fixed order, so that numpy and torch (on the GPU when there is one, for the
    large meshes) give the same bits."""
    try:
        import torch
        dev = "cuda" if torch.cuda.is_available() else None
    except ImportError:
        dev = None
    if dev:
        xp = torch.from_numpy(np.array(x, np.float64)).to(dev)
        tp = torch.from_numpy(np.array(t, np.float64)).to(dev)
        sqrt = torch.sqrt
    else:
        xp, tp, sqrt = np.asarray(x, np.float64), np.asarray(t, np.float64), np.sqrt
    X, Y, Z = xp[:, 0], xp[:, 1], xp[:, 2]
    ax = ay = az = 0.0
    for c, m in sources:
        rx, ry, rz = X - c[0], Y - c[1], Z - c[2]
        d2 = rx * rx
        d2 = d2 + ry * ry
        d2 = d2 + rz * rz
        d2 = d2 + soft * soft
        inv = 1.0 / (d2 * sqrt(d2))
        ax = ax + (m[1] * rz - m[2] * ry) * inv
        ay = ay + (m[2] * rx - m[0] * rz) * inv
        az = az + (m[0] * ry - m[1] * rx) * inv
    A = ax * tp[:, 0]
    A = A + ay * tp[:, 1]
    A = A + az * tp[:, 2]
    return A.cpu().numpy() if dev else A


def ten_ion(ncube=96, nr=128, r_in=1.0, r_out=8.0, seed=0, device_geometry=False):
    """The ten-ion multi-fluid shell: r in [r_in, r_out], 6 x ncube^2 x nr hexahedra x 6 tetrahedra (96, 128: the
    42.5M-cell case), ion masses 1, 2, 4, 12, 14, 16, 28, 30, 32, 44; H+ upstream density 1 and the others seeded
    log-uniform in [1e-4, 1] relative to it, each with the seeded exosphere profile of shell(); the crustal
    background field of crustal_background; wall inside, far field outside; no model sources."""
    m, stretch = shell_mesh(ncube, nr, r_in, r_out, device_geometry=device_geometry)
    u_inf = (-8.0, 0.0, 0.0)
    wl = Workload(name="", mesh=m, n_species=10, gamma=GAMMA, U=[], Phi=np.zeros(m.n_faces), PhiAdd=None, fs=[],
                  mass=list(TEN_ION_MASSES), u_inf=u_inf, B_imf=(0.0, 0.0, -0.5), cfl=0.4, extra=dict(stretch=stretch))
    # upstream densities log-uniform in [1e-4, 1] relative to H+ (seeded); inside, the free stream enhanced by the
    # seeded exosphere profile 1 + lognormal(0, 0.5) exp(-(r - r_in)/0.2); pressure 0.05 rho, flow u_inf.  The
    # densities come from one seeded stream, the profiles from one child stream per species (SeedSequence.spawn),
    # so the species are generated in parallel threads and the state does not depend on the thread count.
    rng = np.random.default_rng(seed + 3)
    rho0s = [1.0] + [10.0 ** rng.uniform(-4.0, 0.0) for _ in range(9)]
    children = np.random.SeedSequence(seed + 4).spawn(10)
    r = np.linalg.norm(np.asarray(m["cell_center"]), axis=1)
    prof = np.exp(-(r - r_in) / 0.2)
    nc = m.n_cells

    def species(s):
        rho0 = rho0s[s]
        W = np.empty((nc, 5))
        W[:, 0] = rho0 if s == 0 else rho0 * (1.0 + np.random.default_rng(children[s]).lognormal(0.0, 0.5, nc) * prof)
        W[:, 1:4] = np.asarray(u_inf)
        W[:, 4] = 0.05 * W[:, 0]
        return to_cons(W, GAMMA).ravel()

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=10) as ex:
        U = list(ex.map(species, range(10)))
    wl.U, wl.fs = U, [(rho0s[s], *u_inf, 0.05 * rho0s[s]) for s in range(10)]
    wl.PhiAdd = crustal_background(m, seed + 5)
    wl.name = f"shell6x{ncube}x{ncube}x{nr}x6_r{r_in:g}-{r_out:g}_10ions"
    wl.steps = 50
    return wl
