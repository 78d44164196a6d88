#!/usr/bin/env python
"""Benchmark of the hot path: explicit SSP-RK2 steps of the two-ion shell workload on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): cubed-sphere shell r in [1, 6], 6 x 64 x 64 surface cells x 96 geometric
radial layers, every hexahedron cut into 6 tetrahedra (14,155,776 cells), two ions (H+, Na+),
inflow u = (-8, 0, 0), IMF (0, 0, -0.5), dipole at (0, 0, 0.2), wall at r = 1; seeded synthetic
state (mpcns_uns_b200/workloads.py).  One step = the reference's Solver::step hot path:
CFL step, half-step exact gyration of the ions, two stages of primitives + cell current + limited
gradients + Rusanov fluxes for both ions + J x B force + ideal UCT EMF + CT, floors, SSP-RK2
average, closing half-step gyration, all on the device (--no-sources: without the J x B force
and the gyration).  Metric: cell-updates/s
(cells x species x 2 stages per step).  Inputs exceed L2 (126 MB) many times over, so no
flush is needed between steps.

The line's "gmres" object is the second half of the metric: the semi-implicit Hall + resistive
induction solve (ImplicitInduction::solve) on the cubed-sphere shell r in [0.8, 6], 6 x 48 x 48 x 96
x 6 tetrahedra (7,962,624 cells, 9,331,392 edge unknowns), eta = 1 below r = 1 and 1e-3 above, Hall
on, dt = 20 x the explicit whistler limit, GMRES(30) with Jacobi to rtol 1e-8, cold start, capped at
--gmres-max-it iterations: seconds per solve in FP64 and mixed precision, per-kernel GB/s, and the
reference's own solve on a bounded sample beside it; its "ilu" object is the same FP64 solve with the
block ILU(0) preconditioner against Jacobi, both capped at --gmres-ilu-max-it iterations.

The "config1" object (left out with --no-config1): config 1 itself, the 24,576-cell box of one ion, 20 steps at
CFL 0.4 in FP64 and mixed precision (device ms per step, div B).

The "semi_implicit" object (left out with --no-semi-implicit): the reference's default run mode, the
semi-implicit step of Solver::step_first_order (forward Euler fluid, EMF from the Hall + resistive solve),
on the same shell in FP64: wall milliseconds per synchronous step and the solve's iterations.

The "ten_ion" object (left out with --no-ten-ion, alone with --ten-ion-only): the ten-ion shell r in
[1, 8], 6 x 96 x 96 x 128 x 6 tetrahedra (42.5M cells), crustal background field: mixed and FP64 steps and
the mixed state's error after 50 steps.

The "adjoint" object: the gradient of J = sum |B_tot|^2 V over the dayside cells with r in [1.2, 1.6]
after 40 FP64 steps on the 6 x 32 x 32 x 64 x 6 shell (2,359,296 cells, two ions, explicit resistive
EMF of a seeded per-cell resistivity) with respect to the resistivity and the inflow velocity: device
seconds of the forward run, the checkpointed adjoint sweep and the tangent-linear run, and the
gradient's agreement with tangent-linear dot products and central differences (--no-adjoint: skip).

Under torchrun (N > 1) every rank runs an independent replica on its own GPU (the hot path
has no data-path exchange on one mesh per GPU); value = all ranks' cell-updates / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s per RK step + GMRES s/solve, mixed vs FP64 GPU at fixed error"
UNIT = "cell-updates/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ algorithmic bytes per launch
def mesh_counts(h):
    return dict(nc=h.n_cells, nf=h.n_faces, ne=h.n_edges, c2f=len(h["c2f_idx"]), f2e=len(h["f2e_idx"]),
                e2f=len(h["e2f_idx"]), ec=len(h["ec_cell"]), f2c=len(h["f2c_idx"]))


def algorithmic_bytes(k, c, nsp, group, precision="fp64", sources=False):
    """Compulsory bytes of one launch of kernel class k: every array the pass needs, counted once
    (perfect reuse within the pass); values 8 bytes (FP64) or 4 (FP32 bulk of the mixed path; the
    state U and the face fluxes Phi stay 8), indices 4, signs / flags 1.  With the two-ion sources:
    * FP64: `prepare` includes the cell-current pass and `update` reads the J x B inputs.
    * Mixed: the face-candidate pass also writes the face terms of J (16 bytes per face), which the
      update gathers with the total field (16 bytes per cell).
    * `gyrate` reads both ions' state and rewrites their momenta and energies, with the total field.
      The opening half step also renews the primitives and u+ of the cells it turns.  FP64 has two
      launches per step (opening, closing) and the figure is their mean.  Mixed has only the opening
      launch, since the update applies the closing half step."""
    base = _algorithmic_bytes(k, c, nsp, group, precision)
    if not sources:
        return base
    nc, nf = c["nc"], c["nf"]
    gyr = 80 * nc + 64 * nc + nc        # U of both ions in, momenta and energies out, material
    if precision == "mixed":
        extra = {"face_candidate": 16 * nf, "update": 16 * nf + 16 * nc,
                 "gyrate": gyr + 16 * nc + 20 * nsp * nc + 16 * nc}
    else:
        extra = {"prepare": 64 * nc + c["c2f"] * 5 + 36 * nf, "update": (2 + 3 + 3) * 8 * nc,
                 "gyrate": gyr + 24 * nc + (40 * nsp * nc + 24 * nc) / 2}
    return base + extra.get(k, 0.0)


def _algorithmic_bytes(k, c, nsp, group, precision="fp64"):
    nc, nf, ne = c["nc"], c["nf"], c["ne"]
    if precision == "mixed":
        g, e2f, f2e, ec = group, c["e2f"], c["f2e"], c["ec"]
        # limited_gradients: primitives (32 B per cell and species), stencil operator K (64 B) and neighbour ids (16 B),
        #   validity, face values out (80 B per cell and species)
        # face_flux: face values of both sides, flux records out, per-face normal, slots, L/R, kind, f2c row
        # update: flux records, face ids and signs, U in and out, U of the averaged stage (stage 2: the mean over
        #   the two launches is 20 B per species), 1/V, material
        # edge_emf: tangent + length, mode, row pointers, E out; per (edge, face) id and the 24-byte plane table;
        #   per (edge, cell) id; the faces' 16-byte EMF records and the cells' velocities
        # ct: the packed face-edge record, Phi in, Phi out, the averaged Phi (mean 4 B), E
        return {
            "prepare": 40 * nsp * nc + 20 * nsp * nc + 16 * nc + 48 * nc + 8 * nf + 16 * nc + 48 * nc + nc,
            "cfl": 20 * nsp * nc + 16 * nc + 16 * nc + 16 * nf + 4 * nc + nc,
            "limited_gradients": 32 * g * nc + 64 * nc + 16 * nc + nc + 80 * g * nc,
            "face_flux": 80 * g * nc + 20 * g * nf + 35 * nf + nc,
            "update": 20 * g * nf + 20 * nc + 40 * g * nc + 40 * g * nc + 20 * g * nc + 4 * nc + nc,
            "face_candidate": 48 * nc + 16 * nf + 16 * nf + 8 * nf + 12 * nf,
            "edge_emf": 29 * ne + 28 * e2f + 4 * ec + 16 * nf + 16 * nc,
            "ct": 36 * nf + 4 * ne,
        }.get(k, 0.0)
    p = 8
    csr_c2f = c["c2f"] * 5 + nc * 4          # idx + sgn + ptr
    if k == "prepare":
        return (10 * nsp * nc + nf * 5 + 3 * nc + 9 * nc) * p + csr_c2f + nc
    if k == "limited_gradients":
        g = group
        return (20 * g * nc + 6 * nc + 3 * c["c2f"] + 3 * nc + 3 * nf) * p + c["c2f"] * 8 + csr_c2f + 2 * nc
    if k == "face_flux":
        g = group
        return (20 * g * nc + 3 * nc + 7 * nf + 5 * g * nf) * p + c["f2c"] * 5 + nf * 4 + 2 * nf * 4 + nf + nc
    if k == "update":
        g = group
        return (5 * g * nf + 12.5 * g * nc + nc) * p + c["c2f"] * 5 + nc * 4 + nc   # stage 1 / 2 averaged (U0 read in stage 2)
    # face_candidate also writes phi_ind / |A| per face for the edge pass; edge_emf reads the per-(edge, slot)
    # face geometry (m, n, sigma, w: 8 values per e2f entry) instead of the faces' centres and areas
    if k == "face_candidate":
        return (9 * nc + 4 * nf + 2 * nf + 3 * nf + nf) * p + c["f2c"] * 5 + nf * 4 + 2 * nf * 4
    if k == "edge_emf":
        return (8 * c["e2f"] + 4 * ne + 3 * nf + nf + 3 * nc + ne) * p + c["e2f"] * 4 + ne * 8 + c["ec"] * 4 + nc + ne
    if k == "ct":
        return (ne + 2.5 * nf) * p + c["f2e"] * 5 + nf * 4 + c["f2c"] * 4 + nf * 4
    if k == "cfl":
        return (5 * nsp * nc + 3 * nc + 4 * nf + nc) * p + csr_c2f + nc
    return 0.0


# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) that one ncu capture measured
# on the 6 x 32 x 32 x 48 x 6 shell of the same construction, with the entity count it scales with;
# the bench line reports it scaled to its own workload (the traffic grows in proportion to that count).
# dram__bytes_read.sum + dram__bytes_write.sum of one launch in the ncu capture of the 6x32x32x48x6 shell
# (1,769,472 cells, 2,082,912 edges), scaled by the entity count the traffic grows with; the update's
# captured launch is a stage-1 launch (the stage-2 launch also reads the step's opening state)
NCU_TRAFFIC = {("edge_emf", "mixed"): (493.91e6, "ne", 2082912), ("update", "mixed"): (543.20e6, "nc", 1769472),
               ("limited_gradients", "mixed"): (511.77e6, "nc", 1769472)}


def ncu_traffic(kernel, precision, counts):
    t = NCU_TRAFFIC.get((kernel, precision))
    if not t:
        return None
    return t[0] / t[2] * counts[t[1]]


# ------------------------------------------------------------------ clocks during the timed region
class ClockSampler:
    def __init__(self, gpu_index):
        self.proc = None
        self.path = None
        try:
            fd, self.path = tempfile.mkstemp(prefix="mhd_clocks_", suffix=".csv")
            self.fh = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(gpu_index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            if self.path:
                self.fh.close()
                os.unlink(self.path)
            return
        # nvidia-smi takes a fraction of a second to start; wait (at most 2 s) for its first sample
        # so that the samples cover the steps that follow, not its start-up
        t0 = time.time()
        while time.time() - t0 < 2.0 and self.proc.poll() is None and os.path.getsize(self.path) == 0:
            time.sleep(0.01)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            lines = fh.readlines()
        os.unlink(self.path)
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ workload
def make_workload(args):
    from mpcns_uns_b200 import workloads
    t = time.time()
    if args.config == "box":
        wl = workloads.box(args.ncube or 16)
    else:
        wl = workloads.shell(args.ncube or 64, args.nr or 96, r_in=1.0, r_out=6.0, sources=not args.no_sources, device_geometry=True)
    log(f"[bench] workload {wl.name}: {wl.mesh.n_cells} cells, {wl.mesh.n_faces} faces, {wl.mesh.n_edges} edges "
        f"(setup {time.time() - t:.1f}s)")
    return wl


def cpu_sample(args):
    """Bounded sample of the same workload for the CPU baseline of this arm: the same shell construction at
    6 x 16 x 16 x 24 (221,184 cells), two ions, built by the reference's own code (reference_workload)."""
    if args.config == "box":
        return reference_workload("box", 12, 0, args)
    return reference_workload("shell", 16, 24, args)


def reference_workload(config, ncube, nr, args):
    """The benchmark's workload built by the reference's own code, with no library of this repository loaded:
    the cubed-sphere shell of uns::make_cubed_sphere_shell cut into tetrahedra and numbered by the reference's
    ComplexBuilder (oracle/_ref: ref_mesh_shell_tets), its uns::compute_geometry and BoundaryInfo::build, and
    the seeded state of workloads.shell_state (numpy) on that mesh.  Entity for entity and bit for bit the
    mesh, metric and state of workloads.shell (same uns::topology_hash; tests/test_oracle.py checks it).
    The box (--config box) has no reference generator with the workload's node jitter, so its sample is the
    reference's unjittered box."""
    from oracle import ref
    from mpcns_uns_b200 import workloads
    if config == "box":
        r = ref.RefMesh.box(ncube, ncube, ncube).boundary("outflow", {}, (1.0, 0.0, 0.0))
        rng = np.random.default_rng(1)
        nc = r.n_cells
        W = np.zeros((nc, 5))
        W[:, 0], W[:, 1], W[:, 4] = 1.0 + 0.01 * rng.uniform(-1, 1, nc), 1.0, 0.1
        return workloads.Workload(name=f"refbox{ncube}^3", mesh=r, n_species=1, gamma=workloads.GAMMA,
                                  U=[workloads.to_cons(W, workloads.GAMMA).ravel()], Phi=np.zeros(r.n_faces),
                                  PhiAdd=np.zeros(r.n_faces), fs=[(1.0, 1.0, 0.0, 0.0, 0.1)], mass=[1.0], u_inf=(1.0, 0.0, 0.0),
                                  B_imf=(0.0, 0.0, 0.0))
    stretch = workloads.shell_stretch(ncube, nr, 1.0, 6.0)
    r = ref.RefMesh.shell_tets(ncube, nr, 1.0, 6.0, stretch)
    r.boundary("outflow", {"inner": "wall", "outer": "farfield"}, (-8.0, 0.0, 0.0))
    return workloads.shell_state(r, f"shell6x{ncube}x{ncube}x{nr}x6", 1.0, stretch, sources=not args.no_sources)


def time_reference(wl, steps, warmup):
    """The reference's own hot-path step (oracle/_ref, np = 1, one core) on workload wl, whose mesh is a
    reference mesh (oracle.ref.RefMesh): seconds per step, median of `steps` after `warmup`."""
    from oracle import ref
    r = wl.mesh
    p = ref.StepParams()
    p.n_species, p.second_order = wl.n_species, 1
    p.gamma, p.rho_floor, p.p_floor, p.cuct, p.M_ref, p.ne_floor, p.rel_limit = wl.gamma, 1e-10, 1e-12, 0.5, 1.0, 0.01, 0.0
    p.u_inf[:] = list(wl.u_inf)
    p.B_imf[:] = list(wl.B_imf)
    for s in range(wl.n_species):
        p.mass[s] = wl.mass[s]
        p.fs[s][:] = list(wl.fs[s])
    p.lorentz, p.induce_coeff, p.inver_MA2 = int(wl.lorentz), wl.induce_coeff, wl.inver_MA2
    U = [np.array(u) for u in wl.U]
    Phi = np.array(wl.Phi)
    Badd = r.cell_vector(wl.PhiAdd)
    dt = None
    times = []
    for k in range(warmup + steps):
        t0 = time.perf_counter()
        W = [r.to_prim(u, wl.gamma) for u in U]
        Btot = r.cell_vector(Phi) + Badd
        if wl.n_species == 2:
            dt = r.local_time_step(wl.gamma, 0.4, 1.0, 1e-2, W[0], W[1], Btot)
        else:
            dt = dt or 0.2 * float(np.min(np.asarray(r["edge_len"])))
        r.rk2_step(p, U, Phi, wl.PhiAdd, Badd, dt)
        if k >= warmup:
            times.append(time.perf_counter() - t0)
        log(f"[bench] reference step {k + 1}/{warmup + steps}: {time.perf_counter() - t0:.2f} s")
    per_step = float(np.median(times))
    return wl.mesh.n_cells * wl.n_species * 2 / per_step, per_step


def gmres_bytes(k, c, precision, steps, launches, reorth=0):
    """Compulsory bytes of one launch of kernel class k of the induction solve, in the form the
    Arnoldi step runs it (preconditioned input, lazily normalised basis vector, Dirichlet mask).
    q = bytes of the operator's arrays (8 FP64, 4 for the FP32 operator of the mixed solve); Krylov
    vectors are FP64.  gram_schmidt: Arnoldi step j (j + 1 basis vectors) reads w and V_0..V_j in its
    dot pass, reads them again and writes w and the next matvec's input (8 bytes, 4 in mixed
    precision) in its update pass, and once more in the second pass where one ran (`reorth` of them);
    `launches` counts the class's launches (three per step, the second pass's gated ones included),
    so the figure is the solve's bytes over its launches."""
    q = 4 if precision == "mixed" else 8
    nc, nf, ne = c["nc"], c["nf"], c["ne"]
    if k == "face_d1":
        return 4 * (nf + 1) + 5 * c["f2e"] + 16 * ne + 8 * nf + 2 * q * nf
    if k == "cell_field":
        return 4 * (nc + 1) + 4 * c["c2f"] + 3 * q * c["c2f"] + q * nf + 3 * q * nc
    if k == "hall_emf":
        return 4 * nc + 5 * c["c2f"] + 4 * nf + 4 * c["f2c"] + 3 * q * nf + 11 * q * nc + nc
    if k == "edge_gather":
        return 8 * ne + 5 * c["e2f"] + q * nf + (4 + q) * c["ec"] + 4 * q * ne + 3 * q * nc + 41 * ne
    if k == "gram_schmidt":
        # steps run in cycles of 30: column j of a cycle has j + 1 basis vectors
        vec = 0.0
        zs = 4 if precision == "mixed" else 8
        for t in range(steps):
            j = t % 30
            vec += (j + 2) * 8 + (j + 2) * 8 + 8 + zs
        if steps:
            jm = sum(t % 30 for t in range(steps)) / steps
            vec += reorth * ((jm + 2) * 8 + 8 + zs)
        return vec * ne / max(launches, 1)
    return 0


def bench_gmres(args, peak):
    """Semi-implicit Hall + resistive induction solve (ImplicitInduction::solve) on the r in [0.8, 6]
    shell: GMRES(30), Jacobi, rtol 1e-8, dt = 20 x the explicit whistler limit, cold start; FP64 and
    mixed (FP32 operator in the Arnoldi, FP64 basis / Hessenberg / true residual)."""
    import torch
    from mpcns_uns_b200 import gpu, workloads
    t = time.time()
    case = workloads.induction_case(args.gmres_ncube, args.gmres_nr, device_geometry=True)
    h = case.mesh
    log(f"[bench] induction workload {case.name}: {h.n_cells} cells, {h.n_edges} edges (setup {time.time() - t:.1f}s)")
    dm = gpu.DeviceMesh(h)
    counts = mesh_counts(h)
    out = {"workload": case.name, "cells": h.n_cells, "faces": h.n_faces, "edges": h.n_edges, "restart": 30, "rtol": 1e-8,
           "max_it": args.gmres_max_it, "dt": case.dt, "dt_over_whistler_limit": case.dt / case.dt_whistler,
           "solves_timed": args.gmres_solves}
    E = {}
    for prec in ("fp64", "mixed"):
        di = gpu.DeviceInduction(dm, case.m_edge, hall=True, hall_coef=case.hall_coef, hall_r_min=case.hall_r_min,
                                 hall_r_max=case.hall_r_max, rtol=1e-8, max_it=args.gmres_max_it, restart=30, precision=prec)
        di.set_frozen_state(case.B0, case.ne)
        di.solve(case.Phi, case.E_expl, case.dirichlet, case.dt, False)  # warm-up (captures the cycle graph)
        torch.cuda.synchronize()
        l0 = di.launches()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(dm.stream)
        for _ in range(args.gmres_solves):
            Ed, it, rr = di.solve(case.Phi, case.E_expl, case.dirichlet, case.dt, False)
        ev1.record(dm.stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1) / args.gmres_solves
        launches = (di.launches() - l0) // args.gmres_solves
        # one more solve with per-kernel events (direct launches instead of the graph)
        di.profile(True)
        di.solve(case.Phi, case.E_expl, case.dirichlet, case.dt, False)
        prof = di.profile_read()
        di.profile(False)
        gs_l = prof.get("gram_schmidt", (0, 0))[1]
        reorth = di.reorth_passes()
        kern = {}
        for k, (kms, n) in prof.items():
            if not n:
                continue
            b = gmres_bytes(k, counts, prec, it, gs_l, reorth)
            kern[k] = {"ms_per_solve": kms, "launches_per_solve": n, "GBps": b / (kms / n / 1e3) / 1e9 if b else None}
        top = max((k for k in kern if kern[k]["GBps"]), key=lambda k: kern[k]["ms_per_solve"])
        E[prec] = Ed.double().cpu().numpy()
        out[prec] = {"s_per_solve": ms / 1e3, "iterations": it, "rel_res": rr, "converged": rr <= 1e-8, "reorth_passes": reorth,
                     "ms_per_iteration": ms / max(it, 1), "gpu_launches_per_solve": launches, "kernels": kern,
                     "roofline": {"bound": "hbm", "kernel": top, "achieved": kern[top]["GBps"], "peak": peak, "unit": "GB/s",
                                  "frac": kern[top]["GBps"] / peak}}
        del di
    out["speedup_mixed"] = out["fp64"]["s_per_solve"] / out["mixed"]["s_per_solve"]
    out["E_rel_l2_mixed_vs_fp64"] = float(np.linalg.norm(E["mixed"] - E["fp64"]) / np.linalg.norm(E["fp64"]))
    out["rel_res_ratio_mixed_vs_fp64"] = out["mixed"]["rel_res"] / out["fp64"]["rel_res"]
    if args.gmres_ilu_max_it > 0:
        out["ilu"] = bench_gmres_ilu(args, case, dm)
    return out


def bench_gmres_ilu(args, case, dm):
    """The same FP64 solve with the block ILU(0) preconditioner (Config::ind_ilu, shift 0.3) against Jacobi, both
    capped at --gmres-ilu-max-it iterations: host pattern time, device time of one factorisation and of one
    application (both triangular solves), seconds per capped solve and the residual each preconditioner reaches."""
    import torch
    from mpcns_uns_b200 import gpu
    il = {"max_it": args.gmres_ilu_max_it, "shift": 0.3}
    for ilu in (False, True):
        di = gpu.DeviceInduction(dm, case.m_edge, hall=True, hall_coef=case.hall_coef, hall_r_min=case.hall_r_min,
                                 hall_r_max=case.hall_r_max, rtol=1e-8, max_it=args.gmres_ilu_max_it, restart=30)
        di.set_frozen_state(case.B0, case.ne)
        if ilu:
            t = time.time()
            di.set_ilu(True, 0.3)
            il["pattern_s"] = time.time() - t
        di.solve(case.Phi, case.E_expl, case.dirichlet, case.dt, False)  # warm-up (captures the cycle graph)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(dm.stream)
        _, it, rr = di.solve(case.Phi, case.E_expl, case.dirichlet, case.dt, False)
        ev1.record(dm.stream)
        ev1.synchronize()
        il["ilu" if ilu else "jacobi"] = {"s_per_solve": ev0.elapsed_time(ev1) / 1e3, "iterations": it, "rel_res": rr}
        if ilu:
            d = torch.tensor(case.dirichlet, device="cuda")
            v = torch.rand(case.mesh.n_edges, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(5))
            evs = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            evs[0].record(dm.stream)
            di.ilu_factor(case.dt, d)
            evs[1].record(dm.stream)
            di.ilu_apply(v, d)
            evs[2].record(dm.stream)
            evs[2].synchronize()
            il["factor_ms"] = evs[0].elapsed_time(evs[1])
            il["apply_ms"] = evs[1].elapsed_time(evs[2])
        del di
    log(f"[bench] ILU(0) {il['max_it']} iterations: {il['ilu']['s_per_solve']:.3f} s, rel_res {il['ilu']['rel_res']:.3e} "
        f"(Jacobi {il['jacobi']['s_per_solve']:.3f} s, {il['jacobi']['rel_res']:.3e}); factor {il['factor_ms']:.1f} ms, "
        f"apply {il['apply_ms']:.2f} ms")
    return il


def bench_adjoint(args):
    """Gradient of J = sum |B_tot|^2 V over the dayside cells with r in [1.2, 1.6] after 40 FP64 steps (fixed CFL
    step of the initial state) on the 6 x 32 x 32 x 64 shell (2.36M tets, two ions, explicit resistive EMF with a
    seeded log-uniform per-cell resistivity 1e-4..1e-2), with respect to the resistivity and the inflow velocity:
    device time of the forward run (checkpoint every 8 steps), the adjoint sweep and the tangent-linear run; the
    adjoint against the tangent-linear run (dot products) and against central differences of the forward run
    (which is bit-identical to the reference's step) along 16 seeded directions in (eta, u_inf) and 6 in eta at
    h = 1e-6 and 1e-7, split by the forward run's switch log into switch-free and switch-crossing directions."""
    import torch
    from mpcns_uns_b200 import gpu, workloads
    t = time.time()
    case = workloads.adjoint_case(args.adj_ncube, args.adj_nr, n_steps=args.adj_steps, checkpoint_every=args.adj_checkpoint,
                                  device_geometry=True)
    wl = case.wl
    h = wl.mesh
    log(f"[bench] adjoint workload {wl.name}: {h.n_cells} cells (setup {time.time() - t:.1f}s)")
    dm = gpu.DeviceMesh(h)
    p = gpu.step_params(wl.n_species, wl.gamma, fs=wl.fs, mass=wl.mass, u_inf=wl.u_inf, B_imf=wl.B_imf, cfl=wl.cfl)
    st = gpu.ResidentState(dm, p)
    st.set(wl.U, wl.Phi, wl.PhiAdd)
    dt = st.cfl_dt()
    free0 = torch.cuda.mem_get_info()[0]
    fn = gpu.DeviceFunction(st, case.eta, case.mask, case.n_steps, case.checkpoint_every, dt)
    fn.forward()
    fn.backward()   # warm-up: allocates the checkpoints and the recorded segment
    torch.cuda.synchronize()
    mem = free0 - torch.cuda.mem_get_info()[0]

    def dev_time(f, reps=2):
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(dm.stream)
            r = f()
            e1.record(dm.stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms)), r

    l0 = st.launches()
    fwd_ms, J = dev_time(fn.forward)
    step_launches = (st.launches() - l0) // 2
    bwd_ms, (ge, gu) = dev_time(fn.backward)
    rng = np.random.default_rng(23)
    nc = h.n_cells
    u0 = np.asarray(wl.u_inf, np.float64)
    d_eta = rng.standard_normal(nc) * case.eta
    d_u = rng.standard_normal(3) * np.linalg.norm(u0)
    fn.tangent(d_eta, d_u)   # warm-up: allocates the tangent arrays
    tan_ms, (Jt, dJ) = dev_time(lambda: fn.tangent(d_eta, d_u), reps=1)
    adj = float(ge @ d_eta + gu @ d_u)
    dots = [abs(adj - dJ) / abs(dJ)]
    for _ in range(2):
        de = rng.standard_normal(nc) * case.eta
        du = rng.standard_normal(3) * np.linalg.norm(u0)
        _, dj = fn.tangent(de, du)
        dots.append(abs(float(ge @ de + gu @ du) - dj) / abs(dj))
    fn.profile(True)
    fn.forward()
    fn.backward()
    prof = fn.profile_read()
    fn.profile(False)
    classes = {k: {"ms": v[0], "launches": v[1]} for k, v in prof.items() if v[1]}
    # Central differences of the forward run (bit-identical to the reference's step; J summed in double-double,
    # so that the difference of two runs is not limited by J's own ulp), split by the forward run's switch log
    # into the directions along which the J(p + h d) and J(p - h d) runs made the same discrete choices
    # everywhere (switch-free) and those that crossed a switch (limiter bound, Rusanov wave-speed side or sign,
    # edge upwind cell or sign, floor), where J is only piecewise smooth.  Directions: --adj-fd-dirs with an
    # eta and an inflow part, and 6 in eta alone (switch-free by construction without model sources).
    fd = {}
    dirs = [(rng.standard_normal(nc) * case.eta, rng.standard_normal(3) * np.linalg.norm(u0)) for _ in range(args.adj_fd_dirs)]
    dirs += [(rng.standard_normal(nc) * case.eta, np.zeros(3)) for _ in range(6)]
    fn.switch_log(True)
    for hh in (1e-6, 1e-7):
        rows = []
        for de, du in dirs:
            fn.set_params(eta=case.eta + hh * de, u_inf=u0 + hh * du)
            fn.forward()
            Jp, sp = fn.last_J(), fn.switches()
            fn.set_params(eta=case.eta - hh * de, u_inf=u0 - hh * du)
            fn.forward()
            Jm, sm = fn.last_J(), fn.switches()
            f = fn.central_difference(Jp, Jm, hh)
            rows.append((abs(float(ge @ de + gu @ du) - f) / abs(f), fn.switch_flips(sp, sm), bool(np.any(du))))
        free = [r for r in rows if sum(r[1].values()) == 0]
        cross = [r for r in rows if sum(r[1].values()) > 0]
        fd[f"h={hh:g}"] = {
            "switch_free": {"directions": len(free), "max_rel_err": max((r[0] for r in free), default=None),
                            "with_inflow_part": sum(r[2] for r in free)},
            "crossing": {"directions": len(cross), "max_rel_err": max((r[0] for r in cross), default=None),
                         "median_rel_err": float(np.median([r[0] for r in cross])) if cross else None,
                         "median_flips": {k: float(np.median([r[1][k] for r in cross])) for k in gpu.DeviceFunction.SWITCH_KINDS} if cross else None},
            "per_direction": [{"rel_err": r[0], "flips": r[1], "inflow_part": r[2]} for r in rows]}
    fn.switch_log(False)
    fn.set_params(eta=case.eta, u_inf=u0)
    out = {"workload": wl.name, "cells": nc, "faces": h.n_faces, "edges": h.n_edges, "n_species": wl.n_species,
           "steps": case.n_steps, "checkpoint_every": case.checkpoint_every, "dt": dt, "J": J,
           "functional": "sum |B_tot|^2 V over the dayside cells with 1.2 <= r <= 1.6",
           "parameters": "per-cell resistivity (log-uniform 1e-4..1e-2) and the inflow velocity (3)",
           "forward_s": fwd_ms / 1e3, "backward_s": bwd_ms / 1e3, "tangent_s": tan_ms / 1e3,
           "backward_over_forward": bwd_ms / fwd_ms, "forward_plus_backward_over_forward": (fwd_ms + bwd_ms) / fwd_ms,
           "tangent_over_forward": tan_ms / fwd_ms, "step_launches_per_forward": step_launches,
           "device_memory_GB": mem / 1e9, "classes_forward_plus_backward": classes,
           "dot_test_rel_err_max": max(dots), "fd": fd, "grad_u": [float(x) for x in gu],
           "grad_eta_abs_max": float(np.abs(ge).max())}
    del fn, st, dm
    torch.cuda.empty_cache()
    return out


def bench_config1(args):
    """Config 1 itself, the reference's CPU-runnable case: the unit cube of 16^3 hexahedra x 6 tetrahedra (24,576
    cells, interior nodes jittered, seed 0), one ion, 20 steps at CFL 0.4 with the device CFL step, outflow
    everywhere; FP64 (reference-exact) and mixed precision, device time of the 20 steps after one warm-up step
    from the same initial state, and div B after them.  A precision that fails is reported, not raised."""
    import torch
    from mpcns_uns_b200 import gpu, workloads
    wl = workloads.box(16)
    h = wl.mesh
    dm = gpu.DeviceMesh(h)
    out = {"workload": wl.name, "cells": h.n_cells, "steps": wl.steps, "cfl": wl.cfl, "n_species": wl.n_species}
    for prec in ("fp64", "mixed"):
        try:
            p = gpu.step_params(wl.n_species, wl.gamma, fs=wl.fs, mass=wl.mass, u_inf=wl.u_inf, B_imf=wl.B_imf, cfl=wl.cfl,
                                precision=prec)
            st = gpu.ResidentState(dm, p)
            st.set(wl.U, wl.Phi, wl.PhiAdd)
            st.step(0.0)
            st.set(wl.U, wl.Phi, wl.PhiAdd)
            torch.cuda.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(dm.stream)
            for _ in range(wl.steps):
                st.step(0.0, sync=False)
            ev1.record(dm.stream)
            ev1.synchronize()
            ms = ev0.elapsed_time(ev1) / wl.steps
            out[prec] = {"ms_per_step": ms, "cell_updates_per_s": h.n_cells * wl.n_species * 2 / (ms / 1e3),
                         "div_b_max_rel": dm.div_b(st.Phi())["max_rel"]}
            del st
        except Exception as e:  # reported, not required
            out[prec] = {"error": str(e)[:200]}
    log(f"[bench] config 1 ({h.n_cells} cells, {wl.steps} steps): " +
        ", ".join(f"{k} {out[k].get('ms_per_step', float('nan')):.3f} ms/step" for k in ("fp64", "mixed")))
    return out


def bench_semi_implicit(args, wl, dm, new_state):
    """The reference's default run mode (Config::time_order = 1, Solver::step_first_order) on the step's shell:
    forward Euler of both ions with the J x B force and the Strang-split gyration, the EMF from the Hall +
    resistive ImplicitInduction::solve (the reference's radial taper from r = 1 to 1.012, eta / star1 with
    eta = 1e-2 below r = 1.2 and 1e-4 above, GMRES(30) to rtol 1e-8 capped at --si-max-it, warm start across
    steps), CT with it; FP64, CFL step.  The Hall coefficient is set so that the initial CFL step is
    --si-whistler-ratio times the explicit whistler limit of the initial state (the stiffness the implicit
    treatment is for; config 3's ratio of 20 stagnates Jacobi GMRES).  Wall time of each synchronous step."""
    import torch
    from mpcns_uns_b200 import gpu, workloads
    h = wl.mesh
    st = new_state("fp64")
    r_e = np.linalg.norm(np.asarray(h["edge_mid"]), axis=1)
    m_edge = np.where(r_e < 1.2, 1e-2, 1e-4) / np.asarray(h["star1"])
    # n_e,eff (M_ref 1, ne_floor 0.01) and |B_tot| of the initial state; whistler limit of hall_coef 1
    nc = h.n_cells
    ne = np.asarray(wl.U[0]).reshape(nc, 5)[:, 0] / wl.mass[0] + np.asarray(wl.U[1]).reshape(nc, 5)[:, 0] / wl.mass[1]
    ne_eff = np.sqrt(ne * ne + 1e-4)
    B = dm.reconstruct_cell_vector(np.asarray(wl.Phi) + np.asarray(wl.PhiAdd)).cpu().numpy()
    dtw1 = workloads.whistler_dt(h, B, ne_eff, 1.0, 1.0)
    hall_coef = args.si_whistler_ratio * dtw1 / st.cfl_dt()
    di = gpu.DeviceInduction(dm, m_edge, hall=True, hall_coef=hall_coef, hall_r_min=1.0, hall_r_max=1.012, rtol=1e-8,
                             max_it=args.si_max_it, restart=30)
    st.step_semi_implicit(di)  # warm-up: the solve's tables and captured restart cycle
    torch.cuda.synchronize()
    ms, its, rrs, dts = [], [], [], []
    for _ in range(args.si_steps):
        t0 = time.perf_counter()
        dt, it, rr = st.step_semi_implicit(di)
        ms.append((time.perf_counter() - t0) * 1e3)
        its.append(it)
        rrs.append(rr)
        dts.append(dt)
    out = {"workload": wl.name, "cells": h.n_cells, "edges": h.n_edges, "steps": args.si_steps, "ms_per_step": float(np.median(ms)),
           "iterations": its, "rel_res": rrs, "dt": dts, "max_it": args.si_max_it, "rtol": 1e-8, "restart": 30, "hall_coef": hall_coef,
           "dt_over_whistler_limit": args.si_whistler_ratio,
           "eta": "1e-2 for r < 1.2, 1e-4 above", "precision": "fp64"}
    log(f"[bench] semi-implicit step: {out['ms_per_step']:.1f} ms per step, iterations {its}, rel_res {max(rrs):.2e}")
    del di, st
    return out


def bench_ten_ion(args, peak):
    """Config 5: the ten-ion shell r in [1, 8], 6 x 96 x 96 x 128 x 6 tetrahedra (42.5M cells), crustal background
    field, no model sources: mixed and FP64 steps (CFL 0.4 on the device), per-kernel times, and the mixed state's
    error against the FP64 state after --ten-accuracy-steps steps from the same start."""
    import torch
    from mpcns_uns_b200 import gpu, workloads
    t = time.time()
    wl = workloads.ten_ion(args.ten_ncube, args.ten_nr, device_geometry=True)
    h = wl.mesh
    log(f"[bench] ten-ion workload {wl.name}: {h.n_cells} cells (setup {time.time() - t:.1f}s)")
    dm = gpu.DeviceMesh(h)
    counts = mesh_counts(h)
    cu = h.n_cells * wl.n_species * 2
    out = {"workload": wl.name, "cells": h.n_cells, "faces": h.n_faces, "edges": h.n_edges, "n_species": wl.n_species,
           "masses": list(wl.mass), "steps_timed": args.ten_steps, "dt": "CFL 0.4 on device", "sources": "none"}
    final = {}
    for prec in ("fp64", "mixed"):
        p = gpu.step_params(wl.n_species, wl.gamma, fs=wl.fs, mass=wl.mass, u_inf=wl.u_inf, B_imf=wl.B_imf, cfl=wl.cfl,
                            precision=prec)
        st = gpu.ResidentState(dm, p)
        st.set(wl.U, wl.Phi, wl.PhiAdd)
        for _ in range(2):
            st.step(0.0)
        torch.cuda.synchronize()
        st.profile(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(dm.stream)
        for _ in range(args.ten_steps):
            st.step(0.0, sync=False)
        e1.record(dm.stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.ten_steps
        prof = st.profile_read()
        st.profile(False)
        kern = {k: {"ms_per_step": v[0] / args.ten_steps,
                    "GBps": algorithmic_bytes(k, counts, wl.n_species, 2, prec, False) / (v[0] / v[1] / 1e3) / 1e9}
                for k, v in prof.items() if v[1]}
        out[prec] = {"ms_per_step": ms, "value": cu / (ms / 1e3), "kernels": kern}
        if args.ten_accuracy_steps > 0:
            st.set(wl.U, wl.Phi, wl.PhiAdd)
            for _ in range(args.ten_accuracy_steps):
                st.step(0.0, sync=False)
            final[prec] = ([st.U(s) for s in range(wl.n_species)], st.Phi())
        del st
        torch.cuda.empty_cache()
    out["speedup_mixed"] = out["mixed"]["value"] / out["fp64"]["value"]
    if final:
        (U64, P64), (U32, P32) = final["fp64"], final["mixed"]
        num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(U32, U64))
        den = sum(float(np.sum(b ** 2)) for b in U64)
        out["accuracy_mixed_vs_fp64"] = {"steps": args.ten_accuracy_steps, "U_all_rel_l2": float(np.sqrt(num / den)),
                                         "U_H_rel_l2": float(np.linalg.norm(U32[0] - U64[0]) / np.linalg.norm(U64[0])),
                                         "Phi_rel_l2": float(np.linalg.norm(P32 - P64) / np.linalg.norm(P64 + wl.PhiAdd)),
                                         "div_b_max_rel_mixed": dm.div_b(P32, wl.PhiAdd)["max_rel"]}
    out["roofline_top_mixed"] = max(out["mixed"]["kernels"].items(), key=lambda kv: kv[1]["ms_per_step"])[0]
    k = out["mixed"]["kernels"][out["roofline_top_mixed"]]
    out["roofline_top_mixed_frac"] = k["GBps"] / peak
    del dm
    torch.cuda.empty_cache()
    return out


def gmres_cpu_baseline(max_it=60):
    """ImplicitInduction::solve of the reference (oracle/_ref, np = 1, one core) on the same construction at
    6 x 16 x 16 x 24 (262,704 edges), cold start, `max_it` iterations: seconds per GMRES iteration."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle import ref
    from helpers import SHELL_TAGS, ref_twin
    from mpcns_uns_b200 import workloads
    case = workloads.induction_case(16, 24)
    r = ref_twin(case.mesh, SHELL_TAGS).boundary("outflow", {"inner": "wall", "outer": "farfield"}, (-8.0, 0.0, 0.0))
    ri = ref.RefInduction(r, hall=True, hall_coef=case.hall_coef, hall_r_min=case.hall_r_min, hall_r_max=case.hall_r_max,
                          rtol=1e-8, max_it=max_it, restart=30)
    ri.set_m(case.m_edge)
    ri.set_frozen_state(case.B0, case.ne)
    t0 = time.perf_counter()
    _, it, rr = ri.solve(case.Phi, case.E_expl, case.dirichlet, case.dt, False)
    el = time.perf_counter() - t0
    return {"ms_per_iteration": 1e3 * el / max(it, 1), "iterations": it, "rel_res": rr, "cores": 1, "kind": "reference",
            "sample": f"{case.name} ({case.mesh.n_edges} edges), one cold solve capped at {max_it} iterations, np=1",
            "edges": case.mesh.n_edges}


def _r(x, d=4):
    """x rounded to d significant digits (None stays None)."""
    if x is None:
        return None
    return float(f"{x:.{d}g}")


def summary(out):
    """The figures of the line in a compact object printed last, so that they survive a cut of the output
    to its last 1500 characters: the mixed and FP64 steps, the mixed state's error after the accuracy run,
    div B, the GMRES solves, the adjoint's cost and checks, and the ten-ion steps when run."""
    sm = {"mixed_ms": _r(out["ms_per_step"]), "fp64_ms": _r(out["fp64"]["ms_per_step"]),
          "speedup_mixed": _r(out["fp64"]["speedup_mixed"]), "e2e": _r(out["e2e"]["value"]),
          "roofline_frac": _r(out["roofline"]["frac"], 3), "roofline_kernel": out["roofline"]["kernel"],
          "clocks_mhz": [(c or {}).get("sm_mhz") for c in (out["clocks"], out["fp64"].get("clocks"))]}
    a = out.get("accuracy_mixed_vs_fp64")
    if a:
        sm["acc"] = {"steps": a["steps"], "U": _r(a["U_all_rel_l2"], 3),
                     "U_sp": [_r(a[k], 3) for k in sorted(a) if k.startswith("U") and k.endswith("_rel_l2") and k[1].isdigit()],
                     "U_sp_fp64_pert": [_r(a[k], 3) for k in sorted(a) if k.endswith("_perturbed_1e-7")],
                     "Phi": _r(a["Phi_rel_l2"], 3), "divB": [_r(a["div_b_max_rel_mixed"], 3), _r(a["div_b_max_rel_fp64"], 3)]}
    g = out.get("gmres")
    if g:
        sm["gmres"] = {p: [_r(g[p]["s_per_solve"]), g[p]["iterations"], _r(g[p]["rel_res"], 3), g[p].get("reorth_passes")]
                       for p in ("fp64", "mixed")}
        sm["gmres"]["speedup_mixed"] = _r(g["speedup_mixed"])
        sm["gmres"]["cols"] = "s_per_solve, iterations, rel_res, Gram-Schmidt second passes"
        il = g.get("ilu")
        if il:
            sm["gmres"]["ilu"] = {"it": il["max_it"], "s": [_r(il["ilu"]["s_per_solve"]), _r(il["jacobi"]["s_per_solve"])],
                                  "rel_res": [_r(il["ilu"]["rel_res"], 3), _r(il["jacobi"]["rel_res"], 3)],
                                  "factor_apply_ms": [_r(il["factor_ms"]), _r(il["apply_ms"])]}
    c1 = out.get("config1")
    if c1:
        sm["config1"] = {k: _r(c1[k].get("ms_per_step"), 3) for k in ("fp64", "mixed") if k in c1}
    si = out.get("semi_implicit")
    if si:
        sm["semi_implicit"] = {"ms": _r(si["ms_per_step"]), "it": si["iterations"], "rel_res": _r(max(si["rel_res"]), 3)}
    d = out.get("adjoint")
    if d:
        fd = d["fd"]
        sm["adjoint"] = {"fwd_s": _r(d["forward_s"]), "fwd_bwd_over_fwd": _r(d["forward_plus_backward_over_forward"]),
                         "dot": _r(d["dot_test_rel_err_max"], 2),
                         "fd": {k: {"free": [v["switch_free"]["directions"], _r(v["switch_free"]["max_rel_err"], 2)],
                                    "crossing": [v["crossing"]["directions"], _r(v["crossing"]["max_rel_err"], 2),
                                                 _r(v["crossing"]["median_rel_err"], 2)]} for k, v in fd.items()},
                         "fd_cols": "free: directions, max rel err; crossing: directions, max, median rel err"}
    t = out.get("ten_ion")
    if t:
        sm["ten_ion"] = {"mixed_ms": _r(t["mixed"]["ms_per_step"]), "fp64_ms": _r(t["fp64"]["ms_per_step"]),
                         "U": _r((t.get("accuracy_mixed_vs_fp64") or {}).get("U_all_rel_l2"), 3)}
    return sm


def max_over_ranks(ms, dist, device):
    """The slowest rank's device time: every rank's K steps count once, the job ends with the last."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="shell", choices=["shell", "box"])
    ap.add_argument("--ncube", type=int, default=0)
    ap.add_argument("--nr", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-max-steps", type=int, default=3, help="cap of the reference arm's timed steps")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--accuracy-steps", type=int, default=100)
    ap.add_argument("--no-gmres", action="store_true")
    ap.add_argument("--no-sources", action="store_true", help="leave out the two-ion J x B force and gyration")
    ap.add_argument("--gmres-ncube", type=int, default=48)
    ap.add_argument("--gmres-nr", type=int, default=96)
    ap.add_argument("--gmres-max-it", type=int, default=300)
    ap.add_argument("--gmres-solves", type=int, default=2)
    ap.add_argument("--gmres-ilu-max-it", type=int, default=60, help="block ILU(0) leg against Jacobi (0: skip)")
    ap.add_argument("--no-semi-implicit", action="store_true", help="leave out the time_order = 1 step")
    ap.add_argument("--no-config1", action="store_true", help="leave out the 24,576-cell box (config 1)")
    ap.add_argument("--si-steps", type=int, default=3)
    ap.add_argument("--si-max-it", type=int, default=100)
    ap.add_argument("--si-whistler-ratio", type=float, default=2.0)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-ten-ion", action="store_true", help="leave out the ten-ion shell (config 5, 42.5M cells)")
    ap.add_argument("--ten-ion-only", action="store_true", help="run only the ten-ion section and print it as its own JSON line")
    ap.add_argument("--ten-ncube", type=int, default=96)
    ap.add_argument("--ten-nr", type=int, default=128)
    ap.add_argument("--ten-steps", type=int, default=5)
    ap.add_argument("--ten-accuracy-steps", type=int, default=50)
    ap.add_argument("--adjoint-only", action="store_true", help="run only the adjoint section and print it as its own JSON line")
    ap.add_argument("--adj-ncube", type=int, default=32)
    ap.add_argument("--adj-nr", type=int, default=64)
    ap.add_argument("--adj-steps", type=int, default=40)
    ap.add_argument("--adj-checkpoint", type=int, default=8)
    ap.add_argument("--adj-fd-dirs", type=int, default=16)
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import ref
        if not ref.available():
            print(json.dumps({"impl": "reference", "unavailable": "reference checker oracle/_ref not built"}))
            return
        # the same workload as this arm's own: the full configuration, built by the reference's code
        t0 = time.time()
        if args.config == "box":
            wl = reference_workload("box", args.ncube or 16, 0, args)
        else:
            wl = reference_workload("shell", args.ncube or 64, args.nr or 96, args)
        setup_s = time.time() - t0
        log(f"[bench] reference workload {wl.name}: {wl.mesh.n_cells} cells (setup {setup_s:.1f}s)")
        # one core takes about half a minute per step of the 14.2M-cell shell: the step count is capped
        steps = max(1, min(args.steps, args.ref_max_steps))
        warm = 1 if args.warmup > 0 else 0
        v, per = time_reference(wl, steps, warm)
        cfgd = {"workload": wl.name, "n_species": wl.n_species, "cells": wl.mesh.n_cells, "faces": wl.mesh.n_faces,
                "edges": wl.mesh.n_edges, "topology_hash": wl.mesh.topology_hash(), "l2": "inputs > L2",
                "sources": "J x B force + Strang-split exact gyration" if wl.lorentz else "none",
                "mesh": "uns::make_cubed_sphere_shell cut into 6 tetrahedra per hexahedron, numbered by the reference's "
                        "ComplexBuilder (no library of this repository loaded)",
                "steps_cap": f"min(--steps, {args.ref_max_steps}) timed steps after min(--warmup, 1) warm-up",
                "setup_s": setup_s}
        print(json.dumps({"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
                          "steps": steps, "warmup": warm, "ms_per_step": per * 1e3, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfgd,
                          "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                                           "sample": f"the full {wl.name} workload, {steps} steps after {warm} warm-up, np=1 "
                                                     "(the reference has no threads; no MPI on this host)"},
                          "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import torch
    torch.cuda.set_device(local)
    if args.adjoint_only or args.ten_ion_only:
        if rank == 0:
            peak, _ = peaks()
            print(json.dumps({"adjoint": bench_adjoint(args)} if args.adjoint_only else {"ten_ion": bench_ten_ion(args, peak)}))
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from mpcns_uns_b200 import gpu
    wl = make_workload(args)
    h = wl.mesh
    dm = gpu.DeviceMesh(h)
    stream = dm.stream
    counts = mesh_counts(h)
    group = min(2, wl.n_species)
    cu_per_step = h.n_cells * wl.n_species * 2

    def new_state(precision):
        p = gpu.step_params(wl.n_species, wl.gamma, fs=wl.fs, mass=wl.mass, u_inf=wl.u_inf, B_imf=wl.B_imf, cfl=wl.cfl,
                            precision=precision, lorentz=wl.lorentz, induce_coeff=wl.induce_coeff, inver_MA2=wl.inver_MA2)
        st = gpu.ResidentState(dm, p)
        st.set(wl.U, wl.Phi, wl.PhiAdd)
        return st

    def timed(st, precision, sampler=None):
        """K device-timed steps (CUDA events on the handle's stream) with live per-kernel events."""
        for _ in range(args.warmup):
            st.step(0.0, sync=True)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = st.launches()
        st.profile(True)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            st.step(0.0, sync=False)
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        prof = st.profile_read()
        st.profile(False)
        launches = st.launches() - l0
        ms = max_over_ranks(ms, dist, "cuda")
        if dist:
            dist.barrier()
        if not np.isfinite(st.cfl_dt()):
            raise RuntimeError("state became invalid")
        kern = max(prof, key=lambda k: prof[k][0])
        k_ms, k_n = prof[kern]
        bl = algorithmic_bytes(kern, counts, wl.n_species, group, precision, wl.lorentz)
        breakdown = {k: {"ms_per_step": v[0] / args.steps, "launches": v[1],
                         "GBps": algorithmic_bytes(k, counts, wl.n_species, group, precision, wl.lorentz) / (v[0] / v[1] / 1e3) / 1e9}
                     for k, v in prof.items() if v[1]}
        return dict(ms=ms, value=cu_per_step * args.steps * world / (ms / 1e3), launches=launches, kernel=kern,
                    bytes_launch=bl, achieved=bl / (k_ms / k_n / 1e3) / 1e9, kernels=breakdown)

    st64 = new_state("fp64")
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    r64 = timed(st64, "fp64")
    clocks64 = sampler.stop() if sampler else None
    st32 = new_state("mixed")
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    rmx = timed(st32, "mixed")
    clocks = sampler.stop() if sampler else None

    # accuracy of the mixed step against the FP64 step (itself bit-identical to the reference)
    acc = None
    if args.accuracy_steps > 0:
        for st in (st64, st32):
            st.set(wl.U, wl.Phi, wl.PhiAdd)
            for _ in range(args.accuracy_steps):
                st.step(0.0, sync=False)
        err = {}
        num = den = 0.0
        U64 = [st64.U(s) for s in range(wl.n_species)]
        P32, P64 = st32.Phi(), st64.Phi()
        for s in range(wl.n_species):
            a, b = st32.U(s), U64[s]
            err[f"U{s}_rel_l2"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
            num += float(np.sum((a - b) ** 2))
            den += float(np.sum(b ** 2))
        err["U_all_rel_l2"] = float(np.sqrt(num / den))
        # conditioning of the problem itself: the FP64 step from a state perturbed by 1e-7 (relative,
        # seeded uniform), the size of single-precision input rounding
        rng = np.random.default_rng(7)
        st64.set([u * (1 + 1e-7 * rng.uniform(-1, 1, u.size)) for u in wl.U], wl.Phi, wl.PhiAdd)
        for _ in range(args.accuracy_steps):
            st64.step(0.0, sync=False)
        for s in range(wl.n_species):
            a = st64.U(s)
            err[f"U{s}_rel_l2_fp64_perturbed_1e-7"] = float(np.linalg.norm(a - U64[s]) / np.linalg.norm(U64[s]))
        err["Phi_rel_l2"] = float(np.linalg.norm(P32 - P64) / np.linalg.norm(P64 + wl.PhiAdd))
        # d2 B relative to the total field the update works with (background flux in the normalisation,
        # as the reference's diagnostics do: MercuryUns/driver/Solver.cpp:577)
        acc = {"steps": args.accuracy_steps, **err, "div_b_max_rel_mixed": dm.div_b(P32, wl.PhiAdd)["max_rel"],
               "div_b_max_rel_fp64": dm.div_b(P64, wl.PhiAdd)["max_rel"]}
    peak, peak_kind = peaks()

    # end to end through the C-ABI with host buffers (pinned), copies inside the timed region
    st = st32
    pin_U = [torch.empty(5 * h.n_cells, dtype=torch.float64).pin_memory() for _ in range(wl.n_species)]
    pin_P = torch.empty(h.n_faces, dtype=torch.float64).pin_memory()
    for s in range(wl.n_species):
        pin_U[s].numpy()[:] = st.U(s)
    pin_P.numpy()[:] = st.Phi()
    e2e_times = []
    for _ in range(args.e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in range(wl.n_species):
            st.upload(gpu.FIELD_U, pin_U[s].numpy(), s)
        st.upload(gpu.FIELD_PHI, pin_P.numpy())
        st.step(0.0, sync=True)
        for s in range(wl.n_species):
            st.download(gpu.FIELD_U, s, out=pin_U[s].numpy())
        st.download(gpu.FIELD_PHI, out=pin_P.numpy())
        e2e_times.append(time.perf_counter() - t0)
    e2e_v = cu_per_step * world / float(np.median(e2e_times))
    io_bytes = (5 * h.n_cells * wl.n_species + h.n_faces) * 8

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            from oracle import ref
            if ref.available():
                swl = cpu_sample(args)
                v, per = time_reference(swl, 3, 1)
                cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                       "sample": f"{swl.name} ({swl.mesh.n_cells} cells, same construction), 3 steps after 1 warm-up, np=1"}
        except Exception as e:  # the baseline is reported, never required
            log(f"[bench] cpu baseline failed: {e}")

    gm = None
    # the configuration sections run once, on a single-GPU run (under torchrun the replicas time the step only)
    if world > 1:
        args.no_gmres = args.no_adjoint = True
        args.no_ten_ion = args.no_semi_implicit = args.no_config1 = True
    c1 = None
    if rank == 0 and not args.no_config1 and args.config != "box":
        try:
            c1 = bench_config1(args)
        except Exception as e:  # reported, not required
            log(f"[bench] config 1 failed: {e}")
    si = None
    if rank == 0 and not args.no_semi_implicit and wl.n_species == 2:
        try:
            si = bench_semi_implicit(args, wl, dm, new_state)
        except Exception as e:  # reported, not required
            log(f"[bench] semi-implicit step failed: {e}")
        torch.cuda.empty_cache()
    if rank == 0 and not args.no_gmres:
        del st64, st32, st
        torch.cuda.empty_cache()
        gm = bench_gmres(args, peak)
        if not args.no_cpu_baseline:
            try:
                from oracle import ref
                if ref.available():
                    gm["cpu_baseline"] = gmres_cpu_baseline()
            except Exception as e:
                log(f"[bench] gmres cpu baseline failed: {e}")

    adj = None
    if rank == 0 and not args.no_adjoint:
        if args.no_gmres:
            del st64, st32, st
            torch.cuda.empty_cache()
        adj = bench_adjoint(args)
    ten = None
    if rank == 0 and not args.no_ten_ion:
        if args.no_gmres and args.no_adjoint:
            del st64, st32, st
        del dm
        torch.cuda.empty_cache()
        ten = bench_ten_ion(args, peak)

    if rank == 0:
        out = {"metric": METRIC, "value": rmx["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": rmx["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32/f64 mixed", "data": "synthetic",
               "config": {"workload": wl.name, "cells": h.n_cells, "faces": h.n_faces, "edges": h.n_edges,
                          "topology_hash": h.topology_hash(),
                          "n_species": wl.n_species, "global_cells": h.n_cells * world,
                          "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                          "dt": "CFL 0.4 on device", "l2": "inputs > L2 (no flush needed)",
                          "precision": "mixed: FP32 reconstruction/limiter/flux/EMF, FP64 state/Phi/CT",
                          "sources": "J x B force + Strang-split exact gyration" if wl.lorentz else "none"},
               "gpu_launches": rmx["launches"],
               "roofline": {"bound": "hbm", "kernel": rmx["kernel"], "achieved": rmx["achieved"], "peak": peak, "unit": "GB/s",
                            "frac": rmx["achieved"] / peak, "peak_kind": peak_kind,
                            "traffic": ncu_traffic(rmx["kernel"], "mixed", counts),
                            "algorithmic_bytes_per_launch": rmx["bytes_launch"]},
               "kernels": rmx["kernels"],
               "fp64": {"value": r64["value"], "ms_per_step": r64["ms"] / args.steps, "speedup_mixed": rmx["value"] / r64["value"],
                        "precision": "fp64 reference-exact", "kernels": r64["kernels"], "clocks": clocks64,
                        "roofline": {"kernel": r64["kernel"], "achieved": r64["achieved"], "frac": r64["achieved"] / peak}},
               "accuracy_mixed_vs_fp64": acc,
               "e2e": {"value": e2e_v, "unit": UNIT, "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes},
               "cpu_baseline": cpu, "clocks": clocks, "config1": c1, "gmres": gm, "semi_implicit": si, "adjoint": adj, "ten_ion": ten}
        out["summary"] = summary(out)
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
