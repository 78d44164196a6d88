// Source terms of the two-ion model, FP64 in the reference's operation order (compiled with
// -fmad=false wherever they are used):
//   * the J x B force of mercury::add_sources_n (MercuryUns/fluid/MercurySources.cpp:20-63);
//   * the exact gyration of mercury::gyrate_n (MercuryUns/physics/Gyration.cpp), which the step
//     applies as half steps around the SSP-RK2 stages (Strang splitting, Solver.cpp:492-510).
// Chemistry and the ambipolar terms of add_sources_n need external source fields and are not here.
#pragma once
#include "fluid.cuh"

namespace mhd
{
struct SrcParams
{
    int on = 0;                         // Config::lorentz_force
    double inver_MA2 = 1, induce = 0;   // Scales::inver_MA2, Scales::induce_coeff
    double M_ref = 1, mH = 1, mNa = 23; // Scales::M_ref, M_H, M_Na
    double ne_floor = 0.01;             // Scales::ne_floor
    double gamma = 5.0 / 3.0, rho_floor = 1e-10, p_floor = 1e-12;
};

struct NumInfo2
{
    double nH, nNa, ne, ne_eff, chiH, chiNa, wH, wNa;
};

// mhd::Scales::numinfo (Common/physics/Scales.cpp:50-62)
__device__ __forceinline__ NumInfo2 numinfo2(const SrcParams &p, double rhoH, double rhoNa)
{
    NumInfo2 n;
    n.nH = dmax(rhoH, 0.0) / p.mH * p.M_ref;
    n.nNa = dmax(rhoNa, 0.0) / p.mNa * p.M_ref;
    n.ne = n.nH + n.nNa;
    n.ne_eff = sqrt(n.ne * n.ne + p.ne_floor * p.ne_floor);
    if (n.ne > 1e-300)
    {
        n.chiH = n.nH / n.ne;
        n.chiNa = n.nNa / n.ne;
    }
    else
    {
        n.chiH = 1.0;
        n.chiNa = 0.0;
    }
    n.wH = n.nH / n.ne_eff;
    n.wNa = n.nNa / n.ne_eff;
    return n;
}

// add_sources_n for one owned fluid cell and species s (:29-47): S = inver_MA2 w_s (J x B),
// rhs_m += S, rhs_E += u.S + dt |S|^2 / (2 rho).  w: primitives of species s; rhoH, rhoNa: the
// primitive densities of the two ions.
__device__ __forceinline__ void lorentz_source(const SrcParams &p, int s, double rhoH, double rhoNa, const double *w, V3 J, V3 B,
                                               double dt, double *r)
{
    const NumInfo2 ni = numinfo2(p, rhoH, rhoNa);
    const double ws = s == 0 ? ni.wH : ni.wNa;
    const double rho = dmax(w[0], 0.0);
    const V3 u = mk(w[1], w[2], w[3]);
    V3 S = mk(0, 0, 0);
    if (p.on) S = S + (p.inver_MA2 * ws) * cross(J, B);
    r[1] += S.x;
    r[2] += S.y;
    r[3] += S.z;
    r[4] += dot(u, S) + (rho > 1e-30 ? 0.5 * dt * dot(S, S) / rho : 0.0);
}

// gyrate_n for one owned fluid cell: the relative velocity w = u_H - u_Na turns by
// th = (a_H chi_Na + a_Na chi_H) |B| dt about B; the ions share the change as f_H, -f_Na; the
// kinetic-energy change goes to the total energy.  uh, un: conservative states, updated in place.
__device__ __forceinline__ void gyrate_cell(const SrcParams &p, V3 b, double dt, double *uh, double *un)
{
    const double aH = p.induce * p.M_ref / p.mH, aN = p.induce * p.M_ref / p.mNa;
    const Prim5 wh = to_prim(uh[0], uh[1], uh[2], uh[3], uh[4], p.gamma, p.rho_floor, p.p_floor);
    const Prim5 wn = to_prim(un[0], un[1], un[2], un[3], un[4], p.gamma, p.rho_floor, p.p_floor);
    const NumInfo2 ni = numinfo2(p, uh[0], un[0]);
    const double bm = sqrt(dot(b, b));
    const double denom = aH * ni.chiNa + aN * ni.chiH;
    if (bm <= 0 || denom <= 0) return;
    const V3 bh = (1.0 / bm) * b;
    const V3 uH = mk(wh.u, wh.v, wh.w), uN = mk(wn.u, wn.v, wn.w);
    const V3 w = uH - uN;
    const V3 wpar = dot(w, bh) * bh, wperp = w - wpar;
    const double th = denom * bm * dt;
    const V3 dw = (cos(th) - 1.0) * wperp + sin(th) * cross(wperp, bh);
    const double fH = aH * ni.chiNa / denom, fN = aN * ni.chiH / denom;
    const V3 dH = fH * dw, dN = (-fN) * dw;
    const V3 uH2 = uH + dH, uN2 = uN + dN;
    double rho = uh[0];
    uh[1] = rho * uH2.x;
    uh[2] = rho * uH2.y;
    uh[3] = rho * uH2.z;
    uh[4] += 0.5 * rho * (dot(uH2, uH2) - dot(uH, uH));
    rho = un[0];
    un[1] = rho * uN2.x;
    un[2] = rho * uN2.y;
    un[3] = rho * uN2.z;
    un[4] += 0.5 * rho * (dot(uN2, uN2) - dot(uN, uN));
}

// Per-cell part of Solver::prepare (Solver.cpp:101-118): primitives of every species and the
// charge-weighted ion velocity u+ (mhd::Scales::numinfo generalised to n species; the number
// densities are recomputed from the primitives just written)
__device__ __forceinline__ void prepare_prims(const FluidParams &p, const double *__restrict__ mass, double M_ref, SField<const double> U,
                                              SField<double> W, int32_t c, bool fluid, double *u)
{
    double ne = 0;
    for (int s = 0; s < p.nsp; ++s)
    {
        const Prim5 w = to_prim(U(s, c, 0), U(s, c, 1), U(s, c, 2), U(s, c, 3), U(s, c, 4), p.gamma, p.rho_floor, p.p_floor);
        W(s, c, 0) = w.rho; W(s, c, 1) = w.u; W(s, c, 2) = w.v; W(s, c, 3) = w.w; W(s, c, 4) = w.p;
        ne += dmax(w.rho, 0.0) / mass[s] * M_ref;
    }
    u[0] = u[1] = u[2] = 0;
    if (fluid)
        for (int s = 0; s < p.nsp; ++s)
        {
            const double ns = dmax(W(s, c, 0), 0.0) / mass[s] * M_ref;
            const double chi = ne > 1e-300 ? ns / ne : (s == 0 ? 1.0 : 0.0);
            for (int a = 0; a < 3; ++a) u[a] += chi * W(s, c, 1 + a);
        }
}

// After the opening half-step gyration the next prepare would only renew what the gyration changed:
// the primitives and u+ (B_ind, B_tot and J depend on Phi alone).  With on, the gyration kernel writes
// them for the cells it turns, so that stage 1 needs no prepare pass.
struct Reprepare
{
    int on = 0;
    FluidParams fp;
    const double *mass = nullptr;
    double M_ref = 1;
    SField<const double> U;
    SField<double> W;
    double *up = nullptr;
};

// the source parameters of a step's parameters (species 0 and 1 are the model's H+ and Na+)
SrcParams src_params(const MhdStepParams &q);

// launchers (sources.cu)
// gyrate_n on the owned fluid cells of species 0 and 1 of a species-major SoA state U (5 per cell and
// species, [(s*5 + m)*nc + c]); the field is B3 (3 doubles per cell) or, if null, B4 (float4 per cell);
// the angle uses scale * (*dtp).
void launch_gyrate(const MeshView &m, const SrcParams &p, const double *B3, const float4 *B4, const double *dtp, double scale,
                   double *U, cudaStream_t s, const Reprepare &rp = Reprepare{});
// mhd::cell_current (induction.cu)
void launch_cell_current(const MeshView &m, const double *B, double *J, cudaStream_t s);
} // namespace mhd
