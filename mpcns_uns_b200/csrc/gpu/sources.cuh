// Source terms of the two-ion model, FP64 in the reference's operation order (compiled with
// -fmad=false wherever they are used):
//   * mercury::add_sources_n (MercuryUns/fluid/MercurySources.cpp:20-63): the J x B force, the
//     electron-pressure (ambipolar) force and the chemistry terms of the external source fields;
//   * mercury::electron_pressure_gradient and the ambipolar edge EMF of mercury::AmbipolarEMF
//     (MercuryUns/physics/Ambipolar.cpp);
//   * the exact gyration of mercury::gyrate_n (MercuryUns/physics/Gyration.cpp), which the step
//     applies as half steps around the SSP-RK2 stages (Strang splitting, Solver.cpp:492-510).
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
    int ambi = 0, chem = 0;             // Config::ambipolar, Config::chemistry
    double pressure_coef = 0;           // Scales::pressure_coef
    double a1_Na = 0, a4 = 0, a5 = 0, a6 = 0, sch = 1, scn = 1, T_ref = 1, Tn0 = 0; // Scales, Config::chem.Tn0
    __host__ __device__ bool any() const { return on || ambi || chem; }
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

// add_sources_n for one owned fluid cell and species s (:29-60).  w: primitives of species s; rhoH,
// rhoNa: the primitive densities of the two ions; dpe (grad p_e), photo and vst: the cell's source
// field values, null where the field is absent.
//   S = inver_MA2 w_s (J x B) - w_s grad p_e;  rhs_m += S, rhs_E += u.S + dt |S|^2 / (2 rho);
//   chemistry: drag, temperature relaxation, thermal drift, Na+ production (legacy AddSourceToRHS_Fluid).
__device__ __forceinline__ void add_sources_cell(const SrcParams &p, int s, double rhoH, double rhoNa, const double *w, V3 J, V3 B,
                                                 const V3 *dpe, const double *photo, const double *vst, double dt, double *r)
{
    const NumInfo2 ni = numinfo2(p, rhoH, rhoNa);
    const double ns = s == 0 ? ni.nH : ni.nNa, ws = s == 0 ? ni.wH : ni.wNa;
    const double rho = dmax(w[0], 0.0);
    const V3 u = mk(w[1], w[2], w[3]);
    V3 S = mk(0, 0, 0);
    if (p.on) S = S + (p.inver_MA2 * ws) * cross(J, B);
    if (p.ambi && dpe) S = S - ws * *dpe;
    r[1] += S.x;
    r[2] += S.y;
    r[3] += S.z;
    r[4] += dot(u, S) + (rho > 1e-30 ? 0.5 * dt * dot(S, S) / rho : 0.0);
    if (p.chem && vst)
    {
        const double v = *vst, u2 = dot(u, u);
        const double Ts = w[4] / (rho > 0 ? rho : 1e-300) / (s == 0 ? p.sch : p.scn) * p.T_ref;
        const double Msum = p.mH + p.mNa;
        const double b1 = v * (p.Tn0 - Ts) * (s == 0 ? p.mH / Msum : 0.5);
        const double b2 = (s == 0 ? p.mNa / Msum : 0.5) * v;
        r[1] -= p.a4 * rho * u.x * v;
        r[2] -= p.a4 * rho * u.y * v;
        r[3] -= p.a4 * rho * u.z * v;
        r[4] -= p.a4 * rho * u2 * v;
        r[4] += p.a5 * ns * b1;
        r[4] += p.a4 * rho * u2 * b2;
        if (s == 1 && photo)
        {
            r[0] += p.a1_Na * *photo;
            r[4] += p.a6 * *photo * p.Tn0;
        }
    }
}

// mercury::electron_pressure_gradient (Ambipolar.cpp:10-31) of one owned fluid cell: Gauss' theorem with
// the face-averaged p_e (the mean with the fluid neighbour across an interior face, the cell's own value
// elsewhere).  pe(c) = p_H + p_Na.
template <class PE>
__device__ __forceinline__ V3 electron_pressure_gradient(const MeshView &m, int32_t c, PE pe)
{
    V3 sum = mk(0, 0, 0);
    const double pc = pe(c);
    for (int32_t k = m.c2f_ptr[c]; k < m.c2f_ptr[c + 1]; ++k)
    {
        const int32_t f = m.c2f_idx[k];
        double pf = pc;
        const int32_t b = m.f2c_ptr[f];
        if (m.f2c_ptr[f + 1] - b == 2)
        {
            const int32_t o = m.f2c_idx[b] == c ? m.f2c_idx[b + 1] : m.f2c_idx[b];
            if (m.material[o] == 0) pf = 0.5 * (pf + pe(o));
        }
        sum = sum + (pf * static_cast<double>(m.c2f_sgn[k])) * ld3(m.face_area, f);
    }
    const double iv = 1.0 / m.cell_volume[c];
    return mk(sum.x * iv, sum.y * iv, sum.z * iv);
}

// nodal p_e of AmbipolarEMF::add (Ambipolar.cpp:57-68): the volume-weighted mean over the node's fluid
// cells (ascending cell order); ok = the node has fluid cells
template <class PE>
__device__ __forceinline__ double node_pressure(const MeshView &m, int32_t v, PE pe, bool &ok)
{
    double s = 0, w = 0;
    const int32_t k0 = m.n2c_ptr[v], k1 = m.n2c_ptr[v + 1];
    for (int32_t k = k0; k < k1; ++k)
    {
        const int32_t c = m.n2c_cell[k];
        s += m.cell_volume[c] * pe(c);
        w += m.cell_volume[c];
    }
    ok = k1 > k0;
    return w > 0 ? s / w : 0.0;
}

// the ambipolar EMF of one owned edge (Ambipolar.cpp:69-87): returns false where the reference adds nothing.
// rho(c, s): primitive density of species s; pn, pok: nodal p_e and its flag
template <class RHO>
__device__ __forceinline__ bool ambipolar_edge(const MeshView &m, const SrcParams &p, int32_t e, RHO rho, const double *__restrict__ pn,
                                               const int8_t *__restrict__ pok, double &out)
{
    double rH = 0, rN = 0, wsum = 0;
    for (int32_t k = m.ec_ptr[e]; k < m.ec_ptr[e + 1]; ++k)
    {
        const int32_t c = m.ec_cell[k];
        if (m.material[c] == 1) continue;
        rH += m.ec_weight[k] * rho(c, 0);
        rN += m.ec_weight[k] * rho(c, 1);
        wsum += m.ec_weight[k];
    }
    if (wsum <= 0) return false;
    const NumInfo2 ni = numinfo2(p, rH / wsum, rN / wsum);
    const int32_t a = m.e_nodes[2 * (int64_t)e], b = m.e_nodes[2 * (int64_t)e + 1];
    if (!pok[a] || !pok[b]) return false;
    out = p.pressure_coef * (pn[b] - pn[a]) / ni.ne_eff;
    return true;
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

// inputs of the ambipolar edge EMF in the step's edge kernel (species-major SoA primitives)
struct AmbArgs
{
    int on = 0;
    SrcParams p;
    const double *W = nullptr; // W[(s*5 + q)*nc + c]
    const double *pn = nullptr;
    const int8_t *pok = nullptr;
};

// launchers (sources.cu)
// grad p_e (3 per cell) of species-major SoA primitives, zero outside the owned fluid cells
void launch_dpe(const MeshView &m, const double *W, double *dpe, cudaStream_t s);
// nodal p_e and its flag of species-major SoA primitives
void launch_node_pressure(const MeshView &m, const double *W, double *pn, int8_t *pok, cudaStream_t s);
// gyrate_n on the owned fluid cells of species 0 and 1 of a species-major SoA state U (5 per cell and
// species, [(s*5 + m)*nc + c]); the field is B3 (3 doubles per cell) or, if null, B4 (float4 per cell);
// the angle uses scale * (*dtp).
void launch_gyrate(const MeshView &m, const SrcParams &p, const double *B3, const float4 *B4, const double *dtp, double scale,
                   double *U, cudaStream_t s, const Reprepare &rp = Reprepare{});
// mhd::cell_current (induction.cu)
void launch_cell_current(const MeshView &m, const double *B, double *J, cudaStream_t s);
} // namespace mhd
