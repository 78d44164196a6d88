// nvcc-flags: -fmad=false
// Magnetic-field side of the explicit step on the device: cell-field reconstruction, the ideal
// UCT edge EMF, boundary edge values, constrained transport (FP64) and the div B diagnostic.
// FP64, reference-exact (see fluid.cu): no multiply-add contraction, reference operation order.
#include <cfloat>
#include <mutex>
#include <vector>

#include "induction.cuh"
#include "kernels.cuh"

namespace mhd
{
__global__ void k_cell_vector(MeshView m, const double *__restrict__ flux, int32_t ncells, double *__restrict__ out)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    st3(out, c, cell_vector(m, flux, c));
}

// Face candidate of mhd::add_ideal_emf (Common/induction/IdealEMF.cpp:32-55):
// E_f = -n x [ 1/2 (F_L + F_R) - 1/2 a_f (B_R^ind - B_L^ind) ],  F_X = (u_X.n) B_X^tot - u_X B_n^tot
// phi_add (optional): static background flux, phi_tot = phi + phi_add as in Solver::prepare (Solver.cpp:119)
// pa (optional): phi_tot / |A| per face (phi_tot before phi_add is added: the induced flux that the edge pass
// divides by |A|, the same quotient).  sw (optional): the switch log of the face's choice of a_f (which side's
// |u . n| is the larger, and the sign of u . n there), one running hash per face.
__global__ void k_face_candidate(MeshView m, const double *__restrict__ u, const double *__restrict__ Bt, const double *__restrict__ Bi,
                                 const double *__restrict__ phi_tot, const double *__restrict__ phi_add, double *__restrict__ Ef,
                                 double *__restrict__ pa, uint32_t *__restrict__ sw)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    const double A = m.face_area_mag[f];
    if (pa) pa[f] = phi_tot[f] / A;
    const V3 n = (1.0 / A) * ld3(m.face_area, f);
    const double pt = phi_add ? phi_tot[f] + phi_add[f] : phi_tot[f];
    const double Bn = pt / A;
    auto flux = [&](int32_t c) {
        const V3 uc = ld3(u, c);
        return dot(uc, n) * ld3(Bt, c) - Bn * uc;
    };
    const int32_t p0 = m.f2c_ptr[f], cnt = m.f2c_ptr[f + 1] - p0;
    V3 F;
    if (cnt == 2)
    {
        const int32_t L = m.face_L[f], R = m.face_R[f];
        const double a = dmax(fabs(dot(ld3(u, L), n)), fabs(dot(ld3(u, R), n)));
        F = 0.5 * (flux(L) + flux(R)) - (0.5 * a) * (ld3(Bi, R) - ld3(Bi, L));
        if (sw)
        {
            const double dL = dot(ld3(u, L), n), dR = dot(ld3(u, R), n);
            const bool r = fabs(dL) < fabs(dR);
            sw[f] = sw_step(sw[f], (r ? 1u : 0u) | ((r ? dR : dL) < 0.0 ? 2u : 0u));
        }
    }
    else
        F = flux(m.f2c_idx[p0]);
    st3(Ef, f, -1.0 * cross(n, F));
}

// Edge loop of mhd::add_ideal_emf (Common/induction/IdealEMF.cpp:59-128), one thread per owned
// edge: central part sum_f w_ef E_f . t, transverse upwind part with the weights omega corrected
// by the 2x2 solve in the plane normal to the edge.
// Returns false for the edges the reference skips (no faces, zero length, no fluid cell).
// MAXV bounds the faces per edge: the per-face values live in registers when the loops over
// [0, MAXV) unroll (MAXV = 8 covers every tetrahedral split mesh), in local memory for MAXV = 32.
// LOG: code receives the switch-log hash of the edge's choices: per face the slot of the cell with the
// largest |u . m| and the sign of u . m there, and whether the 2x2 solve ran.
template <int MAXV, bool LOG = false>
__device__ __forceinline__ bool edge_uct(const MeshView &m, int32_t e, const double *__restrict__ Ef, const double *__restrict__ u,
                                         const double *__restrict__ phi_ind, double cuct, double &out, uint32_t *code = nullptr)
{
    const int32_t f0 = m.e2f_ptr[e], nf = m.e2f_ptr[e + 1] - f0;
    const double L = m.edge_len[e];
    if (nf == 0 || L <= 0) return false;
    const int32_t q0 = m.ec_ptr[e], q1 = m.ec_ptr[e + 1];
    bool any_fluid = false;
    for (int32_t k = q0; k < q1 && !any_fluid; ++k) any_fluid = m.material[m.ec_cell[k]] == 0;
    if (!any_fluid) return false;
    const V3 t = ld3(m.edge_vec, e);
    const V3 th = (1.0 / L) * t;
    const V3 mid = ld3(m.edge_mid, e);
    // plane basis (IdealEMF.cpp:14-20)
    const V3 ax = fabs(th.x) < 0.9 ? mk(1, 0, 0) : mk(0, 1, 0);
    V3 e1 = cross(th, ax);
    e1 = (1.0 / sqrt(dot(e1, e1))) * e1;
    const V3 e2 = cross(th, e1);
    double w[MAXV], aef[MAXV], sg[MAXV], qa[MAXV], qb[MAXV];
    double Ec = 0, M11 = 0, M12 = 0, M22 = 0, g1 = 0, g2 = 0;
#pragma unroll
    for (int i = 0; i < MAXV; ++i)
    {
        if (i >= nf) break;
        const int32_t f = m.e2f_idx[f0 + i];
        w[i] = m.ef_weight[f0 + i];
        Ec += w[i] * dot(ld3(Ef, f), t);
        V3 v = ld3(m.face_center, f) - mid;
        v = v - dot(v, th) * th;
        const double nv = sqrt(dot(v, v));
        const V3 mi = nv > 0 ? (1.0 / nv) * v : mk(0, 0, 0);
        const V3 nrm = (1.0 / m.face_area_mag[f]) * ld3(m.face_area, f);
        double a = 0;
        if (LOG)
        {
            int ka = 31;
            bool neg = false;
            for (int32_t k = q0; k < q1; ++k)
            {
                const double d = dot(ld3(u, m.ec_cell[k]), mi);
                if (a < fabs(d))
                {
                    ka = k - q0;
                    neg = d < 0;
                }
                a = dmax(a, fabs(d));
            }
            *code = sw_step(*code, uint32_t(ka & 31) | (neg ? 32u : 0u));
        }
        else
            for (int32_t k = q0; k < q1; ++k) a = dmax(a, fabs(dot(ld3(u, m.ec_cell[k]), mi)));
        aef[i] = a;
        sg[i] = dot(th, cross(mi, nrm));
        const V3 qv = (a * sg[i]) * nrm;
        qa[i] = dot(qv, e1);
        qb[i] = dot(qv, e2);
        M11 += w[i] * qa[i] * qa[i];
        M12 += w[i] * qa[i] * qb[i];
        M22 += w[i] * qb[i] * qb[i];
        g1 += w[i] * qa[i];
        g2 += w[i] * qb[i];
    }
    const double tr = M11 + M22;
    const double eps = 1e-14 * tr;
    const double det = (M11 + eps) * (M22 + eps) - M12 * M12;
    double l1 = 0, l2 = 0;
    if (LOG) *code = sw_step(*code, tr > 0 && det > 0 ? 64u : 128u);
    if (tr > 0 && det > 0)
    {
        l1 = ((M22 + eps) * g1 - M12 * g2) / det;
        l2 = ((M11 + eps) * g2 - M12 * g1) / det;
    }
    double Eu = 0;
#pragma unroll
    for (int i = 0; i < MAXV; ++i)
    {
        if (i >= nf) break;
        const int32_t f = m.e2f_idx[f0 + i];
        const double omega = w[i] * (1.0 - (qa[i] * l1 + qb[i] * l2));
        Eu += omega * aef[i] * sg[i] * (phi_ind[f] / m.face_area_mag[f]);
    }
    out = Ec + 2.0 * cuct * L * Eu;
    return true;
}

// The geometry of edge_uct's face loop, once per (edge e, slot i < 8 of its e2f row), formed by the same
// operations in the same order: the face's unit in-plane direction m away from the edge, its unit normal n,
// sigma = t.(m x n) and the weight w_ef, component c (m.x m.y m.z n.x n.y n.z sigma w) of slot i at
// geo[(8 * c + i) * ne + e], so that a warp's edges read each component of a slot as consecutive words.
// Slots past an edge's row and edges that edge_uct skips (no faces, zero length, more than 8 faces) are
// left unset and never read.
constexpr int kGeoSlots = 8;
__global__ void k_edge_face_geo(MeshView m, double *__restrict__ geo)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    const int32_t f0 = m.e2f_ptr[e], nf = m.e2f_ptr[e + 1] - f0;
    const double L = m.edge_len[e];
    if (nf == 0 || nf > kGeoSlots || L <= 0) return;
    const int64_t ne = m.ne;
    const V3 t = ld3(m.edge_vec, e);
    const V3 th = (1.0 / L) * t;
    const V3 mid = ld3(m.edge_mid, e);
    for (int32_t i = 0; i < nf; ++i)
    {
        const int32_t f = m.e2f_idx[f0 + i];
        V3 v = ld3(m.face_center, f) - mid;
        v = v - dot(v, th) * th;
        const double nv = sqrt(dot(v, v));
        const V3 mi = nv > 0 ? (1.0 / nv) * v : mk(0, 0, 0);
        const V3 nrm = (1.0 / m.face_area_mag[f]) * ld3(m.face_area, f);
        const double c8[8] = {mi.x, mi.y, mi.z, nrm.x, nrm.y, nrm.z, dot(th, cross(mi, nrm)), m.ef_weight[f0 + i]};
        for (int c = 0; c < 8; ++c) geo[(8 * c + i) * ne + e] = c8[c];
    }
}

void build_edge_face_geo(const MeshView &m, double *geo, cudaStream_t s)
{
    if (!m.ne) return;
    k_edge_face_geo<<<grid_for(m.ne, 128), 128, 0, s>>>(m, geo);
    MHD_LAUNCH_CHECK();
}

// edge_uct from the per-slot geometry table, for edges of at most kGeoCells cells and kGeoSlots faces: the
// cells' velocities are staged once in this thread's column of shared memory (su[(3 * k + a) * 128 + lane]),
// and the face loop runs twice, the second pass forming each face's upwind terms again from the table instead of
// holding them, so that no per-face array lives in registers.  Every value and every sum is formed by
// the operations of edge_uct in its order: the results are the same bits.
constexpr int kGeoCells = 8;
// pa: phi_ind / |A| per face (k_face_candidate's pa)
template <bool LOG>
__device__ __forceinline__ bool edge_uct_geo(const MeshView &m, int32_t e, const double *__restrict__ Ef, const double *__restrict__ u,
                                             const double *__restrict__ pa, double cuct, const double *__restrict__ geo,
                                             double *__restrict__ su, double &out, uint32_t *code)
{
    const int32_t f0 = m.e2f_ptr[e], nf = m.e2f_ptr[e + 1] - f0;
    const double L = m.edge_len[e];
    if (nf == 0 || L <= 0) return false;
    const int32_t q0 = m.ec_ptr[e], q1 = m.ec_ptr[e + 1];
    bool any_fluid = false;
    for (int32_t k = q0; k < q1 && !any_fluid; ++k) any_fluid = m.material[m.ec_cell[k]] == 0;
    if (!any_fluid) return false;
    const int nce = q1 - q0;
    // unrolled over the bound so that every cell's id and velocity loads are in flight together
#pragma unroll
    for (int k = 0; k < kGeoCells; ++k)
        if (k < nce)
        {
            const V3 uk = ld3(u, m.ec_cell[q0 + k]);
            su[(3 * k) * 128] = uk.x;
            su[(3 * k + 1) * 128] = uk.y;
            su[(3 * k + 2) * 128] = uk.z;
        }
    const V3 t = ld3(m.edge_vec, e);
    const V3 th = (1.0 / L) * t;
    // plane basis (IdealEMF.cpp:14-20)
    const V3 ax = fabs(th.x) < 0.9 ? mk(1, 0, 0) : mk(0, 1, 0);
    V3 e1 = cross(th, ax);
    e1 = (1.0 / sqrt(dot(e1, e1))) * e1;
    const V3 e2 = cross(th, e1);
    // the face's largest |u . m| over the edge's cells (and, logged, which cell and its sign)
    auto a_ef = [&](V3 mi) {
        double a = 0;
        int ka = 31;
        bool neg = false;
#pragma unroll
        for (int k = 0; k < kGeoCells; ++k)
        {
            if (k >= nce) break;
            const double d = dot(mk(su[(3 * k) * 128], su[(3 * k + 1) * 128], su[(3 * k + 2) * 128]), mi);
            if (LOG && a < fabs(d))
            {
                ka = k;
                neg = d < 0;
            }
            a = dmax(a, fabs(d));
        }
        if (LOG) *code = sw_step(*code, uint32_t(ka & 31) | (neg ? 32u : 0u));
        return a;
    };
    struct Face
    {
        V3 mi, nrm;
        double sg, w;
    };
    const int64_t ne = m.ne;
    auto face = [&](int32_t i) {
        const double *g = geo + i * ne + e;
        return Face{mk(g[0], g[8 * ne], g[16 * ne]), mk(g[24 * ne], g[32 * ne], g[40 * ne]), g[48 * ne], g[56 * ne]};
    };
    double Ec = 0, M11 = 0, M12 = 0, M22 = 0, g1 = 0, g2 = 0;
    // the face ids of the row, loaded together
    int32_t fid[kGeoSlots];
#pragma unroll
    for (int i = 0; i < kGeoSlots; ++i) fid[i] = i < nf ? m.e2f_idx[f0 + i] : 0;
#pragma unroll
    for (int32_t i = 0; i < kGeoSlots; ++i)
    {
        if (i >= nf) break;
        const int32_t f = fid[i];
        const Face F = face(i);
        Ec += F.w * dot(ld3(Ef, f), t);
        const double a = a_ef(F.mi);
        const V3 qv = (a * F.sg) * F.nrm;
        const double qa = dot(qv, e1), qb = dot(qv, e2);
        M11 += F.w * qa * qa;
        M12 += F.w * qa * qb;
        M22 += F.w * qb * qb;
        g1 += F.w * qa;
        g2 += F.w * qb;
    }
    const double tr = M11 + M22;
    const double eps = 1e-14 * tr;
    const double det = (M11 + eps) * (M22 + eps) - M12 * M12;
    double l1 = 0, l2 = 0;
    if (LOG) *code = sw_step(*code, tr > 0 && det > 0 ? 64u : 128u);
    if (tr > 0 && det > 0)
    {
        l1 = ((M22 + eps) * g1 - M12 * g2) / det;
        l2 = ((M11 + eps) * g2 - M12 * g1) / det;
    }
    double Eu = 0;
#pragma unroll
    for (int32_t i = 0; i < kGeoSlots; ++i)
    {
        if (i >= nf) break;
        const int32_t f = fid[i];
        const Face F = face(i);
        double a = 0;
#pragma unroll
        for (int k = 0; k < kGeoCells; ++k)
        {
            if (k >= nce) break;
            a = dmax(a, fabs(dot(mk(su[(3 * k) * 128], su[(3 * k + 1) * 128], su[(3 * k + 2) * 128]), F.mi)));
        }
        const V3 qv = (a * F.sg) * F.nrm;
        const double qa = dot(qv, e1), qb = dot(qv, e2);
        const double omega = F.w * (1.0 - (qa * l1 + qb * l2));
        Eu += omega * a * F.sg * pa[f];
    }
    out = Ec + 2.0 * cuct * L * Eu;
    return true;
}

template <int MAXV>
__global__ void __launch_bounds__(128) k_edge_uct(MeshView m, const double *__restrict__ Ef, const double *__restrict__ u,
                                                   const double *__restrict__ phi_ind, double cuct, double *__restrict__ E)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.no_edges) return;
    double v;
    if (edge_uct<MAXV>(m, e, Ef, u, phi_ind, cuct, v)) E[e] += v;
}

// EdgeEMF::begin (zero) + add_ideal_emf + the boundary edge values of Solver::rhs (Solver.cpp:150-167).
// Wall and inflow edges are overwritten by the reference, so their UCT value is not evaluated.
// With mres, the explicit resistive EMF m_e (d1^T star2 Phi)_e is added on every owned edge: the resistive
// part of ImplicitInduction::apply_F (ImplicitInduction.cpp:133-137) with its sum m p0 + p1 + p2 (:182), the
// faces of an edge in ascending order (the e2f rows), as the reference's face loop scatters them.
// GEO: the UCT value from the per-entry geometry table (edge_uct_geo; edges of at most kGeoCells cells)
template <int MAXV, bool LOG, bool GEO>
__global__ void __launch_bounds__(128, GEO ? 6 : 4) k_edge_emf_assign(MeshView m, const double *__restrict__ Ef, const double *__restrict__ u,
                                                                    const double *__restrict__ phi_ind, double cuct, V3 E_inf,
                                                                    const double *__restrict__ mres, AmbArgs amb, double *__restrict__ E,
                                                                    uint32_t *__restrict__ sw, const double *__restrict__ geo,
                                                                    const double *__restrict__ pa)
{
    __shared__ double su[GEO ? 3 * kGeoCells * 128 : 1];
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    double val = 0.0;
    if (e < m.no_edges)
    {
        const int mode = m.edge_mode[e];
        if (mode == 1) val = 0.0;
        else if (mode == 2) val = dot(E_inf, ld3(m.edge_vec, e));
        else
        {
            double v;
            uint32_t code = 0;
            bool ok;
            if constexpr (GEO) ok = edge_uct_geo<LOG>(m, e, Ef, u, pa, cuct, geo, su + threadIdx.x, v, &code);
            else ok = edge_uct<MAXV, LOG>(m, e, Ef, u, phi_ind, cuct, v, &code);
            if (ok) val += v;
            if (LOG) sw_log(sw, e, code);
            // AmbipolarEMF::add (Ambipolar.cpp:69-87) after the ideal EMF; on wall and inflow edges the
            // reference overwrites it with the boundary value
            if (amb.on)
            {
                const int64_t nc = m.nc;
                if (ambipolar_edge(m, amb.p, e, [&](int32_t c, int s) { return amb.W[(s * 5) * nc + c]; }, amb.pn, amb.pok, v)) val -= v;
            }
        }
        if (mres) val += mres[e] * resistive_p0(m, phi_ind, e) + 0.0 + 0.0;
    }
    E[e] = val;
}

void launch_face_candidate(const MeshView &m, const double *u, const double *Bt, const double *Bi, const double *phi_tot,
                           const double *phi_add, double *Ef, cudaStream_t s, double *pa, uint32_t *sw)
{
    if (!m.nf) return;
    k_face_candidate<<<grid_for(m.nf, 128), 128, 0, s>>>(m, u, Bt, Bi, phi_tot, phi_add, Ef, pa, sw);
    MHD_LAUNCH_CHECK();
}

void launch_edge_emf_assign(const MeshView &m, const double *Ef, const double *u, const double *phi_ind, double cuct, V3 E_inf,
                            double *E, cudaStream_t s, const double *mres, const AmbArgs &amb, uint32_t *sw, const double *geo,
                            const double *pa)
{
    if (!m.ne) return;
    const int g = grid_for(m.ne, 128);
    if (geo && pa && m.max_edge_cells <= kGeoCells && m.max_valence <= kGeoSlots)
        (sw ? k_edge_emf_assign<8, true, true> : k_edge_emf_assign<8, false, true>)<<<g, 128, 0, s>>>(m, Ef, u, phi_ind, cuct, E_inf, mres,
                                                                                                      amb, E, sw, geo, pa);
    else if (m.max_valence <= 8)
        (sw ? k_edge_emf_assign<8, true, false> : k_edge_emf_assign<8, false, false>)<<<g, 128, 0, s>>>(m, Ef, u, phi_ind, cuct, E_inf, mres,
                                                                                                        amb, E, sw, nullptr, nullptr);
    else
        (sw ? k_edge_emf_assign<kMaxValence, true, false>
            : k_edge_emf_assign<kMaxValence, false, false>)<<<g, 128, 0, s>>>(m, Ef, u, phi_ind, cuct, E_inf, mres, amb, E, sw, nullptr,
                                                                               nullptr);
    MHD_LAUNCH_CHECK();
}

// Boundary edge values of mercury::Solver::rhs (MercuryUns/driver/Solver.cpp:162-167)
__global__ void k_edge_modes(MeshView m, V3 E_inf, double *__restrict__ E)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.no_edges) return;
    const int mode = m.edge_mode[e];
    if (mode == 1) E[e] = 0.0;
    else if (mode == 2) E[e] = dot(E_inf, ld3(m.edge_vec, e));
}

// mhd::faraday_update (Common/induction/Faraday.cpp:15-24) over mhd::active_faces (:7-13), FP64
__global__ void k_faraday(MeshView m, const double *__restrict__ E, const double *__restrict__ dt_edge, double dt, double *__restrict__ B)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    bool active = false;
    for (int32_t k = m.f2c_ptr[f]; k < m.f2c_ptr[f + 1]; ++k) active |= m.f2c_idx[k] < m.no_cells;
    if (!active) return;
    double circ = 0.0;
    if (dt_edge)
    {
        for (int32_t k = m.f2e_ptr[f]; k < m.f2e_ptr[f + 1]; ++k)
        {
            const int32_t e = m.f2e_idx[k];
            circ += m.f2e_sgn[k] * dt_edge[e] * E[e];
        }
        B[f] -= circ;
    }
    else
    {
        for (int32_t k = m.f2e_ptr[f]; k < m.f2e_ptr[f + 1]; ++k) circ += m.f2e_sgn[k] * E[m.f2e_idx[k]];
        B[f] -= dt * circ;
    }
}

// mhd::div_b (Common/diagnostics/DivB.cpp:8-24): block partial (max |s|, its cell, max rel)
struct DivPart
{
    double max_abs, worst, max_rel;
};
__device__ __forceinline__ void div_combine(DivPart &a, const DivPart &b)
{
    // the reference keeps the first cell (lowest id) reaching the maximum
    if (b.max_abs > a.max_abs || (b.max_abs == a.max_abs && b.worst >= 0 && (a.worst < 0 || b.worst < a.worst)))
    {
        a.max_abs = b.max_abs;
        a.worst = b.worst;
    }
    a.max_rel = dmax(a.max_rel, b.max_rel);
}
__device__ __forceinline__ DivPart div_block_reduce(DivPart v)
{
    __shared__ DivPart sh[32];
    for (int o = 16; o > 0; o >>= 1)
    {
        DivPart w{__shfl_down_sync(0xffffffffu, v.max_abs, o), __shfl_down_sync(0xffffffffu, v.worst, o),
                  __shfl_down_sync(0xffffffffu, v.max_rel, o)};
        div_combine(v, w);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0)
    {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : DivPart{0.0, -1.0, 0.0};
        for (int o = 16; o > 0; o >>= 1)
        {
            DivPart w{__shfl_down_sync(0xffffffffu, v.max_abs, o), __shfl_down_sync(0xffffffffu, v.worst, o),
                      __shfl_down_sync(0xffffffffu, v.max_rel, o)};
            div_combine(v, w);
        }
    }
    return v;
}

__global__ void __launch_bounds__(256) k_div_b_partial(MeshView m, const double *__restrict__ B, const double *__restrict__ extra,
                                                        DivPart *__restrict__ part)
{
    DivPart v{0.0, -1.0, 0.0};
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < m.no_cells; c += gridDim.x * blockDim.x)
    {
        double s = 0, a = 0;
        for (int32_t k = m.c2f_ptr[c]; k < m.c2f_ptr[c + 1]; ++k)
        {
            const int32_t f = m.c2f_idx[k];
            s += m.c2f_sgn[k] * B[f];
            a += fabs(B[f]) + (extra ? fabs(extra[f]) : 0.0);
        }
        const double rel = a > 0 ? fabs(s) / a : 0.0;
        div_combine(v, DivPart{fabs(s), fabs(s) > 0 ? double(c) : -1.0, rel});
    }
    v = div_block_reduce(v);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
}

__global__ void __launch_bounds__(1024) k_div_b_final(const DivPart *__restrict__ part, int n, double *__restrict__ out)
{
    DivPart v{0.0, -1.0, 0.0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) div_combine(v, part[i]);
    v = div_block_reduce(v);
    if (threadIdx.x == 0)
    {
        out[0] = v.max_abs;
        out[1] = v.max_rel;
        out[2] = v.worst;
    }
}

// mhd::cell_current (Common/induction/Current.cpp:9-31)
__global__ void k_cell_current(MeshView m, const double *__restrict__ B, double *__restrict__ J)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    if (c >= m.no_cells)
    {
        st3(J, c, mk(0, 0, 0));
        return;
    }
    const V3 bc = ld3(B, c);
    V3 sum = mk(0, 0, 0);
    for (int32_t k = m.c2f_ptr[c]; k < m.c2f_ptr[c + 1]; ++k)
    {
        const int32_t f = m.c2f_idx[k];
        V3 bf = bc;
        const int32_t p0 = m.f2c_ptr[f];
        if (m.f2c_ptr[f + 1] - p0 == 2)
        {
            const int32_t o = m.f2c_idx[p0] == c ? m.f2c_idx[p0 + 1] : m.f2c_idx[p0];
            bf = 0.5 * (bc + ld3(B, o));
        }
        sum = sum + cross(double(m.c2f_sgn[k]) * ld3(m.face_area, f), bf);
    }
    const double invV = 1.0 / m.cell_volume[c];
    st3(J, c, mk(sum.x * invV, sum.y * invV, sum.z * invV));
}

int div_b_blocks(const MeshView &m) { return static_cast<int>(std::min<int64_t>(grid_for(m.no_cells, 256), 4 * 148)); }

// ---------------------------------------------------------------- div B without allocation
// Static scratch of mhd_gpu_div_b_noalloc: MHD_NOALLOC_DIVB_MAX_BLOCKS block partials, then the
// 3-value result.  Host code must not take this name as a device address: the address comes from
// cudaGetSymbolAddress (noalloc_scratch below), per device.
constexpr int kNoAllocCellsPerBlock = 1024; // 256 threads x 4 cells
static __device__ __align__(256) double g_divb_scratch[3 * MHD_NOALLOC_DIVB_MAX_BLOCKS + 4];

// one partial per block of 1024 consecutive owned cells (no grid-stride: the block count is the
// scratch index, bounded by the mesh-size check of the entry point)
__global__ void __launch_bounds__(256) k_div_b_block(MeshView m, const double *__restrict__ B, const double *__restrict__ extra,
                                                      DivPart *__restrict__ part)
{
    DivPart v{0.0, -1.0, 0.0};
    const int64_t base = (int64_t)blockIdx.x * kNoAllocCellsPerBlock;
    for (int i = 0; i < kNoAllocCellsPerBlock / 256; ++i)
    {
        const int64_t cc = base + i * 256 + threadIdx.x;
        if (cc >= m.no_cells) break;
        const int32_t c = static_cast<int32_t>(cc);
        double s = 0, a = 0;
        for (int32_t k = m.c2f_ptr[c]; k < m.c2f_ptr[c + 1]; ++k)
        {
            const int32_t f = m.c2f_idx[k];
            s += m.c2f_sgn[k] * B[f];
            a += fabs(B[f]) + (extra ? fabs(extra[f]) : 0.0);
        }
        const double rel = a > 0 ? fabs(s) / a : 0.0;
        div_combine(v, DivPart{fabs(s), fabs(s) > 0 ? double(c) : -1.0, rel});
    }
    v = div_block_reduce(v);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// Device address of g_divb_scratch on the current device, looked up once per device.
double *noalloc_scratch()
{
    static std::mutex mu;
    static std::vector<double *> addr;
    int dev = 0;
    MHD_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (static_cast<int>(addr.size()) <= dev) addr.resize(dev + 1, nullptr);
    if (!addr[dev])
    {
        void *p = nullptr;
        MHD_CUDA(cudaGetSymbolAddress(&p, g_divb_scratch));
        addr[dev] = static_cast<double *>(p);
    }
    return addr[dev];
}

void launch_cell_current(const MeshView &m, const double *B, double *J, cudaStream_t s)
{
    if (!m.nc) return;
    k_cell_current<<<grid_for(m.nc, 128), 128, 0, s>>>(m, B, J);
    MHD_LAUNCH_CHECK();
}

void ideal_emf_enqueue(const MeshView &m, const double *u, const double *Bt, const double *Bi, const double *phi_tot,
                       const double *phi_ind, double cuct, double *face3, double *E, cudaStream_t s)
{
    if (!m.nf) return;
    k_face_candidate<<<grid_for(m.nf, 128), 128, 0, s>>>(m, u, Bt, Bi, phi_tot, nullptr, face3, nullptr, nullptr);
    if (m.no_edges)
    {
        if (m.max_valence <= 8)
            k_edge_uct<8><<<grid_for(m.no_edges, 128), 128, 0, s>>>(m, face3, u, phi_ind, cuct, E);
        else
            k_edge_uct<kMaxValence><<<grid_for(m.no_edges, 128), 128, 0, s>>>(m, face3, u, phi_ind, cuct, E);
    }
}
} // namespace mhd

using namespace mhd;

extern "C" {

int mhd_gpu_cell_vector(MhdMesh *mesh, const double *flux, int32_t ncells, double *out)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && MHD_ARR(flux, mesh->v.nf) && MHD_ARR(out, ncells), "bad argument");
        MHD_REQUIRE(ncells >= 0 && ncells <= mesh->v.nc, "ncells out of range");
        if (!ncells) return;
        k_cell_vector<<<grid_for(ncells, 128), 128, 0, mesh->stream>>>(mesh->v, flux, ncells, out);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_ideal_emf(MhdMesh *mesh, const double *u, const double *Bt, const double *Bi, const double *phi_tot, const double *phi_ind,
                      double cuct, double *E)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && MHD_ARR(u, mesh->v.nc) && MHD_ARR(Bt, mesh->v.nc) && MHD_ARR(Bi, mesh->v.nc) && MHD_ARR(phi_tot, mesh->v.nf) &&
                        MHD_ARR(phi_ind, mesh->v.nf) && MHD_ARR(E, mesh->v.ne),
                    "bad argument");
        const MeshView &m = mesh->v;
        if (!m.nf) return;
        mesh->scratch_face3.alloc(3 * static_cast<size_t>(m.nf));
        ideal_emf_enqueue(m, u, Bt, Bi, phi_tot, phi_ind, cuct, mesh->scratch_face3.p, E, mesh->stream);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_edge_modes(MhdMesh *mesh, const double *u_inf, const double *B_imf, double *E)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && u_inf && B_imf && MHD_ARR(E, mesh->v.ne), "bad argument");
        if (!mesh->v.no_edges) return;
        const V3 ui = mk(u_inf[0], u_inf[1], u_inf[2]), bi = mk(B_imf[0], B_imf[1], B_imf[2]);
        const V3 Einf = -1.0 * cross(ui, bi);
        k_edge_modes<<<grid_for(mesh->v.no_edges, 256), 256, 0, mesh->stream>>>(mesh->v, Einf, E);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_faraday(MhdMesh *mesh, const double *E, double *B, double dt)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && MHD_ARR(E, mesh->v.ne) && MHD_ARR(B, mesh->v.nf), "bad argument");
        if (!mesh->v.nf) return;
        k_faraday<<<grid_for(mesh->v.nf, 256), 256, 0, mesh->stream>>>(mesh->v, E, nullptr, dt, B);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_faraday_edge_dt(MhdMesh *mesh, const double *E, const double *dt_edge, double *B)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && MHD_ARR(E, mesh->v.ne) && MHD_ARR(B, mesh->v.nf) && MHD_ARR(dt_edge, mesh->v.ne), "bad argument");
        if (!mesh->v.nf) return;
        k_faraday<<<grid_for(mesh->v.nf, 256), 256, 0, mesh->stream>>>(mesh->v, E, dt_edge, 0.0, B);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_div_b(MhdMesh *mesh, const double *B, const double *extra, double *host_out)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && host_out && MHD_ARR(B, mesh->v.nf), "bad argument");
        const MeshView &m = mesh->v;
        if (!m.no_cells)
        {
            host_out[0] = host_out[1] = 0.0;
            host_out[2] = -1.0;
            return;
        }
        const int nb = div_b_blocks(m);
        mesh->scratch_red.alloc(3 * static_cast<size_t>(nb) + 3);
        DivPart *part = reinterpret_cast<DivPart *>(mesh->scratch_red.p);
        double *res = mesh->scratch_red.p + 3 * nb;
        k_div_b_partial<<<nb, 256, 0, mesh->stream>>>(m, B, extra, part);
        MHD_LAUNCH_CHECK();
        k_div_b_final<<<1, 1024, 0, mesh->stream>>>(part, nb, res);
        MHD_LAUNCH_CHECK();
        MHD_CUDA(cudaMemcpyAsync(mesh->pinned, res, 3 * sizeof(double), cudaMemcpyDeviceToHost, mesh->stream));
        MHD_CUDA(cudaStreamSynchronize(mesh->stream));
        host_out[0] = mesh->pinned[0];
        host_out[1] = mesh->pinned[1];
        host_out[2] = mesh->pinned[2];
    });
}

int mhd_gpu_div_b_noalloc_blocks(int64_t n_owned_cells, int64_t *blocks)
{
    return guarded([&] {
        MHD_REQUIRE(blocks && n_owned_cells >= 0, "bad argument");
        const int64_t nb = (n_owned_cells + kNoAllocCellsPerBlock - 1) / kNoAllocCellsPerBlock;
        MHD_REQUIRE(nb <= MHD_NOALLOC_DIVB_MAX_BLOCKS,
                    "div_b_noalloc: the static scratch holds " + std::to_string(MHD_NOALLOC_DIVB_MAX_BLOCKS) +
                        " block partials, i.e. at most " +
                        std::to_string(static_cast<int64_t>(MHD_NOALLOC_DIVB_MAX_BLOCKS) * kNoAllocCellsPerBlock) +
                        " owned cells; this mesh has " + std::to_string(n_owned_cells));
        *blocks = nb;
    });
}

int mhd_gpu_alloc_calls(int64_t *out)
{
    return guarded([&] {
        MHD_REQUIRE(out, "bad argument");
        *out = g_alloc_calls.load(std::memory_order_relaxed);
    });
}

int mhd_gpu_div_b_noalloc(MhdMesh *mesh, const double *B, const double *extra, double *host_out)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && host_out && MHD_ARR(B, mesh->v.nf), "bad argument");
        const MeshView &m = mesh->v;
        if (!m.no_cells)
        {
            host_out[0] = host_out[1] = 0.0;
            host_out[2] = -1.0;
            return;
        }
        int64_t nb = 0;
        const int rc = mhd_gpu_div_b_noalloc_blocks(m.no_cells, &nb);
        if (rc != MHD_OK) throw ApiError(rc, mhd_gpu_last_error());
        double *scratch = noalloc_scratch();
        DivPart *part = reinterpret_cast<DivPart *>(scratch);
        double *res = scratch + 3 * MHD_NOALLOC_DIVB_MAX_BLOCKS;
        k_div_b_block<<<static_cast<int>(nb), 256, 0, mesh->stream>>>(m, B, extra, part);
        MHD_LAUNCH_CHECK();
        k_div_b_final<<<1, 1024, 0, mesh->stream>>>(part, static_cast<int>(nb), res);
        MHD_LAUNCH_CHECK();
        // into the handle's pinned buffer, allocated when the mesh was created
        MHD_CUDA(cudaMemcpyAsync(mesh->pinned, res, 3 * sizeof(double), cudaMemcpyDeviceToHost, mesh->stream));
        MHD_CUDA(cudaStreamSynchronize(mesh->stream));
        host_out[0] = mesh->pinned[0];
        host_out[1] = mesh->pinned[1];
        host_out[2] = mesh->pinned[2];
    });
}

int mhd_gpu_cell_current(MhdMesh *mesh, const double *B, double *J)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && B && J, "bad argument");
        if (!mesh->v.nc) return;
        k_cell_current<<<grid_for(mesh->v.nc, 128), 128, 0, mesh->stream>>>(mesh->v, B, J);
        MHD_LAUNCH_CHECK();
    });
}

} // extern "C"
