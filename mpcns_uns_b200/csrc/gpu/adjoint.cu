// nvcc-flags: -fmad=false
// Differentiated explicit run: forward / tangent-linear / adjoint of the FP64 SSP-RK2 step with the
// explicit resistive EMF, for a scalar functional of the final field
//     J = sum over marked cells of |B_tot,c|^2 V_c,
// with respect to the per-cell resistivity eta_c (m_e = mean of eta over the edge's cells / star1_e)
// and the inflow velocity u_inf (the free-stream velocity of every species and the inflow edge EMF
// -u_inf x B_imf).  The reference has no adjoint; the forward map is the reference's step (pinned bit
// for bit by the parity tests), differentiated at a fixed step size.
//
// Tangent-linear kernels (k_t_*) run the stage on dual numbers (value, tangent): their values equal
// the FP64 step's.  Adjoint kernels (k_a_*) are hand-written reverse sweeps of each stage kernel; they
// recompute what they need from the stage input, its primitives, limited gradients and cell fields.
// The backward sweep restores checkpoints every `checkpoint_every` steps, recomputes a segment while
// recording its stage inputs and floor flags, then reverses it step by step.
#include <math_constants.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "induction.cuh"
#include "kernels.cuh"
#include "state.cuh"
#include "tangent.cuh"

namespace mhd
{
namespace
{
constexpr int kMaxFnSpecies = 2; // the stage keeps the gradients of all species at once

__host__ __device__ __forceinline__ int64_t ui(int s, int q, int64_t c, int64_t n) { return (s * 5 + q) * n + c; }
__host__ __device__ __forceinline__ int64_t gi(int s, int q, int64_t c, int64_t n) { return (s * 15 + q) * n + c; }

// tangent of the free-stream state per species (the inflow velocity's direction on components 1..3)
struct FsTan
{
    double d[kMaxSpecies][5];
};

__device__ __forceinline__ DPrim fs_dual(const FluidParams &p, const FsTan &t, int s)
{
    const Prim5 &f = p.fs[s];
    return DPrim{{f.rho, t.d[s][0]}, {f.u, t.d[s][1]}, {f.v, t.d[s][2]}, {f.w, t.d[s][3]}, {f.p, t.d[s][4]}};
}

__device__ __forceinline__ bool face_active(const MeshView &m, int32_t f)
{
    bool a = false;
    for (int32_t k = m.f2c_ptr[f]; k < m.f2c_ptr[f + 1]; ++k) a |= m.f2c_idx[k] < m.no_cells;
    return a;
}

// ================================================================ tangent-linear stage
// Solver::prepare (k_prepare) on duals
__global__ void __launch_bounds__(128) k_t_prepare(MeshView m, FluidParams p, const double *__restrict__ mass, double M_ref, DCPtr U,
                                                    DPtr W, DCPtr phi, const double *__restrict__ Badd, DPtr bind, DPtr btot, DPtr up)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int64_t n = m.nc;
    Dual ne = dl(0);
    for (int s = 0; s < p.nsp; ++s)
    {
        const DPrim w = to_prim_d(U.get(ui(s, 0, c, n)), U.get(ui(s, 1, c, n)), U.get(ui(s, 2, c, n)), U.get(ui(s, 3, c, n)),
                                  U.get(ui(s, 4, c, n)), p.gamma, p.rho_floor, p.p_floor);
        W.put(ui(s, 0, c, n), w.rho); W.put(ui(s, 1, c, n), w.u); W.put(ui(s, 2, c, n), w.v); W.put(ui(s, 3, c, n), w.w);
        W.put(ui(s, 4, c, n), w.p);
        ne += dmax(w.rho, dl(0.0)) / mass[s] * M_ref;
    }
    Dual u[3] = {dl(0), dl(0), dl(0)};
    if (m.material[c] == 0)
        for (int s = 0; s < p.nsp; ++s)
        {
            const Dual ns = dmax(W.get(ui(s, 0, c, n)), dl(0.0)) / mass[s] * M_ref;
            const Dual chi = ne.v > 1e-300 ? ns / ne : dl(s == 0 ? 1.0 : 0.0);
            for (int a = 0; a < 3; ++a) u[a] += chi * W.get(ui(s, 1 + a, c, n));
        }
    const DV3 b = cell_vector_d(m, DCPtr{phi.v, phi.d}, c);
    dst3(bind, c, b);
    dst3(btot, c, dmk(b.x + Badd[3 * (int64_t)c], b.y + Badd[3 * (int64_t)c + 1], b.z + Badd[3 * (int64_t)c + 2]));
    dst3(up, c, dmk(u[0], u[1], u[2]));
}

// k_limited_gradients_tet on duals, one thread per (cell, species = blockIdx.y)
__global__ void __launch_bounds__(128) k_t_grad(MeshView m, FluidParams p, FsTan ft, DCPtr W, DPtr G)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (c >= m.nc || s >= p.nsp) return;
    const int64_t n = m.nc;
    if (c >= m.no_cells || !m.st_valid[c])
    {
        for (int q = 0; q < 15; ++q) G.put(gi(s, q, c, n), dl(0.0));
        return;
    }
    int32_t nb[4];
    Dual wc[5], wn[4][5];
    for (int j = 0; j < 4; ++j) nb[j] = m.t_nb[j * n + c];
    for (int q = 0; q < 5; ++q) wc[q] = W.get(ui(s, q, c, n));
    for (int j = 0; j < 4; ++j)
        if (nb[j] >= 0)
            for (int q = 0; q < 5; ++q) wn[j][q] = W.get(ui(s, q, nb[j], n));
    const DPrim wcp{wc[0], wc[1], wc[2], wc[3], wc[4]};
    const DPrim fs = fs_dual(p, ft, s);
    for (int j = 0; j < 4; ++j)
        if (nb[j] < 0 && nb[j] != INT32_MIN)
        {
            const int32_t f = -(nb[j] + 1);
            const V3 nrm = (double(m.t_sg[j * n + c]) / m.face_area_mag[f]) * ld3(m.face_area, f);
            const DPrim g = ghost_state_d(m.face_kind[f], p.absorb[s] != 0, wcp, nrm, fs);
            wn[j][0] = g.rho; wn[j][1] = g.u; wn[j][2] = g.v; wn[j][3] = g.w; wn[j][4] = g.p;
        }
    const double I00 = m.t_inv[c], I01 = m.t_inv[n + c], I02 = m.t_inv[2 * n + c], I11 = m.t_inv[3 * n + c], I12 = m.t_inv[4 * n + c],
                 I22 = m.t_inv[5 * n + c];
    for (int q = 0; q < 5; ++q)
    {
        Dual r0 = dl(0), r1 = dl(0), r2 = dl(0), lo = wc[q], hi = wc[q];
        for (int j = 0; j < 4; ++j)
        {
            if (nb[j] == INT32_MIN) continue;
            const Dual dq = wn[j][q] - wc[q];
            r0 += m.t_wd[(3 * j) * n + c] * dq;
            r1 += m.t_wd[(3 * j + 1) * n + c] * dq;
            r2 += m.t_wd[(3 * j + 2) * n + c] * dq;
            lo = dmin(lo, wn[j][q]);
            hi = dmax(hi, wn[j][q]);
        }
        const Dual g0 = I00 * r0 + I01 * r1 + I02 * r2;
        const Dual g1 = I01 * r0 + I11 * r1 + I12 * r2;
        const Dual g2 = I02 * r0 + I12 * r1 + I22 * r2;
        Dual psi = dl(1.0);
        if (p.limit)
        {
            for (int j = 0; j < 4; ++j)
            {
                const Dual d = g0 * m.t_dx[(3 * j) * n + c] + g1 * m.t_dx[(3 * j + 1) * n + c] + g2 * m.t_dx[(3 * j + 2) * n + c];
                if (d.v > 1e-300) psi = dmin(psi, (hi - wc[q]) / d);
                else if (d.v < -1e-300) psi = dmin(psi, (lo - wc[q]) / d);
            }
            if (p.rel_limit > 0 && (q == 0 || q == 4))
                for (int j = 0; j < 4; ++j)
                {
                    const Dual d =
                        dabs(g0 * m.t_dx[(3 * j) * n + c] + g1 * m.t_dx[(3 * j + 1) * n + c] + g2 * m.t_dx[(3 * j + 2) * n + c]);
                    if (d.v > 1e-300) psi = dmin(psi, p.rel_limit * wc[q] / d);
                }
        }
        const Dual ps = dmax(dl(0.0), dmin(dl(1.0), psi));
        G.put(gi(s, 3 * q, c, n), ps * g0);
        G.put(gi(s, 3 * q + 1, c, n), ps * g1);
        G.put(gi(s, 3 * q + 2, c, n), ps * g2);
    }
}

// k_face_flux on duals; F[(s*5 + q)*nf + f]
__global__ void __launch_bounds__(128) k_t_flux(MeshView m, FluidParams p, FsTan ft, DCPtr W, DCPtr G, DPtr F)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (f >= m.nf || s >= p.nsp) return;
    const int64_t nf = m.nf, n = m.nc;
    const int kind = m.face_kind[f];
    const int32_t p0 = m.f2c_ptr[f], cnt = m.f2c_ptr[f + 1] - p0;
    bool any_owned = false;
    for (int q = 0; q < cnt; ++q)
    {
        const int32_t cc = m.f2c_idx[p0 + q];
        any_owned |= cc < m.no_cells && m.material[cc] == 0;
    }
    if (kind == 4 || !any_owned)
    {
        for (int q = 0; q < 5; ++q) F.put((s * 5 + q) * nf + f, dl(0.0));
        return;
    }
    const double A = m.face_area_mag[f];
    const V3 nv = (1.0 / A) * ld3(m.face_area, f);
    const V3 xf = ld3(m.face_center, f);
    const bool interior = cnt == 2 && kind == 0;
    auto state_of = [&](int32_t cc) {
        const DPrim w{W.get(ui(s, 0, cc, n)), W.get(ui(s, 1, cc, n)), W.get(ui(s, 2, cc, n)), W.get(ui(s, 3, cc, n)),
                      W.get(ui(s, 4, cc, n))};
        Dual g[15];
        for (int q = 0; q < 15; ++q) g[q] = G.get(gi(s, q, cc, n));
        return face_state_d(w, g, xf - ld3(m.cell_center, cc));
    };
    DPrim L, R;
    if (interior)
    {
        L = state_of(m.face_L[f]);
        R = state_of(m.face_R[f]);
    }
    else
    {
        int32_t c = m.f2c_idx[p0];
        int sgn = m.f2c_sgn[p0];
        if (cnt == 2 && m.material[c] != 0)
        {
            c = m.f2c_idx[p0 + 1];
            sgn = m.f2c_sgn[p0 + 1];
        }
        const DPrim in = state_of(c);
        const DPrim gh = ghost_state_d(kind, p.absorb[s] != 0, in, double(sgn) * nv, fs_dual(p, ft, s));
        if (sgn > 0) { L = in; R = gh; }
        else { R = in; L = gh; }
    }
    Dual Fl[5];
    rusanov_d(L, R, nv, p.gamma, Fl);
    for (int q = 0; q < 5; ++q) F.put((s * 5 + q) * nf + f, Fl[q] * A);
}

// k_update<4> on duals (no sources): Uo = floors(Ub + dt rhs), no stage-2 average (k_t_average does it)
__global__ void __launch_bounds__(128) k_t_update(MeshView m, FluidParams p, DCPtr F, DCPtr Ub, DPtr Uo, double dt)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (c >= m.nc || s >= p.nsp) return;
    const int64_t n = m.nc, nf = m.nf;
    const bool live = c < m.no_cells && m.material[c] == 0;
    Dual u[5];
    for (int q = 0; q < 5; ++q) u[q] = Ub.get(ui(s, q, c, n));
    if (live)
    {
        const double V = m.cell_volume[c];
        Dual r[5] = {dl(0), dl(0), dl(0), dl(0), dl(0)};
        for (int j = 0; j < 4; ++j)
        {
            const int32_t f = m.cfa_idx[4 * c + j];
            const bool out = m.cfa_sgn[4 * c + j] > 0;
            for (int q = 0; q < 5; ++q)
            {
                const Dual v = F.get((s * 5 + q) * nf + f) / V;
                r[q] = out ? r[q] - v : r[q] + v;
            }
        }
        for (int q = 0; q < 5; ++q) u[q] += dt * r[q];
        const Dual ke = u[0].v > 0 ? 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0] : dl(0.0);
        if (!(u[0].v >= p.rho_floor)) to_cons_d(DPrim{dl(p.rho_floor), dl(0), dl(0), dl(0), dl(p.p_floor)}, p.gamma, u);
        else if (((p.gamma - 1.0) * (u[4] - ke)).v < p.p_floor)
            to_cons_d(to_prim_d(u[0], u[1], u[2], u[3], u[4], p.gamma, p.rho_floor, p.p_floor), p.gamma, u);
    }
    for (int q = 0; q < 5; ++q) Uo.put(ui(s, q, c, n), u[q]);
}

// k_face_candidate on duals
__global__ void __launch_bounds__(128) k_t_face_cand(MeshView m, DCPtr u, DCPtr Bt, DCPtr Bi, DCPtr phi, const double *__restrict__ phi_add,
                                                      DPtr Ef)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    const double A = m.face_area_mag[f];
    const V3 n = (1.0 / A) * ld3(m.face_area, f);
    const Dual pt = phi_add ? phi.get(f) + phi_add[f] : phi.get(f);
    const Dual Bn = pt / A;
    auto flux = [&](int32_t c) {
        const DV3 uc = dld3(u, c);
        return dot(uc, n) * dld3(Bt, c) - Bn * uc;
    };
    const int32_t p0 = m.f2c_ptr[f], cnt = m.f2c_ptr[f + 1] - p0;
    DV3 F;
    if (cnt == 2)
    {
        const int32_t L = m.face_L[f], R = m.face_R[f];
        const Dual a = dmax(dabs(dot(dld3(u, L), n)), dabs(dot(dld3(u, R), n)));
        F = 0.5 * (flux(L) + flux(R)) - (0.5 * a) * (dld3(Bi, R) - dld3(Bi, L));
    }
    else
        F = flux(m.f2c_idx[p0]);
    dst3(Ef, f, -1.0 * cross(n, F));
}

// edge_uct on duals (MAXV faces per edge at most)
template <int MAXV>
__device__ __forceinline__ bool edge_uct_d(const MeshView &m, int32_t e, DCPtr Ef, DCPtr u, DCPtr phi_ind, double cuct, Dual &out)
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
    const V3 ax = fabs(th.x) < 0.9 ? mk(1, 0, 0) : mk(0, 1, 0);
    V3 e1 = mhd::cross(th, ax);
    e1 = (1.0 / sqrt(mhd::dot(e1, e1))) * e1;
    const V3 e2 = mhd::cross(th, e1);
    double w[MAXV], sg[MAXV];
    Dual aef[MAXV], qa[MAXV], qb[MAXV];
    Dual Ec = dl(0), M11 = dl(0), M12 = dl(0), M22 = dl(0), g1 = dl(0), g2 = dl(0);
#pragma unroll
    for (int i = 0; i < MAXV; ++i)
    {
        if (i >= nf) break;
        const int32_t f = m.e2f_idx[f0 + i];
        w[i] = m.ef_weight[f0 + i];
        Ec += w[i] * dot(dld3(Ef, f), t);
        V3 v = ld3(m.face_center, f) - mid;
        v = v - mhd::dot(v, th) * th;
        const double nv = sqrt(mhd::dot(v, v));
        const V3 mi = nv > 0 ? (1.0 / nv) * v : mk(0, 0, 0);
        const V3 nrm = (1.0 / m.face_area_mag[f]) * ld3(m.face_area, f);
        Dual a = dl(0);
        for (int32_t k = q0; k < q1; ++k) a = dmax(a, dabs(dot(dld3(u, m.ec_cell[k]), mi)));
        aef[i] = a;
        sg[i] = mhd::dot(th, mhd::cross(mi, nrm));
        const DV3 qv = (a * sg[i]) * nrm;
        qa[i] = dot(qv, e1);
        qb[i] = dot(qv, e2);
        M11 += w[i] * qa[i] * qa[i];
        M12 += w[i] * qa[i] * qb[i];
        M22 += w[i] * qb[i] * qb[i];
        g1 += w[i] * qa[i];
        g2 += w[i] * qb[i];
    }
    const Dual tr = M11 + M22;
    const Dual eps = 1e-14 * tr;
    const Dual det = (M11 + eps) * (M22 + eps) - M12 * M12;
    Dual l1 = dl(0), l2 = dl(0);
    if (tr.v > 0 && det.v > 0)
    {
        l1 = ((M22 + eps) * g1 - M12 * g2) / det;
        l2 = ((M11 + eps) * g2 - M12 * g1) / det;
    }
    Dual Eu = dl(0);
#pragma unroll
    for (int i = 0; i < MAXV; ++i)
    {
        if (i >= nf) break;
        const int32_t f = m.e2f_idx[f0 + i];
        const Dual omega = w[i] * (1.0 - (qa[i] * l1 + qb[i] * l2));
        Eu += omega * aef[i] * sg[i] * (phi_ind.get(f) / m.face_area_mag[f]);
    }
    out = Ec + 2.0 * cuct * L * Eu;
    return true;
}

// k_edge_emf_assign on duals: modes, UCT, explicit resistive EMF (m is a dual: its tangent follows eta)
template <int MAXV>
__global__ void __launch_bounds__(128) k_t_edge(MeshView m, DCPtr Ef, DCPtr u, DCPtr phi, double cuct, DV3 E_inf, DCPtr mres, DPtr E)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    Dual val = dl(0.0);
    if (e < m.no_edges)
    {
        const int mode = m.edge_mode[e];
        if (mode == 1) val = dl(0.0);
        else if (mode == 2) val = dot(E_inf, ld3(m.edge_vec, e));
        else
        {
            Dual v;
            if (edge_uct_d<MAXV>(m, e, Ef, u, phi, cuct, v)) val += v;
        }
        if (mres.v)
        {
            Dual p0 = dl(0.0);
            for (int32_t k = m.e2f_ptr[e]; k < m.e2f_ptr[e + 1]; ++k)
            {
                const int32_t f = m.e2f_idx[k];
                p0 += m.e2f_sgn[k] * (m.star2[f] * phi.get(f));
            }
            val += mres.get(e) * p0 + 0.0 + 0.0;
        }
    }
    E.put(e, val);
}

// k_ct on duals without the stage-2 average
__global__ void __launch_bounds__(256) k_t_ct(MeshView m, DCPtr E, DCPtr phis, DPtr phio, double dt)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    Dual v = phis.get(f);
    if (face_active(m, f))
    {
        Dual circ = dl(0.0);
        for (int32_t k = m.f2e_ptr[f]; k < m.f2e_ptr[f + 1]; ++k) circ += m.f2e_sgn[k] * E.get(m.f2e_idx[k]);
        v -= dt * circ;
    }
    phio.put(f, v);
}

// the SSP-RK2 average a = (b + a) / 2 of values and tangents (b: the step's start)
__global__ void k_average(int64_t n, const double *__restrict__ bv, double *__restrict__ av, const double *__restrict__ bd,
                          double *__restrict__ ad)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    av[i] = 0.5 * (bv[i] + av[i]);
    if (ad) ad[i] = 0.5 * (bd[i] + ad[i]);
}

// The run's initial state moving with the free stream (uniform_flow): per species and fluid cell the
// primitives of X0 with the velocity shifted by sh = u_inf - u_inf at creation, back to conservative
// variables (to_cons order); dU (if given) its derivative along du.
__global__ void k_init_flow(MeshView m, FluidParams p, const double *__restrict__ X0, V3 sh, V3 du, double *__restrict__ U,
                            double *__restrict__ dU)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (c >= m.nc || s >= p.nsp) return;
    const int64_t n = m.nc;
    double v[5];
    for (int q = 0; q < 5; ++q) v[q] = X0[ui(s, q, c, n)];
    double d[5] = {0, 0, 0, 0, 0};
    if (m.material[c] == 0)
    {
        const Prim5 w = to_prim(v[0], v[1], v[2], v[3], v[4], p.gamma, p.rho_floor, p.p_floor);
        const V3 u = mk(w.u + sh.x, w.v + sh.y, w.w + sh.z);
        v[0] = w.rho;
        v[1] = w.rho * u.x;
        v[2] = w.rho * u.y;
        v[3] = w.rho * u.z;
        v[4] = w.p / (p.gamma - 1.0) + 0.5 * w.rho * (u.x * u.x + u.y * u.y + u.z * u.z);
        d[1] = w.rho * du.x;
        d[2] = w.rho * du.y;
        d[3] = w.rho * du.z;
        d[4] = w.rho * (u.x * du.x + u.y * du.y + u.z * du.z);
    }
    for (int q = 0; q < 5; ++q)
    {
        U[ui(s, q, c, n)] = v[q];
        if (dU) dU[ui(s, q, c, n)] = d[q];
    }
}

// transpose of k_init_flow with respect to u_inf: block sums of sum_s rho (lU1, lU2, lU3) + lU4 rho u over
// the fluid cells (u the shifted velocity), added to out[0..2]
__global__ void __launch_bounds__(256) k_init_flow_T(MeshView m, FluidParams p, const double *__restrict__ X0, V3 sh,
                                                      const double *__restrict__ lU, double *__restrict__ out)
{
    double a[3] = {0, 0, 0};
    const int64_t n = m.nc;
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < m.nc; c += gridDim.x * blockDim.x)
    {
        if (m.material[c] != 0) continue;
        for (int s = 0; s < p.nsp; ++s)
        {
            const Prim5 w = to_prim(X0[ui(s, 0, c, n)], X0[ui(s, 1, c, n)], X0[ui(s, 2, c, n)], X0[ui(s, 3, c, n)], X0[ui(s, 4, c, n)],
                                    p.gamma, p.rho_floor, p.p_floor);
            const double rho = w.rho;
            const V3 u = mk(w.u + sh.x, w.v + sh.y, w.w + sh.z);
            const double l4 = lU[ui(s, 4, c, n)];
            a[0] += rho * (lU[ui(s, 1, c, n)] + l4 * u.x);
            a[1] += rho * (lU[ui(s, 2, c, n)] + l4 * u.y);
            a[2] += rho * (lU[ui(s, 3, c, n)] + l4 * u.z);
        }
    }
    for (int k = 0; k < 3; ++k)
    {
        double v = a[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(out + k, v);
    }
}

// m_e = (sum of eta over the edge's cells / count) / star1_e, and the same linear map of a tangent
__global__ void k_eta_to_m(MeshView m, const double *__restrict__ eta, double *__restrict__ mres)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    const int32_t a = m.ec_ptr[e], b = m.ec_ptr[e + 1];
    double acc = 0.0;
    for (int32_t k = a; k < b; ++k) acc += eta[m.ec_cell[k]];
    mres[e] = b > a ? (acc / (b - a)) / m.star1[e] : 0.0;
}

// transpose of k_eta_to_m: grad_eta[c] += sum over the edges of c of lm_e / count_e / star1_e
__global__ void k_m_to_eta(MeshView m, const double *__restrict__ lm, double *__restrict__ geta)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    const int32_t a = m.ec_ptr[e], b = m.ec_ptr[e + 1];
    if (b <= a || lm[e] == 0.0) return;
    const double w = (1.0 / (b - a)) / m.star1[e];
    for (int32_t k = a; k < b; ++k) atomicAdd(geta + m.ec_cell[k], w * lm[e]);
}

// ================================================================ functional J = sum_mask |B_tot|^2 V
// block partial sums (deterministic: a fixed grid, then k_sum_final adds the parts in order)
// Knuth's TwoSum: s + e == a + b exactly (additions only, so contraction cannot alter it)
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e)
{
    s = a + b;
    const double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// (hi, lo) += (bh, bl) in double-double, renormalised so that |lo| <= ulp(hi) / 2
__device__ __forceinline__ void dd_add(double &hi, double &lo, double bh, double bl)
{
    double s, e;
    two_sum(hi, bh, s, e);
    e += lo + bl;
    hi = s + e;
    lo = e - (hi - s);
}

// J = sum over the marked cells of |B_tot|^2 V (and its tangent), the value summed in double-double: the
// run's J differs from a neighbouring run's by far less than J's own ulp when the parameters move by 1e-6,
// and the unevaluated sum hi + lo keeps that difference (part: per block hi, lo, tangent)
__global__ void __launch_bounds__(256) k_J_partial(MeshView m, DCPtr phi, const double *__restrict__ Badd, const int8_t *__restrict__ mask,
                                                    double *__restrict__ part)
{
    double jh = 0, jl = 0, jd = 0;
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < m.nc; c += gridDim.x * blockDim.x)
    {
        if (!mask[c]) continue;
        const DV3 b = cell_vector_d(m, phi, c);
        const DV3 bt = dmk(b.x + Badd[3 * (int64_t)c], b.y + Badd[3 * (int64_t)c + 1], b.z + Badd[3 * (int64_t)c + 2]);
        const Dual j = dot(bt, bt) * m.cell_volume[c];
        dd_add(jh, jl, j.v, 0.0);
        jd += j.d;
    }
    __shared__ double sh[3][8];
    for (int o = 16; o > 0; o >>= 1)
    {
        const double oh = __shfl_down_sync(0xffffffffu, jh, o), ol = __shfl_down_sync(0xffffffffu, jl, o);
        dd_add(jh, jl, oh, ol);
        jd += __shfl_down_sync(0xffffffffu, jd, o);
    }
    if ((threadIdx.x & 31) == 0)
    {
        sh[0][threadIdx.x >> 5] = jh;
        sh[1][threadIdx.x >> 5] = jl;
        sh[2][threadIdx.x >> 5] = jd;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double h = 0, l = 0, d = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
        {
            dd_add(h, l, sh[0][w], sh[1][w]);
            d += sh[2][w];
        }
        part[3 * blockIdx.x] = h;
        part[3 * blockIdx.x + 1] = l;
        part[3 * blockIdx.x + 2] = d;
    }
}

// out: J (hi), its tangent, J's low part
__global__ void k_sum_final(const double *__restrict__ part, int nparts, double *__restrict__ out)
{
    double h = 0, l = 0, d = 0;
    for (int i = 0; i < nparts; ++i)
    {
        dd_add(h, l, part[3 * i], part[3 * i + 1]);
        d += part[3 * i + 2];
    }
    out[0] = h;
    out[1] = d;
    out[2] = l;
}

// dJ/dB_c = 2 V_c B_tot,c on the marked cells, into lB
__global__ void k_a_J(MeshView m, const double *__restrict__ phi, const double *__restrict__ Badd, const int8_t *__restrict__ mask,
                      double *__restrict__ lB)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    V3 g = mk(0, 0, 0);
    if (mask[c])
    {
        const V3 b = cell_vector(m, phi, c);
        const V3 bt = mk(b.x + Badd[3 * (int64_t)c], b.y + Badd[3 * (int64_t)c + 1], b.z + Badd[3 * (int64_t)c + 2]);
        g = (2.0 * m.cell_volume[c]) * bt;
    }
    st3(lB, c, g);
}

// ================================================================ adjoint stage
// y_c = I_c^T lB_c (the transpose of the cell fit B_c = I_c sum_k n_k Phi_k); lB is cleared for the next stage
__device__ __forceinline__ V3 recon_T(const MeshView &m, int32_t c, V3 lb)
{
    double I[3][3];
    if (!cell_vector_inverse(m, c, I)) return mk(0, 0, 0);
    return mk(I[0][0] * lb.x + I[1][0] * lb.y + I[2][0] * lb.z, I[0][1] * lb.x + I[1][1] * lb.y + I[2][1] * lb.z,
              I[0][2] * lb.x + I[1][2] * lb.y + I[2][2] * lb.z);
}

// lphi_f += n_f . (y_L + y_R), n_f = A_f / |A_f| (faces with |A_f| > 0)
__device__ __forceinline__ double recon_T_face(const MeshView &m, const double *__restrict__ y, int32_t f)
{
    const double A = m.face_area_mag[f];
    if (A <= 0) return 0.0;
    const V3 n = (1.0 / A) * ld3(m.face_area, f);
    double acc = 0.0;
    for (int32_t k = m.f2c_ptr[f]; k < m.f2c_ptr[f + 1]; ++k) acc += mhd::dot(n, ld3(y, m.f2c_idx[k]));
    return acc;
}

__global__ void k_a_recon_cells(MeshView m, double *__restrict__ lB, double *__restrict__ y)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    st3(y, c, recon_T(m, c, ld3(lB, c)));
    st3(lB, c, mk(0, 0, 0));
}

__global__ void k_a_recon_faces(MeshView m, const double *__restrict__ y, double *__restrict__ lphi)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    lphi[f] += recon_T_face(m, y, f);
}

// CT transpose: lE_e = -scale sum over the active faces of e of sgn lphi_f
__global__ void k_a_ct(MeshView m, const int8_t *__restrict__ active, const double *__restrict__ lphi, double scale, double *__restrict__ lE)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    double acc = 0.0;
    for (int32_t k = m.e2f_ptr[e]; k < m.e2f_ptr[e + 1]; ++k)
    {
        const int32_t f = m.e2f_idx[k];
        if (active[f]) acc += m.e2f_sgn[k] * lphi[f];
    }
    lE[e] = -scale * acc;
}

// K0: transpose of U~ = floors(U_in + dt rhs).  lUt: adjoint of U~; Ut: U~ itself (after the floors).
// lU += d/dU_in, lrV = dt (d/dU_pre) / V on the owned fluid cells (0 elsewhere)
__global__ void __launch_bounds__(128) k_a_floors(MeshView m, FluidParams p, const int8_t *__restrict__ flags, const double *__restrict__ Ut,
                                                   const double *__restrict__ lUt, double dt, double *__restrict__ lrV, double *__restrict__ lU)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (c >= m.nc || s >= p.nsp) return;
    const int64_t n = m.nc;
    const bool live = c < m.no_cells && m.material[c] == 0;
    double l[5];
    for (int q = 0; q < 5; ++q) l[q] = lUt[ui(s, q, c, n)];
    if (!live)
    {
        for (int q = 0; q < 5; ++q)
        {
            lU[ui(s, q, c, n)] += l[q];
            lrV[ui(s, q, c, n)] = 0.0;
        }
        return;
    }
    const int fl = flags ? flags[s * n + c] : 0;
    if (fl == 1)
        for (int q = 0; q < 5; ++q) l[q] = 0.0;
    else if (fl == 2)
    {
        // U4' = p_floor / (gamma - 1) + |m|^2 / (2 rho): U0..3 pass, U4 depends on them only
        const double r = Ut[ui(s, 0, c, n)], mx = Ut[ui(s, 1, c, n)], my = Ut[ui(s, 2, c, n)], mz = Ut[ui(s, 3, c, n)];
        const double l4 = l[4];
        l[0] += l4 * (-0.5 * (mx * mx + my * my + mz * mz) / (r * r));
        l[1] += l4 * (mx / r);
        l[2] += l4 * (my / r);
        l[3] += l4 * (mz / r);
        l[4] = 0.0;
    }
    const double sc = dt / m.cell_volume[c];
    for (int q = 0; q < 5; ++q)
    {
        lU[ui(s, q, c, n)] += l[q];
        lrV[ui(s, q, c, n)] = sc * l[q];
    }
}

// K1: edge adjoint of k_edge_emf_assign.  Per edge: the resistive part (lres = m lE for the faces, lm += p0 lE),
// the inflow edge value (lpar[0..2] += t lE), and the reverse of edge_uct: lc = lE (the central part, gathered by
// the faces), efphi per e2f entry (the upwind part's Phi_ind derivative), lup (atomic) through a_ef.
template <int MAXV>
__global__ void __launch_bounds__(128, 4) k_a_edge(MeshView m, const double *__restrict__ u, const double *__restrict__ phi, double cuct,
                                                 const double *__restrict__ mres, const double *__restrict__ lE, double *__restrict__ lc,
                                                 double *__restrict__ efphi, double *__restrict__ lres, double *__restrict__ lm,
                                                 double *__restrict__ lpar, double *__restrict__ lup)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    const int32_t f0 = m.e2f_ptr[e], nf = m.e2f_ptr[e + 1] - f0;
    for (int i = 0; i < nf; ++i) efphi[f0 + i] = 0.0;
    const double le = e < m.no_edges ? lE[e] : 0.0;
    double c_out = 0.0, r_out = 0.0;
    if (le != 0.0)
    {
        if (mres)
        {
            r_out = mres[e] * le;
            lm[e] += resistive_p0(m, phi, e) * le;
        }
        const int mode = m.edge_mode[e];
        if (mode == 2)
        {
            const V3 t = ld3(m.edge_vec, e);
            atomicAdd(lpar, t.x * le);
            atomicAdd(lpar + 1, t.y * le);
            atomicAdd(lpar + 2, t.z * le);
        }
        else if (mode == 0 && nf > 0 && nf <= MAXV && m.edge_len[e] > 0)
        {
            const int32_t q0 = m.ec_ptr[e], q1 = m.ec_ptr[e + 1];
            bool any_fluid = false;
            for (int32_t k = q0; k < q1 && !any_fluid; ++k) any_fluid = m.material[m.ec_cell[k]] == 0;
            if (any_fluid)
            {
                const double L = m.edge_len[e];
                const V3 t = ld3(m.edge_vec, e);
                const V3 th = (1.0 / L) * t;
                const V3 mid = ld3(m.edge_mid, e);
                const V3 ax = fabs(th.x) < 0.9 ? mk(1, 0, 0) : mk(0, 1, 0);
                V3 e1 = cross(th, ax);
                e1 = (1.0 / sqrt(dot(e1, e1))) * e1;
                const V3 e2 = cross(th, e1);
                double w[MAXV], aef[MAXV], sg[MAXV], qa[MAXV], qb[MAXV], na[MAXV], nb[MAXV], mx[MAXV], my[MAXV], mz[MAXV];
                int arg[MAXV];
                double M11 = 0, M12 = 0, M22 = 0, g1 = 0, g2 = 0;
#pragma unroll
                for (int i = 0; i < MAXV; ++i)
                {
                    if (i >= nf) break;
                    const int32_t f = m.e2f_idx[f0 + i];
                    w[i] = m.ef_weight[f0 + i];
                    V3 v = ld3(m.face_center, f) - mid;
                    v = v - dot(v, th) * th;
                    const double nv = sqrt(dot(v, v));
                    const V3 mi = nv > 0 ? (1.0 / nv) * v : mk(0, 0, 0);
                    const V3 nrm = (1.0 / m.face_area_mag[f]) * ld3(m.face_area, f);
                    double a = 0;
                    int ka = -1;
                    for (int32_t k = q0; k < q1; ++k)
                    {
                        const double x = fabs(dot(ld3(u, m.ec_cell[k]), mi));
                        if (a < x)
                        {
                            a = x;
                            ka = k;
                        }
                    }
                    aef[i] = a;
                    arg[i] = ka;
                    mx[i] = mi.x; my[i] = mi.y; mz[i] = mi.z;
                    sg[i] = dot(th, cross(mi, nrm));
                    const V3 qv = (a * sg[i]) * nrm;
                    qa[i] = dot(qv, e1);
                    qb[i] = dot(qv, e2);
                    na[i] = sg[i] * dot(nrm, e1);
                    nb[i] = sg[i] * dot(nrm, e2);
                    M11 += w[i] * qa[i] * qa[i];
                    M12 += w[i] * qa[i] * qb[i];
                    M22 += w[i] * qb[i] * qb[i];
                    g1 += w[i] * qa[i];
                    g2 += w[i] * qb[i];
                }
                const double tr = M11 + M22;
                const double eps = 1e-14 * tr;
                const double P = M11 + eps, Q = M22 + eps;
                const double det = P * Q - M12 * M12;
                const bool solved = tr > 0 && det > 0;
                double l1 = 0, l2 = 0;
                if (solved)
                {
                    l1 = (Q * g1 - M12 * g2) / det;
                    l2 = (P * g2 - M12 * g1) / det;
                }
                const double lEu = 2.0 * cuct * L * le;
                c_out = le;
                double ll1 = 0, ll2 = 0, lqa[MAXV], lqb[MAXV];
#pragma unroll
                for (int i = 0; i < MAXV; ++i)
                {
                    if (i >= nf) break;
                    const int32_t f = m.e2f_idx[f0 + i];
                    const double A = m.face_area_mag[f];
                    const double phiA = phi[f] / A;
                    const double omega = w[i] * (1.0 - (qa[i] * l1 + qb[i] * l2));
                    const double lom = lEu * aef[i] * sg[i] * phiA;
                    efphi[f0 + i] = lEu * omega * aef[i] * sg[i] / A;
                    aef[i] = lEu * omega * sg[i] * phiA; // from here on: the adjoint of a_ef
                    lqa[i] = -w[i] * l1 * lom;
                    lqb[i] = -w[i] * l2 * lom;
                    ll1 -= w[i] * qa[i] * lom;
                    ll2 -= w[i] * qb[i] * lom;
                }
                if (solved)
                {
                    const double lN1 = ll1 / det, lN2 = ll2 / det, ldet = -(ll1 * l1 + ll2 * l2) / det;
                    const double lP = ldet * Q + lN2 * g2, lQ = ldet * P + lN1 * g1;
                    const double lM12 = -2.0 * M12 * ldet - lN1 * g2 - lN2 * g1;
                    const double lg1 = lN1 * Q - lN2 * M12, lg2 = -lN1 * M12 + lN2 * P;
                    const double leps = lP + lQ;
                    const double lM11 = lP + 1e-14 * leps, lM22 = lQ + 1e-14 * leps;
#pragma unroll
                    for (int i = 0; i < MAXV; ++i)
                    {
                        if (i >= nf) break;
                        lqa[i] += w[i] * (2.0 * qa[i] * lM11 + qb[i] * lM12 + lg1);
                        lqb[i] += w[i] * (2.0 * qb[i] * lM22 + qa[i] * lM12 + lg2);
                    }
                }
#pragma unroll
                for (int i = 0; i < MAXV; ++i)
                {
                    if (i >= nf) break;
                    const double la = aef[i] + na[i] * lqa[i] + nb[i] * lqb[i];
                    if (arg[i] < 0 || la == 0.0) continue;
                    const int32_t c = m.ec_cell[arg[i]];
                    const V3 mi = mk(mx[i], my[i], mz[i]);
                    const double x = dot(ld3(u, c), mi);
                    const double g = (x < 0 ? -la : la);
                    atomicAdd(lup + 3 * (int64_t)c, g * mi.x);
                    atomicAdd(lup + 3 * (int64_t)c + 1, g * mi.y);
                    atomicAdd(lup + 3 * (int64_t)c + 2, g * mi.z);
                }
            }
        }
    }
    lc[e] = c_out;
    lres[e] = r_out;
}

// K2: face adjoint of k_face_candidate.  lEf_f = sum over the face's edges of w_ef lc_e t_e (fw: w_ef by f2e
// entry), then E_f = -n x F back to u, B_tot, B_ind of the face's cells (atomic) and Phi_f; plus the edges'
// upwind (efphi through efpos: the e2f entry of each f2e entry) and resistive (star2 sgn lres) terms.
__global__ void __launch_bounds__(128) k_a_face_cand(MeshView m, const double *__restrict__ u, const double *__restrict__ Bt,
                                                      const double *__restrict__ Bi, const double *__restrict__ phi,
                                                      const double *__restrict__ phi_add, const double *__restrict__ lc,
                                                      const double *__restrict__ fw, const int32_t *__restrict__ efpos,
                                                      const double *__restrict__ efphi, const double *__restrict__ lres,
                                                      double *__restrict__ lup, double *__restrict__ lB, double *__restrict__ lphi)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    V3 lEf = mk(0, 0, 0);
    double lp = 0.0, rsum = 0.0;
    for (int32_t k = m.f2e_ptr[f]; k < m.f2e_ptr[f + 1]; ++k)
    {
        const int32_t e = m.f2e_idx[k];
        const double lce = lc[e];
        if (lce != 0.0) lEf = lEf + (fw[k] * lce) * ld3(m.edge_vec, e);
        if (efpos[k] >= 0) lp += efphi[efpos[k]];
        rsum += m.f2e_sgn[k] * lres[e];
    }
    lp += m.star2[f] * rsum;
    if (lEf.x != 0.0 || lEf.y != 0.0 || lEf.z != 0.0)
    {
        const double A = m.face_area_mag[f];
        const V3 n = (1.0 / A) * ld3(m.face_area, f);
        const double pt = phi_add ? phi[f] + phi_add[f] : phi[f];
        const double Bn = pt / A;
        const V3 lF = cross(n, lEf); // E = -n x F
        double lBn = 0.0;
        auto flux_T = [&](int32_t c, V3 lFX, V3 &lu, V3 &lbt) {
            const V3 uc = ld3(u, c);
            lu = dot(ld3(Bt, c), lFX) * n - Bn * lFX;
            lbt = dot(uc, n) * lFX;
            lBn -= dot(uc, lFX);
        };
        const int32_t p0 = m.f2c_ptr[f], cnt = m.f2c_ptr[f + 1] - p0;
        auto add = [&](double *a, int32_t c, V3 v) {
            atomicAdd(a + 3 * (int64_t)c, v.x);
            atomicAdd(a + 3 * (int64_t)c + 1, v.y);
            atomicAdd(a + 3 * (int64_t)c + 2, v.z);
        };
        if (cnt == 2)
        {
            const int32_t L = m.face_L[f], R = m.face_R[f];
            const double xL = dot(ld3(u, L), n), xR = dot(ld3(u, R), n);
            const bool rwin = fabs(xL) < fabs(xR);
            const double a = rwin ? fabs(xR) : fabs(xL);
            const V3 dBi = ld3(Bi, R) - ld3(Bi, L);
            const V3 half = 0.5 * lF;
            const double la = -0.5 * dot(lF, dBi);
            V3 luL, lbL, luR, lbR;
            flux_T(L, half, luL, lbL);
            flux_T(R, half, luR, lbR);
            const V3 lbi = (0.5 * a) * lF; // d/dBi_L = +a/2 lF, d/dBi_R = -a/2 lF
            if (rwin) luR = luR + ((xR < 0 ? -la : la) * n);
            else luL = luL + ((xL < 0 ? -la : la) * n);
            add(lup, L, luL);
            add(lup, R, luR);
            add(lB, L, lbL + lbi);
            add(lB, R, lbR - lbi);
        }
        else
        {
            const int32_t c = m.f2c_idx[p0];
            V3 lu, lb;
            flux_T(c, lF, lu, lb);
            add(lup, c, lu);
            add(lB, c, lb);
        }
        lp += lBn / A;
    }
    lphi[f] += lp;
}

// K3: per cell, y = I^T lB (cleared afterwards) and the transpose of the charge-weighted ion velocity
// u+ = sum_s chi_s u_s into lW (primitive adjoints; lup cleared afterwards)
__global__ void __launch_bounds__(128) k_a_cell(MeshView m, int nsp, const double *__restrict__ mass, double M_ref,
                                                 const double *__restrict__ W, double *__restrict__ lup, double *__restrict__ lB,
                                                 double *__restrict__ y, double *__restrict__ lW)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int64_t n = m.nc;
    st3(y, c, recon_T(m, c, ld3(lB, c)));
    st3(lB, c, mk(0, 0, 0));
    const V3 lu = ld3(lup, c);
    st3(lup, c, mk(0, 0, 0));
    for (int s = 0; s < nsp; ++s)
        for (int q = 0; q < 5; ++q) lW[ui(s, q, c, n)] = 0.0;
    if (m.material[c] != 0 || (lu.x == 0.0 && lu.y == 0.0 && lu.z == 0.0)) return;
    double ns[kMaxFnSpecies], lchi[kMaxFnSpecies], ne = 0;
    for (int s = 0; s < nsp; ++s)
    {
        ns[s] = dmax(W[ui(s, 0, c, n)], 0.0) / mass[s] * M_ref;
        ne += ns[s];
    }
    double chil = 0;
    for (int s = 0; s < nsp; ++s)
    {
        const double chi = ne > 1e-300 ? ns[s] / ne : (s == 0 ? 1.0 : 0.0);
        const V3 us = mk(W[ui(s, 1, c, n)], W[ui(s, 2, c, n)], W[ui(s, 3, c, n)]);
        lW[ui(s, 1, c, n)] = chi * lu.x;
        lW[ui(s, 2, c, n)] = chi * lu.y;
        lW[ui(s, 3, c, n)] = chi * lu.z;
        lchi[s] = dot(us, lu);
        chil += chi * lchi[s];
    }
    if (ne > 1e-300)
        for (int s = 0; s < nsp; ++s)
            if (W[ui(s, 0, c, n)] >= 0) lW[ui(s, 0, c, n)] = (lchi[s] - chil) / ne / mass[s] * M_ref;
}

// reverse of mhd::rusanov: lF (5, per unit area) -> lL, lR (primitive adjoints of the two face states)
__device__ __forceinline__ void rusanov_T(const Prim5 &L, const Prim5 &R, V3 n, double gamma, const double *lF, double *lL, double *lR)
{
    double UL[5], UR[5];
    auto cons = [&](const Prim5 &W, double *U) {
        U[0] = W.rho; U[1] = W.rho * W.u; U[2] = W.rho * W.v; U[3] = W.rho * W.w;
        U[4] = W.p / (gamma - 1.0) + 0.5 * W.rho * (W.u * W.u + W.v * W.v + W.w * W.w);
    };
    cons(L, UL);
    cons(R, UR);
    const double unL = L.u * n.x + L.v * n.y + L.w * n.z, unR = R.u * n.x + R.v * n.y + R.w * n.z;
    const double cL = sqrt(gamma * L.p / L.rho), cR = sqrt(gamma * R.p / R.rho);
    const double sL = fabs(unL) + cL, sR = fabs(unR) + cR;
    const bool rwin = sL < sR;
    const double s = rwin ? sR : sL;
    double ls = 0;
    for (int q = 0; q < 5; ++q) ls -= 0.5 * lF[q] * (UR[q] - UL[q]);
    auto side = [&](const Prim5 &W, const double *U, double un, double c, double sign_u, bool win, double *lw) {
        // lFX = lF / 2, lUX = -/+ s lF / 2
        double lU[5], lun = 0;
        for (int q = 0; q < 5; ++q) lU[q] = sign_u * 0.5 * s * lF[q];
        const double h0 = 0.5 * lF[0], h1 = 0.5 * lF[1], h2 = 0.5 * lF[2], h3 = 0.5 * lF[3], h4 = 0.5 * lF[4];
        double lr = un * h0 + un * W.u * h1 + un * W.v * h2 + un * W.w * h3;
        lun += W.rho * h0 + W.rho * W.u * h1 + W.rho * W.v * h2 + W.rho * W.w * h3 + (U[4] + W.p) * h4;
        double lu = W.rho * un * h1, lv = W.rho * un * h2, lwv = W.rho * un * h3;
        double lp = n.x * h1 + n.y * h2 + n.z * h3 + un * h4;
        lU[4] += un * h4;
        if (win)
        {
            lun += (un < 0 ? -ls : ls);
            if (c > 0)
            {
                lp += ls * gamma / (2.0 * c * W.rho);
                lr -= ls * gamma * W.p / (2.0 * c * W.rho * W.rho);
            }
        }
        // conservative variables
        lr += lU[0] + W.u * lU[1] + W.v * lU[2] + W.w * lU[3] + 0.5 * (W.u * W.u + W.v * W.v + W.w * W.w) * lU[4];
        lu += W.rho * lU[1] + W.rho * W.u * lU[4];
        lv += W.rho * lU[2] + W.rho * W.v * lU[4];
        lwv += W.rho * lU[3] + W.rho * W.w * lU[4];
        lp += lU[4] / (gamma - 1.0);
        lu += n.x * lun;
        lv += n.y * lun;
        lwv += n.z * lun;
        lw[0] = lr; lw[1] = lu; lw[2] = lv; lw[3] = lwv; lw[4] = lp;
    };
    side(L, UL, unL, cL, 1.0, !rwin, lL);
    side(R, UR, unR, cR, -1.0, rwin, lR);
}

// reverse of mhd::ghost_state with respect to the inside state (lin +=) and the free stream (lfs +=)
__device__ __forceinline__ void ghost_T(int kind, bool absorb, V3 n, const double *lg, double *lin, double *lfs)
{
    if (kind == 1)
    {
        if (absorb) return;
        const double d = lg[1] * n.x + lg[2] * n.y + lg[3] * n.z;
        lin[0] += lg[0];
        lin[1] += lg[1] - 2 * d * n.x;
        lin[2] += lg[2] - 2 * d * n.y;
        lin[3] += lg[3] - 2 * d * n.z;
        lin[4] += lg[4];
        return;
    }
    if (kind == 2)
    {
        for (int q = 0; q < 5; ++q)
            if (lg[q] != 0.0) atomicAdd(lfs + q, lg[q]);
        return;
    }
    for (int q = 0; q < 5; ++q) lin[q] += lg[q];
}

// K4: face adjoint of the flux and its gather, per (face, species): lF = sum over the face's cells of -/+ lrV,
// the reverse Rusanov flux, the ghost state; writes the adjoint of each cell's face state into its slot
// lface[((s*2 + side)*5 + q)*nf + f] (side 0: the cell with c2f sign +1).  Species 0 also adds the cell-fit
// transpose n_f . (y_L + y_R) to lphi.
__global__ void __launch_bounds__(128) k_a_flux(MeshView m, FluidParams p, const double *__restrict__ W, const double *__restrict__ G,
                                                 const double *__restrict__ lrV, double *__restrict__ lface, double *__restrict__ lfs,
                                                 const double *__restrict__ y, double *__restrict__ lphi)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (f >= m.nf || s >= p.nsp) return;
    const int64_t nf = m.nf, n = m.nc;
    if (s == 0) lphi[f] += recon_T_face(m, y, f);
    double *o0 = lface + (int64_t)(s * 2) * 5 * nf + f, *o1 = lface + (int64_t)(s * 2 + 1) * 5 * nf + f;
    const int kind = m.face_kind[f];
    const int32_t p0 = m.f2c_ptr[f], cnt = m.f2c_ptr[f + 1] - p0;
    bool any_owned = false;
    double lF[5] = {0, 0, 0, 0, 0};
    for (int k = 0; k < cnt; ++k)
    {
        const int32_t cc = m.f2c_idx[p0 + k];
        any_owned |= cc < m.no_cells && m.material[cc] == 0;
        const double sg = m.f2c_sgn[p0 + k] > 0 ? -1.0 : 1.0;
        for (int q = 0; q < 5; ++q) lF[q] += sg * lrV[ui(s, q, cc, n)];
    }
    const bool zero = lF[0] == 0.0 && lF[1] == 0.0 && lF[2] == 0.0 && lF[3] == 0.0 && lF[4] == 0.0;
    if (kind == 4 || !any_owned || zero)
    {
        for (int q = 0; q < 5; ++q) o0[q * nf] = o1[q * nf] = 0.0;
        return;
    }
    const double A = m.face_area_mag[f];
    for (int q = 0; q < 5; ++q) lF[q] *= A;
    const V3 nv = (1.0 / A) * ld3(m.face_area, f);
    const V3 xf = ld3(m.face_center, f);
    auto state_of = [&](int32_t cc) {
        const Prim5 w{W[ui(s, 0, cc, n)], W[ui(s, 1, cc, n)], W[ui(s, 2, cc, n)], W[ui(s, 3, cc, n)], W[ui(s, 4, cc, n)]};
        double g[15];
        for (int q = 0; q < 15; ++q) g[q] = G[gi(s, q, cc, n)];
        return face_state(w, g, xf - ld3(m.cell_center, cc));
    };
    double lL[5], lR[5];
    if (cnt == 2 && kind == 0)
    {
        const Prim5 L = state_of(m.face_L[f]), R = state_of(m.face_R[f]);
        rusanov_T(L, R, nv, p.gamma, lF, lL, lR);
        for (int q = 0; q < 5; ++q)
        {
            o0[q * nf] = lL[q];
            o1[q * nf] = lR[q];
        }
        return;
    }
    int32_t c = m.f2c_idx[p0];
    int sgn = m.f2c_sgn[p0];
    if (cnt == 2 && m.material[c] != 0)
    {
        c = m.f2c_idx[p0 + 1];
        sgn = m.f2c_sgn[p0 + 1];
    }
    const Prim5 in = state_of(c);
    const V3 nn = double(sgn) * nv;
    const Prim5 gh = ghost_state(kind, p.absorb[s] != 0, in, nn, p.fs[s]);
    double lin[5], lg[5];
    if (sgn > 0)
    {
        rusanov_T(in, gh, nv, p.gamma, lF, lin, lg);
    }
    else
    {
        rusanov_T(gh, in, nv, p.gamma, lF, lg, lin);
    }
    ghost_T(kind, p.absorb[s] != 0, nn, lg, lin, lfs + 5 * s);
    double *mine = sgn > 0 ? o0 : o1, *other = sgn > 0 ? o1 : o0;
    for (int q = 0; q < 5; ++q)
    {
        mine[q * nf] = lin[q];
        other[q * nf] = 0.0;
    }
}

// K5: per (cell, species): the face-state transpose (lW, lG from the cell's four face slots), then the
// reverse of k_limited_gradients_tet.  lW holds the u+ part on entry and the cell's own total on exit;
// slot[((s*4 + j)*5 + q)*nc + c] receives the adjoint of neighbour j's primitive q as this cell's stencil saw it.
// Every loop over the four slots and five variables is unrolled and the winning slots of the min / max
// terms are selected by predicates, so the per-thread arrays stay in registers.
__global__ void __launch_bounds__(128, 3) k_a_grad(MeshView m, FluidParams p, const double *__restrict__ W, const double *__restrict__ G,
                                                 const double *__restrict__ lface, double *__restrict__ lW, double *__restrict__ slot,
                                                 double *__restrict__ lfs)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (c >= m.nc || s >= p.nsp) return;
    const int64_t n = m.nc, nf = m.nf;
    double wc[5], g[15], lw[5], lG[15];
#pragma unroll
    for (int q = 0; q < 5; ++q)
    {
        wc[q] = W[ui(s, q, c, n)];
        lw[q] = lW[ui(s, q, c, n)];
    }
#pragma unroll
    for (int q = 0; q < 15; ++q)
    {
        g[q] = G[gi(s, q, c, n)];
        lG[q] = 0.0;
    }
    const V3 xc = ld3(m.cell_center, c);
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
        const int32_t f = m.c2f_idx[4 * c + j];
        const int side = m.c2f_sgn[4 * c + j] > 0 ? 0 : 1;
        double lf[5];
        bool any = false;
#pragma unroll
        for (int q = 0; q < 5; ++q)
        {
            lf[q] = lface[((int64_t)(s * 2 + side) * 5 + q) * nf + f];
            any |= lf[q] != 0.0;
        }
        if (!any) continue;
        const V3 dx = ld3(m.face_center, f) - xc;
        // face_state extrapolates unless the extrapolated density or pressure is not positive
        const bool extrap = wc[0] + g[0] * dx.x + g[1] * dx.y + g[2] * dx.z > 0 && wc[4] + g[12] * dx.x + g[13] * dx.y + g[14] * dx.z > 0;
#pragma unroll
        for (int q = 0; q < 5; ++q)
        {
            lw[q] += lf[q];
            if (extrap)
            {
                lG[3 * q] += lf[q] * dx.x;
                lG[3 * q + 1] += lf[q] * dx.y;
                lG[3 * q + 2] += lf[q] * dx.z;
            }
        }
    }
    double lwn[4][5];
    int32_t nb[4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
        nb[j] = m.t_nb[j * n + c];
#pragma unroll
        for (int q = 0; q < 5; ++q) lwn[j][q] = 0.0;
    }
    const bool valid = c < m.no_cells && m.st_valid[c];
    if (valid)
    {
        const Prim5 wcp{wc[0], wc[1], wc[2], wc[3], wc[4]};
        double wn[4][5], wd[12], dxs[12];
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            if (nb[j] >= 0)
            {
#pragma unroll
                for (int q = 0; q < 5; ++q) wn[j][q] = W[ui(s, q, nb[j], n)];
            }
            else if (nb[j] != INT32_MIN)
            {
                const int32_t f = -(nb[j] + 1);
                const V3 nrm = (double(m.t_sg[j * n + c]) / m.face_area_mag[f]) * ld3(m.face_area, f);
                const Prim5 gh = ghost_state(m.face_kind[f], p.absorb[s] != 0, wcp, nrm, p.fs[s]);
                wn[j][0] = gh.rho; wn[j][1] = gh.u; wn[j][2] = gh.v; wn[j][3] = gh.w; wn[j][4] = gh.p;
            }
            else
            {
#pragma unroll
                for (int q = 0; q < 5; ++q) wn[j][q] = 0.0;
            }
        }
#pragma unroll
        for (int i = 0; i < 12; ++i)
        {
            wd[i] = m.t_wd[i * n + c];
            dxs[i] = m.t_dx[i * n + c];
        }
        const double I00 = m.t_inv[c], I01 = m.t_inv[n + c], I02 = m.t_inv[2 * n + c], I11 = m.t_inv[3 * n + c],
                     I12 = m.t_inv[4 * n + c], I22 = m.t_inv[5 * n + c];
#pragma unroll
        for (int q = 0; q < 5; ++q)
        {
            if (lG[3 * q] == 0.0 && lG[3 * q + 1] == 0.0 && lG[3 * q + 2] == 0.0) continue;
            double r0 = 0, r1 = 0, r2 = 0, lo = wc[q], hi = wc[q];
            int jlo = -1, jhi = -1;
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                if (nb[j] == INT32_MIN) continue;
                const double dq = wn[j][q] - wc[q];
                r0 += wd[3 * j] * dq;
                r1 += wd[3 * j + 1] * dq;
                r2 += wd[3 * j + 2] * dq;
                if (wn[j][q] < lo)
                {
                    lo = wn[j][q];
                    jlo = j;
                }
                if (hi < wn[j][q])
                {
                    hi = wn[j][q];
                    jhi = j;
                }
            }
            const double g0 = I00 * r0 + I01 * r1 + I02 * r2;
            const double g1 = I01 * r0 + I11 * r1 + I12 * r2;
            const double g2 = I02 * r0 + I12 * r1 + I22 * r2;
            double psi = 1.0, wdl = 0, wx = 0, wy = 0, wz = 0;
            int wtype = -1; // the limiter term that set psi: 0 hi, 1 lo, 2 relative
            if (p.limit)
            {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    const double d = g0 * dxs[3 * j] + g1 * dxs[3 * j + 1] + g2 * dxs[3 * j + 2];
                    double x = psi;
                    int ty = -1;
                    if (d > 1e-300) { x = (hi - wc[q]) / d; ty = 0; }
                    else if (d < -1e-300) { x = (lo - wc[q]) / d; ty = 1; }
                    if (ty >= 0 && x < psi)
                    {
                        psi = x; wtype = ty; wdl = d;
                        wx = dxs[3 * j]; wy = dxs[3 * j + 1]; wz = dxs[3 * j + 2];
                    }
                }
                if (p.rel_limit > 0 && (q == 0 || q == 4))
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                    {
                        const double d = g0 * dxs[3 * j] + g1 * dxs[3 * j + 1] + g2 * dxs[3 * j + 2];
                        const double da = fabs(d);
                        if (da > 1e-300)
                        {
                            const double x = p.rel_limit * wc[q] / da;
                            if (x < psi)
                            {
                                psi = x; wtype = 2; wdl = d;
                                wx = dxs[3 * j]; wy = dxs[3 * j + 1]; wz = dxs[3 * j + 2];
                            }
                        }
                    }
            }
            const double ps = dmax(0.0, dmin(1.0, psi));
            double lg0 = ps * lG[3 * q], lg1 = ps * lG[3 * q + 1], lg2 = ps * lG[3 * q + 2];
            double lwc = 0, lhi = 0, llo = 0;
            if (psi < 1.0 && 0.0 < psi && wtype >= 0)
            {
                const double lpsi = lG[3 * q] * g0 + lG[3 * q + 1] * g1 + lG[3 * q + 2] * g2;
                double ldl;
                if (wtype == 2)
                {
                    const double da = fabs(wdl);
                    lwc += p.rel_limit * lpsi / da;
                    ldl = -psi * lpsi / da * (wdl < 0 ? -1.0 : 1.0);
                }
                else
                {
                    if (wtype == 0) lhi += lpsi / wdl;
                    else llo += lpsi / wdl;
                    lwc -= lpsi / wdl;
                    ldl = -psi * lpsi / wdl;
                }
                lg0 += ldl * wx;
                lg1 += ldl * wy;
                lg2 += ldl * wz;
            }
            if (jhi < 0) lwc += lhi;
            if (jlo < 0) lwc += llo;
            const double lr0 = I00 * lg0 + I01 * lg1 + I02 * lg2;
            const double lr1 = I01 * lg0 + I11 * lg1 + I12 * lg2;
            const double lr2 = I02 * lg0 + I12 * lg1 + I22 * lg2;
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                double a = (j == jhi ? lhi : 0.0) + (j == jlo ? llo : 0.0);
                if (nb[j] != INT32_MIN)
                {
                    const double d = wd[3 * j] * lr0 + wd[3 * j + 1] * lr1 + wd[3 * j + 2] * lr2;
                    a += d;
                    lwc -= d;
                }
                lwn[j][q] += a;
            }
            lw[q] += lwc;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (nb[j] < 0 && nb[j] != INT32_MIN)
            {
                const int32_t f = -(nb[j] + 1);
                const V3 nrm = (double(m.t_sg[j * n + c]) / m.face_area_mag[f]) * ld3(m.face_area, f);
                ghost_T(m.face_kind[f], p.absorb[s] != 0, nrm, lwn[j], lw, lfs + 5 * s);
            }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 0; q < 5; ++q) slot[((int64_t)(s * 4 + j) * 5 + q) * n + c] = nb[j] >= 0 ? lwn[j][q] : 0.0;
#pragma unroll
    for (int q = 0; q < 5; ++q) lW[ui(s, q, c, n)] = lw[q];
}

// K6: per cell: lW + the neighbours' stencil slots pointing here (rslot: the slot of neighbour j that holds
// this cell, -1 if none), then the reverse of to_prim into lU (+=)
__global__ void __launch_bounds__(128) k_a_prim(MeshView m, FluidParams p, const double *__restrict__ U, const double *__restrict__ lW,
                                                 const double *__restrict__ slot, const int8_t *__restrict__ rslot, double *__restrict__ lU)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (c >= m.nc || s >= p.nsp) return;
    const int64_t n = m.nc;
    double l[5];
    for (int q = 0; q < 5; ++q) l[q] = lW[ui(s, q, c, n)];
    for (int j = 0; j < 4; ++j)
    {
        const int32_t nb = m.t_nb[j * n + c];
        const int r = rslot[j * n + c];
        if (nb < 0 || r < 0) continue;
        for (int q = 0; q < 5; ++q) l[q] += slot[((int64_t)(s * 4 + r) * 5 + q) * n + nb];
    }
    const double U0 = U[ui(s, 0, c, n)], U1 = U[ui(s, 1, c, n)], U2 = U[ui(s, 2, c, n)], U3 = U[ui(s, 3, c, n)], U4 = U[ui(s, 4, c, n)];
    const double rho = dmax(U0, p.rho_floor);
    const double u = U1 / rho, v = U2 / rho, w = U3 / rho;
    const double ke = 0.5 * rho * (u * u + v * v + w * w);
    const double pr = (p.gamma - 1.0) * (U4 - ke);
    double lrho = l[0], lu = l[1], lv = l[2], lw = l[3], lU4 = 0;
    if (!(pr < p.p_floor))
    {
        lU4 = (p.gamma - 1.0) * l[4];
        const double lke = -(p.gamma - 1.0) * l[4];
        lrho += 0.5 * (u * u + v * v + w * w) * lke;
        lu += rho * u * lke;
        lv += rho * v * lke;
        lw += rho * w * lke;
    }
    const double lU1 = lu / rho, lU2 = lv / rho, lU3 = lw / rho;
    lrho -= (lu * u + lv * v + lw * w) / rho;
    const double lU0 = U0 < p.rho_floor ? 0.0 : lrho;
    lU[ui(s, 0, c, n)] += lU0;
    lU[ui(s, 1, c, n)] += lU1;
    lU[ui(s, 2, c, n)] += lU2;
    lU[ui(s, 3, c, n)] += lU3;
    lU[ui(s, 4, c, n)] += lU4;
}

// ---------------------------------------------------------------- setup tables
// fw[k]: w_ef of the f2e entry k (its e2f twin), efpos[k]: that twin's e2f position
__global__ void k_fw_tables(MeshView m, double *__restrict__ fw, int32_t *__restrict__ efpos)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    for (int32_t k = m.f2e_ptr[f]; k < m.f2e_ptr[f + 1]; ++k)
    {
        const int32_t e = m.f2e_idx[k];
        int32_t pos = -1;
        for (int32_t j = m.e2f_ptr[e]; j < m.e2f_ptr[e + 1]; ++j)
            if (m.e2f_idx[j] == f) pos = j;
        efpos[k] = pos;
        fw[k] = pos >= 0 ? m.ef_weight[pos] : 0.0;
    }
}

// rslot[j*nc + c]: the stencil slot of neighbour t_nb[j][c] that points back at c (-1 if none)
__global__ void k_rslot(MeshView m, int8_t *__restrict__ rslot)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int64_t n = m.nc;
    for (int j = 0; j < 4; ++j)
    {
        const int32_t nb = m.t_nb[j * n + c];
        int r = -1;
        if (nb >= 0)
            for (int i = 0; i < 4; ++i)
                if (m.t_nb[i * n + nb] == c) r = i;
        rslot[j * n + c] = (int8_t)r;
    }
}

__global__ void k_active(MeshView m, int8_t *__restrict__ a)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < m.nf) a[f] = face_active(m, f) ? 1 : 0;
}

__global__ void k_scale2(int64_t n, const double *__restrict__ src, double a, double *__restrict__ d1, double b, double *__restrict__ d2)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = src[i];
    d1[i] = a * v;
    if (d2) d2[i] = b * v;
}

__global__ void k_axpy(int64_t n, double a, const double *__restrict__ x, double *__restrict__ y)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) y[i] += a * x[i];
}

__global__ void k_set_scalar(double *p, double v) { *p = v; }

inline int g128(int64_t n) { return grid_for(n, 128); }
inline int g256(int64_t n) { return grid_for(n, 256); }
constexpr int kJBlocks = 296; // 2 x 148 SMs: fixed, so the functional's sum has a fixed order
} // namespace
} // namespace mhd

using namespace mhd;

// kernel classes of the differentiated run, timed with CUDA events while profiling is on
enum FnKernel { FN_FORWARD = 0, FN_RECORD, FN_ADJ_FLOORS, FN_ADJ_EDGE, FN_ADJ_FACE, FN_ADJ_CELL, FN_ADJ_FLUX, FN_ADJ_GRAD, FN_ADJ_PRIM,
                FN_ADJ_MISC, FN_TANGENT, FN_COUNT };
static const char *const kFnKernelNames[FN_COUNT] = {"forward_steps", "record_steps", "adj_floors", "adj_edge_emf", "adj_face_candidate",
                                                     "adj_cell", "adj_face_flux", "adj_limited_gradients", "adj_prim", "adj_misc",
                                                     "tangent_steps"};

struct MhdFn
{
    MhdState *st = nullptr;
    MhdFnParams prm{};
    int nsp = 0;
    double u_inf[3] = {0, 0, 0}, u_create[3] = {0, 0, 0};
    DBuf<double> eta, X0U, X0P;
    DBuf<int8_t> mask, active, rslot;
    DBuf<double> fw;
    DBuf<int32_t> efpos;
    std::vector<std::unique_ptr<DBuf<double>>> ckU, ckP;
    // recorded segment: per step the stage inputs, U~ of stage 2 and the floor flags of both stages
    // a stage's primitives, limited gradients and cell fields, as the stage left them in the state's buffers
    struct StageFields
    {
        DBuf<double> W, G, up, bind, btot;
    };
    struct TapeStep
    {
        DBuf<double> U0, P0, U1, P1, Ut2;
        DBuf<int8_t> fl1, fl2;
        StageFields sf[2];
    };
    std::vector<std::unique_ptr<TapeStep>> tape;
    int tape_seg = -1; // the segment whose steps the tape holds (-1: none)
    mhd::EventProfiler<FN_COUNT> prof;
    // adjoint work arrays
    DBuf<double> lU, lP, lU1, lP1, lUt, lE, lrV, lc, efphi, lres, lm, lup, lB, y, lW, lface, slot, lpar, geta, part, red, phiscratch;
    // tangent arrays
    DBuf<double> deta, dm, tU[3], dU[3], tP[3], dP[3], dW, dG, dF, dup, dbi, dbt, dEf, dE;
    bool forward_done = false;
    double J_hi = 0.0, J_lo = 0.0; // the last J (forward or tangent run) as the double-double hi + lo
    bool J_valid = false;
    // switch log of the forward run (mhd_gpu_fn_switch_log): limiter, flux, edge, floor and face-EMF hashes
    DBuf<uint32_t> sw[5];
    bool sw_on = false;
    double *pinned = nullptr;
    ~MhdFn()
    {
        if (pinned) cudaFreeHost(pinned);
    }
};

namespace mhd
{
namespace
{
cudaStream_t stream_of(MhdFn *fn) { return fn->st->mesh->stream; }

void fill_zero(DBuf<double> &b, cudaStream_t s)
{
    if (b.n) MHD_CUDA(cudaMemsetAsync(b.p, 0, b.n * sizeof(double), s));
}

void set_dt(MhdFn *fn)
{
    k_set_scalar<<<1, 1, 0, stream_of(fn)>>>(fn->st->scal.p, fn->prm.dt);
    MHD_LAUNCH_CHECK();
}

void apply_params(MhdFn *fn)
{
    MhdState *st = fn->st;
    for (int s = 0; s < fn->nsp; ++s)
    {
        st->fp.fs[s].u = fn->u_inf[0];
        st->fp.fs[s].v = fn->u_inf[1];
        st->fp.fs[s].w = fn->u_inf[2];
        st->prm.fs[s].u = fn->u_inf[0];
        st->prm.fs[s].v = fn->u_inf[1];
        st->prm.fs[s].w = fn->u_inf[2];
    }
    for (int a = 0; a < 3; ++a) st->prm.u_inf[a] = fn->u_inf[a];
    const MeshView &m = st->mesh->v;
    if (m.ne) k_eta_to_m<<<g256(m.ne), 256, 0, stream_of(fn)>>>(m, fn->eta.p, st->mres.p);
    MHD_LAUNCH_CHECK();
}

// J (and its tangent when dphi is given) of the face flux phi
void functional(MhdFn *fn, const double *phi, const double *dphi, double *J, double *dJ)
{
    MhdState *st = fn->st;
    const MeshView &m = st->mesh->v;
    cudaStream_t s = stream_of(fn);
    fn->part.alloc(3 * kJBlocks);
    fn->red.alloc(3);
    if (!dphi)
    {
        fn->phiscratch.alloc(m.nf);
        fill_zero(fn->phiscratch, s);
        dphi = fn->phiscratch.p;
    }
    k_J_partial<<<kJBlocks, 256, 0, s>>>(m, DCPtr{phi, dphi}, st->badd.p, fn->mask.p, fn->part.p);
    k_sum_final<<<1, 1, 0, s>>>(fn->part.p, kJBlocks, fn->red.p);
    MHD_LAUNCH_CHECK();
    MHD_CUDA(cudaMemcpyAsync(fn->pinned, fn->red.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    MHD_CUDA(cudaStreamSynchronize(s));
    *J = fn->J_hi = fn->pinned[0];
    fn->J_lo = fn->pinned[2];
    fn->J_valid = true;
    if (dJ) *dJ = fn->pinned[1];
}

void copy_d(double *dst, const double *src, size_t n, cudaStream_t s)
{
    if (n) MHD_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
}

// u_inf - u_inf at creation (the shift of the initial flow)
V3 flow_shift(MhdFn *fn)
{
    return mk(fn->u_inf[0] - fn->u_create[0], fn->u_inf[1] - fn->u_create[1], fn->u_inf[2] - fn->u_create[2]);
}

// the run's initial state (and its tangent along du) into U, Phi
void initial_state(MhdFn *fn, double *U, double *P, const double *du, double *dU)
{
    MhdState *st = fn->st;
    const MeshView &m = st->mesh->v;
    cudaStream_t s = stream_of(fn);
    const size_t nU = 5 * (size_t)fn->nsp * m.nc;
    copy_d(P, fn->X0P.p, m.nf, s);
    if (fn->prm.uniform_flow && m.nc)
    {
        const V3 d = du ? mk(du[0], du[1], du[2]) : mk(0, 0, 0);
        k_init_flow<<<dim3(g128(m.nc), fn->nsp), 128, 0, s>>>(m, st->fp, fn->X0U.p, flow_shift(fn), d, U, dU);
        MHD_LAUNCH_CHECK();
    }
    else
    {
        copy_d(U, fn->X0U.p, nU, s);
        if (dU && nU) MHD_CUDA(cudaMemsetAsync(dU, 0, nU * sizeof(double), s));
    }
}

// forward step on the state's buffers (in place on st->U0, st->phi0), flags optional
void plain_step(MhdFn *fn)
{
    MhdState *st = fn->st;
    st->floor_flags = nullptr;
    fp64_stage(st, st->U0.p, st->phi0.p, st->U1.p, st->phi1.p, false);
    fp64_stage(st, st->U1.p, st->phi1.p, st->U0.p, st->phi0.p, true);
}

// ---------------------------------------------------------------- tangent-linear stage
struct TanBufs
{
    const double *U, *dUv;  // stage input
    const double *P, *dPv;
    double *Uo, *dUo;       // U~ (no average)
    double *Po, *dPo;       // Phi out (no average)
};

FsTan fs_tangent(MhdFn *fn, const double *du)
{
    FsTan t{};
    for (int s = 0; s < fn->nsp; ++s)
        for (int a = 0; a < 3; ++a) t.d[s][1 + a] = du ? du[a] : 0.0;
    return t;
}

void tangent_stage(MhdFn *fn, const TanBufs &b, const double *du)
{
    MhdState *st = fn->st;
    const MeshView &m = st->mesh->v;
    cudaStream_t s = stream_of(fn);
    const int64_t nc = m.nc;
    const FsTan ft = fs_tangent(fn, du);
    const int nsp = fn->nsp;
    if (nc)
    {
        k_t_prepare<<<g128(nc), 128, 0, s>>>(m, st->fp, st->mass.p, st->prm.M_ref, DCPtr{b.U, b.dUv}, DPtr{st->W.p, fn->dW.p},
                                             DCPtr{b.P, b.dPv}, st->badd.p, DPtr{st->bind.p, fn->dbi.p}, DPtr{st->btot.p, fn->dbt.p},
                                             DPtr{st->up.p, fn->dup.p});
        if (st->prm.second_order)
            k_t_grad<<<dim3(g128(nc), nsp), 128, 0, s>>>(m, st->fp, ft, DCPtr{st->W.p, fn->dW.p}, DPtr{st->grad.p, fn->dG.p});
        else
        {
            MHD_CUDA(cudaMemsetAsync(st->grad.p, 0, 15 * nc * nsp * sizeof(double), s));
            MHD_CUDA(cudaMemsetAsync(fn->dG.p, 0, 15 * nc * nsp * sizeof(double), s));
        }
    }
    if (m.nf)
        k_t_flux<<<dim3(g128(m.nf), nsp), 128, 0, s>>>(m, st->fp, ft, DCPtr{st->W.p, fn->dW.p}, DCPtr{st->grad.p, fn->dG.p},
                                                        DPtr{st->F.p, fn->dF.p});
    if (nc)
        k_t_update<<<dim3(g128(nc), nsp), 128, 0, s>>>(m, st->fp, DCPtr{st->F.p, fn->dF.p}, DCPtr{b.U, b.dUv}, DPtr{b.Uo, b.dUo},
                                                        fn->prm.dt);
    if (m.nf)
        k_t_face_cand<<<g128(m.nf), 128, 0, s>>>(m, DCPtr{st->up.p, fn->dup.p}, DCPtr{st->btot.p, fn->dbt.p},
                                                  DCPtr{st->bind.p, fn->dbi.p}, DCPtr{b.P, b.dPv}, st->phi_add.p,
                                                  DPtr{st->Ef.p, fn->dEf.p});
    const V3 ui = mk(st->prm.u_inf[0], st->prm.u_inf[1], st->prm.u_inf[2]), bi = mk(st->prm.B_imf[0], st->prm.B_imf[1], st->prm.B_imf[2]);
    const V3 dui = du ? mk(du[0], du[1], du[2]) : mk(0, 0, 0);
    const V3 Ev = -1.0 * cross(ui, bi), Ed = -1.0 * cross(dui, bi);
    const DV3 Einf{{Ev.x, Ed.x}, {Ev.y, Ed.y}, {Ev.z, Ed.z}};
    if (m.ne)
    {
        const DCPtr mr{st->mres.n ? st->mres.p : nullptr, fn->dm.p};
        if (m.max_valence <= 8)
            k_t_edge<8><<<g128(m.ne), 128, 0, s>>>(m, DCPtr{st->Ef.p, fn->dEf.p}, DCPtr{st->up.p, fn->dup.p}, DCPtr{b.P, b.dPv},
                                                    st->prm.cuct, Einf, mr, DPtr{st->E.p, fn->dE.p});
        else
            k_t_edge<kMaxValence><<<g128(m.ne), 128, 0, s>>>(m, DCPtr{st->Ef.p, fn->dEf.p}, DCPtr{st->up.p, fn->dup.p},
                                                              DCPtr{b.P, b.dPv}, st->prm.cuct, Einf, mr, DPtr{st->E.p, fn->dE.p});
    }
    if (m.nf && b.Po)
        k_t_ct<<<g256(m.nf), 256, 0, s>>>(m, DCPtr{st->E.p, fn->dE.p}, DCPtr{b.P, b.dPv}, DPtr{b.Po, b.dPo}, fn->prm.dt);
    MHD_LAUNCH_CHECK();
}

// ---------------------------------------------------------------- adjoint stage
// Reverse of (U~, E) = stage(U_in, Phi_in) at the primitives / gradients / cell fields already in st's
// buffers for that input.  lUt, lE: adjoints of U~ and E (lUt is read, lE consumed); lUin, lPin += the
// input adjoints; parameter adjoints accumulate in fn->lm and fn->lpar.
void adjoint_stage(MhdFn *fn, const double *Uin, const double *Pin, const double *Ut, const int8_t *flags, const double *lUt,
                   double *lUin, double *lPin)
{
    MhdState *st = fn->st;
    const MeshView &m = st->mesh->v;
    cudaStream_t s = stream_of(fn);
    const int64_t nc = m.nc;
    const int nsp = fn->nsp;
    auto &P = fn->prof;
    if (nc)
    {
        P.begin(FN_ADJ_FLOORS, s);
        k_a_floors<<<dim3(g128(nc), nsp), 128, 0, s>>>(m, st->fp, flags, Ut, lUt, fn->prm.dt, fn->lrV.p, lUin);
        P.end(FN_ADJ_FLOORS, s);
    }
    if (m.ne)
    {
        const double *mr = st->mres.n ? st->mres.p : nullptr;
        P.begin(FN_ADJ_EDGE, s);
        if (m.max_valence <= 8)
            k_a_edge<8><<<g128(m.ne), 128, 0, s>>>(m, st->up.p, Pin, st->prm.cuct, mr, fn->lE.p, fn->lc.p, fn->efphi.p, fn->lres.p,
                                                    fn->lm.p, fn->lpar.p, fn->lup.p);
        else
            k_a_edge<kMaxValence><<<g128(m.ne), 128, 0, s>>>(m, st->up.p, Pin, st->prm.cuct, mr, fn->lE.p, fn->lc.p, fn->efphi.p,
                                                              fn->lres.p, fn->lm.p, fn->lpar.p, fn->lup.p);
        P.end(FN_ADJ_EDGE, s);
    }
    if (m.nf)
    {
        P.begin(FN_ADJ_FACE, s);
        k_a_face_cand<<<g128(m.nf), 128, 0, s>>>(m, st->up.p, st->btot.p, st->bind.p, Pin, st->phi_add.p, fn->lc.p, fn->fw.p,
                                                  fn->efpos.p, fn->efphi.p, fn->lres.p, fn->lup.p, fn->lB.p, lPin);
        P.end(FN_ADJ_FACE, s);
    }
    if (nc)
    {
        P.begin(FN_ADJ_CELL, s);
        k_a_cell<<<g128(nc), 128, 0, s>>>(m, nsp, st->mass.p, st->prm.M_ref, st->W.p, fn->lup.p, fn->lB.p, fn->y.p, fn->lW.p);
        P.end(FN_ADJ_CELL, s);
    }
    if (m.nf)
    {
        P.begin(FN_ADJ_FLUX, s);
        k_a_flux<<<dim3(g128(m.nf), nsp), 128, 0, s>>>(m, st->fp, st->W.p, st->grad.p, fn->lrV.p, fn->lface.p, fn->lpar.p + 3, fn->y.p,
                                                        lPin);
        P.end(FN_ADJ_FLUX, s);
    }
    if (nc)
    {
        P.begin(FN_ADJ_GRAD, s);
        k_a_grad<<<dim3(g128(nc), nsp), 128, 0, s>>>(m, st->fp, st->W.p, st->grad.p, fn->lface.p, fn->lW.p, fn->slot.p, fn->lpar.p + 3);
        P.end(FN_ADJ_GRAD, s);
        P.begin(FN_ADJ_PRIM, s);
        k_a_prim<<<dim3(g128(nc), nsp), 128, 0, s>>>(m, st->fp, Uin, fn->lW.p, fn->slot.p, fn->rslot.p, lUin);
        P.end(FN_ADJ_PRIM, s);
    }
    MHD_LAUNCH_CHECK();
}

// exchange the state's stage buffers with a recorded set (equal sizes: ownership stays consistent)
void swap_fields(MhdState *st, MhdFn::StageFields &f)
{
    std::swap(st->W.p, f.W.p);
    std::swap(st->grad.p, f.G.p);
    std::swap(st->up.p, f.up.p);
    std::swap(st->bind.p, f.bind.p);
    std::swap(st->btot.p, f.btot.p);
}

void alloc_step(MhdFn *fn, MhdFn::TapeStep &T)
{
    const MeshView &m = fn->st->mesh->v;
    const size_t nc = m.nc, nf = m.nf, nU = 5 * (size_t)fn->nsp * nc;
    T.U0.alloc(nU); T.P0.alloc(nf); T.U1.alloc(nU); T.P1.alloc(nf); T.Ut2.alloc(nU);
    T.fl1.alloc(fn->nsp * nc); T.fl2.alloc(fn->nsp * nc);
    for (auto &f : T.sf)
    {
        f.W.alloc(fn->st->W.n); f.G.alloc(fn->st->grad.n); f.up.alloc(3 * nc); f.bind.alloc(3 * nc); f.btot.alloc(3 * nc);
    }
}

// one step from (T.U0, T.P0), recording both stages' inputs, floor flags and fields; the step's result
// (the SSP-RK2 average) goes to (Uout, Pout).  Bit-identical to the plain step.
void record_step(MhdFn *fn, MhdFn::TapeStep &T, double *Uout, double *Pout)
{
    MhdState *st = fn->st;
    const MeshView &m = st->mesh->v;
    cudaStream_t s = stream_of(fn);
    const size_t nU = 5 * (size_t)fn->nsp * m.nc, nf = m.nf;
    swap_fields(st, T.sf[0]);
    st->floor_flags = T.fl1.p;
    fp64_stage(st, T.U0.p, T.P0.p, T.U1.p, T.P1.p, false);
    swap_fields(st, T.sf[0]);
    swap_fields(st, T.sf[1]);
    st->floor_flags = T.fl2.p;
    fp64_stage(st, T.U1.p, T.P1.p, T.Ut2.p, st->phi1.p, false);
    swap_fields(st, T.sf[1]);
    st->floor_flags = nullptr;
    copy_d(Uout, T.U0.p, nU, s);
    copy_d(Pout, T.P0.p, nf, s);
    if (nU) k_average<<<g256(nU), 256, 0, s>>>(nU, T.Ut2.p, Uout, nullptr, nullptr);
    if (nf) k_average<<<g256(nf), 256, 0, s>>>(nf, st->phi1.p, Pout, nullptr, nullptr);
    MHD_LAUNCH_CHECK();
}

// steps [n0, n1) from (U, P), recorded in the tape; the result of the last goes to (Uend, Pend)
void record_segment(MhdFn *fn, int n0, int n1, const double *U, const double *P, double *Uend, double *Pend)
{
    MhdState *st = fn->st;
    const MeshView &m = st->mesh->v;
    cudaStream_t s = stream_of(fn);
    const size_t nU = 5 * (size_t)fn->nsp * m.nc;
    while ((int)fn->tape.size() < n1 - n0) fn->tape.emplace_back(new MhdFn::TapeStep);
    for (int n = n0; n < n1; ++n) alloc_step(fn, *fn->tape[n - n0]);
    copy_d(fn->tape[0]->U0.p, U, nU, s);
    copy_d(fn->tape[0]->P0.p, P, m.nf, s);
    for (int n = n0; n < n1; ++n)
    {
        MhdFn::TapeStep &T = *fn->tape[n - n0];
        const bool last = n + 1 == n1;
        record_step(fn, T, last ? Uend : fn->tape[n + 1 - n0]->U0.p, last ? Pend : fn->tape[n + 1 - n0]->P0.p);
    }
}

void alloc_adjoint(MhdFn *fn)
{
    const MeshView &m = fn->st->mesh->v;
    const size_t nc = m.nc, nf = m.nf, ne = m.ne, ns = fn->nsp;
    fn->lU.alloc(5 * ns * nc); fn->lU1.alloc(5 * ns * nc); fn->lUt.alloc(5 * ns * nc); fn->lrV.alloc(5 * ns * nc);
    fn->lP.alloc(nf); fn->lP1.alloc(nf);
    fn->lE.alloc(ne); fn->lc.alloc(ne); fn->lres.alloc(ne); fn->lm.alloc(ne);
    fn->lup.alloc(3 * nc); fn->lB.alloc(3 * nc); fn->y.alloc(3 * nc); fn->lW.alloc(5 * ns * nc);
    fn->lface.alloc(10 * ns * nf); fn->slot.alloc(20 * ns * nc); fn->lpar.alloc(3 + 5 * ns + 3); fn->geta.alloc(nc);
    cudaStream_t s = stream_of(fn);
    if (nc)
    {
        MHD_CUDA(cudaMemsetAsync(fn->lup.p, 0, 3 * nc * sizeof(double), s));
        MHD_CUDA(cudaMemsetAsync(fn->lB.p, 0, 3 * nc * sizeof(double), s));
    }
}

void alloc_tangent(MhdFn *fn)
{
    const MeshView &m = fn->st->mesh->v;
    const size_t nc = m.nc, nf = m.nf, ne = m.ne, ns = fn->nsp;
    for (int i = 0; i < 3; ++i)
    {
        fn->tU[i].alloc(5 * ns * nc); fn->dU[i].alloc(5 * ns * nc);
        fn->tP[i].alloc(nf); fn->dP[i].alloc(nf);
    }
    fn->dW.alloc(5 * ns * nc); fn->dG.alloc(15 * ns * nc); fn->dF.alloc(5 * ns * nf);
    fn->dup.alloc(3 * nc); fn->dbi.alloc(3 * nc); fn->dbt.alloc(3 * nc); fn->dEf.alloc(3 * nf); fn->dE.alloc(ne);
    fn->dm.alloc(ne); fn->deta.alloc(nc);
}

void finish_gradient(MhdFn *fn, double *grad_eta, double *grad_u)
{
    MhdState *st = fn->st;
    const MeshView &m = st->mesh->v;
    cudaStream_t s = stream_of(fn);
    fill_zero(fn->geta, s);
    if (m.ne) k_m_to_eta<<<g256(m.ne), 256, 0, s>>>(m, fn->lm.p, fn->geta.p);
    MHD_LAUNCH_CHECK();
    std::vector<double> par(3 + 5 * fn->nsp + 3);
    MHD_CUDA(cudaMemcpyAsync(par.data(), fn->lpar.p, par.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (grad_eta && m.nc) MHD_CUDA(cudaMemcpyAsync(grad_eta, fn->geta.p, (size_t)m.nc * sizeof(double), cudaMemcpyDeviceToHost, s));
    MHD_CUDA(cudaStreamSynchronize(s));
    if (grad_u)
    {
        // E_inf = -u x B_imf: d(E_inf . a)/du = -(B_imf x a)
        const V3 a = mk(par[0], par[1], par[2]), b = mk(st->prm.B_imf[0], st->prm.B_imf[1], st->prm.B_imf[2]);
        const V3 g = -1.0 * cross(b, a);
        grad_u[0] = g.x; grad_u[1] = g.y; grad_u[2] = g.z;
        for (int sp = 0; sp < fn->nsp; ++sp)
            for (int q = 0; q < 3; ++q) grad_u[q] += par[3 + 5 * sp + 1 + q];
        for (int q = 0; q < 3; ++q) grad_u[q] += par[3 + 5 * fn->nsp + q]; // the initial free stream
    }
}
} // namespace
} // namespace mhd

extern "C" {

int mhd_gpu_state_set_resistivity(MhdState *st, const double *m_edge)
{
    return guarded([&] {
        MHD_REQUIRE(st, "null state");
        if (!m_edge)
        {
            st->mres.release();
            return;
        }
        MHD_REQUIRE(!st->mixed, "the explicit resistive EMF is part of the FP64 step");
        const MeshView &m = st->mesh->v;
        st->mres.alloc(m.ne);
        if (m.ne) MHD_CUDA(cudaMemcpy(st->mres.p, m_edge, (size_t)m.ne * sizeof(double), cudaMemcpyHostToDevice));
    });
}

int mhd_gpu_fn_create(MhdState *st, const MhdFnParams *p, const double *eta, const int8_t *mask, MhdFn **out)
{
    MhdFn *fn = nullptr;
    int rc = guarded([&] {
        MHD_REQUIRE(st && p && eta && mask && out, "null argument");
        const MeshView &m = st->mesh->v;
        MHD_REQUIRE(!st->mixed, "the differentiated run is FP64");
        MHD_REQUIRE(!st->fp.wall_slot, "the differentiated run has no Dirichlet wall table");
        MHD_REQUIRE(!st->src.any(), "the differentiated run has no model sources (lorentz, ambipolar and chemistry must be 0)");
        MHD_REQUIRE(st->nsp <= kMaxFnSpecies, "the differentiated run supports one or two species");
        MHD_REQUIRE(m.faces_per_cell == 4, "the differentiated run needs a tetrahedral mesh");
        MHD_REQUIRE(p->n_steps >= 1 && p->checkpoint_every >= 1 && p->dt > 0, "need n_steps >= 1, checkpoint_every >= 1, dt > 0");
        fn = new MhdFn;
        fn->st = st;
        fn->prm = *p;
        fn->nsp = st->nsp;
        for (int a = 0; a < 3; ++a) fn->u_inf[a] = fn->u_create[a] = st->prm.u_inf[a];
        cudaStream_t s = st->mesh->stream;
        const size_t nc = m.nc, nf = m.nf, ne = m.ne;
        fn->eta.upload(eta, nc);
        fn->mask.upload(mask, nc);
        fn->X0U.alloc(5 * fn->nsp * nc);
        fn->X0P.alloc(nf);
        copy_d(fn->X0U.p, st->U0.p, 5 * fn->nsp * nc, s);
        copy_d(fn->X0P.p, st->phi0.p, nf, s);
        st->mres.alloc(ne);
        fn->active.alloc(nf);
        fn->rslot.alloc(4 * nc);
        // f2e entries: as many as the e2f entries
        int32_t nent = 0;
        if (nf) MHD_CUDA(cudaMemcpy(&nent, m.f2e_ptr + nf, sizeof(int32_t), cudaMemcpyDeviceToHost));
        fn->fw.alloc(nent);
        fn->efpos.alloc(nent);
        fn->efphi.alloc(nent);
        if (nf)
        {
            k_active<<<g256(nf), 256, 0, s>>>(m, fn->active.p);
            k_fw_tables<<<g256(nf), 256, 0, s>>>(m, fn->fw.p, fn->efpos.p);
        }
        if (nc) k_rslot<<<g256(nc), 256, 0, s>>>(m, fn->rslot.p);
        MHD_LAUNCH_CHECK();
        MHD_CUDA(cudaMallocHost(&fn->pinned, 4 * sizeof(double)));
        apply_params(fn);
        MHD_CUDA(cudaStreamSynchronize(s));
        *out = fn;
    });
    if (rc != MHD_OK) delete fn;
    return rc;
}

int mhd_gpu_fn_destroy(MhdFn *fn)
{
    return guarded([&] {
        if (!fn) return;
        cudaStreamSynchronize(stream_of(fn));
        delete fn;
    });
}

int mhd_gpu_fn_set_params(MhdFn *fn, const double *eta, const double *u_inf)
{
    return guarded([&] {
        MHD_REQUIRE(fn, "null function");
        const MeshView &m = fn->st->mesh->v;
        if (eta && m.nc) MHD_CUDA(cudaMemcpy(fn->eta.p, eta, (size_t)m.nc * sizeof(double), cudaMemcpyHostToDevice));
        if (u_inf)
            for (int a = 0; a < 3; ++a) fn->u_inf[a] = u_inf[a];
        apply_params(fn);
        fn->forward_done = false;
        MHD_CUDA(cudaStreamSynchronize(stream_of(fn)));
    });
}

int mhd_gpu_fn_reset(MhdFn *fn)
{
    return guarded([&] {
        MHD_REQUIRE(fn, "null function");
        MhdState *st = fn->st;
        initial_state(fn, st->U0.p, st->phi0.p, nullptr, nullptr);
        MHD_CUDA(cudaStreamSynchronize(stream_of(fn)));
    });
}

namespace mhd
{
namespace
{
// The switch log's arrays on the state's kernels for the duration of one forward run: cleared first, taken
// off the state again however the run ends (the backward sweep's recomputed segments are not logged).
struct SwitchScope
{
    MhdFn *fn;
    explicit SwitchScope(MhdFn *f) : fn(f)
    {
        if (!fn->sw_on) return;
        MhdState *st = fn->st;
        for (auto &b : fn->sw)
            if (b.n) MHD_CUDA(cudaMemsetAsync(b.p, 0, b.n * sizeof(uint32_t), stream_of(fn)));
        st->fp.sw_lim = fn->sw[0].p;
        st->fp.sw_flux = fn->sw[1].p;
        st->sw_edge = fn->sw[2].p;
        st->fp.sw_floor = fn->sw[3].p;
        st->sw_face = fn->sw[4].p;
    }
    ~SwitchScope()
    {
        MhdState *st = fn->st;
        st->fp.sw_lim = st->fp.sw_flux = st->fp.sw_floor = nullptr;
        st->sw_edge = st->sw_face = nullptr;
    }
};

size_t switch_size(const MhdFn *fn, int kind)
{
    const MeshView &m = fn->st->mesh->v;
    const size_t ns = fn->nsp;
    switch (kind)
    {
    case 0: return ns * 5 * m.nc;
    case 1: return ns * m.nf;
    case 2: return m.ne;
    case 4: return m.nf;
    default: return ns * m.nc;
    }
}
} // namespace
} // namespace mhd

int mhd_gpu_fn_switch_log(MhdFn *fn, int32_t enable)
{
    return guarded([&] {
        MHD_REQUIRE(fn, "null function");
        fn->sw_on = enable != 0;
        for (int k = 0; k < 5; ++k)
        {
            if (fn->sw_on) fn->sw[k].alloc(switch_size(fn, k));
            else fn->sw[k].release();
        }
    });
}

int mhd_gpu_fn_switch_read(MhdFn *fn, int32_t kind, uint32_t *out, int64_t n)
{
    return guarded([&] {
        MHD_REQUIRE(fn && out, "null argument");
        MHD_REQUIRE(fn->sw_on, "the switch log is off (mhd_gpu_fn_switch_log)");
        MHD_REQUIRE(kind >= 0 && kind < 5, "kind: 0 limiter, 1 flux, 2 edge, 3 floor, 4 face EMF");
        MHD_REQUIRE(n == (int64_t)switch_size(fn, kind), "n must be the size of the kind's table");
        if (n)
            MHD_CUDA(cudaMemcpyAsync(out, fn->sw[kind].p, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_of(fn)));
        MHD_CUDA(cudaStreamSynchronize(stream_of(fn)));
    });
}

int mhd_gpu_fn_last_J(MhdFn *fn, double *J_hi_lo)
{
    return guarded([&] {
        MHD_REQUIRE(fn && J_hi_lo, "null argument");
        MHD_REQUIRE(fn->J_valid, "no forward or tangent run yet");
        J_hi_lo[0] = fn->J_hi;
        J_hi_lo[1] = fn->J_lo;
    });
}

int mhd_gpu_fn_forward(MhdFn *fn, double *J)
{
    return guarded([&] {
        MHD_REQUIRE(fn && J, "null argument");
        MhdState *st = fn->st;
        const MeshView &m = st->mesh->v;
        cudaStream_t s = stream_of(fn);
        const size_t nU = 5 * (size_t)fn->nsp * m.nc, nf = m.nf;
        const SwitchScope sw_scope(fn);
        apply_params(fn);
        set_dt(fn);
        initial_state(fn, st->U0.p, st->phi0.p, nullptr, nullptr);
        const int K = fn->prm.checkpoint_every, N = fn->prm.n_steps;
        const int nck = (N + K - 1) / K;
        while ((int)fn->ckU.size() < nck)
        {
            fn->ckU.emplace_back(new DBuf<double>);
            fn->ckP.emplace_back(new DBuf<double>);
        }
        // every segment but the last runs plain steps after its checkpoint; the last is recorded for the
        // backward sweep as it runs
        const int last_seg = (N - 1) / K;
        fn->prof.begin(FN_FORWARD, s);
        for (int n = 0; n < last_seg * K; ++n)
        {
            if (n % K == 0)
            {
                const int i = n / K;
                fn->ckU[i]->alloc(nU);
                fn->ckP[i]->alloc(nf);
                copy_d(fn->ckU[i]->p, st->U0.p, nU, s);
                copy_d(fn->ckP[i]->p, st->phi0.p, nf, s);
            }
            plain_step(fn);
        }
        fn->ckU[last_seg]->alloc(nU);
        fn->ckP[last_seg]->alloc(nf);
        copy_d(fn->ckU[last_seg]->p, st->U0.p, nU, s);
        copy_d(fn->ckP[last_seg]->p, st->phi0.p, nf, s);
        fn->prof.end(FN_FORWARD, s);
        fn->prof.begin(FN_RECORD, s);
        record_segment(fn, last_seg * K, N, st->U0.p, st->phi0.p, st->U0.p, st->phi0.p);
        fn->prof.end(FN_RECORD, s);
        fn->tape_seg = last_seg;
        functional(fn, st->phi0.p, nullptr, J, nullptr);
        fn->forward_done = true;
    });
}

int mhd_gpu_fn_backward(MhdFn *fn, double *grad_eta, double *grad_u)
{
    return guarded([&] {
        MHD_REQUIRE(fn, "null function");
        MHD_REQUIRE(fn->forward_done, "backward needs a forward run with the current parameters");
        MhdState *st = fn->st;
        const MeshView &m = st->mesh->v;
        cudaStream_t s = stream_of(fn);
        const int64_t nc = m.nc;
        const size_t nU = 5 * (size_t)fn->nsp * nc, nf = m.nf;
        alloc_adjoint(fn);
        set_dt(fn);
        fill_zero(fn->lm, s);
        fill_zero(fn->lpar, s);
        fill_zero(fn->lU, s);
        fill_zero(fn->lP, s);
        // dJ/dPhi of the final state (st->phi0 holds it after the forward run)
        if (nc)
        {
            k_a_J<<<g128(nc), 128, 0, s>>>(m, st->phi0.p, st->badd.p, fn->mask.p, fn->lB.p);
            k_a_recon_cells<<<g128(nc), 128, 0, s>>>(m, fn->lB.p, fn->y.p);
        }
        if (nf) k_a_recon_faces<<<g256(nf), 256, 0, s>>>(m, fn->y.p, fn->lP.p);
        MHD_LAUNCH_CHECK();
        const int K = fn->prm.checkpoint_every, N = fn->prm.n_steps;
        const double dt = fn->prm.dt;
        for (int seg = (N - 1) / K; seg >= 0; --seg)
        {
            const int n0 = seg * K, n1 = std::min(N, n0 + K);
            if (fn->tape_seg != seg)
            {
                // recompute the segment from its checkpoint, recording it (the end state is not needed)
                fn->prof.begin(FN_RECORD, s);
                fn->phiscratch.alloc(nf);
                record_segment(fn, n0, n1, fn->ckU[seg]->p, fn->ckP[seg]->p, st->U1.p, fn->phiscratch.p);
                fn->prof.end(FN_RECORD, s);
                fn->tape_seg = seg;
            }
            for (int n = n1 - 1; n >= n0; --n)
            {
                MhdFn::TapeStep &T = *fn->tape[n - n0];
                // stage 2: U = (U0 + U~2)/2, Phi = (Phi0 + Phi1 - dt d1 E1)/2
                fn->prof.begin(FN_ADJ_MISC, s);
                if (nU) k_scale2<<<g256(nU), 256, 0, s>>>(nU, fn->lU.p, 0.5, fn->lUt.p, 0.5, fn->lU.p);
                if (m.ne) k_a_ct<<<g256(m.ne), 256, 0, s>>>(m, fn->active.p, fn->lP.p, 0.5 * dt, fn->lE.p);
                if (nf) k_scale2<<<g256(nf), 256, 0, s>>>(nf, fn->lP.p, 0.5, fn->lP1.p, 0.5, fn->lP.p);
                MHD_LAUNCH_CHECK();
                fill_zero(fn->lU1, s);
                fn->prof.end(FN_ADJ_MISC, s);
                swap_fields(st, T.sf[1]);
                adjoint_stage(fn, T.U1.p, T.P1.p, T.Ut2.p, T.fl2.p, fn->lUt.p, fn->lU1.p, fn->lP1.p);
                swap_fields(st, T.sf[1]);
                // stage 1: U1 = U~1, Phi1 = Phi0 - dt d1 E0
                fn->prof.begin(FN_ADJ_MISC, s);
                if (m.ne) k_a_ct<<<g256(m.ne), 256, 0, s>>>(m, fn->active.p, fn->lP1.p, dt, fn->lE.p);
                if (nf) k_axpy<<<g256(nf), 256, 0, s>>>(nf, 1.0, fn->lP1.p, fn->lP.p);
                MHD_LAUNCH_CHECK();
                fn->prof.end(FN_ADJ_MISC, s);
                swap_fields(st, T.sf[0]);
                adjoint_stage(fn, T.U0.p, T.P0.p, T.U1.p, T.fl1.p, fn->lU1.p, fn->lU.p, fn->lP.p);
                swap_fields(st, T.sf[0]);
            }
        }
        if (fn->prm.uniform_flow && nc)
        {
            k_init_flow_T<<<kJBlocks, 256, 0, s>>>(m, st->fp, fn->X0U.p, flow_shift(fn), fn->lU.p, fn->lpar.p + 3 + 5 * fn->nsp);
            MHD_LAUNCH_CHECK();
        }
        finish_gradient(fn, grad_eta, grad_u);
    });
}

int mhd_gpu_fn_tangent(MhdFn *fn, const double *d_eta, const double *d_u, double *J, double *dJ)
{
    return guarded([&] {
        MHD_REQUIRE(fn && J && dJ, "null argument");
        MhdState *st = fn->st;
        const MeshView &m = st->mesh->v;
        cudaStream_t s = stream_of(fn);
        const size_t nU = 5 * (size_t)fn->nsp * m.nc, nf = m.nf;
        alloc_tangent(fn);
        apply_params(fn);
        set_dt(fn);
        if (d_eta && m.nc) MHD_CUDA(cudaMemcpyAsync(fn->deta.p, d_eta, (size_t)m.nc * sizeof(double), cudaMemcpyHostToDevice, s));
        else fill_zero(fn->deta, s);
        if (m.ne) k_eta_to_m<<<g256(m.ne), 256, 0, s>>>(m, fn->deta.p, fn->dm.p);
        MHD_LAUNCH_CHECK();
        initial_state(fn, fn->tU[0].p, fn->tP[0].p, d_u, fn->dU[0].p);
        fill_zero(fn->dP[0], s);
        fill_zero(fn->dP[2], s);
        fn->prof.begin(FN_TANGENT, s);
        for (int n = 0; n < fn->prm.n_steps; ++n)
        {
            tangent_stage(fn, TanBufs{fn->tU[0].p, fn->dU[0].p, fn->tP[0].p, fn->dP[0].p, fn->tU[1].p, fn->dU[1].p, fn->tP[1].p, fn->dP[1].p},
                          d_u);
            tangent_stage(fn, TanBufs{fn->tU[1].p, fn->dU[1].p, fn->tP[1].p, fn->dP[1].p, fn->tU[2].p, fn->dU[2].p, fn->tP[2].p, fn->dP[2].p},
                          d_u);
            // U0 <- (U0 + U~2)/2 etc.: k_average writes a = (b + a)/2, so average into the stage-2 outputs and swap
            if (nU) k_average<<<g256(nU), 256, 0, s>>>(nU, fn->tU[0].p, fn->tU[2].p, fn->dU[0].p, fn->dU[2].p);
            if (nf) k_average<<<g256(nf), 256, 0, s>>>(nf, fn->tP[0].p, fn->tP[2].p, fn->dP[0].p, fn->dP[2].p);
            MHD_LAUNCH_CHECK();
            std::swap(fn->tU[0].p, fn->tU[2].p);
            std::swap(fn->dU[0].p, fn->dU[2].p);
            std::swap(fn->tP[0].p, fn->tP[2].p);
            std::swap(fn->dP[0].p, fn->dP[2].p);
        }
        fn->prof.end(FN_TANGENT, s);
        functional(fn, fn->tP[0].p, fn->dP[0].p, J, dJ);
        // the final state of the tangent run's values, for comparison with the forward run
        copy_d(st->U0.p, fn->tU[0].p, nU, s);
        copy_d(st->phi0.p, fn->tP[0].p, nf, s);
        MHD_CUDA(cudaStreamSynchronize(s));
    });
}

int mhd_gpu_fn_stage_tangent(MhdFn *fn, const double *U, const double *Phi, const double *dU, const double *dPhi, const double *d_eta,
                             const double *d_u, double *dUt, double *dE)
{
    return guarded([&] {
        MHD_REQUIRE(fn && U && Phi && dU && dPhi && dUt && dE, "null argument");
        MhdState *st = fn->st;
        const MeshView &m = st->mesh->v;
        cudaStream_t s = stream_of(fn);
        const size_t nU = 5 * (size_t)fn->nsp * m.nc, nf = m.nf;
        alloc_tangent(fn);
        apply_params(fn);
        set_dt(fn);
        MHD_CUDA(cudaMemcpyAsync(fn->tU[0].p, U, nU * sizeof(double), cudaMemcpyHostToDevice, s));
        MHD_CUDA(cudaMemcpyAsync(fn->dU[0].p, dU, nU * sizeof(double), cudaMemcpyHostToDevice, s));
        MHD_CUDA(cudaMemcpyAsync(fn->tP[0].p, Phi, nf * sizeof(double), cudaMemcpyHostToDevice, s));
        MHD_CUDA(cudaMemcpyAsync(fn->dP[0].p, dPhi, nf * sizeof(double), cudaMemcpyHostToDevice, s));
        if (d_eta && m.nc) MHD_CUDA(cudaMemcpyAsync(fn->deta.p, d_eta, (size_t)m.nc * sizeof(double), cudaMemcpyHostToDevice, s));
        else fill_zero(fn->deta, s);
        if (m.ne) k_eta_to_m<<<g256(m.ne), 256, 0, s>>>(m, fn->deta.p, fn->dm.p);
        tangent_stage(fn, TanBufs{fn->tU[0].p, fn->dU[0].p, fn->tP[0].p, fn->dP[0].p, fn->tU[1].p, fn->dU[1].p, nullptr, nullptr}, d_u);
        MHD_CUDA(cudaMemcpyAsync(dUt, fn->dU[1].p, nU * sizeof(double), cudaMemcpyDeviceToHost, s));
        MHD_CUDA(cudaMemcpyAsync(dE, fn->dE.p, (size_t)m.ne * sizeof(double), cudaMemcpyDeviceToHost, s));
        MHD_CUDA(cudaStreamSynchronize(s));
    });
}

int mhd_gpu_fn_stage_adjoint(MhdFn *fn, const double *U, const double *Phi, const double *lUt, const double *lE, double *lU, double *lPhi,
                             double *l_eta, double *l_u)
{
    return guarded([&] {
        MHD_REQUIRE(fn && U && Phi && lUt && lE && lU && lPhi, "null argument");
        MhdState *st = fn->st;
        const MeshView &m = st->mesh->v;
        cudaStream_t s = stream_of(fn);
        const size_t nU = 5 * (size_t)fn->nsp * m.nc, nf = m.nf;
        alloc_adjoint(fn);
        apply_params(fn);
        set_dt(fn);
        fn->tape.emplace_back(new MhdFn::TapeStep);
        MhdFn::TapeStep &T = *fn->tape.back();
        T.U0.alloc(nU); T.P0.alloc(nf); T.U1.alloc(nU); T.P1.alloc(nf); T.fl1.alloc(fn->nsp * (size_t)m.nc);
        MHD_CUDA(cudaMemcpyAsync(T.U0.p, U, nU * sizeof(double), cudaMemcpyHostToDevice, s));
        MHD_CUDA(cudaMemcpyAsync(T.P0.p, Phi, nf * sizeof(double), cudaMemcpyHostToDevice, s));
        MHD_CUDA(cudaMemcpyAsync(fn->lUt.p, lUt, nU * sizeof(double), cudaMemcpyHostToDevice, s));
        MHD_CUDA(cudaMemcpyAsync(fn->lE.p, lE, (size_t)m.ne * sizeof(double), cudaMemcpyHostToDevice, s));
        fill_zero(fn->lm, s);
        fill_zero(fn->lpar, s);
        fill_zero(fn->lU, s);
        fill_zero(fn->lP, s);
        st->floor_flags = T.fl1.p;
        fp64_stage(st, T.U0.p, T.P0.p, T.U1.p, T.P1.p, false); // leaves the input's primitives, gradients, cell fields
        st->floor_flags = nullptr;
        adjoint_stage(fn, T.U0.p, T.P0.p, T.U1.p, T.fl1.p, fn->lUt.p, fn->lU.p, fn->lP.p);
        MHD_CUDA(cudaMemcpyAsync(lU, fn->lU.p, nU * sizeof(double), cudaMemcpyDeviceToHost, s));
        MHD_CUDA(cudaMemcpyAsync(lPhi, fn->lP.p, nf * sizeof(double), cudaMemcpyDeviceToHost, s));
        fn->tape.pop_back();
        finish_gradient(fn, l_eta, l_u);
    });
}

int mhd_gpu_fn_profile(MhdFn *fn, int32_t enable)
{
    return guarded([&] {
        MHD_REQUIRE(fn, "null function");
        MHD_CUDA(cudaStreamSynchronize(stream_of(fn)));
        fn->prof.on = enable != 0;
        for (auto &u : fn->prof.used) u = 0;
    });
}

int mhd_gpu_fn_profile_read(MhdFn *fn, int32_t max_kernels, char *names, double *ms_total, int64_t *count, int32_t *n_out)
{
    return guarded([&] {
        MHD_REQUIRE(fn && names && ms_total && count && n_out, "null argument");
        MHD_CUDA(cudaStreamSynchronize(stream_of(fn)));
        int n = 0;
        for (int k = 0; k < FN_COUNT && n < max_kernels; ++k, ++n)
        {
            std::strncpy(names + 32 * n, kFnKernelNames[k], 31);
            names[32 * n + 31] = 0;
            fn->prof.read(k, ms_total[n], count[n]);
        }
        *n_out = n;
    });
}

} // extern "C"
