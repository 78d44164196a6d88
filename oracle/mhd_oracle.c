/* CPU restatement of the reference's hot path (TEST INFRASTRUCTURE ONLY; see mhd_oracle.h).
 * Plain C11, the reference's operation order, no fused multiply-add (x86-64 baseline): on the same
 * inputs the results equal the compiled reference's bit for bit, which tests/test_oracle.py checks. */
#include "mhd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double x, y, z; } v3;
static inline v3 mk3(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 ld(const double *a, int64_t i) { return mk3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
static inline v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 scl(double s, v3 a) { return mk3(a.x * s, a.y * s, a.z * s); }
static inline double dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross3(v3 a, v3 b) { return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static inline double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */

/* mhd::to_prim (Common/physics/Euler.h:13-21) */
static OrPrim to_prim1(const double *U, double gamma, double rho_floor, double p_floor)
{
    OrPrim W;
    W.rho = dmax(U[0], rho_floor);
    W.u = U[1] / W.rho; W.v = U[2] / W.rho; W.w = U[3] / W.rho;
    const double ke = 0.5 * W.rho * (W.u * W.u + W.v * W.v + W.w * W.w);
    W.p = dmax((gamma - 1.0) * (U[4] - ke), p_floor);
    return W;
}

/* mhd::to_cons (Euler.h:22-26) */
static void to_cons1(OrPrim W, double gamma, double *U)
{
    U[0] = W.rho; U[1] = W.rho * W.u; U[2] = W.rho * W.v; U[3] = W.rho * W.w;
    U[4] = W.p / (gamma - 1.0) + 0.5 * W.rho * (W.u * W.u + W.v * W.v + W.w * W.w);
}

void or_to_prim(const double *U, int64_t n, double gamma, double rho_floor, double p_floor, double *W)
{
    for (int64_t c = 0; c < n; ++c)
    {
        const OrPrim w = to_prim1(U + 5 * c, gamma, rho_floor, p_floor);
        W[5 * c] = w.rho; W[5 * c + 1] = w.u; W[5 * c + 2] = w.v; W[5 * c + 3] = w.w; W[5 * c + 4] = w.p;
    }
}

/* mhd::ghost_state (Common/fluid/Reconstruction.cpp:9-24); kind 1 wall, 2 inflow */
static OrPrim ghost(int kind, int absorb, OrPrim in, v3 n, OrPrim fs)
{
    if (kind == 1)
    {
        if (absorb) { OrPrim g = {1e-12, 0, 0, 0, 1e-12}; return g; }
        const double un = in.u * n.x + in.v * n.y + in.w * n.z;
        OrPrim g = in;
        g.u -= 2 * un * n.x; g.v -= 2 * un * n.y; g.w -= 2 * un * n.z;
        return g;
    }
    if (kind == 2) return fs;
    return in;
}

static int f2c_count(const OrMesh *m, int32_t f) { return (int)(m->f2c_ptr[f + 1] - m->f2c_ptr[f]); }

/* mhd::Stencil::Stencil + limited_gradients (Common/fluid/Reconstruction.cpp:26-78, :80-142).  The
 * stencil of each cell is rebuilt here with the constructor's arithmetic (the reference keeps it). */
void or_limited_gradients(const OrMesh *m, const double *W, int32_t absorb, const OrPrim *fs, int32_t limit, double rel_limit, double *grad)
{
    memset(grad, 0, sizeof(double) * 15 * (size_t)m->n_cells);
    for (int32_t c = 0; c < m->n_owned_cells; ++c)
    {
        if (m->cell_material[c] == 1) continue;
        const int64_t k0 = m->c2f_ptr[c], k1 = m->c2f_ptr[c + 1];
        double M[3][3] = {{0}}, wk[64], dk[64][3];
        int32_t nbk[64];
        int64_t kk_of[64];
        int ns = 0;
        const v3 xc = ld(m->cell_center, c);
        for (int64_t k = k0; k < k1; ++k)
        {
            const int32_t f = m->c2f_idx[k];
            const int kind = m->face_kind[f];
            if (kind == 4) continue;
            v3 d;
            int32_t nb;
            if (f2c_count(m, f) == 2 && kind == 0)
            {
                const int64_t p0 = m->f2c_ptr[f];
                nb = m->f2c_idx[p0] == c ? m->f2c_idx[p0 + 1] : m->f2c_idx[p0];
                d = sub3(ld(m->cell_center, nb), xc);
            }
            else
            {
                const v3 n = scl(m->c2f_sgn[k] / m->face_area_mag[f], ld(m->face_area, f));
                d = scl(2.0 * dot3(sub3(ld(m->face_center, f), xc), n), n);
                nb = -(f + 1);
            }
            const double w = 1.0 / dot3(d, d);
            nbk[ns] = nb; wk[ns] = w; dk[ns][0] = d.x; dk[ns][1] = d.y; dk[ns][2] = d.z; kk_of[ns] = k;
            ++ns;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) M[a][b] += w * dk[ns - 1][a] * dk[ns - 1][b];
        }
        const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        const double sc = dmax(dmax(dmax(M[0][0], M[1][1]), M[2][2]), 1e-300);
        if (fabs(det) < 1e-9 * sc * sc * sc) continue;
        double I[9];
        I[0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det;
        I[1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
        I[2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det;
        I[3] = I[1];
        I[4] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det;
        I[5] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
        I[6] = I[2];
        I[7] = I[5];
        I[8] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
        const double *wp = W + 5 * (int64_t)c;
        const OrPrim wc = {wp[0], wp[1], wp[2], wp[3], wp[4]};
        const double wcv[5] = {wc.rho, wc.u, wc.v, wc.w, wc.p};
        double r[5][3] = {{0}}, lo[5], hi[5];
        for (int q = 0; q < 5; ++q) lo[q] = hi[q] = wcv[q];
        for (int i = 0; i < ns; ++i)
        {
            OrPrim wn;
            if (nbk[i] >= 0)
            {
                const double *np = W + 5 * (int64_t)nbk[i];
                wn.rho = np[0]; wn.u = np[1]; wn.v = np[2]; wn.w = np[3]; wn.p = np[4];
            }
            else
            {
                const int32_t f = -(nbk[i] + 1);
                const v3 n = scl(m->c2f_sgn[kk_of[i]] / m->face_area_mag[f], ld(m->face_area, f));
                wn = ghost(m->face_kind[f], absorb, wc, n, *fs);
            }
            const double wnv[5] = {wn.rho, wn.u, wn.v, wn.w, wn.p};
            for (int q = 0; q < 5; ++q)
            {
                const double dq = wnv[q] - wcv[q];
                r[q][0] += wk[i] * dk[i][0] * dq; r[q][1] += wk[i] * dk[i][1] * dq; r[q][2] += wk[i] * dk[i][2] * dq;
                lo[q] = dmin(lo[q], wnv[q]);
                hi[q] = dmax(hi[q], wnv[q]);
            }
        }
        for (int q = 0; q < 5; ++q)
        {
            const double g[3] = {I[0] * r[q][0] + I[1] * r[q][1] + I[2] * r[q][2], I[3] * r[q][0] + I[4] * r[q][1] + I[5] * r[q][2],
                                 I[6] * r[q][0] + I[7] * r[q][1] + I[8] * r[q][2]};
            double psi = 1.0;
            if (limit)
                for (int64_t kf = k0; kf < k1; ++kf)
                {
                    const v3 dx = sub3(ld(m->face_center, m->c2f_idx[kf]), xc);
                    const double dl = g[0] * dx.x + g[1] * dx.y + g[2] * dx.z;
                    if (dl > 1e-300) psi = dmin(psi, (hi[q] - wcv[q]) / dl);
                    else if (dl < -1e-300) psi = dmin(psi, (lo[q] - wcv[q]) / dl);
                }
            if (limit && rel_limit > 0 && (q == 0 || q == 4))
                for (int64_t kf = k0; kf < k1; ++kf)
                {
                    const v3 dx = sub3(ld(m->face_center, m->c2f_idx[kf]), xc);
                    const double dl = fabs(g[0] * dx.x + g[1] * dx.y + g[2] * dx.z);
                    if (dl > 1e-300) psi = dmin(psi, rel_limit * wcv[q] / dl);
                }
            psi = dmax(0.0, dmin(1.0, psi));
            double *out = grad + 15 * (int64_t)c + 3 * q;
            out[0] = psi * g[0]; out[1] = psi * g[1]; out[2] = psi * g[2];
        }
    }
}

/* face_state of Common/fluid/FluxRHS.cpp:16-27 */
static OrPrim face_state(const double *W, const double *grad, int32_t c, v3 dx)
{
    const double *w = W + 5 * (int64_t)c, *g = grad + 15 * (int64_t)c;
    OrPrim wc = {w[0], w[1], w[2], w[3], w[4]}, r;
    r.rho = wc.rho + g[0] * dx.x + g[1] * dx.y + g[2] * dx.z;
    r.u = wc.u + g[3] * dx.x + g[4] * dx.y + g[5] * dx.z;
    r.v = wc.v + g[6] * dx.x + g[7] * dx.y + g[8] * dx.z;
    r.w = wc.w + g[9] * dx.x + g[10] * dx.y + g[11] * dx.z;
    r.p = wc.p + g[12] * dx.x + g[13] * dx.y + g[14] * dx.z;
    return (r.rho > 0 && r.p > 0) ? r : wc;
}

/* mhd::rusanov (Common/physics/Euler.h:30-49) */
static void rusanov(OrPrim L, OrPrim R, const double n[3], double gamma, double *F)
{
    double UL[5], UR[5], FL[5], FR[5];
    to_cons1(L, gamma, UL);
    to_cons1(R, gamma, UR);
    const OrPrim *Ws[2] = {&L, &R};
    double *Us[2] = {UL, UR}, *Fs[2] = {FL, FR};
    for (int i = 0; i < 2; ++i)
    {
        const OrPrim W = *Ws[i];
        const double un = W.u * n[0] + W.v * n[1] + W.w * n[2];
        Fs[i][0] = W.rho * un;
        Fs[i][1] = W.rho * un * W.u + W.p * n[0];
        Fs[i][2] = W.rho * un * W.v + W.p * n[1];
        Fs[i][3] = W.rho * un * W.w + W.p * n[2];
        Fs[i][4] = un * (Us[i][4] + W.p);
    }
    const double sL = fabs(L.u * n[0] + L.v * n[1] + L.w * n[2]) + sqrt(gamma * L.p / L.rho);
    const double sR = fabs(R.u * n[0] + R.v * n[1] + R.w * n[2]) + sqrt(gamma * R.p / R.rho);
    const double s = dmax(sL, sR);
    for (int q = 0; q < 5; ++q) F[q] = 0.5 * (FL[q] + FR[q]) - 0.5 * s * (UR[q] - UL[q]);
}

/* mhd::fluid_flux_rhs (Common/fluid/FluxRHS.cpp:30-74) */
void or_flux_rhs(const OrMesh *m, double gamma, int32_t absorb, const OrPrim *fs, const double *W, const double *grad, double *rhs)
{
    const int32_t no = m->n_owned_cells;
    memset(rhs, 0, sizeof(double) * 5 * (size_t)m->n_cells);
    for (int32_t f = 0; f < m->n_faces; ++f)
    {
        const int kind = m->face_kind[f];
        if (kind == 4) continue;
        const int64_t k0 = m->f2c_ptr[f];
        const int nc = f2c_count(m, f);
        int any = 0;
        for (int q = 0; q < nc; ++q) any |= m->f2c_idx[k0 + q] < no && m->cell_material[m->f2c_idx[k0 + q]] == 0;
        if (!any) continue;
        const double A = m->face_area_mag[f];
        const v3 n = scl(1.0 / A, ld(m->face_area, f));
        const double nv[3] = {n.x, n.y, n.z};
        const v3 xf = ld(m->face_center, f);
        OrPrim L, R;
        int32_t cL = -1, cR = -1;
        if (nc == 2 && kind == 0)
        {
            cL = m->f2c_idx[k0]; cR = m->f2c_idx[k0 + 1];
            if (m->f2c_sgn[k0] < 0) { const int32_t t = cL; cL = cR; cR = t; }
            L = face_state(W, grad, cL, sub3(xf, ld(m->cell_center, cL)));
            R = face_state(W, grad, cR, sub3(xf, ld(m->cell_center, cR)));
        }
        else
        {
            int32_t c = m->f2c_idx[k0];
            int sgn = m->f2c_sgn[k0];
            if (nc == 2 && m->cell_material[c] == 1) { c = m->f2c_idx[k0 + 1]; sgn = m->f2c_sgn[k0 + 1]; }
            const OrPrim in = face_state(W, grad, c, sub3(xf, ld(m->cell_center, c)));
            const OrPrim gh = ghost(kind, absorb, in, scl((double)sgn, n), *fs);
            if (sgn > 0) { cL = c; L = in; R = gh; }
            else { cR = c; R = in; L = gh; }
        }
        double F[5];
        rusanov(L, R, nv, gamma, F);
        for (int q = 0; q < 5; ++q) F[q] *= A;
        if (cL >= 0 && cL < no)
            for (int q = 0; q < 5; ++q) rhs[5 * (int64_t)cL + q] -= F[q] / m->cell_volume[cL];
        if (cR >= 0 && cR < no)
            for (int q = 0; q < 5; ++q) rhs[5 * (int64_t)cR + q] += F[q] / m->cell_volume[cR];
    }
}

/* uns::reconstruct_cell_vector (src/uns/geometry/Reconstruct.cpp:8-46) */
void or_cell_vector(const OrMesh *m, const double *flux, int32_t ncells, double *out)
{
    for (int32_t c = 0; c < ncells; ++c)
    {
        double M[3][3] = {{0}}, r[3] = {0, 0, 0};
        out[3 * (int64_t)c] = out[3 * (int64_t)c + 1] = out[3 * (int64_t)c + 2] = 0.0;
        for (int64_t k = m->c2f_ptr[c]; k < m->c2f_ptr[c + 1]; ++k)
        {
            const int32_t f = m->c2f_idx[k];
            const double A = m->face_area_mag[f];
            if (A <= 0) continue;
            const v3 n = scl(m->c2f_sgn[k] / A, ld(m->face_area, f));
            const double nv[3] = {n.x, n.y, n.z};
            const double phi = m->c2f_sgn[k] * flux[f];
            for (int i = 0; i < 3; ++i)
            {
                r[i] += nv[i] * phi;
                for (int j = 0; j < 3; ++j) M[i][j] += A * nv[i] * nv[j];
            }
        }
        const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        const double sc = dmax(dmax(dmax(M[0][0], M[1][1]), M[2][2]), 1e-300);
        if (fabs(det) < 1e-12 * sc * sc * sc) continue;
        double I[3][3];
        I[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det;
        I[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
        I[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det;
        I[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) / det;
        I[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det;
        I[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
        I[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) / det;
        I[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) / det;
        I[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
        for (int a = 0; a < 3; ++a) out[3 * (int64_t)c + a] = I[a][0] * r[0] + I[a][1] * r[1] + I[a][2] * r[2];
    }
}

/* mhd::add_ideal_emf (Common/induction/IdealEMF.cpp:25-129), adds into E */
void or_ideal_emf(const OrMesh *m, const double *u, const double *Bt, const double *Bi, const double *phi_tot, const double *phi_ind,
                  double cuct, double *E)
{
    double *Ef = (double *)malloc(sizeof(double) * 3 * (size_t)(m->n_faces > 0 ? m->n_faces : 1));
    char *have = (char *)calloc((size_t)(m->n_faces > 0 ? m->n_faces : 1), 1);
    for (int32_t e = 0; e < m->n_owned_edges; ++e)
    {
        const int64_t f0 = m->e2f_ptr[e], f1 = m->e2f_ptr[e + 1];
        const int nf = (int)(f1 - f0);
        if (nf == 0 || m->edge_len[e] <= 0) continue;
        int any = 0;
        for (int64_t k = m->ec_ptr[e]; k < m->ec_ptr[e + 1] && !any; ++k) any = m->cell_material[m->ec_cell[k]] == 0;
        if (!any) continue;
        const v3 t = ld(m->edge_vec, e);
        const double L = m->edge_len[e];
        const v3 th = scl(1.0 / L, t);
        double Ec = 0, w[64], aef[64];
        v3 mm[64], nrm[64];
        for (int i = 0; i < nf; ++i)
        {
            const int32_t f = m->e2f_idx[f0 + i];
            if (!have[f])
            {
                /* face candidate (:32-55) */
                have[f] = 1;
                const double A = m->face_area_mag[f];
                const v3 n = scl(1.0 / A, ld(m->face_area, f));
                const double Bn = phi_tot[f] / A;
                const int64_t p0 = m->f2c_ptr[f];
                v3 F;
                if (f2c_count(m, f) == 2)
                {
                    int32_t cl = m->f2c_idx[p0], cr = m->f2c_idx[p0 + 1];
                    if (m->f2c_sgn[p0] < 0) { const int32_t tt = cl; cl = cr; cr = tt; }
                    const v3 uL = ld(u, cl), uR = ld(u, cr);
                    const double a = dmax(fabs(dot3(uL, n)), fabs(dot3(uR, n)));
                    const v3 FL = sub3(scl(dot3(uL, n), ld(Bt, cl)), scl(Bn, uL));
                    const v3 FR = sub3(scl(dot3(uR, n), ld(Bt, cr)), scl(Bn, uR));
                    F = sub3(scl(0.5, add3(FL, FR)), scl(0.5 * a, sub3(ld(Bi, cr), ld(Bi, cl))));
                }
                else
                {
                    const int32_t c = m->f2c_idx[p0];
                    const v3 uc = ld(u, c);
                    F = sub3(scl(dot3(uc, n), ld(Bt, c)), scl(Bn, uc));
                }
                const v3 Ev = scl(-1.0, cross3(n, F));
                Ef[3 * (int64_t)f] = Ev.x; Ef[3 * (int64_t)f + 1] = Ev.y; Ef[3 * (int64_t)f + 2] = Ev.z;
            }
            w[i] = m->ef_weight[f0 + i];
            Ec += w[i] * dot3(ld(Ef, f), t);
            v3 v = sub3(ld(m->face_center, f), ld(m->edge_mid, e));
            v = sub3(v, scl(dot3(v, th), th));
            const double nv = sqrt(dot3(v, v));
            mm[i] = nv > 0 ? scl(1.0 / nv, v) : mk3(0, 0, 0);
            nrm[i] = scl(1.0 / m->face_area_mag[f], ld(m->face_area, f));
            aef[i] = 0.0;
        }
        for (int64_t k = m->ec_ptr[e]; k < m->ec_ptr[e + 1]; ++k)
        {
            const v3 uc = ld(u, m->ec_cell[k]);
            for (int i = 0; i < nf; ++i) aef[i] = dmax(aef[i], fabs(dot3(uc, mm[i])));
        }
        const v3 ax = fabs(th.x) < 0.9 ? mk3(1, 0, 0) : mk3(0, 1, 0);
        v3 e1 = cross3(th, ax);
        e1 = scl(1.0 / sqrt(dot3(e1, e1)), e1);
        const v3 e2 = cross3(th, e1);
        double M11 = 0, M12 = 0, M22 = 0, g1 = 0, g2 = 0, qa[64], qb[64];
        for (int i = 0; i < nf; ++i)
        {
            const v3 qv = scl(aef[i] * dot3(th, cross3(mm[i], nrm[i])), nrm[i]);
            qa[i] = dot3(qv, e1);
            qb[i] = dot3(qv, e2);
            M11 += w[i] * qa[i] * qa[i];
            M12 += w[i] * qa[i] * qb[i];
            M22 += w[i] * qb[i] * qb[i];
            g1 += w[i] * qa[i];
            g2 += w[i] * qb[i];
        }
        const double tr = M11 + M22, eps = 1e-14 * tr, det = (M11 + eps) * (M22 + eps) - M12 * M12;
        double l1 = 0, l2 = 0;
        if (tr > 0 && det > 0)
        {
            l1 = ((M22 + eps) * g1 - M12 * g2) / det;
            l2 = ((M11 + eps) * g2 - M12 * g1) / det;
        }
        double Eu = 0;
        for (int i = 0; i < nf; ++i)
        {
            const int32_t f = m->e2f_idx[f0 + i];
            const double omega = w[i] * (1.0 - (qa[i] * l1 + qb[i] * l2));
            const double sig = dot3(th, cross3(mm[i], nrm[i]));
            Eu += omega * aef[i] * sig * (phi_ind[f] / m->face_area_mag[f]);
        }
        E[e] += Ec + 2.0 * cuct * L * Eu;
    }
    free(Ef);
    free(have);
}

/* boundary edge values of mercury::Solver::rhs (MercuryUns/driver/Solver.cpp:162-167) */
void or_edge_modes(const OrMesh *m, const double *u_inf, const double *B_imf, double *E)
{
    const v3 Einf = scl(-1.0, cross3(mk3(u_inf[0], u_inf[1], u_inf[2]), mk3(B_imf[0], B_imf[1], B_imf[2])));
    for (int32_t e = 0; e < m->n_owned_edges; ++e)
    {
        if (m->edge_mode[e] == 1) E[e] = 0.0;
        else if (m->edge_mode[e] == 2) E[e] = dot3(Einf, ld(m->edge_vec, e));
    }
}

/* mhd::faraday_update / faraday_update_edge_dt (Common/induction/Faraday.cpp:15-36) over active_faces (:7-13) */
void or_faraday(const OrMesh *m, const double *E, const double *dt_edge, double dt, double *B)
{
    for (int32_t f = 0; f < m->n_faces; ++f)
    {
        int active = 0;
        for (int64_t k = m->f2c_ptr[f]; k < m->f2c_ptr[f + 1]; ++k) active |= m->f2c_idx[k] < m->n_owned_cells;
        if (!active) continue;
        double circ = 0.0;
        if (dt_edge)
        {
            for (int64_t k = m->f2e_ptr[f]; k < m->f2e_ptr[f + 1]; ++k) circ += m->f2e_sgn[k] * dt_edge[m->f2e_idx[k]] * E[m->f2e_idx[k]];
            B[f] -= circ;
        }
        else
        {
            for (int64_t k = m->f2e_ptr[f]; k < m->f2e_ptr[f + 1]; ++k) circ += m->f2e_sgn[k] * E[m->f2e_idx[k]];
            B[f] -= dt * circ;
        }
    }
}

/* mhd::div_b (Common/diagnostics/DivB.cpp:8-24): max_abs, max_rel, worst cell */
void or_div_b(const OrMesh *m, const double *B, const double *extra, double *out3)
{
    double max_abs = 0, max_rel = 0, worst = -1;
    for (int32_t c = 0; c < m->n_owned_cells; ++c)
    {
        double s = 0, a = 0;
        for (int64_t k = m->c2f_ptr[c]; k < m->c2f_ptr[c + 1]; ++k)
        {
            const int32_t f = m->c2f_idx[k];
            s += m->c2f_sgn[k] * B[f];
            a += fabs(B[f]) + (extra ? fabs(extra[f]) : 0.0);
        }
        const double rel = a > 0 ? fabs(s) / a : 0.0;
        if (fabs(s) > max_abs) { max_abs = fabs(s); worst = c; }
        max_rel = dmax(max_rel, rel);
    }
    out3[0] = max_abs; out3[1] = max_rel; out3[2] = worst;
}

/* mhd::cell_current (Common/induction/Current.cpp:9-31) */
void or_cell_current(const OrMesh *m, const double *B, double *J)
{
    memset(J, 0, sizeof(double) * 3 * (size_t)m->n_cells);
    for (int32_t c = 0; c < m->n_owned_cells; ++c)
    {
        v3 sum = mk3(0, 0, 0);
        const v3 bc = ld(B, c);
        for (int64_t k = m->c2f_ptr[c]; k < m->c2f_ptr[c + 1]; ++k)
        {
            const int32_t f = m->c2f_idx[k];
            v3 bf = bc;
            const int64_t p0 = m->f2c_ptr[f];
            if (f2c_count(m, f) == 2)
            {
                const int32_t o = m->f2c_idx[p0] == c ? m->f2c_idx[p0 + 1] : m->f2c_idx[p0];
                bf = scl(0.5, add3(bc, ld(B, o)));
            }
            sum = add3(sum, cross3(scl((double)m->c2f_sgn[k], ld(m->face_area, f)), bf));
        }
        const double invV = 1.0 / m->cell_volume[c];
        J[3 * (int64_t)c] = sum.x * invV; J[3 * (int64_t)c + 1] = sum.y * invV; J[3 * (int64_t)c + 2] = sum.z * invV;
    }
}

/* mercury::cell_time_steps + local_time_step (MercuryUns/fluid/MercurySources.cpp:65-116) for n species
 * (no gyration limit); the wave speeds use the summed density as the reference does for its two ions */
double or_local_time_step(const OrMesh *m, int32_t ns, const double *const *W, const double *B, double gamma, double cfl, double inver_MA2,
                          double rho_floor_dt)
{
    double gdt = INFINITY;
    for (int32_t c = 0; c < m->n_owned_cells; ++c)
    {
        if (m->cell_material[c] == 1) continue;
        double dt = INFINITY;
        const v3 b = ld(B, c);
        const double B2 = dot3(b, b);
        double rs = W[0][5 * (int64_t)c];
        for (int s = 1; s < ns; ++s) rs = rs + W[s][5 * (int64_t)c];
        const double rho_tot = dmax(rs, rho_floor_dt);
        for (int s = 0; s < ns; ++s)
        {
            const double *w = W[s] + 5 * (int64_t)c;
            const double cs2 = gamma * w[4] / dmax(w[0], 1e-30);
            double denom = 0;
            for (int64_t k = m->c2f_ptr[c]; k < m->c2f_ptr[c + 1]; ++k)
            {
                const int32_t f = m->c2f_idx[k];
                const double A = m->face_area_mag[f];
                const v3 n = scl(1.0 / A, ld(m->face_area, f));
                const double vA2 = inver_MA2 * B2 / rho_tot;
                const double vAn2 = inver_MA2 * dot3(b, n) * dot3(b, n) / rho_tot;
                const double term = cs2 + vA2;
                const double cf = sqrt(0.5 * (term + sqrt(dmax(0.0, term * term - 4 * cs2 * vAn2))));
                denom += (fabs(w[1] * n.x + w[2] * n.y + w[3] * n.z) + cf) * A;
            }
            if (denom > 0) dt = dmin(dt, cfl * m->cell_volume[c] / denom);
        }
        gdt = dmin(gdt, dt);
    }
    return gdt;
}

/* one SSP-RK2 step of the hot path: mercury::Solver::step (MercuryUns/driver/Solver.cpp:481-516) with
 * prepare (:94-125, no current), rhs (:132-169, no model sources), advance (:194-206) and floors (:171-191) */
static void floors(const OrMesh *m, const OrStepParams *p, double *const *U)
{
    for (int k = 0; k < p->n_species; ++k)
        for (int32_t c = 0; c < m->n_owned_cells; ++c)
        {
            if (m->cell_material[c] == 1) continue;
            double *u = U[k] + 5 * (int64_t)c;
            const double ke = u[0] > 0 ? 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0] : 0.0;
            if (!(u[0] >= p->rho_floor)) { const OrPrim f = {p->rho_floor, 0, 0, 0, p->p_floor}; to_cons1(f, p->gamma, u); }
            else if ((p->gamma - 1.0) * (u[4] - ke) < p->p_floor) to_cons1(to_prim1(u, p->gamma, p->rho_floor, p->p_floor), p->gamma, u);
        }
}

/* mhd::Scales::numinfo (Common/physics/Scales.cpp:50-62) */
typedef struct { double nH, nNa, ne, ne_eff, chiH, chiNa, wH, wNa; } OrNumInfo;
static OrNumInfo numinfo(const OrStepParams *p, double rhoH, double rhoNa)
{
    OrNumInfo n;
    n.nH = dmax(rhoH, 0.0) / p->mass[0] * p->M_ref;
    n.nNa = dmax(rhoNa, 0.0) / p->mass[1] * p->M_ref;
    n.ne = n.nH + n.nNa;
    n.ne_eff = sqrt(n.ne * n.ne + p->ne_floor * p->ne_floor);
    if (n.ne > 1e-300) { n.chiH = n.nH / n.ne; n.chiNa = n.nNa / n.ne; }
    else { n.chiH = 1.0; n.chiNa = 0.0; }
    n.wH = n.nH / n.ne_eff;
    n.wNa = n.nNa / n.ne_eff;
    return n;
}

/* mercury::add_sources_n (MercuryUns/fluid/MercurySources.cpp:20-63) with the Lorentz force only:
 * S = inver_MA2 w_s (J x B); rhs_m += S, rhs_E += u.S + dt |S|^2 / (2 rho) (mid-point velocity work) */
void or_add_sources(const OrMesh *m, const OrStepParams *p, int32_t s, const double *WH, const double *WNa, const double *B,
                    const double *J, const double *dpe, const double *photo, const double *vst, double dt, double *rhs)
{
    const double *W = s == 0 ? WH : WNa;
    for (int32_t c = 0; c < m->n_owned_cells; ++c)
    {
        if (m->cell_material[c] == 1) continue;
        const size_t i = (size_t)c;
        const OrNumInfo ni = numinfo(p, WH[5 * i], WNa[5 * i]);
        const double ns = s == 0 ? ni.nH : ni.nNa, ws = s == 0 ? ni.wH : ni.wNa;
        const double rho = dmax(W[5 * i], 0.0);
        const v3 u = mk3(W[5 * i + 1], W[5 * i + 2], W[5 * i + 3]);
        double *r = rhs + 5 * i;
        v3 S = mk3(0, 0, 0);
        if (p->lorentz) S = add3(S, scl(p->inver_MA2 * ws, cross3(ld(J, c), ld(B, c))));
        if (p->ambipolar && dpe) S = sub3(S, scl(ws, ld(dpe, c)));
        r[1] += S.x; r[2] += S.y; r[3] += S.z;
        r[4] += dot3(u, S) + (rho > 1e-30 ? 0.5 * dt * dot3(S, S) / rho : 0.0);
        if (p->chemistry && vst)
        {
            /* drag, temperature relaxation, thermal drift, Na+ production (MercurySources.cpp:48-60) */
            const double v = vst[i], u2 = dot3(u, u);
            const double Ts = W[5 * i + 4] / (rho > 0 ? rho : 1e-300) / (s == 0 ? p->state_coeff_H : p->state_coeff_Na) * p->T_ref;
            const double Msum = p->mass[0] + p->mass[1];
            const double b1 = v * (p->Tn0 - Ts) * (s == 0 ? p->mass[0] / Msum : 0.5);
            const double b2 = (s == 0 ? p->mass[1] / Msum : 0.5) * v;
            r[1] -= p->a4 * rho * u.x * v; r[2] -= p->a4 * rho * u.y * v; r[3] -= p->a4 * rho * u.z * v;
            r[4] -= p->a4 * rho * u2 * v;
            r[4] += p->a5 * ns * b1;
            r[4] += p->a4 * rho * u2 * b2;
            if (s == 1 && photo)
            {
                r[0] += p->a1_Na * photo[i];
                r[4] += p->a6 * photo[i] * p->Tn0;
            }
        }
    }
}

static double pe_of(const double *WH, const double *WNa, int32_t c) { return WH[5 * (size_t)c + 4] + WNa[5 * (size_t)c + 4]; }

void or_electron_pressure_gradient(const OrMesh *m, const double *WH, const double *WNa, double *dpe)
{
    memset(dpe, 0, 3 * sizeof(double) * (size_t)m->n_cells);
    for (int32_t c = 0; c < m->n_owned_cells; ++c)
    {
        if (m->cell_material[c] == 1) continue;
        v3 sum = mk3(0, 0, 0);
        for (int64_t k = m->c2f_ptr[c]; k < m->c2f_ptr[c + 1]; ++k)
        {
            const int32_t f = m->c2f_idx[k];
            double pf = pe_of(WH, WNa, c);
            const int64_t b = m->f2c_ptr[f];
            if (m->f2c_ptr[f + 1] - b == 2)
            {
                const int32_t o = m->f2c_idx[b] == c ? m->f2c_idx[b + 1] : m->f2c_idx[b];
                if (m->cell_material[o] == 0) pf = 0.5 * (pf + pe_of(WH, WNa, o));
            }
            sum = add3(sum, scl(pf * (double)m->c2f_sgn[k], ld(m->face_area, f)));
        }
        const double iv = 1.0 / m->cell_volume[c];
        dpe[3 * (size_t)c] = sum.x * iv; dpe[3 * (size_t)c + 1] = sum.y * iv; dpe[3 * (size_t)c + 2] = sum.z * iv;
    }
}

static int cmp_i32(const void *a, const void *b)
{
    const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

void or_ambipolar_emf(const OrMesh *m, const OrStepParams *p, const double *WH, const double *WNa, double *E)
{
    const int32_t nn = m->n_nodes, nc = m->n_cells;
    /* per node its fluid cells, ascending: a cell's nodes are the sorted end points of its faces' edges */
    int64_t *cnt = (int64_t *)calloc((size_t)nn + 1, sizeof(int64_t));
    int64_t npairs = 0;
    int32_t buf[512];
    for (int pass = 0; pass < 2; ++pass)
    {
        int32_t *cells = NULL;
        int64_t *fill = NULL;
        if (pass == 1)
        {
            for (int32_t v = 0; v < nn; ++v) cnt[v + 1] += cnt[v];
            npairs = cnt[nn];
            cells = (int32_t *)malloc(sizeof(int32_t) * (size_t)(npairs > 0 ? npairs : 1));
            fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nn > 0 ? nn : 1));
            for (int32_t v = 0; v < nn; ++v) fill[v] = cnt[v];
        }
        for (int32_t c = 0; c < nc; ++c)
        {
            if (m->cell_material[c] == 1) continue;
            int n = 0;
            for (int64_t k = m->c2f_ptr[c]; k < m->c2f_ptr[c + 1]; ++k)
            {
                const int32_t f = m->c2f_idx[k];
                for (int64_t q = m->f2e_ptr[f]; q < m->f2e_ptr[f + 1] && n + 2 <= 512; ++q)
                {
                    buf[n++] = m->edge_nodes[2 * (size_t)m->f2e_idx[q]];
                    buf[n++] = m->edge_nodes[2 * (size_t)m->f2e_idx[q] + 1];
                }
            }
            qsort(buf, (size_t)n, sizeof(int32_t), cmp_i32);
            for (int i = 0; i < n; ++i)
            {
                if (i > 0 && buf[i] == buf[i - 1]) continue;
                if (pass == 0) ++cnt[buf[i] + 1];
                else cells[fill[buf[i]]++] = c;
            }
        }
        if (pass == 1)
        {
            double *pn = (double *)malloc(sizeof(double) * (size_t)(nn > 0 ? nn : 1));
            for (int32_t v = 0; v < nn; ++v)
            {
                double sp = 0, w = 0;
                for (int64_t k = cnt[v]; k < cnt[v + 1]; ++k)
                {
                    const int32_t cc = cells[k];
                    sp += m->cell_volume[cc] * pe_of(WH, WNa, cc);
                    w += m->cell_volume[cc];
                }
                pn[v] = w > 0 ? sp / w : 0.0;
            }
            for (int32_t e = 0; e < m->n_owned_edges; ++e)
            {
                double rH = 0, rN = 0, wsum = 0;
                for (int64_t k = m->ec_ptr[e]; k < m->ec_ptr[e + 1]; ++k)
                {
                    const int32_t cc = m->ec_cell[k];
                    if (m->cell_material[cc] == 1) continue;
                    rH += m->ec_weight[k] * WH[5 * (size_t)cc];
                    rN += m->ec_weight[k] * WNa[5 * (size_t)cc];
                    wsum += m->ec_weight[k];
                }
                if (wsum <= 0) continue;
                const OrNumInfo ni = numinfo(p, rH / wsum, rN / wsum);
                const int32_t a = m->edge_nodes[2 * (size_t)e], b = m->edge_nodes[2 * (size_t)e + 1];
                if (cnt[a + 1] == cnt[a] || cnt[b + 1] == cnt[b]) continue;
                E[e] -= p->pressure_coef * (pn[b] - pn[a]) / ni.ne_eff;
            }
            free(pn);
            free(cells);
            free(fill);
        }
    }
    free(cnt);
}

/* mercury::gyrate_n (MercuryUns/physics/Gyration.cpp): w = u_H - u_Na rotated by
 * th = (a_H chi_Na + a_Na chi_H) |B| dt about b = B/|B|, split f_H, -f_Na between the ions; the
 * kinetic-energy change goes to the total energy */
void or_gyrate(const OrMesh *m, const OrStepParams *p, const double *B, double dt, double *UH, double *UNa)
{
    if (p->induce_coeff <= 0 || !p->lorentz) return;
    const double aH = p->induce_coeff * p->M_ref / p->mass[0], aN = p->induce_coeff * p->M_ref / p->mass[1];
    for (int32_t c = 0; c < m->n_owned_cells; ++c)
    {
        if (m->cell_material[c] == 1) continue;
        double *uh = UH + 5 * (size_t)c, *un = UNa + 5 * (size_t)c;
        const OrPrim wh = to_prim1(uh, p->gamma, p->rho_floor, p->p_floor), wn = to_prim1(un, p->gamma, p->rho_floor, p->p_floor);
        const OrNumInfo ni = numinfo(p, uh[0], un[0]);
        const v3 b = ld(B, c);
        const double bm = sqrt(dot3(b, b));
        const double denom = aH * ni.chiNa + aN * ni.chiH;
        if (bm <= 0 || denom <= 0) continue;
        const v3 bh = scl(1.0 / bm, b);
        const v3 uH = mk3(wh.u, wh.v, wh.w), uN = mk3(wn.u, wn.v, wn.w);
        const v3 w = sub3(uH, uN);
        const v3 wpar = scl(dot3(w, bh), bh), wperp = sub3(w, wpar);
        const double th = denom * bm * dt;
        const v3 dw = add3(scl(cos(th) - 1.0, wperp), scl(sin(th), cross3(wperp, bh)));
        const double fH = aH * ni.chiNa / denom, fN = aN * ni.chiH / denom;
        const v3 dH = scl(fH, dw), dN = scl(-fN, dw);
        const v3 uH2 = add3(uH, dH), uN2 = add3(uN, dN);
        double rho = uh[0];
        uh[1] = rho * uH2.x; uh[2] = rho * uH2.y; uh[3] = rho * uH2.z;
        uh[4] += 0.5 * rho * (dot3(uH2, uH2) - dot3(uH, uH));
        rho = un[0];
        un[1] = rho * uN2.x; un[2] = rho * uN2.y; un[3] = rho * uN2.z;
        un[4] += 0.5 * rho * (dot3(uN2, uN2) - dot3(uN, uN));
    }
}

/* E_e += m_e p0_e + 0 + 0, p0 = d1^T star2 Phi scattered face by face in ascending order: the resistive part of
 * ImplicitInduction::apply_F (ImplicitInduction.cpp:133-137) and its sum out = m p0 + p1 + p2 (:182) with the Hall
 * and ideal parts off, added to the owned edges' EMF */
void or_resistive_emf(const OrMesh *m, const double *m_res, const double *phi, double *E)
{
    double *p0 = (double *)calloc((size_t)(m->n_edges > 0 ? m->n_edges : 1), sizeof(double));
    for (int32_t f = 0; f < m->n_faces; ++f)
    {
        const double v = m->star2[f] * phi[f];
        for (int64_t k = m->f2e_ptr[f]; k < m->f2e_ptr[f + 1]; ++k) p0[m->f2e_idx[k]] += m->f2e_sgn[k] * v;
    }
    for (int32_t e = 0; e < m->n_owned_edges; ++e) E[e] += m_res[e] * p0[e] + 0.0 + 0.0;
    free(p0);
}

/* One step of the hot path: the SSP-RK2 step of Solver::step (ind NULL), or with ind the semi-implicit step of
 * Solver::step_first_order (Solver.cpp:228-277): one forward Euler stage whose EMF is ind's solve */
static int step_impl(const OrMesh *m, const OrStepParams *p, OrInduction *ind, double *const *U, double *Phi, const double *PhiAdd,
                     const double *BaddCell, double dt, int32_t *iterations, double *rel_res)
{
    const int32_t nc = m->n_cells, nf = m->n_faces, ne = m->n_edges, ns = p->n_species;
    const size_t c5 = 5 * (size_t)nc;
    double *mem = (double *)malloc(sizeof(double) * (ns * (5 + 15 + 5 + 5 + 5) * (size_t)nc + 9 * (size_t)nc + 3 * (size_t)nf + ne));
    if (!mem) return -1;
    double *W = mem, *G = W + ns * c5, *R = G + 3 * ns * c5, *U1 = R + ns * c5, *U2 = U1 + ns * c5;
    double *Bi = U2 + ns * c5, *Bt = Bi + 3 * (size_t)nc, *up = Bt + 3 * (size_t)nc, *Pt = up + 3 * (size_t)nc, *P1 = Pt + nf, *P2 = P1 + nf;
    double *E = P2 + nf;
    double *Us[16], *U1s[16], *U2s[16];
    const int lorentz = p->lorentz != 0, split = lorentz && p->induce_coeff > 0;
    if ((lorentz || p->ambipolar || p->chemistry) && ns != 2) { free(mem); return -1; }
    double *Jc = lorentz ? (double *)malloc(sizeof(double) * 3 * (size_t)(nc > 0 ? nc : 1)) : NULL;
    double *dpe = p->ambipolar ? (double *)malloc(sizeof(double) * 3 * (size_t)(nc > 0 ? nc : 1)) : NULL;
    for (int s = 0; s < ns; ++s) { Us[s] = U[s]; U1s[s] = U1 + s * c5; U2s[s] = U2 + s * c5; }
    if (split)
    {
        /* the opening half-step gyration with Btot of prepare(U^n) (Solver.cpp:492-498) */
        or_cell_vector(m, Phi, nc, Bi);
        for (size_t i = 0; i < 3 * (size_t)nc; ++i) Bt[i] = Bi[i] + BaddCell[i];
        or_gyrate(m, p, Bt, 0.5 * dt, Us[0], Us[1]);
    }
    double *Eimp = ind ? (double *)malloc(sizeof(double) * ((size_t)ne + 1)) : NULL;
    double *nec = ind ? (double *)malloc(sizeof(double) * ((size_t)nc + 1)) : NULL;
    int8_t *dirv = ind ? (int8_t *)malloc((size_t)ne + 1) : NULL;
    for (int st = 0; st < (ind ? 1 : 2); ++st)
    {
        double *const *Ui = st == 0 ? Us : U1s;
        double *const *Uo = st == 0 ? U1s : U2s;
        const double *phis = st == 0 ? Phi : P1;
        double *phio = st == 0 ? P1 : P2;
        for (int s = 0; s < ns; ++s) or_to_prim(Ui[s], nc, p->gamma, p->rho_floor, p->p_floor, W + s * c5);
        or_cell_vector(m, phis, nc, Bi);
        for (int32_t c = 0; c < nc; ++c)
        {
            for (int a = 0; a < 3; ++a) Bt[3 * (int64_t)c + a] = Bi[3 * (int64_t)c + a] + BaddCell[3 * (int64_t)c + a];
            double u3[3] = {0, 0, 0};
            if (m->cell_material[c] == 0)
            {
                double nsv[16], ne_ = 0;
                for (int s = 0; s < ns; ++s) { nsv[s] = dmax(W[s * c5 + 5 * (size_t)c], 0.0) / p->mass[s] * p->M_ref; ne_ += nsv[s]; }
                for (int s = 0; s < ns; ++s)
                {
                    const double chi = ne_ > 1e-300 ? nsv[s] / ne_ : (s == 0 ? 1.0 : 0.0);
                    for (int a = 0; a < 3; ++a) u3[a] += chi * W[s * c5 + 5 * (size_t)c + 1 + a];
                }
            }
            for (int a = 0; a < 3; ++a) up[3 * (int64_t)c + a] = u3[a];
        }
        for (int32_t f = 0; f < nf; ++f) Pt[f] = phis[f] + PhiAdd[f];
        for (int s = 0; s < ns; ++s)
        {
            if (p->second_order) or_limited_gradients(m, W + s * c5, p->absorb[s], &p->fs[s], 1, p->rel_limit, G + 3 * s * c5);
            else memset(G + 3 * s * c5, 0, sizeof(double) * 3 * c5);
            or_flux_rhs(m, p->gamma, p->absorb[s], &p->fs[s], W + s * c5, G + 3 * s * c5, R + s * c5);
        }
        if (lorentz) or_cell_current(m, Bi, Jc); /* Solver::prepare (Solver.cpp:123) */
        if (p->ambipolar) or_electron_pressure_gradient(m, W, W + c5, dpe); /* :124 */
        if (lorentz || p->ambipolar || p->chemistry) /* Solver::rhs (Solver.cpp:146-149): sources after both flux passes */
            for (int s = 0; s < ns; ++s)
                or_add_sources(m, p, s, W, W + c5, Bt, Jc, p->ambipolar ? dpe : NULL, p->photo, p->vst, dt, R + s * c5);
        memset(E, 0, sizeof(double) * (size_t)ne);
        or_ideal_emf(m, up, Bt, Bi, Pt, phis, p->cuct, E);
        if (p->ambipolar) or_ambipolar_emf(m, p, W, W + c5, E); /* Solver.cpp:158 */
        or_edge_modes(m, p->u_inf, p->B_imf, E);
        if (p->m_res) or_resistive_emf(m, p->m_res, phis, E);
        if (ind)
        {
            /* the implicit linear terms with the total EMF as the unknown (Solver.cpp:252-265): frozen total field
             * and n_e,eff of the fluid cells, inflow edges Dirichlet, E_expl the rhs's EMF, warm start */
            for (int32_t c = 0; c < nc; ++c)
                nec[c] = m->cell_material[c] == 0 ? numinfo(p, W[5 * (size_t)c], W[c5 + 5 * (size_t)c]).ne_eff : 0.0;
            for (int32_t e = 0; e < ne; ++e) dirv[e] = m->edge_mode[e] == 2;
            or_ind_set_frozen(ind, Bt, nec);
            double rr = 0;
            const int32_t it = or_ind_solve(ind, phis, E, dirv, dt, 1, Eimp, &rr);
            if (iterations) *iterations = it;
            if (rel_res) *rel_res = rr;
            memcpy(E, Eimp, sizeof(double) * (size_t)ne);
        }
        for (int s = 0; s < ns; ++s)
        {
            memcpy(Uo[s], Ui[s], sizeof(double) * c5);
            for (int32_t c = 0; c < m->n_owned_cells; ++c)
            {
                if (m->cell_material[c] == 1) continue;
                for (int q = 0; q < 5; ++q) Uo[s][5 * (size_t)c + q] += dt * R[s * c5 + 5 * (size_t)c + q];
            }
        }
        memcpy(phio, phis, sizeof(double) * (size_t)nf);
        or_faraday(m, E, NULL, dt, phio);
        floors(m, p, Uo);
    }
    if (ind)
    {
        /* the forward Euler result; the closing half step with Btot of the step's prepare (Solver.cpp:274) */
        for (int s = 0; s < ns; ++s) memcpy(U[s], U1s[s], sizeof(double) * c5);
        memcpy(Phi, P1, sizeof(double) * (size_t)nf);
    }
    else
    {
        for (int s = 0; s < ns; ++s)
            for (size_t i = 0; i < c5; ++i) U[s][i] = 0.5 * (U[s][i] + U2s[s][i]);
        for (int32_t f = 0; f < nf; ++f) Phi[f] = 0.5 * (Phi[f] + P2[f]);
    }
    /* the closing half step with Btot of the last stage's input (Solver.cpp:510) */
    if (split) or_gyrate(m, p, Bt, 0.5 * dt, Us[0], Us[1]);
    free(Jc);
    free(dpe);
    free(Eimp);
    free(nec);
    free(dirv);
    free(mem);
    return 0;
}

int or_rk2_step(const OrMesh *m, const OrStepParams *p, double *const *U, double *Phi, const double *PhiAdd, const double *BaddCell, double dt)
{
    return step_impl(m, p, NULL, U, Phi, PhiAdd, BaddCell, dt, NULL, NULL);
}

int or_first_order_step(const OrMesh *m, const OrStepParams *p, OrInduction *ind, double *const *U, double *Phi, const double *PhiAdd,
                        const double *BaddCell, double dt, int32_t *iterations, double *rel_res)
{
    if (!ind || p->n_species != 2) return -1;
    return step_impl(m, p, ind, U, Phi, PhiAdd, BaddCell, dt, iterations, rel_res);
}

/* ------------------------------------------------------------------ semi-implicit induction
 * mhd::ImplicitInduction (Common/induction/ImplicitInduction.cpp): constructor tables (:10-103),
 * set_frozen_state (:105-111), apply_F (:127-183), apply_A (:185-198), dot_owned (:200-207) and the
 * restarted GMRES(m) with modified Gram-Schmidt, Givens rotations and the Jacobi right
 * preconditioner (:299-390), or the block-Jacobi ILU(0) (:209-297).  The resistive coefficient
 * m_e = eta_e / star1_e is an input (the reference fills it from its tanh window). */
struct OrInduction
{
    const OrMesh *m;
    OrIndParams p;
    int resistive, hall;
    double *m_edge, *taper, *alpha, *B0, *recon, *d2, *ce_wt, *corr;
    int64_t *ce_ptr;
    int32_t *ce_edge;
    double *phi, *bcell, *part, *tmp;
    /* the implicit ideal part (set_ideal_state, :112-116): frozen cell velocities, the edges that carry it */
    int ideal;
    double cuct;
    double *u_ideal, *ide;
    int8_t *imask;
    /* block-Jacobi ILU(0) of the owned edges (:209-297) */
    int ilu;
    double shift;
    int64_t *pc_ptr, *pc_diag;
    int32_t *pc_col;
    double *pc_coef, *pc_val;
};

OrInduction *or_ind_create(const OrMesh *m, const OrIndParams *p, const double *m_edge)
{
    OrInduction *s = (OrInduction *)calloc(1, sizeof(OrInduction));
    const int32_t ne = m->n_edges, nc = m->n_cells, no = m->n_owned_cells;
    s->m = m;
    s->p = *p;
    s->hall = p->hall && p->hall_coef > 0;
    s->m_edge = (double *)calloc((size_t)ne + 1, sizeof(double));
    if (m_edge)
        for (int32_t e = 0; e < ne; ++e) { s->m_edge[e] = m_edge[e]; s->resistive |= m_edge[e] != 0.0; }
    s->taper = (double *)calloc((size_t)nc + 1, sizeof(double));
    s->alpha = (double *)calloc((size_t)nc + 1, sizeof(double));
    s->B0 = (double *)calloc(3 * (size_t)nc + 1, sizeof(double));
    const double mid = 0.5 * (p->hall_r_min + p->hall_r_max), width = p->hall_r_max - p->hall_r_min;
    for (int32_t c = 0; c < nc; ++c)
    {
        if (m->cell_material[c] == 1) continue;
        const double r = sqrt(dot3(ld(m->cell_center, c), ld(m->cell_center, c)));
        s->taper[c] = width <= 0 ? (r >= p->hall_r_min ? 1.0 : 0.0) : 0.5 * (1.0 + tanh(2.0 * (r - mid) / width));
    }
    const int64_t nnz = m->c2f_ptr[nc];
    s->recon = (double *)calloc(3 * (size_t)nnz + 1, sizeof(double));
    for (int32_t c = 0; c < nc; ++c)
    {
        double M[3][3] = {{0}};
        for (int64_t k = m->c2f_ptr[c]; k < m->c2f_ptr[c + 1]; ++k)
        {
            const int32_t f = m->c2f_idx[k];
            const double A = m->face_area_mag[f];
            if (A <= 0) continue;
            const v3 n = scl(1.0 / A, ld(m->face_area, f));
            const double nv[3] = {n.x, n.y, n.z};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) M[i][j] += A * nv[i] * nv[j];
        }
        const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        const double sc = dmax(dmax(dmax(M[0][0], M[1][1]), M[2][2]), 1e-300);
        if (fabs(det) < 1e-12 * sc * sc * sc) continue;
        double I[3][3];
        I[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det; I[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
        I[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det; I[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) / det;
        I[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det; I[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
        I[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) / det; I[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) / det;
        I[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
        for (int64_t k = m->c2f_ptr[c]; k < m->c2f_ptr[c + 1]; ++k)
        {
            const int32_t f = m->c2f_idx[k];
            const double A = m->face_area_mag[f];
            if (A <= 0) continue;
            const v3 n = scl(1.0 / A, ld(m->face_area, f));
            for (int i = 0; i < 3; ++i) s->recon[3 * k + i] = I[i][0] * n.x + I[i][1] * n.y + I[i][2] * n.z;
        }
    }
    /* owned fluid cell -> (edge, w_ec t_e) */
    s->ce_ptr = (int64_t *)calloc((size_t)no + 1, sizeof(int64_t));
    size_t cap = 1024, cnt = 0;
    s->ce_edge = (int32_t *)malloc(cap * sizeof(int32_t));
    s->ce_wt = (double *)malloc(3 * cap * sizeof(double));
    int32_t es[256];
    for (int32_t c = 0; c < no; ++c)
    {
        int nes = 0;
        if (m->cell_material[c] == 0)
            for (int64_t kf = m->c2f_ptr[c]; kf < m->c2f_ptr[c + 1]; ++kf)
                for (int64_t ke = m->f2e_ptr[m->c2f_idx[kf]]; ke < m->f2e_ptr[m->c2f_idx[kf] + 1]; ++ke)
                    if (nes < 256) es[nes++] = m->f2e_idx[ke];
        qsort(es, (size_t)nes, sizeof(int32_t), cmp_i32);
        int u = 0;
        for (int i = 0; i < nes; ++i)
            if (i == 0 || es[i] != es[i - 1]) es[u++] = es[i];
        for (int i = 0; i < u; ++i)
        {
            const int32_t e = es[i];
            int64_t lo = m->ec_ptr[e], hi = m->ec_ptr[e + 1];
            while (lo < hi) { const int64_t mid2 = (lo + hi) / 2; if (m->ec_cell[mid2] < c) lo = mid2 + 1; else hi = mid2; }
            if (lo == m->ec_ptr[e + 1] || m->ec_cell[lo] != c) continue;
            if (cnt == cap)
            {
                cap *= 2;
                s->ce_edge = (int32_t *)realloc(s->ce_edge, cap * sizeof(int32_t));
                s->ce_wt = (double *)realloc(s->ce_wt, 3 * cap * sizeof(double));
            }
            const v3 wt = scl(m->ec_weight[lo], ld(m->edge_vec, e));
            s->ce_edge[cnt] = e;
            s->ce_wt[3 * cnt] = wt.x; s->ce_wt[3 * cnt + 1] = wt.y; s->ce_wt[3 * cnt + 2] = wt.z;
            ++cnt;
        }
        s->ce_ptr[c + 1] = (int64_t)cnt;
    }
    s->d2 = (double *)calloc((size_t)ne + 1, sizeof(double));
    for (int32_t f = 0; f < m->n_faces; ++f) /* every face is owned on one rank */
        for (int64_t k = m->f2e_ptr[f]; k < m->f2e_ptr[f + 1]; ++k) s->d2[m->f2e_idx[k]] += m->star2[f];
    s->phi = (double *)calloc((size_t)m->n_faces + 1, sizeof(double));
    s->bcell = (double *)calloc(3 * (size_t)nc + 1, sizeof(double));
    s->part = (double *)calloc(3 * (size_t)ne + 1, sizeof(double));
    s->tmp = (double *)calloc((size_t)ne + 1, sizeof(double));
    return s;
}

void or_ind_free(OrInduction *s)
{
    if (!s) return;
    free(s->m_edge); free(s->taper); free(s->alpha); free(s->B0); free(s->recon); free(s->d2); free(s->ce_wt); free(s->corr);
    free(s->ce_ptr); free(s->ce_edge); free(s->phi); free(s->bcell); free(s->part); free(s->tmp);
    free(s->pc_ptr); free(s->pc_diag); free(s->pc_col); free(s->pc_coef); free(s->pc_val);
    free(s->u_ideal); free(s->ide); free(s->imask);
    free(s);
}

/* build_precond_pattern (:209-242): per owned row e the entries (e2, m_e s_e,f s_e2,f star2_f) of every face of
 * e and every owned edge e2 of that face, plus (e, 0), sorted by column (insertion sort: ties keep the
 * gathering order), equal columns summed in that order */
void or_ind_set_ilu(OrInduction *s, int32_t enable, double shift)
{
    const OrMesh *m = s->m;
    const int32_t no = m->n_owned_edges;
    s->shift = shift;
    s->ilu = enable != 0 && (s->resistive || s->hall);
    if (!s->ilu || s->pc_ptr) return;
    int64_t cap = 1024, nnz = 0;
    s->pc_ptr = (int64_t *)calloc((size_t)no + 1, sizeof(int64_t));
    s->pc_col = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
    s->pc_coef = (double *)malloc((size_t)cap * sizeof(double));
    int32_t rc[1024];
    double rv[1024];
    for (int32_t e = 0; e < no; ++e)
    {
        int n = 0;
        rc[n] = e; rv[n] = 0.0; ++n;
        for (int64_t kf = m->e2f_ptr[e]; kf < m->e2f_ptr[e + 1]; ++kf)
        {
            const int32_t f = m->e2f_idx[kf];
            const double se = m->e2f_sgn[kf];
            for (int64_t k = m->f2e_ptr[f]; k < m->f2e_ptr[f + 1]; ++k)
            {
                const int32_t e2 = m->f2e_idx[k];
                if (e2 >= no || n >= 1024) continue;
                rc[n] = e2; rv[n] = s->m_edge[e] * se * m->f2e_sgn[k] * m->star2[f]; ++n;
            }
        }
        for (int i = 1; i < n; ++i)
        {
            const int32_t c = rc[i];
            const double v = rv[i];
            int j = i - 1;
            while (j >= 0 && rc[j] > c) { rc[j + 1] = rc[j]; rv[j + 1] = rv[j]; --j; }
            rc[j + 1] = c; rv[j + 1] = v;
        }
        for (int i = 0; i < n;)
        {
            int j = i;
            double sum = 0;
            for (; j < n && rc[j] == rc[i]; ++j) sum += rv[j];
            if (nnz == cap)
            {
                cap *= 2;
                s->pc_col = (int32_t *)realloc(s->pc_col, (size_t)cap * sizeof(int32_t));
                s->pc_coef = (double *)realloc(s->pc_coef, (size_t)cap * sizeof(double));
            }
            s->pc_col[nnz] = rc[i];
            s->pc_coef[nnz] = sum;
            ++nnz;
            i = j;
        }
        s->pc_ptr[e + 1] = nnz;
    }
    s->pc_val = (double *)calloc((size_t)nnz + 1, sizeof(double));
    s->pc_diag = (int64_t *)calloc((size_t)no + 1, sizeof(int64_t));
    for (int32_t e = 0; e < no; ++e)
        for (int64_t k = s->pc_ptr[e]; k < s->pc_ptr[e + 1]; ++k)
            if (s->pc_col[k] == e) s->pc_diag[e] = k;
}

int64_t or_ind_ilu_pattern(OrInduction *s, int64_t *ptr, int32_t *col, double *coef)
{
    if (!s->pc_ptr) return -1;
    const int32_t no = s->m->n_owned_edges;
    const int64_t nnz = s->pc_ptr[no];
    if (ptr) memcpy(ptr, s->pc_ptr, ((size_t)no + 1) * sizeof(int64_t));
    if (col) memcpy(col, s->pc_col, (size_t)nnz * sizeof(int32_t));
    if (coef) memcpy(coef, s->pc_coef, (size_t)nnz * sizeof(double));
    return nnz;
}

/* factor_precond (:247-275): Dirichlet rows and columns removed, the relaxed diagonal, IKJ elimination with the
 * breakdown guard */
static void ilu_factor(OrInduction *s, double dt, const int8_t *dir)
{
    const int32_t no = s->m->n_owned_edges;
    const int64_t *P = s->pc_ptr, *D = s->pc_diag;
    const int32_t *C = s->pc_col;
    double *V = s->pc_val;
    for (int32_t e = 0; e < no; ++e)
        for (int64_t k = P[e]; k < P[e + 1]; ++k)
        {
            const int32_t c = C[k];
            const int de = dir && dir[e], dc = dir && dir[c];
            V[k] = (de || dc) ? (c == e ? 1.0 : 0.0) : (c == e ? 1.0 : 0.0) + dt * s->pc_coef[k];
            if (c == e && !de) V[k] += s->shift * dt * s->pc_coef[k];
        }
    int64_t *pos = (int64_t *)malloc(((size_t)s->m->n_edges + 1) * sizeof(int64_t));
    for (int32_t e = 0; e <= s->m->n_edges; ++e) pos[e] = -1;
    for (int32_t i = 0; i < no; ++i)
    {
        for (int64_t k = P[i]; k < P[i + 1]; ++k) pos[C[k]] = k;
        for (int64_t kk = P[i]; kk < P[i + 1] && C[kk] < i; ++kk)
        {
            const int32_t k = C[kk];
            V[kk] /= V[D[k]];
            const double lik = V[kk];
            for (int64_t jj = D[k] + 1; jj < P[k + 1]; ++jj)
            {
                const int64_t q = pos[C[jj]];
                if (q >= 0) V[q] -= lik * V[jj];
            }
        }
        if (!(fabs(V[D[i]]) > 1e-12)) V[D[i]] = 1.0;
        for (int64_t k = P[i]; k < P[i + 1]; ++k) pos[C[k]] = -1;
    }
    free(pos);
}

/* apply_precond (:277-297): unit lower, then upper; z = 0 on the non-owned edges */
static void ilu_apply(const OrInduction *s, const double *v, double *z, const int8_t *dir)
{
    const int32_t no = s->m->n_owned_edges, ne = s->m->n_edges;
    const int64_t *P = s->pc_ptr, *D = s->pc_diag;
    const int32_t *C = s->pc_col;
    const double *V = s->pc_val;
    for (int32_t i = 0; i < no; ++i)
    {
        double t = (dir && dir[i]) ? 0.0 : v[i];
        for (int64_t k = P[i]; k < D[i]; ++k) t -= V[k] * z[C[k]];
        z[i] = t;
    }
    for (int32_t i = no; i-- > 0;)
    {
        double t = z[i];
        for (int64_t k = D[i] + 1; k < P[i + 1]; ++k) t -= V[k] * z[C[k]];
        z[i] = (dir && dir[i]) ? 0.0 : t / V[D[i]];
    }
    for (int32_t e = no; e < ne; ++e) z[e] = 0.0;
}

void or_ind_ilu_precond(OrInduction *s, double dt, const int8_t *dir, const double *v, double *z)
{
    if (!s->pc_ptr) return;
    ilu_factor(s, dt, dir);
    ilu_apply(s, v, z, dir);
}

void or_ind_set_frozen(OrInduction *s, const double *B0, const double *ne)
{
    const int32_t nc = s->m->n_cells;
    memcpy(s->B0, B0, 3 * (size_t)nc * sizeof(double));
    for (int32_t c = 0; c < nc; ++c) s->alpha[c] = (s->hall && ne[c] > 0) ? s->taper[c] * s->p.hall_coef / ne[c] : 0.0;
}

/* apply_F (:127-183) with the resistive and Hall parts as given (ideal_linear, :118-124, turns both off) */
static void apply_F_parts(OrInduction *s, const double *phi, double *out, int resistive, int hall)
{
    const OrMesh *m = s->m;
    const int32_t ne = m->n_edges, nc = m->n_cells;
    memset(s->part, 0, 3 * (size_t)ne * sizeof(double));
    if (resistive)
        for (int32_t f = 0; f < m->n_faces; ++f)
        {
            const double v = m->star2[f] * phi[f];
            for (int64_t k = m->f2e_ptr[f]; k < m->f2e_ptr[f + 1]; ++k) s->part[3 * (int64_t)m->f2e_idx[k]] += m->f2e_sgn[k] * v;
        }
    if (hall || s->ideal) /* the cell field from the face fluxes (:138-149) */
        for (int32_t c = 0; c < nc; ++c)
        {
            double b[3] = {0, 0, 0};
            for (int64_t k = m->c2f_ptr[c]; k < m->c2f_ptr[c + 1]; ++k)
            {
                const double v = phi[m->c2f_idx[k]];
                b[0] += s->recon[3 * k] * v; b[1] += s->recon[3 * k + 1] * v; b[2] += s->recon[3 * k + 2] * v;
            }
            s->bcell[3 * (int64_t)c] = b[0]; s->bcell[3 * (int64_t)c + 1] = b[1]; s->bcell[3 * (int64_t)c + 2] = b[2];
        }
    if (s->ideal) /* the ideal EMF of the frozen velocities and that field, on the masked edges (:150-158) */
    {
        memset(s->ide, 0, (size_t)ne * sizeof(double));
        or_ideal_emf(m, s->u_ideal, s->bcell, s->bcell, phi, phi, s->cuct, s->ide);
        for (int32_t e = 0; e < ne; ++e) s->part[3 * (int64_t)e + 2] = s->imask[e] ? s->ide[e] : 0.0;
    }
    if (hall)
    {
        for (int32_t c = 0; c < m->n_owned_cells; ++c)
        {
            if (s->alpha[c] == 0.0) continue;
            v3 sum = mk3(0, 0, 0);
            const v3 bc = ld(s->bcell, c);
            for (int64_t k = m->c2f_ptr[c]; k < m->c2f_ptr[c + 1]; ++k)
            {
                const int32_t f = m->c2f_idx[k];
                v3 bf = bc;
                const int64_t p0 = m->f2c_ptr[f];
                if (f2c_count(m, f) == 2)
                {
                    const int32_t o = m->f2c_idx[p0] == c ? m->f2c_idx[p0 + 1] : m->f2c_idx[p0];
                    bf = scl(0.5, add3(bc, ld(s->bcell, o)));
                }
                sum = add3(sum, cross3(scl((double)m->c2f_sgn[k], ld(m->face_area, f)), bf));
            }
            const v3 J = scl(1.0 / m->cell_volume[c], sum);
            const v3 g = scl(s->alpha[c], cross3(J, ld(s->B0, c)));
            for (int64_t q = s->ce_ptr[c]; q < s->ce_ptr[c + 1]; ++q) s->part[3 * (int64_t)s->ce_edge[q] + 1] += dot3(g, ld(s->ce_wt, q));
        }
    }
    for (int32_t e = 0; e < ne; ++e) out[e] = s->m_edge[e] * s->part[3 * (int64_t)e] + s->part[3 * (int64_t)e + 1] + s->part[3 * (int64_t)e + 2];
}

void or_ind_apply_F(OrInduction *s, const double *phi, double *out) { apply_F_parts(s, phi, out, s->resistive, s->hall); }

void or_ind_ideal_linear(OrInduction *s, const double *phi, double *out) { apply_F_parts(s, phi, out, 0, 0); }

void or_ind_set_ideal(OrInduction *s, const double *u_cell, const int8_t *mask, double cuct)
{
    const OrMesh *m = s->m;
    s->ideal = u_cell != NULL;
    if (!s->ideal) return;
    if (!s->u_ideal)
    {
        s->u_ideal = (double *)calloc(3 * (size_t)m->n_cells + 1, sizeof(double));
        s->ide = (double *)calloc((size_t)m->n_edges + 1, sizeof(double));
        s->imask = (int8_t *)calloc((size_t)m->n_edges + 1, 1);
    }
    memcpy(s->u_ideal, u_cell, 3 * (size_t)m->n_cells * sizeof(double));
    memcpy(s->imask, mask, (size_t)m->n_edges);
    s->cuct = cuct;
}

/* apply_A (:185-198): y = x + dt F(d1 x), or with the per-edge step dte y = x + F(d1 diag(dte) x) */
static void apply_A_dte(OrInduction *s, const double *x, double dt, const double *dte, double *y)
{
    const OrMesh *m = s->m;
    for (int32_t f = 0; f < m->n_faces; ++f)
    {
        double v = 0;
        if (dte)
            for (int64_t k = m->f2e_ptr[f]; k < m->f2e_ptr[f + 1]; ++k) v += m->f2e_sgn[k] * dte[m->f2e_idx[k]] * x[m->f2e_idx[k]];
        else
            for (int64_t k = m->f2e_ptr[f]; k < m->f2e_ptr[f + 1]; ++k) v += m->f2e_sgn[k] * x[m->f2e_idx[k]];
        s->phi[f] = v;
    }
    or_ind_apply_F(s, s->phi, s->tmp);
    if (dte) for (int32_t e = 0; e < m->n_edges; ++e) y[e] = x[e] + s->tmp[e];
    else for (int32_t e = 0; e < m->n_edges; ++e) y[e] = x[e] + dt * s->tmp[e];
}

void or_ind_apply_A(OrInduction *s, const double *x, double dt, double *y) { apply_A_dte(s, x, dt, NULL, y); }

static double dot_owned(const OrMesh *m, const double *a, const double *b)
{
    double s = 0;
    for (int32_t e = 0; e < m->n_owned_edges; ++e) s += a[e] * b[e];
    return s;
}

static int32_t solve_impl(OrInduction *s, const double *Phi, const double *Eexp, const int8_t *dir, double dt, const double *dte, int32_t warm,
                          double *E, double *rel_res)
{
    const OrMesh *m = s->m;
    const int32_t ne = m->n_edges, mr = s->p.restart < 2 ? 2 : s->p.restart;
    const size_t nb = sizeof(double) * (size_t)(ne > 0 ? ne : 1);
    double *x0 = (double *)malloc(nb), *b = (double *)malloc(nb), *r = (double *)malloc(nb), *Ax = (double *)malloc(nb);
    double *Fn = (double *)malloc(nb), *idg = (double *)malloc(nb), *delta = (double *)calloc((size_t)ne + 1, sizeof(double));
    double *w = (double *)malloc(nb), *z = (double *)malloc(nb), *comb = (double *)malloc(nb);
    double *V = (double *)malloc(nb * (size_t)(mr + 1));
    double *H = (double *)calloc((size_t)(mr + 1) * (size_t)mr, sizeof(double));
    double *cs = (double *)calloc((size_t)mr, sizeof(double)), *sn = (double *)calloc((size_t)mr, sizeof(double));
    double *g = (double *)calloc((size_t)mr + 1, sizeof(double)), *yv = (double *)calloc((size_t)mr, sizeof(double));
#define HH(i, j) H[(size_t)(i) * (size_t)mr + (size_t)(j)]
    memcpy(x0, Eexp, nb);
    if (!warm && s->corr) { free(s->corr); s->corr = NULL; }
    if (s->corr)
        for (int32_t e = 0; e < ne; ++e)
            if (!dir[e]) x0[e] += s->corr[e];
    or_ind_apply_F(s, Phi, Fn);
    for (int32_t e = 0; e < ne; ++e) b[e] = Eexp[e] + Fn[e];
    apply_A_dte(s, x0, dt, dte, Ax);
    for (int32_t e = 0; e < ne; ++e) r[e] = dir[e] ? 0.0 : b[e] - Ax[e];
    for (int32_t e = 0; e < ne; ++e) idg[e] = 1.0 / (1.0 + (dte ? dte[e] : dt) * s->m_edge[e] * s->d2[e]);
    /* ILU(0) for a scalar dt (:317-318), built only without the ideal part (:102) */
    const int ilu = s->ilu && s->pc_ptr && !dte && !s->ideal;
    if (ilu) ilu_factor(s, dt, dir);
    const double bnorm = sqrt(dmax(dot_owned(m, b, b), 1e-300));
    double beta = sqrt(dot_owned(m, r, r));
    int total = 0;
    while (beta > s->p.rtol * bnorm && total < s->p.max_it)
    {
        for (int32_t e = 0; e < ne; ++e) V[e] = r[e] / beta;
        memset(g, 0, sizeof(double) * ((size_t)mr + 1));
        g[0] = beta;
        int j = 0;
        for (; j < mr && total < s->p.max_it; ++j, ++total)
        {
            const double *Vj = V + (size_t)j * (size_t)ne;
            if (ilu) ilu_apply(s, Vj, z, dir);
            else for (int32_t e = 0; e < ne; ++e) z[e] = dir[e] ? 0.0 : Vj[e] * idg[e];
            apply_A_dte(s, z, dt, dte, w);
            for (int32_t e = 0; e < ne; ++e)
                if (dir[e]) w[e] = 0.0;
            for (int i = 0; i <= j; ++i)
            {
                const double *Vi = V + (size_t)i * (size_t)ne;
                HH(i, j) = dot_owned(m, w, Vi);
                for (int32_t e = 0; e < ne; ++e) w[e] -= HH(i, j) * Vi[e];
            }
            HH(j + 1, j) = sqrt(dot_owned(m, w, w));
            if (HH(j + 1, j) > 1e-300)
            {
                double *Vn = V + (size_t)(j + 1) * (size_t)ne;
                for (int32_t e = 0; e < ne; ++e) Vn[e] = w[e] / HH(j + 1, j);
            }
            for (int i = 0; i < j; ++i)
            {
                const double t = cs[i] * HH(i, j) + sn[i] * HH(i + 1, j);
                HH(i + 1, j) = -sn[i] * HH(i, j) + cs[i] * HH(i + 1, j);
                HH(i, j) = t;
            }
            const double den = hypot(HH(j, j), HH(j + 1, j));
            cs[j] = den > 0 ? HH(j, j) / den : 1.0;
            sn[j] = den > 0 ? HH(j + 1, j) / den : 0.0;
            HH(j, j) = den;
            HH(j + 1, j) = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            if (fabs(g[j + 1]) <= s->p.rtol * bnorm) { ++j; ++total; break; }
        }
        for (int i = j - 1; i >= 0; --i)
        {
            double t = g[i];
            for (int k = i + 1; k < j; ++k) t -= HH(i, k) * yv[k];
            yv[i] = t / HH(i, i);
        }
        for (int32_t e = 0; e < ne; ++e)
        {
            double t = 0;
            for (int i = 0; i < j; ++i) t += yv[i] * V[(size_t)i * (size_t)ne + e];
            comb[e] = t;
        }
        if (ilu)
        {
            ilu_apply(s, comb, z, dir);
            for (int32_t e = 0; e < ne; ++e) delta[e] += z[e];
        }
        else
            for (int32_t e = 0; e < ne; ++e) delta[e] += dir[e] ? 0.0 : comb[e] * idg[e];
        for (int32_t e = 0; e < ne; ++e) z[e] = x0[e] + delta[e];
        apply_A_dte(s, z, dt, dte, Ax);
        for (int32_t e = 0; e < ne; ++e) r[e] = dir[e] ? 0.0 : b[e] - Ax[e];
        beta = sqrt(dot_owned(m, r, r));
    }
#undef HH
    for (int32_t e = 0; e < ne; ++e) E[e] = x0[e] + delta[e];
    if (!s->corr) s->corr = (double *)malloc(nb);
    for (int32_t e = 0; e < ne; ++e) s->corr[e] = dir[e] ? 0.0 : E[e] - Eexp[e];
    if (rel_res) *rel_res = beta / bnorm;
    free(x0); free(b); free(r); free(Ax); free(Fn); free(idg); free(delta); free(w); free(z); free(comb); free(V); free(H);
    free(cs); free(sn); free(g); free(yv);
    return total;
}

int32_t or_ind_solve(OrInduction *s, const double *Phi, const double *Eexp, const int8_t *dir, double dt, int32_t warm, double *E, double *rel_res)
{
    return solve_impl(s, Phi, Eexp, dir, dt, NULL, warm, E, rel_res);
}

int32_t or_ind_solve_dte(OrInduction *s, const double *Phi, const double *Eexp, const int8_t *dir, const double *dte, int32_t warm, double *E,
                         double *rel_res)
{
    return solve_impl(s, Phi, Eexp, dir, 0.0, dte, warm, E, rel_res);
}
