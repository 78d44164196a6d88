// Dual-number forms of the stage's local functions (tangent-linear model).  Each follows its FP64
// counterpart in fluid.cuh / induction.cuh / step.cu operation for operation, so the value part of a
// dual evaluation equals the plain FP64 result and the tangent part is its exact directional
// derivative (one-sided at the reference's max/min/limiter switches, on the branch the value takes).
// Include only from files compiled with -fmad=false.
#pragma once
#include "dual.cuh"
#include "fluid.cuh"

namespace mhd
{
struct DPrim
{
    Dual rho, u, v, w, p;
};

__device__ __forceinline__ DPrim to_prim_d(Dual U0, Dual U1, Dual U2, Dual U3, Dual U4, double gamma, double rho_floor,
                                           double p_floor)
{
    DPrim W;
    W.rho = dmax(U0, dl(rho_floor));
    W.u = U1 / W.rho;
    W.v = U2 / W.rho;
    W.w = U3 / W.rho;
    const Dual ke = 0.5 * W.rho * (W.u * W.u + W.v * W.v + W.w * W.w);
    W.p = dmax((gamma - 1.0) * (U4 - ke), dl(p_floor));
    return W;
}

__device__ __forceinline__ void to_cons_d(const DPrim &W, double gamma, Dual *U)
{
    U[0] = W.rho;
    U[1] = W.rho * W.u;
    U[2] = W.rho * W.v;
    U[3] = W.rho * W.w;
    U[4] = W.p / (gamma - 1.0) + 0.5 * W.rho * (W.u * W.u + W.v * W.v + W.w * W.w);
}

__device__ __forceinline__ DPrim ghost_state_d(int kind, bool absorb, const DPrim &in, V3 n, const DPrim &fs)
{
    if (kind == 1)
    {
        if (absorb) return DPrim{dl(1e-12), dl(0), dl(0), dl(0), dl(1e-12)};
        const Dual un = in.u * n.x + in.v * n.y + in.w * n.z;
        DPrim g = in;
        g.u -= 2 * un * n.x;
        g.v -= 2 * un * n.y;
        g.w -= 2 * un * n.z;
        return g;
    }
    if (kind == 2) return fs;
    return in;
}

__device__ __forceinline__ void rusanov_d(const DPrim &L, const DPrim &R, V3 n, double gamma, Dual *F)
{
    Dual UL[5], UR[5];
    to_cons_d(L, gamma, UL);
    to_cons_d(R, gamma, UR);
    const Dual unL = L.u * n.x + L.v * n.y + L.w * n.z, unR = R.u * n.x + R.v * n.y + R.w * n.z;
    const Dual FL[5] = {L.rho * unL, L.rho * unL * L.u + L.p * n.x, L.rho * unL * L.v + L.p * n.y, L.rho * unL * L.w + L.p * n.z,
                        unL * (UL[4] + L.p)};
    const Dual FR[5] = {R.rho * unR, R.rho * unR * R.u + R.p * n.x, R.rho * unR * R.v + R.p * n.y, R.rho * unR * R.w + R.p * n.z,
                        unR * (UR[4] + R.p)};
    const Dual sL = dabs(unL) + dsqrt(gamma * L.p / L.rho);
    const Dual sR = dabs(unR) + dsqrt(gamma * R.p / R.rho);
    const Dual s = dmax(sL, sR);
    for (int q = 0; q < 5; ++q) F[q] = 0.5 * (FL[q] + FR[q]) - 0.5 * s * (UR[q] - UL[q]);
}

__device__ __forceinline__ DPrim face_state_d(const DPrim &w, const Dual *g, V3 dx)
{
    DPrim r;
    r.rho = w.rho + g[0] * dx.x + g[1] * dx.y + g[2] * dx.z;
    r.u = w.u + g[3] * dx.x + g[4] * dx.y + g[5] * dx.z;
    r.v = w.v + g[6] * dx.x + g[7] * dx.y + g[8] * dx.z;
    r.w = w.w + g[9] * dx.x + g[10] * dx.y + g[11] * dx.z;
    r.p = w.p + g[12] * dx.x + g[13] * dx.y + g[14] * dx.z;
    return (r.rho.v > 0 && r.p.v > 0) ? r : w;
}

__device__ __forceinline__ DV3 operator*(Dual s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ DV3 cross(DV3 a, V3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// uns::reconstruct_cell_vector of a dual flux (the normal matrix is geometry: plain FP64)
__device__ __forceinline__ DV3 cell_vector_d(const MeshView &m, DCPtr flux, int32_t c)
{
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    Dual r[3] = {dl(0), dl(0), dl(0)};
    for (int32_t k = m.c2f_ptr[c]; k < m.c2f_ptr[c + 1]; ++k)
    {
        const int32_t f = m.c2f_idx[k];
        const double A = m.face_area_mag[f];
        if (A <= 0) continue;
        const double s = m.c2f_sgn[k];
        const V3 n = (s / A) * ld3(m.face_area, f);
        const double nv[3] = {n.x, n.y, n.z};
        const Dual phi = s * flux.get(f);
        for (int i = 0; i < 3; ++i)
        {
            r[i] += nv[i] * phi;
            for (int j = 0; j < 3; ++j) M[i][j] += A * nv[i] * nv[j];
        }
    }
    const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                       M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    const double sc = dmax(dmax(dmax(M[0][0], M[1][1]), M[2][2]), 1e-300);
    if (fabs(det) < 1e-12 * sc * sc * sc) return dmk(dl(0), dl(0), dl(0));
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
    return dmk(I[0][0] * r[0] + I[0][1] * r[1] + I[0][2] * r[2], I[1][0] * r[0] + I[1][1] * r[1] + I[1][2] * r[2],
               I[2][0] * r[0] + I[2][1] * r[1] + I[2][2] * r[2]);
}

// The inverse normal matrix of uns::reconstruct_cell_vector: B_c = I_c sum_k n_k phi_k (n_k the face's
// unit normal as stored, phi_k its flux).  Returns false where the reference returns a zero vector.
__device__ __forceinline__ bool cell_vector_inverse(const MeshView &m, int32_t c, double I[3][3])
{
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int32_t k = m.c2f_ptr[c]; k < m.c2f_ptr[c + 1]; ++k)
    {
        const int32_t f = m.c2f_idx[k];
        const double A = m.face_area_mag[f];
        if (A <= 0) continue;
        const double s = m.c2f_sgn[k];
        const V3 n = (s / A) * ld3(m.face_area, f);
        const double nv[3] = {n.x, n.y, n.z};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) M[i][j] += A * nv[i] * nv[j];
    }
    const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                       M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    const double sc = dmax(dmax(dmax(M[0][0], M[1][1]), M[2][2]), 1e-300);
    if (fabs(det) < 1e-12 * sc * sc * sc) return false;
    I[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det;
    I[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
    I[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det;
    I[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) / det;
    I[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det;
    I[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
    I[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) / det;
    I[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) / det;
    I[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
    return true;
}
} // namespace mhd
