// nvcc-flags: -prec-div=false -prec-sqrt=false
// Mixed-precision stage of the explicit step (tetrahedral meshes).
//
// FP32: primitives, least-squares gradients with the Barth-Jespersen limiter, Rusanov face fluxes,
//       cell field fit, charge-weighted velocity, CFL step, face EMF candidates and the UCT edge EMF.
// FP64: the conservative state U (U += dt rhs and the floors), the face fluxes Phi, the CT update
//       Phi -= dt d1 E (the edge values are summed in FP64, so d2 Phi stays at FP64 round-off for any
//       E) and the SSP-RK2 averages.
// The algorithm is the reference's (see step.cu for the per-kernel citations); the geometry enters
// through single-precision tables derived once from the FP64 mesh, laid out as structures of arrays
// over cells, faces and edges so that every warp load is coalesced and every gather is independent.
#include <math_constants.h>

#include <algorithm>
#include <cmath>

#include "state.cuh"

namespace mhd
{
namespace
{
struct F5
{
    float rho, u, v, w, p;
};

struct MV
{
    int32_t nc, nf, ne, no_cells, no_edges;
    const int32_t *c2f_idx, *cfa_idx, *t_nb, *face_L, *face_R, *f2c_ptr, *f2c_idx, *f2e_ptr, *f2e_idx, *e2f_ptr, *e2f_idx, *ec_ptr,
        *ec_cell;
    const int8_t *c2f_sgn, *cfa_sgn, *t_sg, *material, *face_kind, *edge_mode, *st_valid, *f2c_sgn, *f2e_sgn, *emode;
    const float *K, *recon, *fdx, *vol_inv;
    const float4 *fn, *eth, *emn;
    const float2 *esw;
    const char2 *fslot;
    const double *cell_volume; // FP64: the update divides the FP64-summed fluxes by it
};

MV make_view(const MeshView &m, const MixedTables &t)
{
    MV v;
    v.nc = m.nc; v.nf = m.nf; v.ne = m.ne; v.no_cells = m.no_cells; v.no_edges = m.no_edges;
    v.c2f_idx = m.c2f_idx; v.cfa_idx = m.cfa_idx; v.t_nb = m.t_nb; v.face_L = m.face_L; v.face_R = m.face_R;
    v.f2c_ptr = m.f2c_ptr; v.f2c_idx = m.f2c_idx; v.f2e_ptr = m.f2e_ptr; v.f2e_idx = m.f2e_idx; v.e2f_ptr = m.e2f_ptr;
    v.e2f_idx = m.e2f_idx; v.ec_ptr = m.ec_ptr; v.ec_cell = m.ec_cell;
    v.c2f_sgn = m.c2f_sgn; v.cfa_sgn = m.cfa_sgn; v.t_sg = m.t_sg; v.material = m.material; v.face_kind = m.face_kind;
    v.edge_mode = m.edge_mode; v.st_valid = m.st_valid; v.f2c_sgn = m.f2c_sgn; v.f2e_sgn = m.f2e_sgn;
    v.K = t.K.p; v.recon = t.recon.p; v.fdx = t.fdx.p; v.vol_inv = t.vol_inv.p;
    v.fn = t.fn.p; v.eth = t.eth.p; v.emn = t.emn.p; v.esw = t.esw.p; v.emode = t.emode.p;
    v.fslot = t.fslot.p;
    v.cell_volume = m.cell_volume;
    return v;
}

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float fdot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 fcross(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// the FP64 electron pressure of cell c that mx_prims leaves in the padding of species 0's pressure slot
__device__ __forceinline__ double mx_pe(const float4 *__restrict__ W, int32_t c)
{
    const float4 b = W[2 * (int64_t)c + 1];
    return __hiloint2double(__float_as_int(b.z), __float_as_int(b.w));
}

// ------------------------------------------------------------------ one-time tables (FP64 in, FP32 out)
__global__ void k_mx_cells(MeshView m, float *K, float *recon, float *vol_inv)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int64_t n = m.nc;
    // The least-squares gradient g = I sum_k wd_k dq_k projected on the face offsets dx_j, dl_j = dx_j . g,
    // is linear in the neighbour differences: dl_j = sum_k K_jk dq_k with K_jk = dx_j^T I wd_k (FP64 here,
    // stored in FP32; skipped faces take no part in the sum)
    {
        const double I00 = m.t_inv[c], I01 = m.t_inv[n + c], I02 = m.t_inv[2 * n + c], I11 = m.t_inv[3 * n + c],
                     I12 = m.t_inv[4 * n + c], I22 = m.t_inv[5 * n + c];
        for (int k = 0; k < 4; ++k)
        {
            const double w0 = m.t_wd[(3 * k) * n + c], w1 = m.t_wd[(3 * k + 1) * n + c], w2 = m.t_wd[(3 * k + 2) * n + c];
            const double h0 = I00 * w0 + I01 * w1 + I02 * w2, h1 = I01 * w0 + I11 * w1 + I12 * w2, h2 = I02 * w0 + I12 * w1 + I22 * w2;
            const bool skip = m.t_nb[k * n + c] == INT32_MIN;
            for (int j = 0; j < 4; ++j)
            {
                const double v = m.t_dx[(3 * j) * n + c] * h0 + m.t_dx[(3 * j + 1) * n + c] * h1 + m.t_dx[(3 * j + 2) * n + c] * h2;
                K[(4 * j + k) * n + c] = skip ? 0.f : static_cast<float>(v);
            }
        }
    }
    vol_inv[c] = static_cast<float>(1.0 / m.cell_volume[c]);
    // cell-field coefficients B_c = sum_j recon_j Phi_j of ImplicitInduction's constructor
    // (Common/induction/ImplicitInduction.cpp:34-62): recon_j = M^-1 n_j, M = sum A n n^T
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    V3 nn[4];
    double A[4];
    for (int j = 0; j < 4; ++j)
    {
        const int32_t f = m.c2f_idx[4 * (int64_t)c + j];
        A[j] = m.face_area_mag[f];
        nn[j] = A[j] > 0 ? (1.0 / A[j]) * ld3(m.face_area, f) : mk(0, 0, 0);
        const double nv[3] = {nn[j].x, nn[j].y, nn[j].z};
        if (A[j] > 0)
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) M[a][b] += A[j] * nv[a] * nv[b];
    }
    const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                       M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    const double sc = fmax(fmax(M[0][0], M[1][1]), fmax(M[2][2], 1e-300));
    double I[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (fabs(det) >= 1e-12 * sc * sc * sc)
    {
        I[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det; I[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
        I[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det; I[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) / det;
        I[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det; I[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
        I[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) / det; I[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) / det;
        I[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
    }
    for (int j = 0; j < 4; ++j)
        for (int a = 0; a < 3; ++a)
            recon[(3 * j + a) * n + c] = A[j] > 0 ? static_cast<float>(I[a][0] * nn[j].x + I[a][1] * nn[j].y + I[a][2] * nn[j].z) : 0.f;
}

__global__ void k_mx_faces(MeshView m, float4 *fn, float *fdx, char2 *fslot)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    // position of f in the c2f rows of its L and R cells (the face-value slot of k_mx_grad)
    {
        const int32_t L = m.face_L[f], R = m.face_R[f];
        signed char jl = 0, jr = 0;
        for (int j = 0; j < 4; ++j)
        {
            if (L >= 0 && m.c2f_idx[4 * (int64_t)L + j] == f) jl = static_cast<signed char>(j);
            if (R >= 0 && m.c2f_idx[4 * (int64_t)R + j] == f) jr = static_cast<signed char>(j);
        }
        fslot[f] = make_char2(jl, jr);
    }
    const int64_t n = m.nf;
    const double A = m.face_area_mag[f];
    const V3 nr = (1.0 / A) * ld3(m.face_area, f);
    fn[f] = make_float4(static_cast<float>(nr.x), static_cast<float>(nr.y), static_cast<float>(nr.z), static_cast<float>(A));
    const V3 xf = ld3(m.face_center, f);
    const int32_t L = m.face_L[f], R = m.face_R[f];
    const V3 dL = L >= 0 ? xf - ld3(m.cell_center, L) : mk(0, 0, 0);
    const V3 dR = R >= 0 ? xf - ld3(m.cell_center, R) : mk(0, 0, 0);
    fdx[0 * n + f] = static_cast<float>(dL.x); fdx[1 * n + f] = static_cast<float>(dL.y); fdx[2 * n + f] = static_cast<float>(dL.z);
    fdx[3 * n + f] = static_cast<float>(dR.x); fdx[4 * n + f] = static_cast<float>(dR.y); fdx[5 * n + f] = static_cast<float>(dR.z);
}

// Orthonormal basis (e1, e2) of the plane normal to the unit tangent th, built in single precision; the
// table builder and the edge pass both call it on the same single-precision tangent, so they pick the
// same helper axis and the same basis up to rounding.
__host__ __device__ __forceinline__ void edge_basis(float3 th, float3 &e1, float3 &e2)
{
    const float3 ax = fabsf(th.x) < 0.9f ? make_float3(1.f, 0.f, 0.f) : make_float3(0.f, 1.f, 0.f);
    e1 = make_float3(th.y * ax.z - th.z * ax.y, th.z * ax.x - th.x * ax.z, th.x * ax.y - th.y * ax.x);
    const float n1 = sqrtf(e1.x * e1.x + e1.y * e1.y + e1.z * e1.z);
    e1 = n1 > 0.f ? make_float3(e1.x / n1, e1.y / n1, e1.z / n1) : make_float3(0.f, 0.f, 0.f);
    e2 = make_float3(th.y * e1.z - th.z * e1.y, th.z * e1.x - th.x * e1.z, th.x * e1.y - th.y * e1.x);
}

__global__ void k_mx_edges(MeshView m, float4 *eth, int8_t *emode, float4 *emn, float2 *esw)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    const double L = m.edge_len[e];
    const V3 th = L > 0 ? (1.0 / L) * ld3(m.edge_vec, e) : mk(0, 0, 0);
    const float4 t4 = make_float4(static_cast<float>(th.x), static_cast<float>(th.y), static_cast<float>(th.z), static_cast<float>(L));
    eth[e] = t4;
    // the edge's mode in the mixed edge pass: edges that are not owned, or have no face, no length or no
    // fluid cell get E = 0 like wall edges (IdealEMF.cpp:59-70 skips them; Solver.cpp:162-167)
    int mode = e < m.no_edges ? m.edge_mode[e] : 1;
    if (mode == 0)
    {
        bool fluid = false;
        for (int32_t k = m.ec_ptr[e]; k < m.ec_ptr[e + 1]; ++k) fluid |= m.material[m.ec_cell[k]] == 0;
        if (!fluid || t4.w <= 0.f || m.e2f_ptr[e + 1] == m.e2f_ptr[e]) mode = 1;
    }
    emode[e] = static_cast<int8_t>(mode);
    float3 e1f, e2f;
    edge_basis(make_float3(t4.x, t4.y, t4.z), e1f, e2f);
    const V3 e1 = mk(e1f.x, e1f.y, e1f.z), e2 = mk(e2f.x, e2f.y, e2f.z);
    const V3 mid = ld3(m.edge_mid, e);
    for (int32_t k = m.e2f_ptr[e]; k < m.e2f_ptr[e + 1]; ++k)
    {
        const int32_t f = m.e2f_idx[k];
        V3 v = ld3(m.face_center, f) - mid;
        v = v - dot(v, th) * th;
        const double nv = sqrt(dot(v, v));
        const V3 mi = nv > 0 ? (1.0 / nv) * v : mk(0, 0, 0);
        const V3 nrm = (1.0 / m.face_area_mag[f]) * ld3(m.face_area, f);
        const double sig = dot(th, cross(mi, nrm));
        emn[k] = make_float4(static_cast<float>(dot(mi, e1)), static_cast<float>(dot(mi, e2)), static_cast<float>(dot(nrm, e1)),
                             static_cast<float>(dot(nrm, e2)));
        esw[k] = make_float2(static_cast<float>(sig), static_cast<float>(m.ef_weight[k]));
    }
}

__global__ void k_mx_badd(const double *badd, float4 *b32, int32_t nc)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    b32[c] = make_float4(static_cast<float>(badd[3 * (int64_t)c]), static_cast<float>(badd[3 * (int64_t)c + 1]),
                         static_cast<float>(badd[3 * (int64_t)c + 2]), 0.f);
}

// ------------------------------------------------------------------ stage kernels
struct MxParams
{
    int nsp, limit;
    float gamma, rel_limit, rho_floor, p_floor;
    double rho_floor_d, p_floor_d, gamma_d;
    F5 fs[kMaxSpecies];
    int8_t absorb[kMaxSpecies];
    float mass[kMaxSpecies];
    float M_ref;
    int src_on;                 // two-ion J x B force (species 0 = H+, 1 = Na+)
    float inver_MA2, ne_floor;
    int ambi, chem;             // ambipolar force, chemistry terms (two-ion model)
    double a1_Na, a4, a5, a6, sch, scn, T_ref, Tn0;
    const int32_t *wall_slot;   // the caller's Dirichlet wall states (FluidParams), global species index
    const double *wall_prim;
    int64_t wall_n;
};

// the caller's wall ghost of face f, species s, in FP32 (FluidParams wall table); false where ghost32 applies
__device__ __forceinline__ bool wall_ghost32(const MxParams &p, int kind, int32_t f, int s, F5 &g)
{
    if (kind != 1 || !p.wall_slot) return false;
    const int32_t k = p.wall_slot[f];
    if (k < 0) return false;
    const double *w = p.wall_prim + 5 * ((int64_t)s * p.wall_n + k);
    g = F5{static_cast<float>(w[0]), static_cast<float>(w[1]), static_cast<float>(w[2]), static_cast<float>(w[3]),
           static_cast<float>(w[4])};
    return true;
}

__device__ __forceinline__ F5 ghost32(int kind, bool absorb, const F5 &in, float3 n, const F5 &fs)
{
    if (kind == 1)
    {
        if (absorb) return F5{1e-12f, 0.f, 0.f, 0.f, 1e-12f};
        const float un = in.u * n.x + in.v * n.y + in.w * n.z;
        F5 g = in;
        g.u -= 2.f * un * n.x;
        g.v -= 2.f * un * n.y;
        g.w -= 2.f * un * n.z;
        return g;
    }
    if (kind == 2) return fs;
    return in;
}

__device__ __forceinline__ void rusanov32(const F5 &L, const F5 &R, float3 n, float gamma, float *F)
{
    const float gm1 = 1.f / (gamma - 1.f);
    const float EL = L.p * gm1 + 0.5f * L.rho * (L.u * L.u + L.v * L.v + L.w * L.w);
    const float ER = R.p * gm1 + 0.5f * R.rho * (R.u * R.u + R.v * R.v + R.w * R.w);
    const float unL = L.u * n.x + L.v * n.y + L.w * n.z, unR = R.u * n.x + R.v * n.y + R.w * n.z;
    const float mL = L.rho * unL, mR = R.rho * unR;
    const float sL = fabsf(unL) + sqrtf(gamma * L.p / L.rho), sR = fabsf(unR) + sqrtf(gamma * R.p / R.rho);
    const float s = fmaxf(sL, sR);
    F[0] = 0.5f * (mL + mR) - 0.5f * s * (R.rho - L.rho);
    F[1] = 0.5f * (mL * L.u + L.p * n.x + mR * R.u + R.p * n.x) - 0.5f * s * (R.rho * R.u - L.rho * L.u);
    F[2] = 0.5f * (mL * L.v + L.p * n.y + mR * R.v + R.p * n.y) - 0.5f * s * (R.rho * R.v - L.rho * L.v);
    F[3] = 0.5f * (mL * L.w + L.p * n.z + mR * R.w + R.p * n.z) - 0.5f * s * (R.rho * R.w - L.rho * L.w);
    F[4] = 0.5f * (unL * (EL + L.p) + unR * (ER + R.p)) - 0.5f * s * (ER - EL);
}

// per-cell primitives (FP32, 32 bytes per species) and the charge-weighted velocity u+ of cell c
__device__ __forceinline__ void mx_prims(const MxParams &p, int64_t n, const double *__restrict__ U, float4 *__restrict__ W,
                                         float4 *__restrict__ up, int32_t c, bool fluid)
{
    float ne = 0.f;
    double pe = 0.0;
    for (int s = 0; s < p.nsp; ++s)
    {
        const double *Us = U + (int64_t)s * 5 * n;
        const double r = fmax(Us[c], p.rho_floor_d);
        const double ir = 1.0 / r;
        const double u = Us[n + c] * ir, v = Us[2 * n + c] * ir, w = Us[3 * n + c] * ir;
        const double pr = fmax((p.gamma_d - 1.0) * (Us[4 * n + c] - 0.5 * r * (u * u + v * v + w * w)), p.p_floor_d);
        float4 *Wc = W + 2 * ((int64_t)s * n + c);
        Wc[0] = make_float4(static_cast<float>(r), static_cast<float>(u), static_cast<float>(v), static_cast<float>(w));
        Wc[1] = make_float4(static_cast<float>(pr), 0.f, 0.f, 0.f);
        ne += static_cast<float>(r) / p.mass[s] * p.M_ref;
        if (s < 2) pe += pr;
    }
    // with the ambipolar terms on, the FP64 electron pressure p_H + p_Na rides in the padding of species 0's
    // pressure slot (.z = high word, .w = low word): the gradients of p_e are differences of nearly equal
    // values that FP32 pressures would not resolve
    if (p.ambi)
        W[2 * (int64_t)c + 1] = make_float4(W[2 * (int64_t)c + 1].x, 0.f, __int_as_float(__double2hiint(pe)),
                                            __int_as_float(__double2loint(pe)));
    float u3[3] = {0.f, 0.f, 0.f};
    if (fluid)
        for (int s = 0; s < p.nsp; ++s)
        {
            // number density and velocity re-read from the primitives this thread has just written
            const float4 wv = W[2 * ((int64_t)s * n + c)];
            const float chi = ne > 1e-30f ? (wv.x / p.mass[s] * p.M_ref) / ne : (s == 0 ? 1.f : 0.f);
            u3[0] += chi * wv.y;
            u3[1] += chi * wv.z;
            u3[2] += chi * wv.w;
        }
    up[c] = make_float4(u3[0], u3[1], u3[2], 0.f);
}

// primitives (FP32), cell field fit, total field, charge-weighted velocity
__global__ void __launch_bounds__(128) k_mx_prepare(MV m, MxParams p, const double *__restrict__ U, const double *__restrict__ phi,
                                                     const float4 *__restrict__ badd, float4 *__restrict__ W, float4 *__restrict__ up,
                                                     float4 *__restrict__ bt, float4 *__restrict__ bi)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int64_t n = m.nc;
    mx_prims(p, n, U, W, up, c, m.material[c] == 0);
    const int4 fi = *reinterpret_cast<const int4 *>(m.c2f_idx + 4 * (int64_t)c);
    const float ph[4] = {static_cast<float>(phi[fi.x]), static_cast<float>(phi[fi.y]), static_cast<float>(phi[fi.z]),
                         static_cast<float>(phi[fi.w])};
    float b[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int a = 0; a < 3; ++a) b[a] += m.recon[(3 * j + a) * n + c] * ph[j];
    const float4 ba = badd[c];
    bi[c] = make_float4(b[0], b[1], b[2], 0.f);
    bt[c] = make_float4(b[0] + ba.x, b[1] + ba.y, b[2] + ba.z, 0.f);
}

// The opening half-step gyration (mercury::gyrate, FP64 on the FP64 state, FP32 total field) with the
// primitives and u+ of the cells it turns renewed, so that stage 1 starts prepared (B_ind and B_tot
// depend on Phi alone)
__global__ void __launch_bounds__(128) k_mx_gyrate(MV m, MxParams p, SrcParams sp, const float4 *__restrict__ bt,
                                                   const double *__restrict__ dtp, double scale, double *__restrict__ U,
                                                   float4 *__restrict__ W, float4 *__restrict__ up)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.no_cells || m.material[c] == 1) return;
    const int64_t n = m.nc;
    double uh[5], un[5];
    for (int q = 0; q < 5; ++q)
    {
        uh[q] = U[q * n + c];
        un[q] = U[(5 + q) * n + c];
    }
    gyrate_cell(sp, mk(bt[c].x, bt[c].y, bt[c].z), scale * *dtp, uh, un);
    for (int q = 1; q < 5; ++q)
    {
        U[q * n + c] = uh[q];
        U[(5 + q) * n + c] = un[q];
    }
    mx_prims(p, n, U, W, up, c, m.material[c] == 0);
}

__global__ void __launch_bounds__(128) k_mx_cfl(MV m, MxParams p, float cfl, float inver_MA2, float rho_floor_dt,
                                                 const float4 *__restrict__ W, const float4 *__restrict__ bt,
                                                 unsigned long long *__restrict__ dt_bits, int *__restrict__ flag)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = m.nc;
    float dt = CUDART_INF_F;
    if (c < m.no_cells && m.material[c] == 0)
    {
        const float3 b = f3(bt[c]);
        const float B2 = fdot(b, b);
        float rs = 0.f;
        for (int s = 0; s < p.nsp; ++s) rs += W[2 * ((int64_t)s * n + c)].x;
        const float rho_tot = fmaxf(rs, rho_floor_dt);
        const int4 fi = *reinterpret_cast<const int4 *>(m.c2f_idx + 4 * (int64_t)c);
        const float4 fn4[4] = {m.fn[fi.x], m.fn[fi.y], m.fn[fi.z], m.fn[fi.w]};
        const float vol = 1.f / m.vol_inv[c];
        for (int s = 0; s < p.nsp; ++s)
        {
            const float4 wa = W[2 * ((int64_t)s * n + c)];
            const float rho = wa.x, u = wa.y, v = wa.z, w = wa.w, pr = W[2 * ((int64_t)s * n + c) + 1].x;
            const float cs2 = p.gamma * pr / fmaxf(rho, 1e-30f);
            const float vA2 = inver_MA2 * B2 / rho_tot;
            float denom = 0.f;
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const float3 nr = f3(fn4[j]);
                const float bn = fdot(b, nr);
                const float vAn2 = inver_MA2 * bn * bn / rho_tot;
                const float term = cs2 + vA2;
                const float cf = sqrtf(0.5f * (term + sqrtf(fmaxf(0.f, term * term - 4.f * cs2 * vAn2))));
                denom += (fabsf(u * nr.x + v * nr.y + w * nr.z) + cf) * fn4[j].w;
            }
            if (denom > 0.f) dt = fminf(dt, cfl * vol / denom);
        }
        if (!(dt > 0.f)) atomicOr(flag, 1);
    }
    __shared__ float sh[32];
    float v = dt > 0.f ? dt : CUDART_INF_F;
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : CUDART_INF_F;
        for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0 && v < CUDART_INF_F)
            atomicMin(dt_bits, static_cast<unsigned long long>(__double_as_longlong(static_cast<double>(v))));
    }
}

// limited face values (see below) of cell c for species s0 + g of a group of ng: FV[(q*n + c)*ng + g] holds
// variable q at the cell's four faces (c2f order) as one float4
__device__ __forceinline__ void mx_grad_one(const MV &m, const MxParams &p, int s0, int g, int ng, int32_t c,
                                            const float4 *__restrict__ W, float4 *__restrict__ FV)
{
    const int s = s0 + g;
    const int64_t n = m.nc;
    // primitives of species s: 8 floats per cell (rho u v w | p - - -), one 32-byte sector per gather
    const float4 *Ws = W + 2 * (int64_t)s * n;
    auto prim = [&](int32_t cc, float *q5) {
        const float4 a = Ws[2 * (int64_t)cc], b = Ws[2 * (int64_t)cc + 1];
        q5[0] = a.x; q5[1] = a.y; q5[2] = a.z; q5[3] = a.w; q5[4] = b.x;
    };
    float4 *out = FV + (int64_t)c * ng + g;
    const int64_t qs = n * ng; // stride of variable q
    if (c >= m.no_cells || !m.st_valid[c])
    {
        // zero gradient: every face value is the cell value
        float w5[5];
        prim(c, w5);
#pragma unroll
        for (int q = 0; q < 5; ++q) out[q * qs] = make_float4(w5[q], w5[q], w5[q], w5[q]);
        return;
    }
    int32_t nb[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) nb[j] = m.t_nb[j * n + c];
    float wc[5], wn[4][5], K[16];
    prim(c, wc);
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (nb[j] >= 0) prim(nb[j], wn[j]);
#pragma unroll
    for (int i = 0; i < 16; ++i) K[i] = m.K[i * n + c];
    const F5 wcp{wc[0], wc[1], wc[2], wc[3], wc[4]};
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
        if (nb[j] == INT32_MIN)
        {
            // skipped face: no neighbour value (its column of K is zero, and it takes no part in the bounds)
#pragma unroll
            for (int q = 0; q < 5; ++q) wn[j][q] = wc[q];
        }
        else if (nb[j] < 0)
        {
            const int32_t f = -(nb[j] + 1);
            const float4 nf = m.fn[f];
            const float sg = m.t_sg[j * n + c];
            F5 gh;
            if (!wall_ghost32(p, m.face_kind[f], f, s, gh))
                gh = ghost32(m.face_kind[f], p.absorb[s] != 0, wcp, make_float3(sg * nf.x, sg * nf.y, sg * nf.z), p.fs[s]);
            wn[j][0] = gh.rho; wn[j][1] = gh.u; wn[j][2] = gh.v; wn[j][3] = gh.w; wn[j][4] = gh.p;
        }
    }
    // Limited face values v_j = w + psi dl_j, dl_j = g . dx_j (the face_state of FluxRHS.cpp:16-27 before its
    // positivity test) instead of the gradient.  The face that sets the Barth-Jespersen psi is snapped to its
    // bound, which exact arithmetic gives (w + (b - w)/dl * dl = b): near an absorbing wall the bound is the
    // 1e-12 floor state and the single-precision sum w + psi dl, with w ~ 1e-3, could not resolve it.
    float fv[5][4];
#pragma unroll
    for (int q = 0; q < 5; ++q)
    {
        float dq[4], lo = wc[q], hi = wc[q];
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            dq[k] = wn[k][q] - wc[q];
            lo = fminf(lo, wn[k][q]);
            hi = fmaxf(hi, wn[k][q]);
        }
        float dl[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) dl[j] = K[4 * j] * dq[0] + K[4 * j + 1] * dq[1] + K[4 * j + 2] * dq[2] + K[4 * j + 3] * dq[3];
        // Barth-Jespersen psi = min over the faces of (hi - w)/dl for dl > 0 and (lo - w)/dl for dl < 0: with
        // hi - w >= 0 >= lo - w the minimum is taken at the largest and at the most negative dl, so two
        // quotients per variable instead of four (likewise one for the relative limiter, at the largest |dl|)
        float dpos = 0.f, dneg = 0.f;
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            dpos = fmaxf(dpos, dl[j]);
            dneg = fminf(dneg, dl[j]);
        }
        // dsel: the extreme dl whose bound sets psi (0: none); every face at that dl is snapped to the bound
        float psi = 1.f, bound = 0.f, dsel = 0.f;
        if (p.limit)
        {
            if (dpos > 1e-30f)
            {
                const float r = (hi - wc[q]) / dpos;
                if (r < psi) { psi = r; dsel = dpos; bound = hi; }
            }
            if (dneg < -1e-30f)
            {
                const float r = (lo - wc[q]) / dneg;
                if (r < psi) { psi = r; dsel = dneg; bound = lo; }
            }
            if (p.rel_limit > 0.f && (q == 0 || q == 4))
            {
                const float a = fmaxf(dpos, -dneg);
                if (a > 1e-30f)
                {
                    const float r = p.rel_limit * wc[q] / a;
                    if (r < psi) { psi = r; dsel = 0.f; }
                }
            }
        }
        if (psi < 0.f) { psi = 0.f; dsel = 0.f; }
        psi = fminf(1.f, psi);
#pragma unroll
        for (int j = 0; j < 4; ++j) fv[q][j] = (dsel != 0.f && dl[j] == dsel) ? bound : wc[q] + psi * dl[j];
    }
    // positivity fallback of face_state: a face with rho <= 0 or p <= 0 takes the cell state
    bool ok[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) ok[j] = fv[0][j] > 0.f && fv[4][j] > 0.f;
#pragma unroll
    for (int q = 0; q < 5; ++q)
        out[q * qs] = make_float4(ok[0] ? fv[q][0] : wc[q], ok[1] ? fv[q][1] : wc[q], ok[2] ? fv[q][2] : wc[q], ok[3] ? fv[q][3] : wc[q]);
}

// Rusanov face flux times |A| of face f for species s0 + g of a group of ng: F[(f*ng + g)*5 + q], so that a
// face's fluxes of the whole group are one contiguous record for the update's gather
__device__ __forceinline__ void mx_flux_one(const MV &m, const MxParams &p, int s0, int g, int ng, int32_t f,
                                            const float *__restrict__ FV, float *__restrict__ F)
{
    const int s = s0 + g;
    const int64_t n = m.nc;
    float *Fo = F + ((int64_t)f * ng + g) * 5;
    const int kind = m.face_kind[f];
    const int32_t p0 = m.f2c_ptr[f], cnt = m.f2c_ptr[f + 1] - p0;
    const int32_t L = m.face_L[f], R = m.face_R[f];
    bool any = false;
    if (L >= 0) any |= L < m.no_cells && m.material[L] == 0;
    if (R >= 0) any |= R < m.no_cells && m.material[R] == 0;
    if (kind == 4 || !any)
    {
#pragma unroll
        for (int q = 0; q < 5; ++q) Fo[q] = 0.f;
        return;
    }
    const float4 nf4 = m.fn[f];
    const float3 nr = f3(nf4);
    const char2 sl = m.fslot[f];
    // reconstructed face state of cell c (positivity fallback already applied by k_mx_grad): slot j of the
    // cell's float4 of each variable
    const int64_t qs = 4 * n * ng;
    auto state = [&](int32_t c, int side) {
        const float *b = FV + ((int64_t)c * ng + g) * 4 + (side == 0 ? sl.x : sl.y);
        return F5{b[0], b[qs], b[2 * qs], b[3 * qs], b[4 * qs]};
    };
    F5 Ls, Rs;
    if (cnt == 2 && kind == 0)
    {
        Ls = state(L, 0);
        Rs = state(R, 1);
    }
    else
    {
        // the one fluid cell of a boundary / interface face (FluxRHS.cpp:58-66)
        int32_t c = m.f2c_idx[p0];
        int sgn = m.f2c_sgn[p0];
        if (cnt == 2 && m.material[c] != 0)
        {
            c = m.f2c_idx[p0 + 1];
            sgn = m.f2c_sgn[p0 + 1];
        }
        const F5 in = state(c, sgn > 0 ? 0 : 1);
        const float sf = static_cast<float>(sgn);
        F5 gh;
        if (!wall_ghost32(p, kind, f, s, gh)) gh = ghost32(kind, p.absorb[s] != 0, in, make_float3(sf * nr.x, sf * nr.y, sf * nr.z), p.fs[s]);
        if (sgn > 0) { Ls = in; Rs = gh; }
        else { Rs = in; Ls = gh; }
    }
    float Fl[5];
    rusanov32(Ls, Rs, nr, p.gamma, Fl);
#pragma unroll
    for (int q = 0; q < 5; ++q) Fo[q] = Fl[q] * nf4.w;
}

// The stage's primitives of one species from its FP64 conservative state, as mx_prims forms them (the same
// FP64 operations, rounded to FP32): the update takes them from the state it holds instead of re-reading
// the FP32 primitive records
struct Prim32
{
    float rho, u, v, w, p;
};
__device__ __forceinline__ Prim32 prims_of(const MxParams &p, const double *u)
{
    const double r = fmax(u[0], p.rho_floor_d);
    const double ir = 1.0 / r;
    const double vx = u[1] * ir, vy = u[2] * ir, vz = u[3] * ir;
    const double pr = fmax((p.gamma_d - 1.0) * (u[4] - 0.5 * r * (vx * vx + vy * vy + vz * vz)), p.p_floor_d);
    return Prim32{static_cast<float>(r), static_cast<float>(vx), static_cast<float>(vy), static_cast<float>(vz), static_cast<float>(pr)};
}

// U (FP64) += dt rhs, floors, SSP-RK2 average in stage 2; cell c, species s0 + g.  u holds the species'
// stage state on entry, r the FP64 sum of its face fluxes (the caller gathered them); ws, nH, nN are the
// stage primitives of this species and the ion number densities, jb = J x B_tot and d = V grad p_e of the
// cell (used by the two-ion sources only).
__device__ __forceinline__ void mx_update_one(const MV &m, const MxParams &p, int s0, int g, int32_t c, bool fluid, const double *r,
                                              double *__restrict__ u, double *__restrict__ Uo, const double *__restrict__ dtp, int stage2,
                                              const Prim32 &ws, float nH, float nN, float3 jb, float3 d, const double *__restrict__ photo,
                                              const double *__restrict__ vst, double *__restrict__ res)
{
    const int s = s0 + g;
    const int64_t n = m.nc;
    double *uo = Uo + (int64_t)s * 5 * n;
    if (fluid)
    {
        const float iv = m.vol_inv[c];
        const double dtv = *dtp * static_cast<double>(iv);
#pragma unroll
        for (int q = 0; q < 5; ++q) u[q] += dtv * r[q];
        if (p.src_on || p.ambi || p.chem)
        {
            // mercury::add_sources_n (MercurySources.cpp:29-60).  The J x B force in FP32 with the work of the
            // mid-point velocity, added to the FP64 update: J_c = (1/V) sum_f s_f G_f (the face terms of
            // k_mx_face_cand, same faces as the flux gather), S = inver_MA2 n_s / n_e,eff (J x B_tot).  The
            // ambipolar force -w_s grad p_e with grad p_e = (1/V) sum_f D_f.  The chemistry terms in FP64
            // from the FP32 primitives.
            const float ne = nH + nN;
            float Sx = 0.f, Sy = 0.f, Sz = 0.f;
            if (p.src_on)
            {
                const float k = p.inver_MA2 * (s == 0 ? nH : nN) / sqrtf(ne * ne + p.ne_floor * p.ne_floor);
                Sx = k * jb.x;
                Sy = k * jb.y;
                Sz = k * jb.z;
            }
            if (p.ambi)
            {
                const float ws = (s == 0 ? nH : nN) / sqrtf(ne * ne + p.ne_floor * p.ne_floor);
                Sx -= ws * iv * d.x;
                Sy -= ws * iv * d.y;
                Sz -= ws * iv * d.z;
            }
            const float rho = fmaxf(ws.rho, 0.f);
            const double dt = *dtp;
            const float work = ws.u * Sx + ws.v * Sy + ws.w * Sz +
                               (rho > 1e-30f ? 0.5f * static_cast<float>(dt) * (Sx * Sx + Sy * Sy + Sz * Sz) / rho : 0.f);
            u[1] += dt * static_cast<double>(Sx);
            u[2] += dt * static_cast<double>(Sy);
            u[3] += dt * static_cast<double>(Sz);
            u[4] += dt * static_cast<double>(work);
            if (p.chem && vst)
            {
                const double v = vst[c], r = rho, ux = ws.u, uy = ws.v, uz = ws.w, ps = ws.p;
                const double u2 = ux * ux + uy * uy + uz * uz;
                const double Ts = ps / (r > 0 ? r : 1e-300) / (s == 0 ? p.sch : p.scn) * p.T_ref;
                const double mH = p.mass[0], mN = p.mass[1], Msum = mH + mN;
                const double b1 = v * (p.Tn0 - Ts) * (s == 0 ? mH / Msum : 0.5);
                const double b2 = (s == 0 ? mN / Msum : 0.5) * v;
                const double ns = s == 0 ? nH : nN;
                u[1] -= dt * (p.a4 * r * ux * v);
                u[2] -= dt * (p.a4 * r * uy * v);
                u[3] -= dt * (p.a4 * r * uz * v);
                u[4] += dt * (-p.a4 * r * u2 * v + p.a5 * ns * b1 + p.a4 * r * u2 * b2);
                if (s == 1 && photo)
                {
                    u[0] += dt * (p.a1_Na * photo[c]);
                    u[4] += dt * (p.a6 * photo[c] * p.Tn0);
                }
            }
        }
        const double ke = u[0] > 0 ? 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0] : 0.0;
        const double gm = p.gamma_d;
        if (!(u[0] >= p.rho_floor_d))
        {
            u[0] = p.rho_floor_d; u[1] = u[2] = u[3] = 0.0;
            u[4] = p.p_floor_d / (gm - 1.0);
        }
        else if ((gm - 1.0) * (u[4] - ke) < p.p_floor_d)
            u[4] = p.p_floor_d / (gm - 1.0) + ke;
    }
    if (stage2)
#pragma unroll
        for (int q = 0; q < 5; ++q) res[q] = 0.5 * (uo[q * n + c] + u[q]);
    else
#pragma unroll
        for (int q = 0; q < 5; ++q) res[q] = u[q];
}

// face EMF candidates E_f = -n x F_f (IdealEMF.cpp:32-55), 3 per face (structure of arrays)
// With G: also the face term of the cell current, G_f = A_f x b_f, b_f = (b_L + b_R)/2 or the one
// cell's b (mhd::cell_current, Common/induction/Current.cpp:9-31); cell c sums +-G over its faces.
__global__ void __launch_bounds__(128) k_mx_face_cand(MV m, const float4 *__restrict__ up, const float4 *__restrict__ bt,
                                                      const float4 *__restrict__ bi, const double *__restrict__ phi,
                                                      const double *__restrict__ phi_add, float4 *__restrict__ Ef,
                                                      float4 *__restrict__ G, const float4 *__restrict__ W, float4 *__restrict__ D)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    const float4 nf4 = m.fn[f];
    const float3 n = f3(nf4);
    const float Bn = static_cast<float>(phi[f] + phi_add[f]) / nf4.w;
    const int32_t L = m.face_L[f], R = m.face_R[f];
    float3 F;
    auto flux = [&](int32_t c) {
        const float3 uc = f3(up[c]), bc = f3(bt[c]);
        const float un = fdot(uc, n);
        return make_float3(un * bc.x - Bn * uc.x, un * bc.y - Bn * uc.y, un * bc.z - Bn * uc.z);
    };
    if (L >= 0 && R >= 0)
    {
        const float a = fmaxf(fabsf(fdot(f3(up[L]), n)), fabsf(fdot(f3(up[R]), n)));
        const float3 FL = flux(L), FR = flux(R);
        const float3 bL = f3(bi[L]), bR = f3(bi[R]);
        F = make_float3(0.5f * (FL.x + FR.x) - 0.5f * a * (bR.x - bL.x), 0.5f * (FL.y + FR.y) - 0.5f * a * (bR.y - bL.y),
                        0.5f * (FL.z + FR.z) - 0.5f * a * (bR.z - bL.z));
    }
    else
        F = flux(L >= 0 ? L : R);
    if (G)
    {
        const float3 bL = L >= 0 ? f3(bi[L]) : f3(bi[R]), bR = R >= 0 ? f3(bi[R]) : bL;
        const float3 bf = L >= 0 && R >= 0 ? make_float3(0.5f * (bL.x + bR.x), 0.5f * (bL.y + bR.y), 0.5f * (bL.z + bR.z)) : bL;
        const float3 g = fcross(make_float3(nf4.w * n.x, nf4.w * n.y, nf4.w * n.z), bf);
        G[f] = make_float4(g.x, g.y, g.z, 0.f);
    }
    if (D)
    {
        // mercury::electron_pressure_gradient (Ambipolar.cpp:10-31) sums p_f s_f A_f over the cell's faces with
        // p_f the mean with a fluid neighbour, the cell's own p_c elsewhere.  As sum (p_f - p_c) s_f A_f (the
        // faces of a cell close: sum s_f A_f = 0) only faces between two fluid cells contribute, and both
        // cells receive the same vector (p_R - p_L) A_f / 2, formed from the FP64 p_e
        float dp = 0.f;
        if (L >= 0 && R >= 0 && m.material[L] == 0 && m.material[R] == 0) dp = static_cast<float>(0.5 * (mx_pe(W, R) - mx_pe(W, L)));
        D[f] = make_float4(dp * nf4.w * n.x, dp * nf4.w * n.y, dp * nf4.w * n.z, 0.f);
    }
    const float3 E = fcross(n, F);
    // with Phi_ind / |A| of the face, which the edge pass needs for its dissipation term: one 16-byte
    // gather per (edge, face) there
    Ef[f] = make_float4(-E.x, -E.y, -E.z, static_cast<float>(phi[f]) / nf4.w);
}

// UCT edge EMF (IdealEMF.cpp:59-128) with the boundary edge values (Solver.cpp:162-167), one thread per
// edge.  The faces' terms enter only through sums, so one pass over the faces accumulates them: with
// q_i = (q_a, q_b), w_i the face weight and x_i = w_i a_i sigma_i Phi_i/|A_i|,
//   M = sum w q q^T, g = sum w q, E_u = sum (1 - q . l) x = sum x - l . sum q x,  l = M^-1 g,
// so no per-face state is kept between two passes.  Everything happens in the plane normal to the edge,
// in the basis (e1, e2) of edge_basis: the in-face directions m_f and the face normals come from the
// per-(edge, face) table in that basis, and the velocities of the edge's cells (at most 8 on the meshes
// the mixed path takes) are projected onto it once and held in registers, so a_f = max_c |u_c . m_f| costs
// no memory traffic per face.  Per face the pass gathers only the 16-byte EMF candidate record.
__global__ void __launch_bounds__(128, 8) k_mx_edge(MV m, const float4 *__restrict__ Ef, const float4 *__restrict__ up,
                                                    float cuct, float3 E_inf, float *__restrict__ E)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    float val = 0.f;
    const float4 t4 = m.eth[e];
    const float Lg = t4.w;
    const float3 th = f3(t4);
    const int mode = m.emode[e];
    if (mode == 2) val = Lg * fdot(E_inf, th);
    else if (mode == 0)
    {
        float3 e1, e2;
        edge_basis(th, e1, e2);
        const int32_t q0 = m.ec_ptr[e], nce = m.ec_ptr[e + 1] - q0;
        const int32_t f0 = m.e2f_ptr[e], nfe = m.e2f_ptr[e + 1] - f0;
        // the velocities of the edge's cells in the plane normal to the edge (the mesh check admits at most 8)
        constexpr int kCells = 8;
        float pa[kCells], pb[kCells];
#pragma unroll
        for (int k = 0; k < kCells; ++k)
        {
            pa[k] = 0.f;
            pb[k] = 0.f;
            if (k < nce)
            {
                const float3 u = f3(up[m.ec_cell[q0 + k]]);
                pa[k] = fdot(u, e1);
                pb[k] = fdot(u, e2);
            }
        }
        float Ec = 0.f, M11 = 0.f, M12 = 0.f, M22 = 0.f, g1 = 0.f, g2 = 0.f, S0 = 0.f, S1 = 0.f, S2 = 0.f;
        // the next face's index is loaded one iteration ahead, so that a face's gather waits on one load
        int32_t f_next = m.e2f_idx[f0];
#pragma unroll 1
        for (int i = 0; i < nfe; ++i)
        {
            const int32_t f = f_next;
            if (i + 1 < nfe) f_next = m.e2f_idx[f0 + i + 1];
            const float4 mn = m.emn[f0 + i];
            const float2 sw = m.esw[f0 + i];
            const float4 ef = Ef[f];
            const float w = sw.y;
            Ec += w * (ef.x * th.x + ef.y * th.y + ef.z * th.z);
            float a = 0.f;
#pragma unroll
            for (int k = 0; k < kCells; ++k) a = fmaxf(a, fabsf(pa[k] * mn.x + pb[k] * mn.y));
            const float as = a * sw.x;
            const float qa = as * mn.z;
            const float qb = as * mn.w;
            const float wx = w * as * ef.w;
            M11 += w * qa * qa;
            M12 += w * qa * qb;
            M22 += w * qb * qb;
            g1 += w * qa;
            g2 += w * qb;
            S0 += wx;
            S1 += qa * wx;
            S2 += qb * wx;
        }
        const float tr = M11 + M22;
        const float eps = 1e-14f * tr;
        const float det = (M11 + eps) * (M22 + eps) - M12 * M12;
        float l1 = 0.f, l2 = 0.f;
        if (tr > 0.f && det > 0.f)
        {
            l1 = ((M22 + eps) * g1 - M12 * g2) / det;
            l2 = ((M11 + eps) * g2 - M12 * g1) / det;
        }
        const float Eu = S0 - (l1 * S1 + l2 * S2);
        val = Lg * Ec + 2.f * cuct * Lg * Eu;
    }
    E[e] = val;
}

// Phi -= dt d1 E on the active faces (mhd::active_faces, Faraday.cpp:7-13), E summed in FP64; stage 2
// averages with Phi0.  The faces of a tetrahedral mesh are triangles: one 16-byte record per face holds its
// three edges (f2e order) and, in the last word, the edges' negative signs (bits 0-2) and the active flag
// (bit 3), so the pass reads one coalesced record instead of the CSR rows of f2e and f2c.
__global__ void __launch_bounds__(256) k_mx_ct(int32_t nf, const int4 *__restrict__ fe, const float *__restrict__ E,
                                               const double *__restrict__ phis, double *__restrict__ phio, const double *__restrict__ dtp,
                                               int stage2)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int4 r = fe[f];
    double v = phis[f];
    if (r.w & 8)
    {
        const double e0 = E[r.x], e1 = E[r.y], e2 = E[r.z];
        const double circ = ((r.w & 1) ? -e0 : e0) + ((r.w & 2) ? -e1 : e1) + ((r.w & 4) ? -e2 : e2);
        v -= *dtp * circ;
    }
    phio[f] = stage2 ? 0.5 * (phio[f] + v) : v;
}

__global__ void k_mx_face_edges(MeshView m, int4 *fe)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    bool active = false;
    for (int32_t k = m.f2c_ptr[f]; k < m.f2c_ptr[f + 1]; ++k) active |= m.f2c_idx[k] < m.no_cells;
    const int32_t k0 = m.f2e_ptr[f];
    int w = active ? 8 : 0;
    for (int i = 0; i < 3; ++i) w |= m.f2e_sgn[k0 + i] < 0 ? (1 << i) : 0;
    fe[f] = make_int4(m.f2e_idx[k0], m.f2e_idx[k0 + 1], m.f2e_idx[k0 + 2], w);
}

__global__ void k_mx_cfl_init(unsigned long long *dt_bits, int *flag)
{
    *dt_bits = static_cast<unsigned long long>(__double_as_longlong(CUDART_INF));
    *flag = 0;
}

__global__ void k_mx_cfl_final(const unsigned long long *dt_bits, double dt_max, double *dt, int *flag)
{
    double g = __longlong_as_double(static_cast<long long>(*dt_bits));
    g = fmin(g, dt_max);
    if (!isfinite(g) || g <= 0) atomicOr(flag, 1);
    *dt = g;
}

// Face values and fluxes: the species of a group run as adjacent threads (thread t: cell or face t / ng,
// species t % ng).  The two threads of a cell read the same stencil tables (one load serves both), write
// the adjacent float4s of its face values, and the two threads of a face read adjacent face values and
// write adjacent halves of the face's flux record, so every gather and store of the pair shares its
// sectors.  The update keeps the group's species in one thread per cell and gathers each face's record
// once for both.
__global__ void __launch_bounds__(128) k_mx_grad(MV m, MxParams p, int s0, int ng, const float4 *__restrict__ W,
                                                 float4 *__restrict__ FV)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t c = ng == 2 ? t >> 1 : t;
    if (c >= m.nc) return;
    mx_grad_one(m, p, s0, ng == 2 ? static_cast<int>(t & 1) : 0, ng, static_cast<int32_t>(c), W, FV);
}

__global__ void __launch_bounds__(128) k_mx_flux(MV m, MxParams p, int s0, int ng, const float *__restrict__ FV, float *__restrict__ F)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t f = ng == 2 ? t >> 1 : t;
    if (f >= m.nf) return;
    mx_flux_one(m, p, s0, ng == 2 ? static_cast<int>(t & 1) : 0, ng, static_cast<int32_t>(f), FV, F);
}

// gyr: the closing half-step gyration of the Strang splitting (mercury::gyrate, FP64 on the averaged
// state, with the total field of the stage-2 prepare) applied to the cell's two ions before they are
// written, instead of in a pass of its own
template <bool GYR>
__global__ void __launch_bounds__(128) k_mx_update(MV m, MxParams p, int s0, int ng, const float *__restrict__ F,
                                                   const double *__restrict__ Ub, double *__restrict__ Uo, const double *__restrict__ dtp,
                                                   int stage2, const float4 *__restrict__ G,
                                                   const float4 *__restrict__ bt, SrcParams sp, int gyr, const float4 *__restrict__ D,
                                                   const double *__restrict__ photo, const double *__restrict__ vst)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int64_t n = m.nc;
    double r0[5], r1[5], u0[5], u1[5];
    const double *ub = Ub + (int64_t)s0 * 5 * n;
    if (stage2)
    {
        // the step's opening state, read at the end of the second stage, on its way to L2 while the flux
        // records are gathered
        const double *un = Uo + (int64_t)s0 * 5 * n + c;
#pragma unroll
        for (int q = 0; q < 10; ++q)
            if (q < 5 * ng) asm volatile("prefetch.global.L2 [%0];" ::"l"(un + q * n));
    }
#pragma unroll
    for (int q = 0; q < 5; ++q)
    {
        u0[q] = ub[q * n + c];
        u1[q] = ng > 1 ? ub[(5 + q) * n + c] : 0.0;
    }
    // the four faces' flux records, summed in FP64 (the rhs is a difference of fluxes that can nearly cancel);
    // with two species a face's record is 10 floats at an 8-byte boundary, read as five float2
    const bool fluid = c < m.no_cells && m.material[c] == 0;
    int32_t ff[4] = {0, 0, 0, 0};
    double sv[4] = {0, 0, 0, 0}, f0[5] = {0, 0, 0, 0, 0}, f1[5] = {0, 0, 0, 0, 0};
    if (fluid)
    {
        const int4 fi = *reinterpret_cast<const int4 *>(m.cfa_idx + 4 * (int64_t)c);
        const char4 sg = *reinterpret_cast<const char4 *>(m.cfa_sgn + 4 * (int64_t)c);
        ff[0] = fi.x; ff[1] = fi.y; ff[2] = fi.z; ff[3] = fi.w;
        sv[0] = sg.x > 0 ? -1.0 : 1.0; sv[1] = sg.y > 0 ? -1.0 : 1.0; sv[2] = sg.z > 0 ? -1.0 : 1.0; sv[3] = sg.w > 0 ? -1.0 : 1.0;
        if (ng == 2)
        {
            const float2 *R = reinterpret_cast<const float2 *>(F);
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const float2 a = R[5 * (int64_t)ff[j]], b = R[5 * (int64_t)ff[j] + 1], d = R[5 * (int64_t)ff[j] + 2],
                             e = R[5 * (int64_t)ff[j] + 3], h = R[5 * (int64_t)ff[j] + 4];
                f0[0] += sv[j] * static_cast<double>(a.x); f0[1] += sv[j] * static_cast<double>(a.y);
                f0[2] += sv[j] * static_cast<double>(b.x); f0[3] += sv[j] * static_cast<double>(b.y);
                f0[4] += sv[j] * static_cast<double>(d.x);
                f1[0] += sv[j] * static_cast<double>(d.y); f1[1] += sv[j] * static_cast<double>(e.x);
                f1[2] += sv[j] * static_cast<double>(e.y); f1[3] += sv[j] * static_cast<double>(h.x);
                f1[4] += sv[j] * static_cast<double>(h.y);
            }
        }
        else
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int q = 0; q < 5; ++q) f0[q] += sv[j] * static_cast<double>(F[5 * (int64_t)ff[j] + q]);
    }
    // the two-ion sources (their switches require exactly the species 0 and 1 in this thread) need the stage
    // primitives of both ions
    Prim32 w0{}, w1{};
    float nH = 0.f, nN = 0.f;
    if (p.src_on || p.ambi || p.chem)
    {
        w0 = prims_of(p, u0);
        w1 = prims_of(p, u1);
        nH = fmaxf(w0.rho, 0.f) / p.mass[0] * p.M_ref;
        nN = fmaxf(w1.rho, 0.f) / p.mass[1] * p.M_ref;
    }
    // the cell current from the face terms of the face-candidate pass, J_c = (1/V) sum_f s_f G_f over the
    // faces of the flux gather, and J x B_tot; the face terms D_f of grad p_e (already oriented: the same
    // vector for both cells of the face)
    float3 jb = make_float3(0.f, 0.f, 0.f), dsum = make_float3(0.f, 0.f, 0.f);
    if (fluid && p.src_on)
    {
        float3 Jc = make_float3(0.f, 0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const float4 g = G[ff[j]];
            const float sj = sv[j] < 0.0 ? 1.f : -1.f; // +1 where the canonical normal points out of c
            Jc.x += sj * g.x;
            Jc.y += sj * g.y;
            Jc.z += sj * g.z;
        }
        const float iv = m.vol_inv[c];
        jb = fcross(make_float3(iv * Jc.x, iv * Jc.y, iv * Jc.z), f3(bt[c]));
    }
    if (fluid && p.ambi)
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const float4 g = D[ff[j]];
            dsum.x += g.x;
            dsum.y += g.y;
            dsum.z += g.z;
        }
    mx_update_one(m, p, s0, 0, c, fluid, f0, u0, Uo, dtp, stage2, w0, nH, nN, jb, dsum, photo, vst, r0);
    if (ng > 1) mx_update_one(m, p, s0, 1, c, fluid, f1, u1, Uo, dtp, stage2, w1, nH, nN, jb, dsum, photo, vst, r1);
    if (GYR && gyr && ng == 2 && c < m.no_cells && m.material[c] != 1) gyrate_cell(sp, mk(bt[c].x, bt[c].y, bt[c].z), 0.5 * *dtp, r0, r1);
    double *uo = Uo + (int64_t)s0 * 5 * n;
#pragma unroll
    for (int q = 0; q < 5; ++q) uo[q * n + c] = r0[q];
    if (ng > 1)
#pragma unroll
        for (int q = 0; q < 5; ++q) uo[(5 + q) * n + c] = r1[q];
}

// nodal p_e of AmbipolarEMF::add (Ambipolar.cpp:57-68) from the FP64 p_e of the cells
__global__ void k_mx_node_pressure(int32_t nn, const int32_t *__restrict__ n2c_ptr, const int32_t *__restrict__ n2c_cell,
                                   const double *__restrict__ vol, const float4 *__restrict__ W, double *__restrict__ pn,
                                   int8_t *__restrict__ pok)
{
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    double s = 0, w = 0;
    for (int32_t k = n2c_ptr[v]; k < n2c_ptr[v + 1]; ++k)
    {
        const int32_t c = n2c_cell[k];
        s += vol[c] * mx_pe(W, c);
        w += vol[c];
    }
    pn[v] = w > 0 ? s / w : 0.0;
    pok[v] = n2c_ptr[v + 1] > n2c_ptr[v] ? 1 : 0;
}

// AmbipolarEMF::add on the owned free edges (the reference overwrites wall and inflow edges), FP32, E in place
__global__ void k_mx_ambipolar(MV m, MxParams p, const float4 *__restrict__ W, const double *__restrict__ ecw, const int32_t *__restrict__ en,
                               const double *__restrict__ pn, const int8_t *__restrict__ pok, float coef, float *__restrict__ E)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.no_edges || m.edge_mode[e] != 0) return;
    float rH = 0.f, rN = 0.f, wsum = 0.f;
    for (int32_t k = m.ec_ptr[e]; k < m.ec_ptr[e + 1]; ++k)
    {
        const int32_t c = m.ec_cell[k];
        if (m.material[c] == 1) continue;
        const float w = static_cast<float>(ecw[k]);
        rH += w * W[2 * (int64_t)c].x;
        rN += w * W[2 * ((int64_t)m.nc + c)].x;
        wsum += w;
    }
    if (wsum <= 0.f) return;
    const float nH = fmaxf(rH / wsum, 0.f) / p.mass[0] * p.M_ref, nN = fmaxf(rN / wsum, 0.f) / p.mass[1] * p.M_ref;
    const float ne = nH + nN;
    const int32_t a = en[2 * (int64_t)e], b = en[2 * (int64_t)e + 1];
    if (!pok[a] || !pok[b]) return;
    E[e] -= coef * static_cast<float>(pn[b] - pn[a]) / sqrtf(ne * ne + p.ne_floor * p.ne_floor);
}

MxParams mx_params(const MhdState *st)
{
    MxParams p{};
    const MhdStepParams &q = st->prm;
    p.nsp = st->nsp;
    p.limit = 1;
    p.gamma = static_cast<float>(q.gamma);
    p.gamma_d = q.gamma;
    p.rel_limit = static_cast<float>(q.rel_limit);
    p.rho_floor = static_cast<float>(q.rho_floor);
    p.p_floor = static_cast<float>(q.p_floor);
    p.rho_floor_d = q.rho_floor;
    p.p_floor_d = q.p_floor;
    p.M_ref = static_cast<float>(q.M_ref);
    p.src_on = st->src.on;
    p.inver_MA2 = static_cast<float>(q.inver_MA2);
    p.ne_floor = static_cast<float>(q.ne_floor);
    p.ambi = st->src.ambi;
    p.chem = st->src.chem;
    p.a1_Na = q.a1_Na; p.a4 = q.a4; p.a5 = q.a5; p.a6 = q.a6;
    p.sch = q.state_coeff_H; p.scn = q.state_coeff_Na; p.T_ref = q.T_ref; p.Tn0 = q.Tn0;
    p.wall_slot = st->fp.wall_slot;
    p.wall_prim = st->fp.wall_prim;
    p.wall_n = st->fp.wall_n;
    for (int s = 0; s < st->nsp; ++s)
    {
        p.fs[s] = F5{static_cast<float>(q.fs[s].rho), static_cast<float>(q.fs[s].u), static_cast<float>(q.fs[s].v),
                     static_cast<float>(q.fs[s].w), static_cast<float>(q.fs[s].p)};
        p.absorb[s] = q.absorb[s];
        p.mass[s] = static_cast<float>(q.mass[s]);
    }
    return p;
}
} // namespace

void mixed_setup(MhdState *st)
{
    MhdMesh *mesh = st->mesh;
    const MeshView &m = mesh->v;
    cudaStream_t s = mesh->stream;
    MixedTables &t = st->mt;
    const size_t nc = m.nc, nf = m.nf, ne = m.ne;
    int32_t nnz_e2f = 0;
    MHD_CUDA(cudaMemcpy(&nnz_e2f, m.e2f_ptr + m.ne, sizeof(int32_t), cudaMemcpyDeviceToHost));
    t.K.alloc(16 * nc); t.recon.alloc(12 * nc); t.vol_inv.alloc(nc);
    if (st->src.on) st->g32.alloc(nf);
    if (st->src.ambi) st->d32.alloc(nf);
    t.fn.alloc(nf); t.fdx.alloc(6 * nf); t.fslot.alloc(nf); t.fe.alloc(nf);
    t.eth.alloc(ne); t.emode.alloc(ne); t.emn.alloc(nnz_e2f); t.esw.alloc(nnz_e2f);
    if (nc) k_mx_cells<<<grid_for(nc, 128), 128, 0, s>>>(m, t.K.p, t.recon.p, t.vol_inv.p);
    if (nf) k_mx_faces<<<grid_for(nf, 256), 256, 0, s>>>(m, t.fn.p, t.fdx.p, t.fslot.p);
    if (nf) k_mx_face_edges<<<grid_for(nf, 256), 256, 0, s>>>(m, t.fe.p);
    if (ne) k_mx_edges<<<grid_for(ne, 128), 128, 0, s>>>(m, t.eth.p, t.emode.p, t.emn.p, t.esw.p);
    MHD_LAUNCH_CHECK();
    st->W32.alloc(8 * nc * st->nsp); // 8 floats per (species, cell): rho u v w | p, padded to 32 bytes
    st->grad32.alloc(20 * nc * st->group); // limited face values, 5 variables x 4 faces per cell
    st->F32.alloc(5 * nf * st->group);
    st->Ef32.alloc(nf);
    st->E32.alloc(ne);
    st->up32.alloc(nc); st->bt32.alloc(nc); st->bi32.alloc(nc); st->badd32.alloc(nc);
    if (nc) MHD_CUDA(cudaMemsetAsync(st->badd32.p, 0, nc * sizeof(float4), s));
    MHD_CUDA(cudaStreamSynchronize(s));
}

void mixed_badd(MhdState *st)
{
    const MeshView &m = st->mesh->v;
    if (!m.nc) return;
    k_mx_badd<<<grid_for(m.nc, 256), 256, 0, st->mesh->stream>>>(st->badd.p, st->badd32.p, m.nc);
    MHD_LAUNCH_CHECK();
}

void mixed_prepare(MhdState *st, const double *Us, const double *phis, bool cfl, double dt_max)
{
    MhdMesh *mesh = st->mesh;
    const MV m = make_view(mesh->v, st->mt);
    cudaStream_t s = mesh->stream;
    Profiler &P = st->prof;
    const MxParams p = mx_params(st);
    const int gc = grid_for(m.nc, 128);
    if (!m.nc) return;
    float4 *W4 = reinterpret_cast<float4 *>(st->W32.p);
    P.begin(KP_PREPARE, s);
    k_mx_prepare<<<gc, 128, 0, s>>>(m, p, Us, phis, st->badd32.p, W4, st->up32.p, st->bt32.p, st->bi32.p);
    MHD_LAUNCH_CHECK();
    ++st->launches;
    P.end(KP_PREPARE, s);
    if (cfl)
    {
        P.begin(KP_CFL, s);
        k_mx_cfl_init<<<1, 1, 0, s>>>(st->dt_bits.p, st->flag.p);
        k_mx_cfl<<<gc, 128, 0, s>>>(m, p, static_cast<float>(st->prm.cfl), static_cast<float>(st->prm.inver_MA2),
                                    static_cast<float>(st->prm.rho_floor_dt), W4, st->bt32.p, st->dt_bits.p, st->flag.p);
        k_mx_cfl_final<<<1, 1, 0, s>>>(st->dt_bits.p, dt_max, st->scal.p, st->flag.p);
        MHD_LAUNCH_CHECK();
        P.end(KP_CFL, s);
        st->launches += 3;
    }
}

void mixed_gyrate_open(MhdState *st)
{
    const MV m = make_view(st->mesh->v, st->mt);
    if (!m.no_cells) return;
    k_mx_gyrate<<<grid_for(m.no_cells, 128), 128, 0, st->mesh->stream>>>(m, mx_params(st), st->src, st->bt32.p, st->scal.p, 0.5,
                                                                            st->U0.p, reinterpret_cast<float4 *>(st->W32.p), st->up32.p);
    MHD_LAUNCH_CHECK();
    ++st->launches;
}

void mixed_stage(MhdState *st, const double *Us, const double *phis, double *Uo, double *phio, bool stage2, bool cfl, double dt_max,
                 bool prepared, bool gyrate_close)
{
    MhdMesh *mesh = st->mesh;
    const MeshView &mv = mesh->v;
    const MV m = make_view(mv, st->mt);
    cudaStream_t s = mesh->stream;
    Profiler &P = st->prof;
    const MxParams p = mx_params(st);
    const int gc = grid_for(m.nc, 128), gf = grid_for(m.nf, 128), ge = grid_for(m.ne, 128);
    if (!m.nc) return;
    float4 *W4 = reinterpret_cast<float4 *>(st->W32.p);
    if (!prepared) mixed_prepare(st, Us, phis, cfl, dt_max);
    // face EMF candidates first: with the J x B force on, this pass also leaves the face terms of the
    // cell current that the update gathers
    P.begin(KP_FACE_CAND, s);
    k_mx_face_cand<<<gf, 128, 0, s>>>(m, st->up32.p, st->bt32.p, st->bi32.p, phis, st->phi_add.p, st->Ef32.p,
                                      st->src.on ? st->g32.p : nullptr, W4, st->src.ambi ? st->d32.p : nullptr);
    MHD_LAUNCH_CHECK();
    P.end(KP_FACE_CAND, s);
    for (int s0 = 0; s0 < st->nsp; s0 += st->group)
    {
        const int ng = std::min(st->group, st->nsp - s0);
        P.begin(KP_GRAD, s);
        k_mx_grad<<<grid_for(static_cast<int64_t>(m.nc) * ng, 128), 128, 0, s>>>(m, p, s0, ng, W4,
                                                                                   reinterpret_cast<float4 *>(st->grad32.p));
        MHD_LAUNCH_CHECK();
        P.end(KP_GRAD, s);
        P.begin(KP_FLUX, s);
        k_mx_flux<<<grid_for(static_cast<int64_t>(m.nf) * ng, 128), 128, 0, s>>>(m, p, s0, ng, st->grad32.p, st->F32.p);
        MHD_LAUNCH_CHECK();
        P.end(KP_FLUX, s);
        P.begin(KP_UPDATE, s);
        // the instance with the closing gyration fused carries its registers; the other stages use the lean one
        auto upd = gyrate_close && s0 == 0 ? k_mx_update<true> : k_mx_update<false>;
        upd<<<gc, 128, 0, s>>>(m, p, s0, ng, st->F32.p, Us, Uo, st->scal.p, stage2 ? 1 : 0, st->g32.p, st->bt32.p, st->src,
                               gyrate_close && s0 == 0 ? 1 : 0, st->src.ambi ? st->d32.p : nullptr,
                               st->src.chem && st->photo.n ? st->photo.p : nullptr, st->src.chem && st->vst.n ? st->vst.p : nullptr);
        MHD_LAUNCH_CHECK();
        P.end(KP_UPDATE, s);
        st->launches += 3;
    }
    const float3 Einf = make_float3(static_cast<float>(-(st->prm.u_inf[1] * st->prm.B_imf[2] - st->prm.u_inf[2] * st->prm.B_imf[1])),
                                    static_cast<float>(-(st->prm.u_inf[2] * st->prm.B_imf[0] - st->prm.u_inf[0] * st->prm.B_imf[2])),
                                    static_cast<float>(-(st->prm.u_inf[0] * st->prm.B_imf[1] - st->prm.u_inf[1] * st->prm.B_imf[0])));
    P.begin(KP_EDGE_EMF, s);
    k_mx_edge<<<ge, 128, 0, s>>>(m, st->Ef32.p, st->up32.p, static_cast<float>(st->prm.cuct), Einf, st->E32.p);
    MHD_LAUNCH_CHECK();
    if (st->src.ambi)
    {
        if (mv.nn)
            k_mx_node_pressure<<<grid_for(mv.nn, 128), 128, 0, s>>>(mv.nn, mv.n2c_ptr, mv.n2c_cell, mv.cell_volume, W4, st->pn.p,
                                                                    st->pok.p);
        k_mx_ambipolar<<<grid_for(m.ne, 128), 128, 0, s>>>(m, p, W4, mv.ec_weight, mv.e_nodes, st->pn.p, st->pok.p,
                                                            static_cast<float>(st->prm.pressure_coef), st->E32.p);
        MHD_LAUNCH_CHECK();
        st->launches += 1 + (mv.nn ? 1 : 0);
    }
    P.end(KP_EDGE_EMF, s);
    P.begin(KP_CT, s);
    k_mx_ct<<<grid_for(m.nf, 256), 256, 0, s>>>(m.nf, st->mt.fe.p, st->E32.p, phis, phio, st->scal.p, stage2 ? 1 : 0);
    MHD_LAUNCH_CHECK();
    P.end(KP_CT, s);
    st->launches += 3;
}
} // namespace mhd
