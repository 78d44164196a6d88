// nvcc-flags: -fmad=false
// Fluid right-hand side on the device: primitives, limited least-squares gradients, Rusanov
// face fluxes, and the deterministic (atomic-free) gather of face fluxes into cells.
// FP64, reference-exact: every expression keeps the reference's operation order and this file
// is compiled without multiply-add contraction, so results round exactly as the host code does.
#include "kernels.cuh"

namespace mhd
{
// mhd::to_prim over n cells
__global__ void k_to_prim(SField<const double> U, SField<double> W, int32_t n, int nsp, double gamma, double rho_floor, double p_floor)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    for (int s = 0; s < nsp; ++s)
    {
        const Prim5 w = to_prim(U(s, c, 0), U(s, c, 1), U(s, c, 2), U(s, c, 3), U(s, c, 4), gamma, rho_floor, p_floor);
        W(s, c, 0) = w.rho; W(s, c, 1) = w.u; W(s, c, 2) = w.v; W(s, c, 3) = w.w; W(s, c, 4) = w.p;
    }
}

// One component of mhd::ghost_state (Common/fluid/Reconstruction.cpp:9-24); (cu, cv, cw) the velocity
// of the inside state, wc its component q.
__device__ __forceinline__ double ghost_component(int kind, bool absorb, int q, double wc, double cu, double cv, double cw, V3 n,
                                                  const Prim5 &fs)
{
    if (kind == 1)
    {
        if (absorb) return (q == 0 || q == 4) ? 1e-12 : 0.0;
        if (q == 0 || q == 4) return wc;
        const double un = cu * n.x + cv * n.y + cw * n.z;
        const double nq = q == 1 ? n.x : (q == 2 ? n.y : n.z);
        return wc - 2 * un * nq;
    }
    if (kind == 2) return q == 0 ? fs.rho : q == 1 ? fs.u : q == 2 ? fs.v : q == 3 ? fs.w : fs.p;
    return wc;
}

// mhd::Stencil::limited_gradients (Common/fluid/Reconstruction.cpp:80-142): least-squares gradient
// from the precomputed w*d and the symmetric inverse, Barth-Jespersen psi over all faces of the cell,
// optional relative limiter on rho and p, clamp to [0, 1]; zero for cells without a valid stencil.
// One thread per (cell, primitive variable): blockDim = (32, 5), warp q of a block handles variable
// q of 32 consecutive cells.  Each variable's fit and limiter are independent of the others (wall
// ghosts only read the velocity), so the per-thread state is small, occupancy high, and the five
// warps share the cell's geometry through L1.  The reference's arithmetic order is kept per variable.
template <bool LOG>
__global__ void __launch_bounds__(160) k_limited_gradients_v(MeshView m, FluidParams p, SField<const double> W, SField<double> G)
{
    const int32_t c = blockIdx.x * 32 + threadIdx.x;
    const int q = threadIdx.y;
    if (c >= m.nc) return;
    if (c >= m.no_cells || !m.st_valid[c])
    {
        for (int s = 0; s < p.nsp; ++s)
            for (int a = 0; a < 3; ++a) G(s, c, 3 * q + a) = 0.0;
        return;
    }
    const int32_t k0 = m.c2f_ptr[c], k1 = m.c2f_ptr[c + 1];
    const V3 xc = ld3(m.cell_center, c);
    const double *Ip = m.st_inv + 6 * (int64_t)c;
    const double I00 = Ip[0], I01 = Ip[1], I02 = Ip[2], I11 = Ip[3], I12 = Ip[4], I22 = Ip[5];
    for (int s = 0; s < p.nsp; ++s)
    {
        const double wc = W(s, c, q);
        double lo = wc, hi = wc, r0 = 0, r1 = 0, r2 = 0;
        int jlo = 7, jhi = 7, jpos = 7, jneg = 7; // switch log: the slots of the extremes
        for (int32_t k = k0; k < k1; ++k)
        {
            const int32_t nb = m.st_nb[k];
            if (nb == INT32_MIN) continue;
            double wn;
            if (nb >= 0) wn = W(s, nb, q);
            else
            {
                const int32_t f = -(nb + 1);
                const int kind = m.face_kind[f];
                const V3 n = (double(m.c2f_sgn[k]) / m.face_area_mag[f]) * ld3(m.face_area, f);
                const bool vel = kind == 1 && !p.absorb[s] && q >= 1 && q <= 3;
                const double *wg = wall_ghost(p, kind, f, s);
                wn = wg ? wg[q]
                        : ghost_component(kind, p.absorb[s] != 0, q, wc, vel ? W(s, c, 1) : 0.0, vel ? W(s, c, 2) : 0.0,
                                          vel ? W(s, c, 3) : 0.0, n, p.fs[s]);
            }
            const double dq = wn - wc;
            r0 += m.st_wd[3 * (int64_t)k] * dq;
            r1 += m.st_wd[3 * (int64_t)k + 1] * dq;
            r2 += m.st_wd[3 * (int64_t)k + 2] * dq;
            if (LOG && wn < lo) jlo = k - k0;
            if (LOG && hi < wn) jhi = k - k0;
            lo = dmin(lo, wn);
            hi = dmax(hi, wn);
        }
        const double g0 = I00 * r0 + I01 * r1 + I02 * r2;
        const double g1 = I01 * r0 + I11 * r1 + I12 * r2;
        const double g2 = I02 * r0 + I12 * r1 + I22 * r2;
        double psi = 1.0;
        if (p.limit)
        {
            // min over the faces of (hi - w)/dl (dl > 0) and (lo - w)/dl (dl < 0): a correctly rounded
            // quotient is monotone in dl, so the minimum is the quotient at the largest and at the most
            // negative dl, bit for bit (min is exact and order-free); likewise for the relative limiter
            double dpos = 0, dneg = 0;
            for (int32_t k = k0; k < k1; ++k)
            {
                const V3 dx = ld3(m.face_center, m.c2f_idx[k]) - xc;
                const double dl = g0 * dx.x + g1 * dx.y + g2 * dx.z;
                if (LOG && dl > dpos) jpos = k - k0;
                if (LOG && dl < dneg) jneg = k - k0;
                if (dl > dpos) dpos = dl;
                if (dl < dneg) dneg = dl;
            }
            if (dpos > 1e-300) psi = dmin(psi, (hi - wc) / dpos);
            if (dneg < -1e-300) psi = dmin(psi, (lo - wc) / dneg);
            if (p.rel_limit > 0 && (q == 0 || q == 4))
            {
                const double a = dmax(dpos, -dneg);
                if (a > 1e-300) psi = dmin(psi, p.rel_limit * wc / a);
            }
            if (LOG)
                sw_log(p.sw_lim, (s * 5 + q) * (int64_t)m.nc + c,
                       limiter_code(psi, wc, lo, hi, dpos, dneg, jlo, jhi, jpos, jneg, p.rel_limit, p.rel_limit > 0 && (q == 0 || q == 4)));
        }
        const double ps = dmax(0.0, dmin(1.0, psi));
        G(s, c, 3 * q) = ps * g0;
        G(s, c, 3 * q + 1) = ps * g1;
        G(s, c, 3 * q + 2) = ps * g2;
    }
}

// The same limited gradients on a tetrahedral mesh: one thread per (cell, species = blockIdx.y), the
// four slots unrolled at compile time so that every stencil load (coalesced structure-of-arrays
// tables) and the twenty neighbour gathers are in flight together.  Per variable the arithmetic and
// its order are those of the reference (slots and faces in c2f order).
template <bool LOG>
__global__ void __launch_bounds__(128, 4) k_limited_gradients_tet(MeshView m, FluidParams p, SField<const double> W, SField<double> G)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (c >= m.nc || s >= p.nsp) return;
    const int64_t n = m.nc;
    if (c >= m.no_cells || !m.st_valid[c])
    {
        for (int q = 0; q < 15; ++q) G(s, c, q) = 0.0;
        return;
    }
    int32_t nb[4];
    double wd[12], dx[12], wc[5], wn[4][5];
#pragma unroll
    for (int j = 0; j < 4; ++j) nb[j] = m.t_nb[j * n + c];
#pragma unroll
    for (int q = 0; q < 5; ++q) wc[q] = W(s, c, q);
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (nb[j] >= 0)
        {
#pragma unroll
            for (int q = 0; q < 5; ++q) wn[j][q] = W(s, nb[j], q);
        }
#pragma unroll
    for (int i = 0; i < 12; ++i)
    {
        wd[i] = m.t_wd[i * n + c];
        dx[i] = m.t_dx[i * n + c];
    }
    const double I00 = m.t_inv[c], I01 = m.t_inv[n + c], I02 = m.t_inv[2 * n + c], I11 = m.t_inv[3 * n + c],
                 I12 = m.t_inv[4 * n + c], I22 = m.t_inv[5 * n + c];
    const Prim5 wcp{wc[0], wc[1], wc[2], wc[3], wc[4]};
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (nb[j] < 0 && nb[j] != INT32_MIN)
        {
            const int32_t f = -(nb[j] + 1);
            const V3 nrm = (double(m.t_sg[j * n + c]) / m.face_area_mag[f]) * ld3(m.face_area, f);
            const double *wg = wall_ghost(p, m.face_kind[f], f, s);
            if (wg)
#pragma unroll
                for (int q = 0; q < 5; ++q) wn[j][q] = wg[q];
            else
                prim_arr(ghost_state(m.face_kind[f], p.absorb[s] != 0, wcp, nrm, p.fs[s]), wn[j]);
        }
#pragma unroll
    for (int q = 0; q < 5; ++q)
    {
        double r0 = 0, r1 = 0, r2 = 0, lo = wc[q], hi = wc[q];
        int jlo = 7, jhi = 7, jpos = 7, jneg = 7; // switch log: the slots of the extremes
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            if (nb[j] == INT32_MIN) continue;
            const double dq = wn[j][q] - wc[q];
            r0 += wd[3 * j] * dq;
            r1 += wd[3 * j + 1] * dq;
            r2 += wd[3 * j + 2] * dq;
            if (LOG && wn[j][q] < lo) jlo = j;
            if (LOG && hi < wn[j][q]) jhi = j;
            lo = dmin(lo, wn[j][q]);
            hi = dmax(hi, wn[j][q]);
        }
        const double g0 = I00 * r0 + I01 * r1 + I02 * r2;
        const double g1 = I01 * r0 + I11 * r1 + I12 * r2;
        const double g2 = I02 * r0 + I12 * r1 + I22 * r2;
        double psi = 1.0;
        if (p.limit)
        {
            // two quotients instead of four: the minimum sits at the largest and the most negative dl
            // (monotone correctly rounded quotients, exact min), bit for bit the reference's psi
            double dpos = 0, dneg = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const double dl = g0 * dx[3 * j] + g1 * dx[3 * j + 1] + g2 * dx[3 * j + 2];
                if (LOG && dl > dpos) jpos = j;
                if (LOG && dl < dneg) jneg = j;
                if (dl > dpos) dpos = dl;
                if (dl < dneg) dneg = dl;
            }
            if (dpos > 1e-300) psi = dmin(psi, (hi - wc[q]) / dpos);
            if (dneg < -1e-300) psi = dmin(psi, (lo - wc[q]) / dneg);
            if (p.rel_limit > 0 && (q == 0 || q == 4))
            {
                const double a = dmax(dpos, -dneg);
                if (a > 1e-300) psi = dmin(psi, p.rel_limit * wc[q] / a);
            }
            if (LOG)
                sw_log(p.sw_lim, (s * 5 + q) * (int64_t)m.nc + c,
                       limiter_code(psi, wc[q], lo, hi, dpos, dneg, jlo, jhi, jpos, jneg, p.rel_limit, p.rel_limit > 0 && (q == 0 || q == 4)));
        }
        const double ps = dmax(0.0, dmin(1.0, psi));
        G(s, c, 3 * q) = ps * g0;
        G(s, c, 3 * q + 1) = ps * g1;
        G(s, c, 3 * q + 2) = ps * g2;
    }
}

// Face loop of mhd::fluid_flux_rhs (Common/fluid/FluxRHS.cpp:36-69): Rusanov flux of the
// reconstructed face states times |A|, per face and species (SoA: F[(s*5 + m)*nf + f]).
// Faces that the reference skips (Skip kind, no owned fluid cell) get zero.
template <bool LOG>
__global__ void __launch_bounds__(128) k_face_flux(MeshView m, FluidParams p, SField<const double> W, SField<const double> G,
                                                   double *__restrict__ F)
{
    // one species per grid row (blockIdx.y)
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (f >= m.nf || s >= p.nsp) return;
    const int64_t nf = m.nf;
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
        for (int q = 0; q < 5; ++q) F[(s * 5 + q) * nf + f] = 0.0;
        return;
    }
    const double A = m.face_area_mag[f];
    const V3 n = (1.0 / A) * ld3(m.face_area, f);
    const V3 xf = ld3(m.face_center, f);
    const bool interior = cnt == 2 && kind == 0;
    int32_t cL = -1, cR = -1, c = -1;
    int sgn = 0;
    if (interior)
    {
        cL = m.face_L[f];
        cR = m.face_R[f];
    }
    else
    {
        c = m.f2c_idx[p0];
        sgn = m.f2c_sgn[p0];
        if (cnt == 2 && m.material[c] != 0)
        {
            c = m.f2c_idx[p0 + 1];
            sgn = m.f2c_sgn[p0 + 1];
        }
    }
    {
        Prim5 L, R;
        double g[15];
        uint32_t code = 0; // switch log: the face states' positivity fallbacks (bits 2, 3), Rusanov's choices
        auto state_of = [&](int32_t cc, uint32_t bit) {
            const Prim5 w{W(s, cc, 0), W(s, cc, 1), W(s, cc, 2), W(s, cc, 3), W(s, cc, 4)};
            for (int q = 0; q < 15; ++q) g[q] = G(s, cc, q);
            if (LOG && face_state_fallback(w, g, xf - ld3(m.cell_center, cc))) code |= bit;
            return face_state(w, g, xf - ld3(m.cell_center, cc));
        };
        if (interior)
        {
            L = state_of(cL, 4u);
            R = state_of(cR, 8u);
        }
        else
        {
            const Prim5 in = state_of(c, 4u);
            const double *wg = wall_ghost(p, kind, f, s);
            const Prim5 gh = wg ? Prim5{wg[0], wg[1], wg[2], wg[3], wg[4]} : ghost_state(kind, p.absorb[s] != 0, in, double(sgn) * n, p.fs[s]);
            if (sgn > 0) { L = in; R = gh; }
            else { R = in; L = gh; }
        }
        double Fl[5];
        rusanov(L, R, n, p.gamma, Fl);
        if (LOG)
            sw_log(p.sw_flux, s * nf + f,
                   code | rusanov_code(L, R, n, p.gamma, !interior && kind == 1 && !p.absorb[s] && !wall_ghost(p, kind, f, s)));
        for (int q = 0; q < 5; ++q) F[(s * 5 + q) * nf + f] = Fl[q] * A;
    }
}

// Scatter of Common/fluid/FluxRHS.cpp:70-72 as a gather: rhs_c = sum_f -s_cf F_f / V_c over the
// faces of each owned fluid cell, zero elsewhere.  The faces are visited in ascending id, the
// order in which the reference's face loop scatters into the cell, so the sum rounds the same.
__global__ void k_gather_rhs(MeshView m, int nsp, const double *__restrict__ F, SField<double> rhs)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int64_t nf = m.nf;
    if (c >= m.no_cells || m.material[c] != 0)
    {
        for (int s = 0; s < nsp; ++s)
            for (int q = 0; q < 5; ++q) rhs(s, c, q) = 0.0;
        return;
    }
    const double V = m.cell_volume[c];
    const int32_t k0 = m.c2f_ptr[c], k1 = m.c2f_ptr[c + 1];
    for (int s = 0; s < nsp; ++s)
    {
        double r[5] = {0, 0, 0, 0, 0};
        for (int32_t k = k0; k < k1; ++k)
        {
            const int32_t f = m.cfa_idx[k];
            const bool out = m.cfa_sgn[k] > 0;
            for (int q = 0; q < 5; ++q)
            {
                const double v = F[(s * 5 + q) * nf + f] / V;
                r[q] = out ? r[q] - v : r[q] + v;
            }
        }
        for (int q = 0; q < 5; ++q) rhs(s, c, q) = r[q];
    }
}

void launch_limited_gradients(const MeshView &m, const FluidParams &p, SField<const double> W, SField<double> G, cudaStream_t s)
{
    if (!m.nc) return;
    const bool log = p.sw_lim && p.limit;
    if (m.faces_per_cell == 4)
        (log ? k_limited_gradients_tet<true> : k_limited_gradients_tet<false>)<<<dim3(grid_for(m.nc, 128), p.nsp), 128, 0, s>>>(m, p, W, G);
    else (log ? k_limited_gradients_v<true> : k_limited_gradients_v<false>)<<<grid_for(m.nc, 32), dim3(32, 5), 0, s>>>(m, p, W, G);
    MHD_LAUNCH_CHECK();
}

void launch_face_flux(const MeshView &m, const FluidParams &p, SField<const double> W, SField<const double> G, double *F, cudaStream_t s)
{
    if (!m.nf) return;
    (p.sw_flux ? k_face_flux<true> : k_face_flux<false>)<<<dim3(grid_for(m.nf, 128), p.nsp), 128, 0, s>>>(m, p, W, G, F);
    MHD_LAUNCH_CHECK();
}

__global__ void k_wall_slots(MeshView m, const int32_t *__restrict__ faces, int32_t n, int32_t *__restrict__ slot, int *__restrict__ err)
{
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t f = faces[i];
    if (f < 0 || f >= m.nf || m.face_kind[f] != 1)
    {
        atomicOr(err, 1);
        return;
    }
    if (atomicCAS(slot + f, -1, i) != -1) atomicOr(err, 2);
}

void build_wall_slots(const MeshView &m, const int32_t *faces, int32_t n, int32_t *slot, cudaStream_t s)
{
    if (m.nf) MHD_CUDA(cudaMemsetAsync(slot, 0xff, (size_t)m.nf * sizeof(int32_t), s));
    if (!n) return;
    DBuf<int> err;
    err.alloc(1);
    MHD_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    k_wall_slots<<<grid_for(n, 128), 128, 0, s>>>(m, faces, n, slot, err.p);
    MHD_LAUNCH_CHECK();
    int h = 0;
    MHD_CUDA(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    MHD_CUDA(cudaStreamSynchronize(s));
    MHD_REQUIRE(!(h & 1), "wall ghost faces must be faces of kind wall");
    MHD_REQUIRE(!(h & 2), "wall ghost faces must be distinct");
}

static FluidParams single_species(int32_t species, const MhdPrim *fs, double gamma, int limit, double rel_limit)
{
    FluidParams p{};
    p.nsp = 1;
    p.limit = limit;
    p.gamma = gamma;
    p.rel_limit = rel_limit;
    if (fs) p.fs[0] = Prim5{fs->rho, fs->u, fs->v, fs->w, fs->p};
    p.absorb[0] = species == 1; // reference ghost_state: species 1 is absorbed at walls
    return p;
}
} // namespace mhd

using namespace mhd;

extern "C" {

int mhd_gpu_to_prim(MhdMesh *mesh, const double *U, int32_t n, double gamma, double rho_floor, double p_floor, double *W)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && n >= 0 && MHD_ARR(U, n) && MHD_ARR(W, n), "bad argument");
        if (!n) return;
        k_to_prim<<<grid_for(n, 256), 256, 0, mesh->stream>>>(SField<const double>{U, 0, 5, 1}, SField<double>{W, 0, 5, 1}, n, 1,
                                                              gamma, rho_floor, p_floor);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_limited_gradients(MhdMesh *mesh, const double *W, int32_t species, const MhdPrim *fs, int32_t limit, double rel_limit,
                              double *grad)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && fs && MHD_ARR(W, mesh->v.nc) && MHD_ARR(grad, mesh->v.nc), "bad argument");
        MHD_REQUIRE(species >= 0, "negative species");
        const MeshView &m = mesh->v;
        if (!m.nc) return;
        const FluidParams p = single_species(species, fs, 0.0, limit, rel_limit);
        launch_limited_gradients(m, p, SField<const double>{W, 0, 5, 1}, SField<double>{grad, 0, 15, 1}, mesh->stream);
    });
}

int mhd_gpu_limited_gradients_wall(MhdMesh *mesh, const double *W, int32_t species, const MhdPrim *fs, int32_t limit, double rel_limit,
                                   int32_t n_wall, const int32_t *wall_faces, const double *wall_prims, double *grad)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && fs && MHD_ARR(W, mesh->v.nc) && MHD_ARR(grad, mesh->v.nc), "bad argument");
        MHD_REQUIRE(species >= 0, "negative species");
        MHD_REQUIRE(n_wall >= 0 && (!n_wall || (wall_faces && wall_prims)), "bad wall ghost table");
        const MeshView &m = mesh->v;
        if (!m.nc) return;
        FluidParams p = single_species(species, fs, 0.0, limit, rel_limit);
        DBuf<int32_t> slot;
        slot.alloc(m.nf ? (size_t)m.nf : 1);
        build_wall_slots(m, wall_faces, n_wall, slot.p, mesh->stream);
        p.wall_slot = slot.p;
        p.wall_prim = wall_prims;
        p.wall_n = n_wall;
        launch_limited_gradients(m, p, SField<const double>{W, 0, 5, 1}, SField<double>{grad, 0, 15, 1}, mesh->stream);
        MHD_CUDA(cudaStreamSynchronize(mesh->stream)); // the slot map is freed on return
    });
}

int mhd_gpu_flux_rhs_wall(MhdMesh *mesh, double gamma, int32_t species, const MhdPrim *fs, const double *W, const double *grad,
                          int32_t n_wall, const int32_t *wall_faces, const double *wall_prims, double *rhs)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && fs && MHD_ARR(W, mesh->v.nc) && MHD_ARR(grad, mesh->v.nc) && MHD_ARR(rhs, mesh->v.nc), "bad argument");
        MHD_REQUIRE(gamma > 1.0, "gamma must exceed 1");
        MHD_REQUIRE(n_wall >= 0 && (!n_wall || (wall_faces && wall_prims)), "bad wall ghost table");
        const MeshView &m = mesh->v;
        if (!m.nc) return;
        FluidParams p = single_species(species, fs, gamma, 1, 0.0);
        DBuf<int32_t> slot;
        slot.alloc(m.nf ? (size_t)m.nf : 1);
        build_wall_slots(m, wall_faces, n_wall, slot.p, mesh->stream);
        p.wall_slot = slot.p;
        p.wall_prim = wall_prims;
        p.wall_n = n_wall;
        mesh->scratch_face.alloc(5 * static_cast<size_t>(m.nf));
        k_face_flux<false><<<grid_for(m.nf, 128), 128, 0, mesh->stream>>>(m, p, SField<const double>{W, 0, 5, 1},
                                                                   SField<const double>{grad, 0, 15, 1}, mesh->scratch_face.p);
        MHD_LAUNCH_CHECK();
        k_gather_rhs<<<grid_for(m.nc, 256), 256, 0, mesh->stream>>>(m, 1, mesh->scratch_face.p, SField<double>{rhs, 0, 5, 1});
        MHD_LAUNCH_CHECK();
        MHD_CUDA(cudaStreamSynchronize(mesh->stream));
    });
}

int mhd_gpu_flux_rhs(MhdMesh *mesh, double gamma, int32_t species, const MhdPrim *fs, const double *W, const double *grad, double *rhs)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && fs && MHD_ARR(W, mesh->v.nc) && MHD_ARR(grad, mesh->v.nc) && MHD_ARR(rhs, mesh->v.nc), "bad argument");
        MHD_REQUIRE(gamma > 1.0, "gamma must exceed 1");
        const MeshView &m = mesh->v;
        if (!m.nc) return;
        const FluidParams p = single_species(species, fs, gamma, 1, 0.0);
        mesh->scratch_face.alloc(5 * static_cast<size_t>(m.nf));
        k_face_flux<false><<<grid_for(m.nf, 128), 128, 0, mesh->stream>>>(m, p, SField<const double>{W, 0, 5, 1},
                                                                   SField<const double>{grad, 0, 15, 1}, mesh->scratch_face.p);
        MHD_LAUNCH_CHECK();
        k_gather_rhs<<<grid_for(m.nc, 256), 256, 0, mesh->stream>>>(m, 1, mesh->scratch_face.p, SField<double>{rhs, 0, 5, 1});
        MHD_LAUNCH_CHECK();
    });
}

} // extern "C"
