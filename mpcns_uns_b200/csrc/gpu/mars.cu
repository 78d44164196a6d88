// nvcc-flags: -fmad=false
// The ten-ion (Mars) source pieces of mars::MarsSolver (MarsUns/driver/MarsSolver.cpp) as device passes in the
// reference's operation order:
//   * the plasma quantities of prepare (n_e, n_e,eff, p_e = sum p_s, u+; :287-303) and grad p_e (:305-325);
//   * the explicit J x B and ambipolar force of fluid_and_sources_ (:400-418);
//   * the ambipolar edge EMF with the nodal p_e (ambipolar_emf_, :529-562);
//   * the CFL step (local_dt_, :330-376): each ion alone and the plasma's fast mode;
//   * the point-implicit sources (implicit_sources_, :420-520): Crank-Nicolson gyration of the coupled ions
//     about B (closed form), ion-neutral drag and thermal relaxation, backward Euler;
//   * the forward-Euler advance (step, :719-726) and the floors (floors_, :686-702).
// Arrays of the ions are species-major, 5 values per cell: U[(s * nc + c) * 5 + m].  One thread per cell.
#include <cfloat>
#include <cstring>

#include "common.cuh"
#include "sources.cuh"

namespace mhd
{
namespace
{
struct MarsP
{
    int nsp, nneu, nstride, ambi;
    double mass[kMaxSpecies];
    double rho_ref, n_ref, p_ref, time_ref, kB, L, U, q, B;
    double mag_scale, pressure_scale, ne_floor, rho_floor, p_floor, gamma;
};

MarsP mars_params(const MhdMarsParams &q)
{
    MHD_REQUIRE(q.n_species >= 1 && q.n_species <= kMaxSpecies, "n_species must be 1..16");
    MHD_REQUIRE(q.n_neutral >= 0 && q.n_neutral <= q.n_species && q.n_neutral <= q.neutral_stride,
                "the reactive neutrals are the first n_neutral entries of the species table (n_neutral <= n_species, <= neutral_stride)");
    MHD_REQUIRE(q.gamma > 1.0, "gamma must exceed 1");
    MarsP p;
    p.nsp = q.n_species;
    p.nneu = q.n_neutral;
    p.nstride = q.neutral_stride;
    p.ambi = q.ambipolar != 0;
    for (int s = 0; s < kMaxSpecies; ++s) p.mass[s] = s < q.n_species ? q.mass[s] : 1.0;
    for (int s = 0; s < q.n_species; ++s) MHD_REQUIRE(q.mass[s] > 0, "species masses must be positive");
    p.rho_ref = q.rho_ref; p.n_ref = q.n_ref; p.p_ref = q.p_ref; p.time_ref = q.time_ref; p.kB = q.kB;
    p.L = q.L; p.U = q.U; p.q = q.q; p.B = q.B;
    p.mag_scale = q.mag_scale; p.pressure_scale = q.pressure_scale; p.ne_floor = q.ne_floor;
    p.rho_floor = q.rho_floor; p.p_floor = q.p_floor; p.gamma = q.gamma;
    return p;
}

// number density of species s relative to n_ref: max(rho, 0) rho_ref / (m_s n_ref)
__device__ __forceinline__ double nrel(const MarsP &p, int s, double rho) { return dmax(rho, 0.0) * p.rho_ref / (p.mass[s] * p.n_ref); }

__device__ __forceinline__ const double *cell5(const double *a, int64_t nc, int s, int32_t c) { return a + ((int64_t)s * nc + c) * 5; }
__device__ __forceinline__ double *cell5(double *a, int64_t nc, int s, int32_t c) { return a + ((int64_t)s * nc + c) * 5; }

// ------------------------------------------------------------------ prepare: n_e, n_e,eff, p_e, u+
__global__ void __launch_bounds__(128) k_mars_plasma(MeshView m, MarsP p, const double *__restrict__ U, const double *__restrict__ W,
                                                     double *__restrict__ ne_o, double *__restrict__ ne_eff_o, double *__restrict__ pe_o,
                                                     double *__restrict__ up_o)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int64_t nc = m.nc;
    double ne = 0, pe = 0, v0 = 0, v1 = 0, v2 = 0;
    for (int s = 0; s < p.nsp; ++s)
    {
        const double *w = cell5(W, nc, s, c);
        const double n = nrel(p, s, cell5(U, nc, s, c)[0]);
        ne += n;
        pe += w[4];
        v0 += n * w[1];
        v1 += n * w[2];
        v2 += n * w[3];
    }
    ne_o[c] = ne;
    ne_eff_o[c] = sqrt(ne * ne + p.ne_floor * p.ne_floor);
    pe_o[c] = pe;
    const double inv = ne > 1e-300 ? 1.0 / ne : 0.0;
    const bool fluid = m.material[c] == 0;
    up_o[3 * (int64_t)c] = fluid ? v0 * inv : 0.0;
    up_o[3 * (int64_t)c + 1] = fluid ? v1 * inv : 0.0;
    up_o[3 * (int64_t)c + 2] = fluid ? v2 * inv : 0.0;
}

// grad p by Gauss' theorem with the face-averaged p (MarsSolver.cpp:305-325, the form of Ambipolar.cpp:10-31)
__global__ void __launch_bounds__(128) k_pressure_gradient(MeshView m, const double *__restrict__ pe, double *__restrict__ dpe)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    V3 g = mk(0, 0, 0);
    if (c < m.no_cells && m.material[c] != 1) g = electron_pressure_gradient(m, c, [&](int32_t o) { return pe[o]; });
    st3(dpe, c, g);
}

// ------------------------------------------------------------------ explicit J x B and ambipolar force
__global__ void __launch_bounds__(128) k_mars_explicit(MeshView m, MarsP p, const double *__restrict__ U, const double *__restrict__ W,
                                                       const double *__restrict__ Btot, const double *__restrict__ J,
                                                       const double *__restrict__ dpe, const double *__restrict__ ne_eff, double *__restrict__ rhs)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.no_cells || m.material[c] == 1) return;
    const int64_t nc = m.nc;
    const V3 b = ld3(Btot, c), j = ld3(J, c), d = ld3(dpe, c);
    const V3 jxb = cross(j, b);
    for (int s = 0; s < p.nsp; ++s)
    {
        const double rho = dmax(cell5(U, nc, s, c)[0], 0.0);
        const double w = rho * p.rho_ref / (p.mass[s] * p.n_ref) / ne_eff[c]; // charge share n_s / n_e,eff
        const double *wp = cell5(W, nc, s, c);
        V3 f = (w * p.mag_scale) * jxb;
        if (p.ambi) f = f - w * d;
        double *r = cell5(rhs, nc, s, c);
        r[1] += f.x;
        r[2] += f.y;
        r[3] += f.z;
        r[4] += dot(f, mk(wp[1], wp[2], wp[3]));
    }
}

// ------------------------------------------------------------------ ambipolar edge EMF
__global__ void __launch_bounds__(128) k_mars_node_p(MeshView m, const double *__restrict__ pe, double *__restrict__ pn, int8_t *__restrict__ pok)
{
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= m.nn) return;
    bool ok;
    pn[v] = node_pressure(m, v, [&](int32_t c) { return pe[c]; }, ok);
    pok[v] = ok ? 1 : 0;
}

__global__ void __launch_bounds__(128) k_mars_ambipolar(MeshView m, MarsP p, const double *__restrict__ ne_c, const double *__restrict__ pn,
                                                        const int8_t *__restrict__ pok, double *__restrict__ E)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.no_edges) return;
    double ne = 0, wsum = 0;
    for (int32_t k = m.ec_ptr[e]; k < m.ec_ptr[e + 1]; ++k)
    {
        const int32_t c = m.ec_cell[k];
        if (m.material[c] == 1) continue;
        ne += m.ec_weight[k] * ne_c[c];
        wsum += m.ec_weight[k];
    }
    if (wsum <= 0) return;
    ne /= wsum;
    const int32_t a = m.e_nodes[2 * (int64_t)e], b = m.e_nodes[2 * (int64_t)e + 1];
    if (!pok[a] || !pok[b]) return;
    E[e] -= p.pressure_scale * (pn[b] - pn[a]) / sqrt(ne * ne + p.ne_floor * p.ne_floor);
}

// ------------------------------------------------------------------ CFL step
__global__ void __launch_bounds__(128) k_mars_dt(MeshView m, MarsP p, double cfl, const double *__restrict__ U, const double *__restrict__ W,
                                                 const double *__restrict__ Btot, const double *__restrict__ up,
                                                 unsigned long long *__restrict__ dt_bits)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nc = m.nc;
    double dt = 1e300;
    if (c < m.no_cells && m.material[c] != 1)
    {
        const double V = m.cell_volume[c];
        const int32_t k0 = m.c2f_ptr[c], k1 = m.c2f_ptr[c + 1];
        // each ion on its own: cfl V / sum_f (|u.A| + c_s |A|)
        for (int s = 0; s < p.nsp; ++s)
        {
            const double *w = cell5(W, nc, s, c);
            const double cs = sqrt(p.gamma * w[4] / w[0]);
            double den = 0;
            for (int32_t k = k0; k < k1; ++k)
            {
                const int32_t f = m.c2f_idx[k];
                const V3 A = ld3(m.face_area, f);
                den += fabs(w[1] * A.x + w[2] * A.y + w[3] * A.z) + cs * m.face_area_mag[f];
            }
            if (den > 0) dt = dmin(dt, cfl * V / den);
        }
        // the charged plasma as one fluid: fast magnetosonic waves of the total field advected with u+
        double rho = 0, pr = 0;
        for (int s = 0; s < p.nsp; ++s)
        {
            rho += dmax(cell5(U, nc, s, c)[0], 0.0);
            pr += dmax(cell5(W, nc, s, c)[4], 0.0);
        }
        rho = dmax(rho, p.rho_floor);
        pr = dmax(pr, p.p_floor);
        const V3 b = ld3(Btot, c), u = ld3(up, c);
        const double cs2 = p.gamma * pr / rho, va2 = p.mag_scale * dot(b, b) / rho;
        double den = 0;
        for (int32_t k = k0; k < k1; ++k)
        {
            const int32_t f = m.c2f_idx[k];
            const double A = m.face_area_mag[f];
            const V3 Av = ld3(m.face_area, f);
            const double bn = dot(b, Av) / A, van2 = p.mag_scale * bn * bn / rho;
            const double sum = cs2 + va2, disc = dmax(0.0, sum * sum - 4.0 * cs2 * van2);
            const double cf = sqrt(0.5 * (sum + sqrt(disc)));
            den += fabs(dot(u, Av)) + cf * A;
        }
        if (den > 0) dt = dmin(dt, cfl * V / den);
    }
    // block minimum (exact), one atomic per block; 1e300 is the reference's "no limit"
    __shared__ double sh[32];
    double v = dt;
    for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 1e300;
        for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0 && v > 0) atomicMin(dt_bits, static_cast<unsigned long long>(__double_as_longlong(v)));
    }
}

// ------------------------------------------------------------------ point-implicit sources
// complex<double> arithmetic as the reference's compiled std::complex: products (ac - bd, ad + bc); quotients
// by Smith's method (R. L. Smith, "Algorithm 116: Complex division", CACM 5(8), 1962), the form of the C
// runtime's complex division for finite operands of moderate size
struct Cx
{
    double re, im;
};
__device__ __forceinline__ Cx cadd(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Cx cmul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Cx cscale(double s, Cx a) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ Cx cdiv(Cx x, Cx y)
{
    const double a = x.re, b = x.im, c = y.re, d = y.im;
    double ratio, denom;
    if (fabs(c) < fabs(d))
    {
        ratio = c / d;
        denom = (c * ratio) + d;
        if (fabs(ratio) > DBL_MIN) return {((a * ratio) + b) / denom, ((b * ratio) - a) / denom};
        return {((c * (a / d)) + b) / denom, ((c * (b / d)) - a) / denom};
    }
    ratio = d / c;
    denom = (d * ratio) + c;
    if (fabs(ratio) > DBL_MIN) return {((b * ratio) + a) / denom, (b - (a * ratio)) / denom};
    return {(a + (d * (b / c))) / denom, (b - (d * (a / c))) / denom};
}
// 1 - a and 1 + a of a complex a (a real minus / plus a complex: imaginary part 0 - a.im, 0 + a.im)
__device__ __forceinline__ Cx one_minus(Cx a) { return {1.0 - a.re, 0.0 - a.im}; }
__device__ __forceinline__ Cx one_plus(Cx a) { return {1.0 + a.re, 0.0 + a.im}; }

__global__ void __launch_bounds__(128) k_mars_implicit(MeshView m, MarsP p, const double *__restrict__ Btot, const double *__restrict__ neutral,
                                                       double dt, double *__restrict__ Ua)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.no_cells || m.material[c] == 1) return;
    const int64_t nc = m.nc;
    const double g = p.gamma;
    const double a5 = 3.0e6 * p.L * p.kB / (p.rho_ref * p.U * p.U * p.U);
    double nr[kMaxSpecies], ntot = 0;
    for (int s = 0; s < p.nsp; ++s)
    {
        nr[s] = nrel(p, s, cell5(Ua, nc, s, c)[0]);
        ntot += nr[s];
    }
    // 1. gyration dz_s/dt = -i Omega_s (z_s - Z) in the plane normal to B, Crank-Nicolson in closed form
    const V3 B = ld3(Btot, c);
    const double Bm = sqrt(dot(B, B));
    if (ntot > 1e-300 && Bm > 1e-30)
    {
        const V3 k = (1.0 / Bm) * B;
        const V3 t = fabs(k.x) < 0.9 ? mk(1, 0, 0) : mk(0, 1, 0);
        V3 e1 = cross(k, t);
        e1 = (1.0 / sqrt(dot(e1, e1))) * e1;
        const V3 e2 = cross(k, e1);
        Cx z[kMaxSpecies], al[kMaxSpecies], Z0{0.0, 0.0};
        for (int s = 0; s < p.nsp; ++s)
        {
            const double *u = cell5(Ua, nc, s, c);
            const double rho = dmax(u[0], p.rho_floor);
            const V3 v = mk(u[1] / rho, u[2] / rho, u[3] / rho);
            z[s] = Cx{dot(v, e1), dot(v, e2)};
            al[s] = Cx{0.0, p.q * p.B * p.L / (p.mass[s] * p.U) * Bm * dt * 0.5}; // i alpha_s / 2
            Z0 = cadd(Z0, cscale(nr[s] / ntot, z[s]));
        }
        Cx Pn{0.0, 0.0}, Qn{0.0, 0.0};
        for (int s = 0; s < p.nsp; ++s)
        {
            const double chi = nr[s] / ntot;
            const Cx a{-al[s].re, -al[s].im};
            Pn = cadd(Pn, cdiv(cscale(chi, cadd(cmul(z[s], one_minus(a)), cmul(a, Z0))), one_plus(a)));
            Qn = cadd(Qn, cdiv(cscale(chi, a), one_plus(a)));
        }
        const Cx Zn = cdiv(Pn, one_minus(Qn));
        for (int s = 0; s < p.nsp; ++s)
        {
            const Cx a{-al[s].re, -al[s].im};
            const Cx zn = cdiv(cadd(cmul(z[s], one_minus(a)), cmul(a, cadd(Z0, Zn))), one_plus(a));
            double *u = cell5(Ua, nc, s, c);
            const double rho = dmax(u[0], p.rho_floor);
            const V3 v = mk(u[1] / rho, u[2] / rho, u[3] / rho);
            const double vpar = dot(v, k);
            const V3 vn = (vpar * k + zn.re * e1) + zn.im * e2;
            u[4] += 0.5 * rho * (dot(vn, vn) - dot(v, v));
            u[1] = rho * vn.x;
            u[2] = rho * vn.y;
            u[3] = rho * vn.z;
        }
    }
    // 2./3. drag (backward Euler, the lost kinetic energy stays as heat) and thermal relaxation to 185 K
    double coll[kMaxSpecies], collision = 0;
    for (int n = 0; n < p.nneu; ++n)
    {
        coll[n] = dmax(neutral[(int64_t)c * p.nstride + n], 0.0) * 2.0e-10;
        collision += coll[n];
    }
    const double nu = p.time_ref * collision;
    for (int s = 0; s < p.nsp; ++s)
    {
        double *u = cell5(Ua, nc, s, c);
        const double ms = p.mass[s];
        const double rho = dmax(u[0], p.rho_floor);
        const V3 v = mk(u[1] / rho, u[2] / rho, u[3] / rho);
        const double ke_old = 0.5 * rho * dot(v, v);
        const double den = 1.0 + nu * dt;
        u[1] /= den;
        u[2] /= den;
        u[3] /= den;
        const double ke = ke_old / (den * den);
        const double pr = dmax((g - 1.0) * (u[4] - ke), p.p_floor);
        double b1c = 0, b2 = 0;
        for (int n = 0; n < p.nneu; ++n)
        {
            const double mm = ms + p.mass[n];
            b1c += ms * coll[n] / mm;
            b2 += p.mass[n] * coll[n] / mm;
        }
        const double n_m3 = rho * p.rho_ref / ms;
        const double ns_cm3 = n_m3 * 1e-6;
        const double kk = a5 * ns_cm3 * b1c;
        const double cT = p.p_ref / (dmax(n_m3, 1.0) * p.kB);
        const double Sf = p.time_ref * rho * dot(v, v) * b2;
        double pn;
        if (pr * cT >= 50.0) pn = (pr + dt * (g - 1.0) * (kk * 185.0 + Sf)) / (1.0 + dt * (g - 1.0) * kk * cT);
        else pn = pr + dt * (g - 1.0) * (kk * (185.0 - 50.0) + Sf);
        u[4] = pn / (g - 1.0) + ke;
    }
}

// ------------------------------------------------------------------ advance and floors
__global__ void __launch_bounds__(128) k_mars_advance(MeshView m, int nsp, const double *__restrict__ rhs, double dt, double *__restrict__ U)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.no_cells || m.material[c] == 1) return;
    const int64_t nc = m.nc;
    for (int s = 0; s < nsp; ++s)
    {
        double *u = cell5(U, nc, s, c);
        const double *r = cell5(rhs, nc, s, c);
        for (int q = 0; q < 5; ++q) u[q] += dt * r[q];
    }
}

__global__ void __launch_bounds__(128) k_mars_floors(MeshView m, MarsP p, double *__restrict__ U)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.no_cells || m.material[c] == 1) return;
    const int64_t nc = m.nc;
    const double g = p.gamma;
    for (int s = 0; s < p.nsp; ++s)
    {
        double *u = cell5(U, nc, s, c);
        double rho = u[0];
        if (!isfinite(rho) || rho < p.rho_floor)
        {
            const double scale = p.rho_floor / dmax(rho, 1e-30);
            for (int q = 1; q < 4; ++q) u[q] *= scale;
            u[0] = rho = p.rho_floor;
        }
        const double ke = 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / rho;
        u[4] = dmax(u[4], ke + p.p_floor / (g - 1.0));
    }
}
} // namespace
} // namespace mhd

using namespace mhd;

extern "C" {

int mhd_gpu_mars_plasma(MhdMesh *mesh, const MhdMarsParams *params, const double *U, const double *W, double *ne, double *ne_eff, double *pe,
                        double *uplus)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && params && U && W && ne && ne_eff && pe && uplus, "null argument");
        const MarsP p = mars_params(*params);
        const MeshView &m = mesh->v;
        if (!m.nc) return;
        k_mars_plasma<<<grid_for(m.nc, 128), 128, 0, mesh->stream>>>(m, p, U, W, ne, ne_eff, pe, uplus);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_pressure_gradient(MhdMesh *mesh, const double *pe, double *dpe)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && pe && dpe, "null argument");
        const MeshView &m = mesh->v;
        if (!m.nc) return;
        k_pressure_gradient<<<grid_for(m.nc, 128), 128, 0, mesh->stream>>>(m, pe, dpe);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_mars_explicit_sources(MhdMesh *mesh, const MhdMarsParams *params, const double *U, const double *W, const double *Btot,
                                  const double *J, const double *dpe, const double *ne_eff, double *rhs)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && params && U && W && Btot && J && dpe && ne_eff && rhs, "null argument");
        const MarsP p = mars_params(*params);
        const MeshView &m = mesh->v;
        if (!m.no_cells) return;
        k_mars_explicit<<<grid_for(m.no_cells, 128), 128, 0, mesh->stream>>>(m, p, U, W, Btot, J, dpe, ne_eff, rhs);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_mars_ambipolar_emf(MhdMesh *mesh, const MhdMarsParams *params, const double *pe, const double *ne, double *E)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && params && pe && ne && E, "null argument");
        const MarsP p = mars_params(*params);
        const MeshView &m = mesh->v;
        MHD_REQUIRE(m.e_nodes && m.n2c_ptr, "the ambipolar EMF needs the mesh's edge_nodes");
        if (!m.no_edges) return;
        DBuf<double> pn;
        DBuf<int8_t> pok;
        pn.alloc(m.nn > 0 ? (size_t)m.nn : 1);
        pok.alloc(m.nn > 0 ? (size_t)m.nn : 1);
        if (m.nn) k_mars_node_p<<<grid_for(m.nn, 128), 128, 0, mesh->stream>>>(m, pe, pn.p, pok.p);
        k_mars_ambipolar<<<grid_for(m.no_edges, 128), 128, 0, mesh->stream>>>(m, p, ne, pn.p, pok.p, E);
        MHD_LAUNCH_CHECK();
        MHD_CUDA(cudaStreamSynchronize(mesh->stream)); // the nodal arrays are freed on return
    });
}

int mhd_gpu_mars_time_step(MhdMesh *mesh, const MhdMarsParams *params, double cfl, const double *U, const double *W, const double *Btot,
                           const double *uplus, double *host_dt)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && params && U && W && Btot && uplus && host_dt, "null argument");
        const MarsP p = mars_params(*params);
        const MeshView &m = mesh->v;
        DBuf<unsigned long long> bits;
        bits.alloc(1);
        const double big = 1e300;
        unsigned long long init;
        std::memcpy(&init, &big, sizeof(init));
        MHD_CUDA(cudaMemcpyAsync(bits.p, &init, sizeof(init), cudaMemcpyHostToDevice, mesh->stream));
        if (m.no_cells) k_mars_dt<<<grid_for(m.no_cells, 128), 128, 0, mesh->stream>>>(m, p, cfl, U, W, Btot, uplus, bits.p);
        MHD_LAUNCH_CHECK();
        unsigned long long h = 0;
        MHD_CUDA(cudaMemcpyAsync(&h, bits.p, sizeof(h), cudaMemcpyDeviceToHost, mesh->stream));
        MHD_CUDA(cudaStreamSynchronize(mesh->stream));
        double d;
        static_assert(sizeof(d) == sizeof(h), "64-bit");
        std::memcpy(&d, &h, sizeof(d));
        *host_dt = d;
    });
}

int mhd_gpu_mars_implicit_sources(MhdMesh *mesh, const MhdMarsParams *params, const double *Btot, const double *neutral, double dt, double *U)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && params && Btot && U && (neutral || params->n_neutral == 0), "null argument");
        const MarsP p = mars_params(*params);
        const MeshView &m = mesh->v;
        if (!m.no_cells) return;
        k_mars_implicit<<<grid_for(m.no_cells, 128), 128, 0, mesh->stream>>>(m, p, Btot, neutral, dt, U);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_mars_advance(MhdMesh *mesh, int32_t n_species, const double *rhs, double dt, double *U)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && rhs && U && n_species >= 1 && n_species <= kMaxSpecies, "bad argument");
        const MeshView &m = mesh->v;
        if (!m.no_cells) return;
        k_mars_advance<<<grid_for(m.no_cells, 128), 128, 0, mesh->stream>>>(m, n_species, rhs, dt, U);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_mars_floors(MhdMesh *mesh, const MhdMarsParams *params, double *U)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && params && U, "null argument");
        const MarsP p = mars_params(*params);
        const MeshView &m = mesh->v;
        if (!m.no_cells) return;
        k_mars_floors<<<grid_for(m.no_cells, 128), 128, 0, mesh->stream>>>(m, p, U);
        MHD_LAUNCH_CHECK();
    });
}

} // extern "C"
