// nvcc-flags: -fmad=false
// Resident state and the fused explicit SSP-RK2 step of the hot path (FP64, reference-exact:
// reference operation order, no multiply-add contraction).
//
// One stage on (Us, Phi_s) -> (Uo, Phi_o):
//   k_prepare      per cell: primitives of every species, B_ind = cell fit of Phi_s, B_tot, u+
//   [k_cell_current] J of B_ind when the two-ion J x B force is on
//   [k_cfl_*]      stage 1, CFL mode: per-cell step, device-wide minimum (no host round trip)
//   per species group: k_limited_gradients, k_face_flux, k_update (gather [+ J x B] + U += dt rhs + floors)
//   k_face_candidate, k_edge_emf_assign (begin + UCT + boundary edge values)
//   k_ct           Phi_o = Phi_s - dt d1 E on the active faces
// Stage 2 writes the SSP-RK2 averages U = (U0 + U2)/2, Phi = (Phi0 + Phi2)/2 in place.  With the
// gyration on, half-step exact gyrations (k_gyrate) wrap the two stages (Strang splitting).
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "induction.cuh"
#include "kernels.cuh"
#include "state.cuh"

namespace mhd
{
namespace
{
constexpr int kGroup = 2; // species whose gradients and face fluxes are held at once

__device__ __forceinline__ void to_cons5(const Prim5 &W, double gamma, double *U)
{
    U[0] = W.rho;
    U[1] = W.rho * W.u;
    U[2] = W.rho * W.v;
    U[3] = W.rho * W.w;
    U[4] = W.p / (gamma - 1.0) + 0.5 * W.rho * (W.u * W.u + W.v * W.v + W.w * W.w);
}

// Solver::prepare (Solver.cpp:94-125) without the halo exchange and the cell current
__global__ void __launch_bounds__(128) k_prepare(MeshView m, FluidParams p, const double *__restrict__ mass, double M_ref,
                                                  SField<const double> U, SField<double> W, const double *__restrict__ phi,
                                                  const double *__restrict__ Badd, double *__restrict__ Bind, double *__restrict__ Btot,
                                                  double *__restrict__ up)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    double u[3];
    prepare_prims(p, mass, M_ref, U, W, c, m.material[c] == 0, u);
    const V3 b = cell_vector(m, phi, c);
    st3(Bind, c, b);
    st3(Btot, c, mk(b.x + Badd[3 * (int64_t)c], b.y + Badd[3 * (int64_t)c + 1], b.z + Badd[3 * (int64_t)c + 2]));
    st3(up, c, mk(u[0], u[1], u[2]));
}

__device__ __forceinline__ double cell_dt(const MeshView &m, const FluidParams &p, double cfl, double inver_MA2, double rho_floor_dt,
                                          const SField<const double> &W, const double *__restrict__ Btot, int32_t c);

// mercury::cell_time_steps (MercuryUns/fluid/MercurySources.cpp:65-106) without the optional gyration
// limit, n species (the wave speeds use the summed density, as the reference does for its two ions);
// the device-wide minimum of mercury::local_time_step (:108-116) is reduced per block first.
__global__ void __launch_bounds__(128) k_cfl_cells(MeshView m, FluidParams p, double cfl, double inver_MA2, double rho_floor_dt,
                                                    SField<const double> W, const double *__restrict__ Btot,
                                                    unsigned long long *__restrict__ dt_bits, int *__restrict__ flag)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    double dt = CUDART_INF;
    if (c < m.no_cells && m.material[c] == 0) dt = cell_dt(m, p, cfl, inver_MA2, rho_floor_dt, W, Btot, c);
    if (!(dt > 0)) atomicOr(flag, 1); // zero, negative or NaN: the reference's "invalid time step"
    // block minimum (min is exact, so the order of the reduction does not matter), one atomic per block
    __shared__ double sh[32];
    double v = dt > 0 ? dt : CUDART_INF;
    for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : CUDART_INF;
        for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0 && v < CUDART_INF) atomicMin(dt_bits, static_cast<unsigned long long>(__double_as_longlong(v)));
    }
}

__device__ __forceinline__ double cell_dt(const MeshView &m, const FluidParams &p, double cfl, double inver_MA2, double rho_floor_dt,
                                          const SField<const double> &W, const double *__restrict__ Btot, int32_t c)
{
    double dt = CUDART_INF;
    const V3 b = ld3(Btot, c);
    const double B2 = dot(b, b);
    double rsum = W(0, c, 0);
    for (int s = 1; s < p.nsp; ++s) rsum = rsum + W(s, c, 0);
    const double rho_tot = dmax(rsum, rho_floor_dt);
    const int32_t k0 = m.c2f_ptr[c], k1 = m.c2f_ptr[c + 1];
    for (int s = 0; s < p.nsp; ++s)
    {
        const double cs2 = p.gamma * W(s, c, 4) / dmax(W(s, c, 0), 1e-30);
        double denom = 0;
        for (int32_t k = k0; k < k1; ++k)
        {
            const int32_t f = m.c2f_idx[k];
            const double A = m.face_area_mag[f];
            const V3 n = (1.0 / A) * ld3(m.face_area, f);
            const double vA2 = inver_MA2 * B2 / rho_tot;
            const double vAn2 = inver_MA2 * dot(b, n) * dot(b, n) / rho_tot;
            const double term = cs2 + vA2;
            const double cf = sqrt(0.5 * (term + sqrt(dmax(0.0, term * term - 4 * cs2 * vAn2))));
            denom += (fabs(W(s, c, 1) * n.x + W(s, c, 2) * n.y + W(s, c, 3) * n.z) + cf) * A;
        }
        if (denom > 0) dt = dmin(dt, cfl * m.cell_volume[c] / denom);
    }
    return dt;
}

__global__ void k_cfl_init(unsigned long long *dt_bits, int *flag)
{
    *dt_bits = static_cast<unsigned long long>(__double_as_longlong(CUDART_INF));
    *flag = 0;
}

// gdt = min(gdt, dt_max); invalid unless finite and positive (Solver.cpp:233-236)
__global__ void k_cfl_final(const unsigned long long *dt_bits, double dt_max, double *dt, int *flag)
{
    double g = __longlong_as_double(static_cast<long long>(*dt_bits));
    g = dmin(g, dt_max);
    if (!isfinite(g) || g <= 0) atomicOr(flag, 1);
    *dt = g;
}

__global__ void k_set_dt(double *dt, double v, int *flag)
{
    *dt = v;
    *flag = 0;
}

// Inputs of the two-ion J x B source added to the gathered rhs (mercury::Solver::rhs, Solver.cpp:146-149)
struct SrcView
{
    SrcParams p;
    SField<const double> W; // primitives of all species
    const double *J, *Bt;   // cell current of the induced field, total cell field
    const double *dpe, *photo, *vst; // source fields (null: absent)
};

// Solver::advance (Solver.cpp:194-206) for one species group: rhs gathered from the face fluxes in the
// reference's scatter order, plus the J x B source when it is on, U = U_base + dt rhs on the owned
// fluid cells, Solver::enforce_floors (:171-191); stage 2 averages with U0 in place (Solver.cpp:505-506).
// NF = 4: tetrahedral mesh, the four faces of the cell unrolled (all flux gathers in flight together);
// NF = 0: any polyhedra.  One thread per (cell, species of the group = blockIdx.y).
// fl (optional): which floor each owned fluid cell and species met, [s*nc + c]: 0 none, 1 density, 2 pressure.
template <int NF>
__global__ void __launch_bounds__(128) k_update(MeshView m, FluidParams p, int s0, int ng, const double *__restrict__ F,
                                                 SField<const double> Ub, SField<double> Uo, const double *__restrict__ dtp, int stage2,
                                                 SrcView sv, int8_t *__restrict__ fl)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (c >= m.nc || g >= ng) return;
    const int64_t nf = m.nf;
    const double dt = *dtp;
    const bool live = c < m.no_cells && m.material[c] == 0;
    const int32_t k0 = NF ? NF * c : m.c2f_ptr[c], k1 = NF ? NF * c + NF : m.c2f_ptr[c + 1];
    const double V = m.cell_volume[c];
    {
        const int s = s0 + g;
        double u[5];
        for (int q = 0; q < 5; ++q) u[q] = Ub(s, c, q);
        if (live)
        {
            double r[5] = {0, 0, 0, 0, 0};
            if constexpr (NF == 4)
            {
                const int4 fi = *reinterpret_cast<const int4 *>(m.cfa_idx + k0);
                const char4 sg = *reinterpret_cast<const char4 *>(m.cfa_sgn + k0);
                const int32_t ff[4] = {fi.x, fi.y, fi.z, fi.w};
                const bool out[4] = {sg.x > 0, sg.y > 0, sg.z > 0, sg.w > 0};
                double Fv[4][5];
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int q = 0; q < 5; ++q) Fv[j][q] = F[(g * 5 + q) * nf + ff[j]];
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int q = 0; q < 5; ++q)
                    {
                        const double v = Fv[j][q] / V;
                        r[q] = out[j] ? r[q] - v : r[q] + v;
                    }
            }
            else
                for (int32_t k = k0; k < k1; ++k)
                {
                    const int32_t f = m.cfa_idx[k];
                    const bool out = m.cfa_sgn[k] > 0;
                    for (int q = 0; q < 5; ++q)
                    {
                        const double v = F[(g * 5 + q) * nf + f] / V;
                        r[q] = out ? r[q] - v : r[q] + v;
                    }
                }
            if (sv.p.any()) // mercury::add_sources after the flux gather (Solver.cpp:146-149)
            {
                const double w[5] = {sv.W(s, c, 0), sv.W(s, c, 1), sv.W(s, c, 2), sv.W(s, c, 3), sv.W(s, c, 4)};
                const V3 d = sv.dpe ? ld3(sv.dpe, c) : mk(0, 0, 0);
                add_sources_cell(sv.p, s, sv.W(0, c, 0), sv.W(1, c, 0), w, sv.p.on ? ld3(sv.J, c) : mk(0, 0, 0),
                                 sv.p.on ? ld3(sv.Bt, c) : mk(0, 0, 0), sv.dpe ? &d : nullptr, sv.photo ? sv.photo + c : nullptr,
                                 sv.vst ? sv.vst + c : nullptr, dt, r);
            }
            for (int q = 0; q < 5; ++q) u[q] += dt * r[q];
            const double ke = u[0] > 0 ? 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0] : 0.0;
            int8_t which = 0;
            if (!(u[0] >= p.rho_floor))
            {
                to_cons5(Prim5{p.rho_floor, 0, 0, 0, p.p_floor}, p.gamma, u);
                which = 1;
            }
            else if ((p.gamma - 1.0) * (u[4] - ke) < p.p_floor)
            {
                to_cons5(to_prim(u[0], u[1], u[2], u[3], u[4], p.gamma, p.rho_floor, p.p_floor), p.gamma, u);
                which = 2;
            }
            if (fl) fl[(int64_t)s * m.nc + c] = which;
            if (p.sw_floor) sw_log(p.sw_floor, (int64_t)s * m.nc + c, static_cast<uint32_t>(which));
        }
        if (stage2)
            for (int q = 0; q < 5; ++q) Uo(s, c, q) = 0.5 * (Uo(s, c, q) + u[q]);
        else
            for (int q = 0; q < 5; ++q) Uo(s, c, q) = u[q];
    }
}

// mhd::faraday_update on the active faces (Faraday.cpp:15-24); stage 2 averages with Phi0 in place (Solver.cpp:507-508)
__global__ void __launch_bounds__(256) k_ct(MeshView m, const double *__restrict__ E, const double *__restrict__ phis,
                                             double *__restrict__ phio, const double *__restrict__ dtp, int stage2)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    bool active = false;
    for (int32_t k = m.f2c_ptr[f]; k < m.f2c_ptr[f + 1]; ++k) active |= m.f2c_idx[k] < m.no_cells;
    double v = phis[f];
    if (active)
    {
        double circ = 0.0;
        for (int32_t k = m.f2e_ptr[f]; k < m.f2e_ptr[f + 1]; ++k) circ += m.f2e_sgn[k] * E[m.f2e_idx[k]];
        v -= *dtp * circ;
    }
    phio[f] = stage2 ? 0.5 * (phio[f] + v) : v;
}

// n_e,eff of the fluid cells, 0 elsewhere (Solver.cpp:257-259: mhd::Scales::numinfo of the two ions' densities)
__global__ void k_ne_eff(MeshView m, SrcParams sp, SField<const double> W, double *__restrict__ ne)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    ne[c] = m.material[c] == 0 ? numinfo2(sp, W(0, c, 0), W(1, c, 0)).ne_eff : 0.0;
}

// the Dirichlet edges of the semi-implicit solve: the inflow edges (Solver.cpp:261-262)
__global__ void k_inflow_dir(MeshView m, int8_t *__restrict__ dir)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < m.ne) dir[e] = m.edge_mode[e] == 2 ? 1 : 0;
}

__global__ void k_aos_to_soa(const double *__restrict__ in, double *__restrict__ out, int32_t n, int ncomp)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * ncomp) return;
    const int64_t c = i / ncomp, q = i % ncomp;
    out[q * n + c] = in[i];
}

__global__ void k_soa_to_aos(const double *__restrict__ in, double *__restrict__ out, int32_t n, int ncomp)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * ncomp) return;
    const int64_t c = i / ncomp, q = i % ncomp;
    out[i] = in[q * n + c];
}

__global__ void k_cell_vector_all(MeshView m, const double *__restrict__ flux, double *__restrict__ out)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    st3(out, c, cell_vector(m, flux, c));
}
} // namespace
} // namespace mhd

namespace mhd
{
namespace
{
SField<double> soa_state(double *p, int64_t nc) { return {p, 5 * nc, 1, nc}; }
SField<const double> soa_cstate(const double *p, int64_t nc) { return {p, 5 * nc, 1, nc}; }

// Solver::prepare of (Us, phis) (with the cell current when the J x B force is on) and, with cfl,
// the device CFL step (mercury::local_time_step) into scal[0]
void prepare_cfl(MhdState *st, const double *Us, const double *phis, bool cfl, double dt_max)
{
    MhdMesh *mesh = st->mesh;
    const MeshView &m = mesh->v;
    cudaStream_t s = mesh->stream;
    const int64_t nc = m.nc;
    Profiler &P = st->prof;
    if (m.nc)
    {
        P.begin(KP_PREPARE, s);
        k_prepare<<<grid_for(m.nc, 128), 128, 0, s>>>(m, st->fp, st->mass.p, st->prm.M_ref, soa_cstate(Us, nc), soa_state(st->W.p, nc),
                                                      phis, st->badd.p, st->bind.p, st->btot.p, st->up.p);
        MHD_LAUNCH_CHECK();
        ++st->launches;
        if (st->src.on) // J of the induced field (Solver.cpp:123)
        {
            launch_cell_current(m, st->bind.p, st->J.p, s);
            ++st->launches;
        }
        if (st->src.ambi && !st->mixed) // grad p_e (Solver.cpp:124) and the nodal p_e of the ambipolar EMF
        {
            launch_dpe(m, st->W.p, st->dpe.p, s);
            launch_node_pressure(m, st->W.p, st->pn.p, st->pok.p, s);
            st->launches += 1 + (m.nn ? 1 : 0);
        }
        P.end(KP_PREPARE, s);
    }
    if (cfl)
    {
        P.begin(KP_CFL, s);
        k_cfl_init<<<1, 1, 0, s>>>(st->dt_bits.p, st->flag.p);
        if (m.no_cells)
            k_cfl_cells<<<grid_for(m.no_cells, 128), 128, 0, s>>>(m, st->fp, st->prm.cfl, st->prm.inver_MA2, st->prm.rho_floor_dt,
                                                                   soa_cstate(st->W.p, nc), st->btot.p, st->dt_bits.p, st->flag.p);
        k_cfl_final<<<1, 1, 0, s>>>(st->dt_bits.p, dt_max, st->scal.p, st->flag.p);
        MHD_LAUNCH_CHECK();
        P.end(KP_CFL, s);
        st->launches += m.no_cells ? 3 : 2;
    }
}

void stage(MhdState *st, const double *Us, const double *phis, double *Uo, double *phio, bool stage2, bool cfl, double dt_max,
           bool prepared = false, bool ct = true)
{
    MhdMesh *mesh = st->mesh;
    const MeshView &m = mesh->v;
    cudaStream_t s = mesh->stream;
    const int64_t nc = m.nc;
    const int nsp = st->nsp;
    Profiler &P = st->prof;
    if (!prepared) prepare_cfl(st, Us, phis, cfl, dt_max);
    const SrcView sv{st->src,
                     soa_cstate(st->W.p, nc),
                     st->J.p,
                     st->btot.p,
                     st->src.ambi ? st->dpe.p : nullptr,
                     st->src.chem && st->photo.n ? st->photo.p : nullptr,
                     st->src.chem && st->vst.n ? st->vst.p : nullptr};
    for (int s0 = 0; s0 < nsp; s0 += st->group)
    {
        const int ng = std::min(st->group, nsp - s0);
        FluidParams gp = st->fp;
        gp.nsp = ng;
        for (int g = 0; g < ng; ++g)
        {
            gp.fs[g] = st->fp.fs[s0 + g];
            gp.absorb[g] = st->fp.absorb[s0 + g];
        }
        if (gp.wall_prim) gp.wall_prim = st->fp.wall_prim + (int64_t)s0 * 5 * st->fp.wall_n;
        if (gp.sw_lim) gp.sw_lim += (int64_t)s0 * 5 * nc;
        if (gp.sw_flux) gp.sw_flux += (int64_t)s0 * m.nf;
        const SField<const double> Wg{st->W.p + (int64_t)s0 * 5 * nc, 5 * nc, 1, nc};
        const SField<double> Gg{st->grad.p, 15 * nc, 1, nc};
        P.begin(KP_GRAD, s);
        if (st->prm.second_order) launch_limited_gradients(m, gp, Wg, Gg, s);
        else MHD_CUDA(cudaMemsetAsync(st->grad.p, 0, (size_t)15 * ng * nc * sizeof(double), s));
        P.end(KP_GRAD, s);
        P.begin(KP_FLUX, s);
        launch_face_flux(m, gp, Wg, SField<const double>{st->grad.p, 15 * nc, 1, nc}, st->F.p, s);
        P.end(KP_FLUX, s);
        if (m.nc)
        {
            P.begin(KP_UPDATE, s);
            const dim3 grid(grid_for(m.nc, 128), ng);
            if (m.faces_per_cell == 4)
                k_update<4><<<grid, 128, 0, s>>>(m, st->fp, s0, ng, st->F.p, soa_cstate(Us, nc), soa_state(Uo, nc), st->scal.p,
                                                 stage2 ? 1 : 0, sv, st->floor_flags);
            else
                k_update<0><<<grid, 128, 0, s>>>(m, st->fp, s0, ng, st->F.p, soa_cstate(Us, nc), soa_state(Uo, nc), st->scal.p,
                                                 stage2 ? 1 : 0, sv, st->floor_flags);
            MHD_LAUNCH_CHECK();
            P.end(KP_UPDATE, s);
        }
        st->launches += (st->prm.second_order && m.nc ? 1 : 0) + (m.nf ? 1 : 0) + (m.nc ? 1 : 0);
    }
    const V3 ui = mk(st->prm.u_inf[0], st->prm.u_inf[1], st->prm.u_inf[2]), bi = mk(st->prm.B_imf[0], st->prm.B_imf[1], st->prm.B_imf[2]);
    const V3 Einf = -1.0 * cross(ui, bi);
    P.begin(KP_FACE_CAND, s);
    launch_face_candidate(m, st->up.p, st->btot.p, st->bind.p, phis, st->phi_add.p, st->Ef.p, s, st->efgeo.n ? st->pa.p : nullptr,
                          st->sw_face);
    P.end(KP_FACE_CAND, s);
    P.begin(KP_EDGE_EMF, s);
    AmbArgs amb;
    amb.on = st->src.ambi;
    amb.p = st->src;
    amb.W = st->W.p;
    amb.pn = st->pn.p;
    amb.pok = st->pok.p;
    launch_edge_emf_assign(m, st->Ef.p, st->up.p, phis, st->prm.cuct, Einf, st->E.p, s, st->mres.n ? st->mres.p : nullptr, amb,
                           st->sw_edge, st->efgeo.n ? st->efgeo.p : nullptr, st->efgeo.n ? st->pa.p : nullptr);
    P.end(KP_EDGE_EMF, s);
    st->launches += (m.nf ? 1 : 0) + (m.ne ? 1 : 0);
    if (ct && m.nf)
    {
        P.begin(KP_CT, s);
        k_ct<<<grid_for(m.nf, 256), 256, 0, s>>>(m, st->E.p, phis, phio, st->scal.p, stage2 ? 1 : 0);
        MHD_LAUNCH_CHECK();
        P.end(KP_CT, s);
        ++st->launches;
    }
}

} // namespace

// One FP64 stage at the step size already in st->scal[0] (no CFL), for the differentiated run
void fp64_stage(MhdState *st, const double *Us, const double *phis, double *Uo, double *phio, bool stage2)
{
    stage(st, Us, phis, Uo, phio, stage2, false, 0.0);
}

// The first half of a stage: primitives, cell fields, u+ and the limited gradients of every species
// (one species group) of (Us, phis), as fp64_stage leaves them
void fp64_prepare_grad(MhdState *st, const double *Us, const double *phis)
{
    MHD_REQUIRE(st->nsp <= st->group, "one species group");
    prepare_cfl(st, Us, phis, false, 0.0);
    const MeshView &m = st->mesh->v;
    const int64_t nc = m.nc;
    const SField<const double> Wg{st->W.p, 5 * nc, 1, nc};
    const SField<double> Gg{st->grad.p, 15 * nc, 1, nc};
    if (st->prm.second_order) launch_limited_gradients(m, st->fp, Wg, Gg, st->mesh->stream);
    else if (nc) MHD_CUDA(cudaMemsetAsync(st->grad.p, 0, (size_t)15 * st->nsp * nc * sizeof(double), st->mesh->stream));
}

namespace
{
void read_dt(MhdState *st, double *dt_host)
{
    cudaStream_t s = st->mesh->stream;
    MHD_CUDA(cudaMemcpyAsync(st->pinned, st->scal.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    MHD_CUDA(cudaMemcpyAsync(st->pinned + 1, st->flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    MHD_CUDA(cudaStreamSynchronize(s));
    int flag;
    std::memcpy(&flag, st->pinned + 1, sizeof(int));
    if (flag) throw ApiError(MHD_ESTATE, "invalid time step");
    *dt_host = st->pinned[0];
}
} // namespace
} // namespace mhd

using namespace mhd;

extern "C" {

int mhd_gpu_state_set_wall_ghosts(MhdState *st, int32_t n_wall, const int32_t *faces, const double *prims)
{
    return guarded([&] {
        MHD_REQUIRE(st, "null state");
        MHD_REQUIRE(n_wall >= 0 && (!n_wall || (faces && prims)), "bad wall ghost table");
        st->fp.wall_slot = nullptr;
        st->fp.wall_prim = nullptr;
        st->fp.wall_n = 0;
        st->wall_slot.release();
        st->wall_prim.release();
        if (!n_wall) return;
        const MeshView &m = st->mesh->v;
        cudaStream_t s = st->mesh->stream;
        DBuf<int32_t> df;
        df.upload(faces, (size_t)n_wall);
        st->wall_slot.alloc(m.nf ? (size_t)m.nf : 1);
        try
        {
            build_wall_slots(m, df.p, n_wall, st->wall_slot.p, s);
        }
        catch (...)
        {
            st->wall_slot.release();
            throw;
        }
        st->wall_prim.upload(prims, (size_t)st->nsp * n_wall * 5);
        MHD_CUDA(cudaStreamSynchronize(s));
        st->fp.wall_slot = st->wall_slot.p;
        st->fp.wall_prim = st->wall_prim.p;
        st->fp.wall_n = n_wall;
    });
}

int mhd_gpu_state_create(MhdMesh *mesh, const MhdStepParams *p, MhdState **out)
{
    MhdState *st = nullptr;
    int rc = guarded([&] {
        MHD_REQUIRE(mesh && p && out, "null argument");
        MHD_REQUIRE(p->n_species >= 1 && p->n_species <= kMaxSpecies, "n_species must be 1..16");
        MHD_REQUIRE(p->gamma > 1.0, "gamma must exceed 1");
        for (int s = 0; s < p->n_species; ++s) MHD_REQUIRE(p->mass[s] > 0, "species masses must be positive");
        MHD_REQUIRE(!p->lorentz || p->n_species == 2, "the J x B force and the gyration are those of the two-ion model (n_species == 2)");
        MHD_REQUIRE(!(p->ambipolar || p->chemistry) || p->n_species == 2,
                    "the ambipolar and chemistry terms are those of the two-ion model (n_species == 2)");
        MHD_REQUIRE(!p->ambipolar || mesh->v.e_nodes, "the ambipolar EMF needs the mesh's edge_nodes");
        st = new MhdState;
        st->mesh = mesh;
        st->prm = *p;
        st->nsp = p->n_species;
        st->group = std::min(kGroup, st->nsp);
        FluidParams &fp = st->fp;
        fp.nsp = st->nsp;
        fp.limit = 1;
        fp.gamma = p->gamma;
        fp.rel_limit = p->rel_limit;
        fp.rho_floor = p->rho_floor;
        fp.p_floor = p->p_floor;
        for (int s = 0; s < st->nsp; ++s)
        {
            fp.fs[s] = Prim5{p->fs[s].rho, p->fs[s].u, p->fs[s].v, p->fs[s].w, p->fs[s].p};
            fp.absorb[s] = p->absorb[s];
        }
        const MeshView &m = mesh->v;
        const size_t nc = m.nc, nf = m.nf, ne = m.ne;
        st->U0.alloc(5 * nc * st->nsp);
        st->U1.alloc(5 * nc * st->nsp);
        st->W.alloc(5 * nc * st->nsp);
        st->grad.alloc(15 * nc * st->group);
        st->F.alloc(5 * nf * st->group);
        st->phi0.alloc(nf);
        st->phi1.alloc(nf);
        st->phi_add.alloc(nf);
        st->badd.alloc(3 * nc);
        st->bind.alloc(3 * nc);
        st->btot.alloc(3 * nc);
        st->up.alloc(3 * nc);
        st->Ef.alloc(3 * nf);
        st->E.alloc(ne);
        st->stage.alloc(std::max<size_t>(5 * nc, 3 * nc));
        st->scal.alloc(4);
        st->dt_bits.alloc(1);
        st->flag.alloc(1);
        st->mass.upload(p->mass, st->nsp);
        st->src = src_params(*p);
        if (st->src.on) st->J.alloc(3 * nc);
        if (st->src.ambi)
        {
            if (p->precision != MHD_PREC_MIXED) st->dpe.alloc(3 * nc); // the mixed update gathers grad p_e itself
            st->pn.alloc(m.nn ? (size_t)m.nn : 1);
            st->pok.alloc(m.nn ? (size_t)m.nn : 1);
        }
        MHD_CUDA(cudaMallocHost(&st->pinned, 8 * sizeof(double)));
        MHD_REQUIRE(p->precision == MHD_PREC_FP64 || p->precision == MHD_PREC_MIXED, "unknown precision");
        st->mixed = p->precision == MHD_PREC_MIXED;
        if (st->mixed)
        {
            MHD_REQUIRE(!m.nc || (m.faces_per_cell == 4 && m.tri_faces), "mixed precision needs a tetrahedral mesh");
            MHD_REQUIRE(m.max_valence <= 8 && m.max_edge_cells <= 8, "mixed precision needs edge valence <= 8");
            mixed_setup(st);
        }
        else
        {
            // the FP64 UCT's face geometry per (edge, slot) (512 bytes per edge), where the memory allows it:
            // without it the edge pass forms the same values inline
            const size_t n_geo = size_t(64) * ne;
            size_t free_b = 0, total_b = 0;
            MHD_CUDA(cudaMemGetInfo(&free_b, &total_b));
            if (n_geo && m.max_edge_cells <= 8 && m.max_valence <= 8 && free_b > n_geo * sizeof(double) + (size_t(8) << 30))
            {
                st->efgeo.alloc(n_geo);
                st->pa.alloc(nf);
                build_edge_face_geo(m, st->efgeo.p, mesh->stream);
            }
        }
        cudaStream_t s = mesh->stream;
        if (nc) MHD_CUDA(cudaMemsetAsync(st->U0.p, 0, 5 * nc * st->nsp * sizeof(double), s));
        if (nf)
        {
            MHD_CUDA(cudaMemsetAsync(st->phi0.p, 0, nf * sizeof(double), s));
            MHD_CUDA(cudaMemsetAsync(st->phi_add.p, 0, nf * sizeof(double), s));
        }
        if (nc) MHD_CUDA(cudaMemsetAsync(st->badd.p, 0, 3 * nc * sizeof(double), s));
        MHD_CUDA(cudaMemsetAsync(st->flag.p, 0, sizeof(int), s));
        MHD_CUDA(cudaStreamSynchronize(s));
        *out = st;
    });
    if (rc != MHD_OK) delete st;
    return rc;
}

int mhd_gpu_state_destroy(MhdState *st)
{
    return guarded([&] {
        if (!st) return;
        cudaStreamSynchronize(st->mesh->stream);
        delete st;
    });
}

// entries of a field's host array (0 for an unknown field)
static size_t field_count(const MhdState *st, int32_t field)
{
    const MeshView &m = st->mesh->v;
    return field == MHD_FIELD_U ? 5 * (size_t)m.nc : field == MHD_FIELD_BADD ? 3 * (size_t)m.nc
                                                                             : (field == MHD_FIELD_PHI || field == MHD_FIELD_PHIADD) ? (size_t)m.nf : 0;
}

int mhd_gpu_state_upload(MhdState *st, int32_t field, int32_t species, const double *host)
{
    return guarded([&] {
        MHD_REQUIRE(st && MHD_ARR(host, field_count(st, field)), "null argument");
        const MeshView &m = st->mesh->v;
        cudaStream_t s = st->mesh->stream;
        if (field == MHD_FIELD_U)
        {
            MHD_REQUIRE(species >= 0 && species < st->nsp, "species out of range");
            if (!m.nc) return;
            MHD_CUDA(cudaMemcpyAsync(st->stage.p, host, 5 * (size_t)m.nc * sizeof(double), cudaMemcpyHostToDevice, s));
            k_aos_to_soa<<<grid_for(5 * (int64_t)m.nc, 256), 256, 0, s>>>(st->stage.p, st->U0.p + (size_t)species * 5 * m.nc, m.nc, 5);
            MHD_LAUNCH_CHECK();
        }
        else if (field == MHD_FIELD_PHI)
        {
            if (m.nf) MHD_CUDA(cudaMemcpyAsync(st->phi0.p, host, (size_t)m.nf * sizeof(double), cudaMemcpyHostToDevice, s));
        }
        else if (field == MHD_FIELD_PHIADD)
        {
            if (m.nf) MHD_CUDA(cudaMemcpyAsync(st->phi_add.p, host, (size_t)m.nf * sizeof(double), cudaMemcpyHostToDevice, s));
            // BaddCell = reconstruct_cell_vector(PhiAdd) (MercuryUns/initial/Initial.cpp:82-83)
            if (m.nc) k_cell_vector_all<<<grid_for(m.nc, 128), 128, 0, s>>>(m, st->phi_add.p, st->badd.p);
            MHD_LAUNCH_CHECK();
            if (st->mixed) mixed_badd(st);
        }
        else
            MHD_REQUIRE(false, "unknown field");
        MHD_CUDA(cudaStreamSynchronize(s)); // the host buffer may be reused on return
    });
}

int mhd_gpu_state_download(MhdState *st, int32_t field, int32_t species, double *host)
{
    return guarded([&] {
        MHD_REQUIRE(st && MHD_ARR(host, field_count(st, field)), "null argument");
        const MeshView &m = st->mesh->v;
        cudaStream_t s = st->mesh->stream;
        if (field == MHD_FIELD_U)
        {
            MHD_REQUIRE(species >= 0 && species < st->nsp, "species out of range");
            if (!m.nc) return;
            k_soa_to_aos<<<grid_for(5 * (int64_t)m.nc, 256), 256, 0, s>>>(st->U0.p + (size_t)species * 5 * m.nc, st->stage.p, m.nc, 5);
            MHD_LAUNCH_CHECK();
            MHD_CUDA(cudaMemcpyAsync(host, st->stage.p, 5 * (size_t)m.nc * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        else if (field == MHD_FIELD_PHI)
        {
            if (m.nf) MHD_CUDA(cudaMemcpyAsync(host, st->phi0.p, (size_t)m.nf * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        else if (field == MHD_FIELD_PHIADD)
        {
            if (m.nf) MHD_CUDA(cudaMemcpyAsync(host, st->phi_add.p, (size_t)m.nf * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        else if (field == MHD_FIELD_BADD)
        {
            if (m.nc) MHD_CUDA(cudaMemcpyAsync(host, st->badd.p, 3 * (size_t)m.nc * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        else
            MHD_REQUIRE(false, "unknown field");
        MHD_CUDA(cudaStreamSynchronize(s));
    });
}

int mhd_gpu_state_set_source_fields(MhdState *st, const double *photo, const double *vst)
{
    return guarded([&] {
        MHD_REQUIRE(st, "null state");
        const size_t nc = st->mesh->v.nc;
        if (photo) st->photo.upload(photo, nc);
        else st->photo.release();
        if (vst) st->vst.upload(vst, nc);
        else st->vst.release();
    });
}

int mhd_gpu_state_device_ptr(MhdState *st, int32_t field, double **out)
{
    return guarded([&] {
        MHD_REQUIRE(st && out, "null argument");
        if (field == MHD_FIELD_U) *out = st->U0.p;
        else if (field == MHD_FIELD_PHI) *out = st->phi0.p;
        else if (field == MHD_FIELD_PHIADD) *out = st->phi_add.p;
        else if (field == MHD_FIELD_BADD) *out = st->badd.p;
        else MHD_REQUIRE(false, "unknown field");
    });
}

int mhd_gpu_cfl_dt(MhdState *st, double dt_max, double *host_dt)
{
    return guarded([&] {
        MHD_REQUIRE(st && host_dt, "null argument");
        MhdMesh *mesh = st->mesh;
        const MeshView &m = mesh->v;
        cudaStream_t s = mesh->stream;
        const int64_t nc = m.nc;
        if (nc)
            k_prepare<<<grid_for(m.nc, 128), 128, 0, s>>>(m, st->fp, st->mass.p, st->prm.M_ref, soa_cstate(st->U0.p, nc),
                                                          soa_state(st->W.p, nc), st->phi0.p, st->badd.p, st->bind.p, st->btot.p,
                                                          st->up.p);
        k_cfl_init<<<1, 1, 0, s>>>(st->dt_bits.p, st->flag.p);
        if (m.no_cells)
            k_cfl_cells<<<grid_for(m.no_cells, 128), 128, 0, s>>>(m, st->fp, st->prm.cfl, st->prm.inver_MA2, st->prm.rho_floor_dt,
                                                                   soa_cstate(st->W.p, nc), st->btot.p, st->dt_bits.p, st->flag.p);
        k_cfl_final<<<1, 1, 0, s>>>(st->dt_bits.p, dt_max, st->scal.p, st->flag.p);
        MHD_LAUNCH_CHECK();
        read_dt(st, host_dt);
    });
}

int mhd_gpu_step_rk2(MhdState *st, double dt_fixed, double dt_max, double *dt_used)
{
    return guarded([&] {
        MHD_REQUIRE(st, "null state");
        MHD_REQUIRE(dt_fixed > 0 || dt_max > 0, "need dt_fixed > 0 or dt_max > 0");
        cudaStream_t s = st->mesh->stream;
        const bool cfl = !(dt_fixed > 0);
        if (!cfl)
        {
            k_set_dt<<<1, 1, 0, s>>>(st->scal.p, dt_fixed, st->flag.p);
            MHD_LAUNCH_CHECK();
            ++st->launches;
        }
        // Strang splitting of the gyration (Solver.cpp:487-510): prepare and CFL step of U^n, half-step
        // gyration with its Btot, the two stages, then the closing half step with the Btot of the last
        // prepare (that of the stage-2 input)
        const bool split = st->src.on && st->src.induce > 0;
        const MeshView &m = st->mesh->v;
        if (st->mixed)
        {
            if (split)
            {
                mixed_prepare(st, st->U0.p, st->phi0.p, cfl, dt_max);
                st->prof.begin(KP_GYRATE, s);
                mixed_gyrate_open(st);
                st->prof.end(KP_GYRATE, s);
            }
            mixed_stage(st, st->U0.p, st->phi0.p, st->U1.p, st->phi1.p, false, cfl && !split, dt_max, split);
            mixed_stage(st, st->U1.p, st->phi1.p, st->U0.p, st->phi0.p, true, false, dt_max, false, split);
        }
        else
        {
            if (split)
            {
                prepare_cfl(st, st->U0.p, st->phi0.p, cfl, dt_max);
                // the gyration renews the primitives and u+ of the cells it turns: stage 1 starts prepared
                Reprepare rp;
                rp.on = 1;
                rp.fp = st->fp;
                rp.mass = st->mass.p;
                rp.M_ref = st->prm.M_ref;
                rp.U = soa_cstate(st->U0.p, m.nc);
                rp.W = soa_state(st->W.p, m.nc);
                rp.up = st->up.p;
                st->prof.begin(KP_GYRATE, s);
                launch_gyrate(m, st->src, st->btot.p, nullptr, st->scal.p, 0.5, st->U0.p, s, rp);
                st->prof.end(KP_GYRATE, s);
                st->launches += m.no_cells ? 1 : 0;
            }
            stage(st, st->U0.p, st->phi0.p, st->U1.p, st->phi1.p, false, cfl && !split, dt_max, split);
            stage(st, st->U1.p, st->phi1.p, st->U0.p, st->phi0.p, true, false, dt_max);
            if (split)
            {
                st->prof.begin(KP_GYRATE, s);
                launch_gyrate(m, st->src, st->btot.p, nullptr, st->scal.p, 0.5, st->U0.p, s);
                st->prof.end(KP_GYRATE, s);
            }
        }
        if (split && m.no_cells && !st->mixed) ++st->launches; // the FP64 closing gyration
        if (dt_used) read_dt(st, dt_used);
    });
}

int mhd_gpu_step_semi_implicit(MhdState *st, MhdInduction *ind, double dt_fixed, double dt_max, double *dt_used, int32_t *iterations,
                               double *rel_res)
{
    int status = MHD_OK;
    const int rc = guarded([&] {
        MHD_REQUIRE(st && ind, "null state or induction handle");
        MHD_REQUIRE(dt_fixed > 0 || dt_max > 0, "need dt_fixed > 0 or dt_max > 0");
        MHD_REQUIRE(!st->mixed, "the semi-implicit step runs on an FP64 state");
        MHD_REQUIRE(st->nsp == 2, "the semi-implicit step is the two-ion model's");
        MHD_REQUIRE(induction_mesh(ind) == st->mesh, "the induction handle belongs to another mesh");
        MhdMesh *mesh = st->mesh;
        const MeshView &m = mesh->v;
        cudaStream_t s = mesh->stream;
        const bool cfl = !(dt_fixed > 0);
        if (!cfl)
        {
            k_set_dt<<<1, 1, 0, s>>>(st->scal.p, dt_fixed, st->flag.p);
            MHD_LAUNCH_CHECK();
            ++st->launches;
        }
        // Solver::step_first_order (Solver.cpp:228-277): prepare and the CFL step; with the J x B force the
        // opening half-step gyration and prepare again
        const bool split = st->src.on && st->src.induce > 0;
        if (split)
        {
            prepare_cfl(st, st->U0.p, st->phi0.p, cfl, dt_max);
            Reprepare rp;
            rp.on = 1;
            rp.fp = st->fp;
            rp.mass = st->mass.p;
            rp.M_ref = st->prm.M_ref;
            rp.U = soa_cstate(st->U0.p, m.nc);
            rp.W = soa_state(st->W.p, m.nc);
            rp.up = st->up.p;
            st->prof.begin(KP_GYRATE, s);
            launch_gyrate(m, st->src, st->btot.p, nullptr, st->scal.p, 0.5, st->U0.p, s, rp);
            st->prof.end(KP_GYRATE, s);
            st->launches += m.no_cells ? 1 : 0;
        }
        // rhs and forward Euler of the fluid with floors, in place; E = the explicit EMF (ideal, ambipolar,
        // boundary values); no CT yet
        stage(st, st->U0.p, st->phi0.p, st->U0.p, st->phi0.p, false, cfl && !split, dt_max, split, false);
        // the implicit linear terms with the total EMF as the unknown (:250-266)
        st->ne_eff.alloc(std::max<size_t>(1, (size_t)m.nc));
        st->E_impl.alloc(std::max<size_t>(1, (size_t)m.ne));
        if (!st->dir_inflow.n)
        {
            st->dir_inflow.alloc(std::max<size_t>(1, (size_t)m.ne));
            if (m.ne) k_inflow_dir<<<grid_for(m.ne, 256), 256, 0, s>>>(m, st->dir_inflow.p);
            ++st->launches;
        }
        if (m.nc)
        {
            k_ne_eff<<<grid_for(m.nc, 256), 256, 0, s>>>(m, st->src, soa_cstate(st->W.p, m.nc), st->ne_eff.p);
            ++st->launches;
        }
        MHD_LAUNCH_CHECK();
        double dt = 0.0;
        read_dt(st, &dt);
        int rcs = mhd_gpu_induction_set_frozen(ind, st->btot.p, st->ne_eff.p);
        if (rcs != MHD_OK) throw ApiError(rcs, std::string("induction: ") + mhd_gpu_last_error());
        int32_t it = 0;
        double rr = 0.0;
        rcs = mhd_gpu_induction_solve(ind, st->phi0.p, st->E.p, st->dir_inflow.p, dt, 1, st->E_impl.p, &it, &rr);
        if (rcs != MHD_OK && rcs != MHD_ENOCONV) throw ApiError(rcs, std::string("induction: ") + mhd_gpu_last_error());
        if (rcs == MHD_ENOCONV) status = MHD_ENOCONV;
        if (iterations) *iterations = it;
        if (rel_res) *rel_res = rr;
        // faraday_update with the implicit EMF (:269), then the closing half-step gyration with the Btot of
        // the step's prepare (:274)
        if (m.nf)
        {
            st->prof.begin(KP_CT, s);
            k_ct<<<grid_for(m.nf, 256), 256, 0, s>>>(m, st->E_impl.p, st->phi0.p, st->phi0.p, st->scal.p, 0);
            MHD_LAUNCH_CHECK();
            st->prof.end(KP_CT, s);
            ++st->launches;
        }
        if (split)
        {
            st->prof.begin(KP_GYRATE, s);
            launch_gyrate(m, st->src, st->btot.p, nullptr, st->scal.p, 0.5, st->U0.p, s);
            st->prof.end(KP_GYRATE, s);
            st->launches += m.no_cells ? 1 : 0;
        }
        if (dt_used) *dt_used = dt;
        MHD_CUDA(cudaStreamSynchronize(s));
    });
    return rc != MHD_OK ? rc : status;
}

int mhd_gpu_state_profile(MhdState *st, int32_t enable)
{
    return guarded([&] {
        MHD_REQUIRE(st, "null state");
        MHD_CUDA(cudaStreamSynchronize(st->mesh->stream));
        st->prof.on = enable != 0;
        for (auto &u : st->prof.used) u = 0;
    });
}

int mhd_gpu_state_profile_read(MhdState *st, int32_t max_kernels, char *names, double *ms_total, int64_t *count, int32_t *n_out)
{
    return guarded([&] {
        MHD_REQUIRE(st && names && ms_total && count && n_out, "null argument");
        MHD_CUDA(cudaStreamSynchronize(st->mesh->stream));
        int n = 0;
        for (int k = 0; k < KP_COUNT && n < max_kernels; ++k, ++n)
        {
            std::strncpy(names + 32 * n, kStepKernelNames[k], 31);
            names[32 * n + 31] = 0;
            st->prof.read(k, ms_total[n], count[n]);
        }
        *n_out = n;
    });
}

int mhd_gpu_state_launches(MhdState *st, int64_t *out)
{
    return guarded([&] {
        MHD_REQUIRE(st && out, "null argument");
        *out = st->launches;
    });
}

} // extern "C"
