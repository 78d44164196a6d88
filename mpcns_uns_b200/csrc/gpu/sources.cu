// nvcc-flags: -fmad=false
// Source terms of the two-ion model (sources.cuh): add_sources_n (J x B, ambipolar force, chemistry), the
// electron-pressure gradient, the ambipolar edge EMF and the exact gyration, as reference-signature entry
// points and as the launchers the fused step uses.
#include "common.cuh"
#include "sources.cuh"

namespace mhd
{
namespace
{
// mercury::gyrate_n (MercuryUns/physics/Gyration.cpp) on the owned fluid cells; UH, UNa addressed
// as SField (AoS or species-major SoA); B as 3 doubles per cell, or float4 per cell when B3 is null;
// angle from dt_val, or scale * (*dtp) when dtp is set
__global__ void __launch_bounds__(128) k_gyrate(MeshView m, SrcParams p, const double *__restrict__ B3, const float4 *__restrict__ B4,
                                                 const double *__restrict__ dtp, double scale, double dt_val, SField<double> UH,
                                                 SField<double> UN, Reprepare rp)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.no_cells || m.material[c] == 1) return;
    const double dt = dtp ? scale * *dtp : dt_val;
    const V3 b = B3 ? ld3(B3, c) : mk(B4[c].x, B4[c].y, B4[c].z);
    double uh[5], un[5];
    for (int q = 0; q < 5; ++q)
    {
        uh[q] = UH(0, c, q);
        un[q] = UN(0, c, q);
    }
    gyrate_cell(p, b, dt, uh, un); // densities unchanged; momenta and energies rewritten (unchanged where nothing turns)
    for (int q = 1; q < 5; ++q)
    {
        UH(0, c, q) = uh[q];
        UN(0, c, q) = un[q];
    }
    if (rp.on)
    {
        double u[3];
        prepare_prims(rp.fp, rp.mass, rp.M_ref, rp.U, rp.W, c, true, u);
        st3(rp.up, c, mk(u[0], u[1], u[2]));
    }
}

// mercury::add_sources (MercurySources.cpp:13-63), reference (AoS) layout, rhs in place
__global__ void __launch_bounds__(128) k_add_sources(MeshView m, SrcParams p, int s, const double *__restrict__ WH,
                                                      const double *__restrict__ WNa, const double *__restrict__ B,
                                                      const double *__restrict__ J, const double *__restrict__ dpe,
                                                      const double *__restrict__ photo, const double *__restrict__ vst, double dt,
                                                      double *__restrict__ rhs)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.no_cells || m.material[c] == 1) return;
    const double *W = (s == 0 ? WH : WNa) + 5 * (int64_t)c;
    const double w[5] = {W[0], W[1], W[2], W[3], W[4]};
    double r[5];
    for (int q = 0; q < 5; ++q) r[q] = rhs[5 * (int64_t)c + q];
    const V3 d = dpe ? ld3(dpe, c) : mk(0, 0, 0);
    add_sources_cell(p, s, WH[5 * (int64_t)c], WNa[5 * (int64_t)c], w, J ? ld3(J, c) : mk(0, 0, 0), B ? ld3(B, c) : mk(0, 0, 0),
                     dpe ? &d : nullptr, photo ? photo + c : nullptr, vst ? vst + c : nullptr, dt, r);
    for (int q = 0; q < 5; ++q) rhs[5 * (int64_t)c + q] = r[q];
}

// electron_pressure_gradient over all cells (zero outside the owned fluid cells); W(s, c, 4) the pressures
__global__ void __launch_bounds__(128) k_dpe(MeshView m, SField<const double> W, double *__restrict__ dpe)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    V3 g = mk(0, 0, 0);
    if (c < m.no_cells && m.material[c] == 0) g = electron_pressure_gradient(m, c, [&](int32_t o) { return W(0, o, 4) + W(1, o, 4); });
    st3(dpe, c, g);
}

__global__ void __launch_bounds__(128) k_node_pressure(MeshView m, SField<const double> W, double *__restrict__ pn, int8_t *__restrict__ pok)
{
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= m.nn) return;
    bool ok;
    pn[v] = node_pressure(m, v, [&](int32_t c) { return W(0, c, 4) + W(1, c, 4); }, ok);
    pok[v] = ok ? 1 : 0;
}

// AmbipolarEMF::add on the owned edges, E in place
__global__ void __launch_bounds__(128) k_ambipolar_emf(MeshView m, SrcParams p, SField<const double> W, const double *__restrict__ pn,
                                                        const int8_t *__restrict__ pok, double *__restrict__ E)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.no_edges) return;
    double v;
    if (ambipolar_edge(m, p, e, [&](int32_t c, int s) { return W(s, c, 0); }, pn, pok, v)) E[e] -= v;
}
} // namespace

void launch_dpe(const MeshView &m, const double *W, double *dpe, cudaStream_t s)
{
    if (!m.nc) return;
    const int64_t nc = m.nc;
    k_dpe<<<grid_for(m.nc, 128), 128, 0, s>>>(m, SField<const double>{W, 5 * nc, 1, nc}, dpe);
    MHD_LAUNCH_CHECK();
}

void launch_node_pressure(const MeshView &m, const double *W, double *pn, int8_t *pok, cudaStream_t s)
{
    if (!m.nn) return;
    const int64_t nc = m.nc;
    k_node_pressure<<<grid_for(m.nn, 128), 128, 0, s>>>(m, SField<const double>{W, 5 * nc, 1, nc}, pn, pok);
    MHD_LAUNCH_CHECK();
}

SrcParams src_params(const MhdStepParams &q)
{
    SrcParams p;
    p.on = q.lorentz != 0;
    p.inver_MA2 = q.inver_MA2;
    p.induce = q.induce_coeff;
    p.M_ref = q.M_ref;
    p.mH = q.mass[0];
    p.mNa = q.n_species > 1 ? q.mass[1] : q.mass[0];
    p.ne_floor = q.ne_floor;
    p.gamma = q.gamma;
    p.rho_floor = q.rho_floor;
    p.p_floor = q.p_floor;
    p.ambi = q.ambipolar != 0;
    p.chem = q.chemistry != 0;
    p.pressure_coef = q.pressure_coef;
    p.a1_Na = q.a1_Na;
    p.a4 = q.a4;
    p.a5 = q.a5;
    p.a6 = q.a6;
    p.sch = q.state_coeff_H;
    p.scn = q.state_coeff_Na;
    p.T_ref = q.T_ref;
    p.Tn0 = q.Tn0;
    return p;
}

void launch_gyrate(const MeshView &m, const SrcParams &p, const double *B3, const float4 *B4, const double *dtp, double scale,
                   double *U, cudaStream_t s, const Reprepare &rp)
{
    if (!m.no_cells || !p.on || !(p.induce > 0)) return;
    const int64_t nc = m.nc;
    k_gyrate<<<grid_for(m.no_cells, 128), 128, 0, s>>>(m, p, B3, B4, dtp, scale, 0.0, SField<double>{U, 0, 1, nc},
                                                        SField<double>{U + 5 * nc, 0, 1, nc}, rp);
    MHD_LAUNCH_CHECK();
}
} // namespace mhd

using namespace mhd;

extern "C" {

int mhd_gpu_add_sources(MhdMesh *mesh, const MhdStepParams *params, int32_t species, const double *WH, const double *WNa, const double *B,
                        const double *J, const double *dpe, const double *photo, const double *vst, double dt, double *rhs)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && params && WH && WNa && rhs, "null argument");
        MHD_REQUIRE(!params->lorentz || (B && J), "the J x B force needs B and J");
        MHD_REQUIRE(params->n_species == 2, "the source terms are those of the two-ion model (n_species == 2)");
        MHD_REQUIRE(species == 0 || species == 1, "species must be 0 (H+) or 1 (Na+)");
        MHD_REQUIRE(params->mass[0] > 0 && params->mass[1] > 0, "species masses must be positive");
        const MeshView &m = mesh->v;
        if (!m.no_cells) return;
        k_add_sources<<<grid_for(m.no_cells, 128), 128, 0, mesh->stream>>>(m, src_params(*params), species, WH, WNa, B, J, dpe, photo,
                                                                            vst, dt, rhs);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_electron_pressure_gradient(MhdMesh *mesh, const double *WH, const double *WNa, double *dpe)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && WH && WNa && dpe, "null argument");
        const MeshView &m = mesh->v;
        if (!m.nc) return;
        // the AoS primitives of the two species as one strided view: species 0 at WH, species 1 at WNa
        const int64_t off = WNa - WH;
        k_dpe<<<grid_for(m.nc, 128), 128, 0, mesh->stream>>>(m, SField<const double>{WH, off, 5, 1}, dpe);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_ambipolar_emf(MhdMesh *mesh, const MhdStepParams *params, const double *WH, const double *WNa, double *E)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && params && WH && WNa && E, "null argument");
        MHD_REQUIRE(params->n_species == 2 && params->mass[0] > 0 && params->mass[1] > 0, "the two-ion model (n_species == 2)");
        const MeshView &m = mesh->v;
        MHD_REQUIRE(m.e_nodes && m.n2c_ptr, "the ambipolar EMF needs the mesh's edge_nodes");
        if (!m.no_edges) return;
        const int64_t off = WNa - WH;
        const SField<const double> W{WH, off, 5, 1};
        DBuf<double> pn;
        DBuf<int8_t> pok;
        pn.alloc(m.nn > 0 ? (size_t)m.nn : 1);
        pok.alloc(m.nn > 0 ? (size_t)m.nn : 1);
        if (m.nn) k_node_pressure<<<grid_for(m.nn, 128), 128, 0, mesh->stream>>>(m, W, pn.p, pok.p);
        k_ambipolar_emf<<<grid_for(m.no_edges, 128), 128, 0, mesh->stream>>>(m, src_params(*params), W, pn.p, pok.p, E);
        MHD_LAUNCH_CHECK();
        MHD_CUDA(cudaStreamSynchronize(mesh->stream)); // the nodal arrays are freed on return
    });
}

int mhd_gpu_gyrate(MhdMesh *mesh, const MhdStepParams *params, const double *B, double dt, double *UH, double *UNa)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && params && B && UH && UNa, "null argument");
        MHD_REQUIRE(params->n_species == 2, "the gyration is that of the two-ion model (n_species == 2)");
        MHD_REQUIRE(params->mass[0] > 0 && params->mass[1] > 0, "species masses must be positive");
        const MeshView &m = mesh->v;
        const SrcParams p = src_params(*params);
        if (!m.no_cells || !p.on || !(p.induce > 0)) return; // gyrate_n returns at once (Gyration.cpp)
        k_gyrate<<<grid_for(m.no_cells, 128), 128, 0, mesh->stream>>>(m, p, B, nullptr, nullptr, 1.0, dt, SField<double>{UH, 0, 5, 1},
                                                                       SField<double>{UNa, 0, 5, 1}, Reprepare{});
        MHD_LAUNCH_CHECK();
    });
}

} // extern "C"
