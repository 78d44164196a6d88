// nvcc-flags: -fmad=false
// Source terms of the two-ion model (sources.cuh): the J x B force and the exact gyration, as
// reference-signature entry points and as the launcher the fused step uses.
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

// mercury::add_sources (MercurySources.cpp:13-63), J x B part, reference (AoS) layout, rhs in place
__global__ void __launch_bounds__(128) k_add_sources(MeshView m, SrcParams p, int s, const double *__restrict__ WH,
                                                      const double *__restrict__ WNa, const double *__restrict__ B,
                                                      const double *__restrict__ J, double dt, double *__restrict__ rhs)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.no_cells || m.material[c] == 1) return;
    const double *W = (s == 0 ? WH : WNa) + 5 * (int64_t)c;
    const double w[5] = {W[0], W[1], W[2], W[3], W[4]};
    double r[5];
    for (int q = 0; q < 5; ++q) r[q] = rhs[5 * (int64_t)c + q];
    lorentz_source(p, s, WH[5 * (int64_t)c], WNa[5 * (int64_t)c], w, ld3(J, c), ld3(B, c), dt, r);
    for (int q = 0; q < 5; ++q) rhs[5 * (int64_t)c + q] = r[q];
}
} // namespace

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
                        const double *J, double dt, double *rhs)
{
    return guarded([&] {
        MHD_REQUIRE(mesh && params && WH && WNa && B && J && rhs, "null argument");
        MHD_REQUIRE(params->n_species == 2, "the source terms are those of the two-ion model (n_species == 2)");
        MHD_REQUIRE(species == 0 || species == 1, "species must be 0 (H+) or 1 (Na+)");
        MHD_REQUIRE(params->mass[0] > 0 && params->mass[1] > 0, "species masses must be positive");
        const MeshView &m = mesh->v;
        if (!m.no_cells) return;
        k_add_sources<<<grid_for(m.no_cells, 128), 128, 0, mesh->stream>>>(m, src_params(*params), species, WH, WNa, B, J, dt, rhs);
        MHD_LAUNCH_CHECK();
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
