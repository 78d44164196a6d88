// Resident state of the fused step, shared by the FP64 (step.cu) and the mixed-precision (mixed.cu)
// translation units.
#pragma once
#include <vector>

#include "fluid.cuh"
#include "sources.cuh"

namespace mhd
{
// Kernel classes of the step, timed with CUDA events on the handle's stream when profiling is on.
enum StepKernel { KP_PREPARE = 0, KP_CFL, KP_GRAD, KP_FLUX, KP_UPDATE, KP_FACE_CAND, KP_EDGE_EMF, KP_CT, KP_GYRATE, KP_COUNT };
static const char *const kStepKernelNames[KP_COUNT] = {"prepare", "cfl",            "limited_gradients", "face_flux", "update",
                                                        "face_candidate", "edge_emf", "ct",                "gyrate"};

using Profiler = EventProfiler<KP_COUNT>;

// Single-precision tables of the mixed path, derived once from the FP64 mesh (tetrahedral meshes):
// structure of arrays over cells / faces / edges so that every warp load is coalesced.
struct MixedTables
{
    DBuf<float> K;              // stencil: dl_j = sum_k K_jk (w_k - w_c), K_jk = dx_j^T I wd_k, [16][nc]
    DBuf<float> recon;          // cell field from face fluxes: B_c = sum_j recon[j] Phi_{f_j}, [12][nc]
    DBuf<float4> fn;            // per face: canonical unit normal, |A|
    DBuf<float> fdx;            // per face: x_f - x_L (3), x_f - x_R (3): [6][nf]
    DBuf<char2> fslot;          // per face: its position in the c2f rows of L and R
    DBuf<int4> fe;              // per (triangular) face: its 3 edges, negative-sign bits 0-2 and active bit 3
    DBuf<float4> eth;           // per edge: unit tangent, length
    DBuf<int8_t> emode;         // per edge: 0 UCT, 1 zero (wall edge, not owned, no fluid cell, no face), 2 inflow
    // per e2f entry, in the orthonormal basis (e1, e2) of the plane normal to the edge that edge_basis builds
    // from the single-precision tangent: the in-face unit direction m away from the edge and the face's unit
    // normal n, (m.e1, m.e2, n.e1, n.e2); and (sigma = t.(m x n), w_ef)
    DBuf<float4> emn;
    DBuf<float2> esw;
    DBuf<float> vol_inv;        // per cell: 1 / V
};
} // namespace mhd

struct MhdState
{
    MhdMesh *mesh = nullptr;
    MhdStepParams prm{};
    mhd::FluidParams fp{};
    int nsp = 0, group = 0;
    bool mixed = false;
    mhd::DBuf<double> U0, U1, W, grad, F, phi0, phi1, phi_add, badd, bind, btot, up, Ef, E, mass, stage;
    mhd::SrcParams src;     // two-ion J x B force and gyration (off unless params.lorentz)
    mhd::DBuf<double> J;    // cell current of the induced field (3 per cell) when the J x B force is on
    mhd::DBuf<double> dpe;  // grad p_e (3 per cell) when the ambipolar terms are on
    mhd::DBuf<double> pn;   // nodal p_e of the ambipolar EMF
    mhd::DBuf<int8_t> pok;  // the node has fluid cells
    mhd::DBuf<double> photo, vst; // source fields of the chemistry terms (empty: absent)
    mhd::DBuf<double> ne_eff, E_impl; // semi-implicit step: n_e,eff per cell, the implicit EMF per edge
    mhd::DBuf<int8_t> dir_inflow;     // semi-implicit step: the Dirichlet (inflow) edges of the solve
    mhd::DBuf<float4> g32;  // mixed precision: face terms A_f x b_f of the cell current (per face)
    mhd::DBuf<float4> d32;  // mixed precision: face terms (p_R - p_L) A_f / 2 of grad p_e (per face)
    mhd::DBuf<int32_t> wall_slot; // the caller's Dirichlet wall states: slot per face (-1: ghost_state)
    mhd::DBuf<double> wall_prim;  // [species][slot][5]
    mhd::DBuf<double> mres; // explicit resistive EMF: m_e = eta_e / star1_e per edge (empty: off)
    int8_t *floor_flags = nullptr; // when set, the update records the floors it applied ([s*nc + c])
    uint32_t *sw_edge = nullptr;   // switch log of the edge EMF (null: off), with fp.sw_lim, sw_flux, sw_floor
    uint32_t *sw_face = nullptr;   // switch log of the face EMF candidates' a_f (null: off)
    mhd::DBuf<double> efgeo;       // FP64 state: the UCT's per-(edge, slot) face geometry (build_edge_face_geo), or empty
    mhd::DBuf<double> pa;          // with efgeo: the stage's phi_ind / |A| per face, left by the face-candidate pass
    mhd::DBuf<double> scal; // [0] dt
    mhd::DBuf<unsigned long long> dt_bits;
    mhd::DBuf<int> flag;
    // mixed precision: FP32 bulk arrays (the state U and the face fluxes Phi stay FP64)
    mhd::MixedTables mt;
    mhd::DBuf<float> W32, grad32, F32, E32;
    mhd::DBuf<float4> Ef32; // per face: EMF candidate E_f (3) and Phi_ind / |A|
    mhd::DBuf<float4> up32, bt32, bi32, badd32;
    double *pinned = nullptr;
    int64_t launches = 0; // kernels launched by the step since creation
    mhd::Profiler prof;
    ~MhdState()
    {
        if (pinned) cudaFreeHost(pinned);
    }
};

namespace mhd
{
void mixed_setup(MhdState *st);
// one FP64 stage (Us, phis) -> (Uo, phio) at the step size in st->scal[0]; stage2 averages with Uo, phio in place
void fp64_stage(MhdState *st, const double *Us, const double *phis, double *Uo, double *phio, bool stage2);
// its first half alone: primitives, cell fields, u+ and limited gradients of (Us, phis) into st's buffers
void fp64_prepare_grad(MhdState *st, const double *Us, const double *phis);
// gyrate_close: stage 2 applies the closing half-step gyration in its update (two-ion sources on)
void mixed_stage(MhdState *st, const double *Us, const double *phis, double *Uo, double *phio, bool stage2, bool cfl, double dt_max,
                 bool prepared = false, bool gyrate_close = false);
// the opening half-step gyration of U0, renewing its primitives and u+ (stage 1 then runs prepared)
void mixed_gyrate_open(MhdState *st);
void mixed_badd(MhdState *st);
// primitives, cell fields (and with cfl the device CFL step) of (Us, phis) in mixed precision
void mixed_prepare(MhdState *st, const double *Us, const double *phis, bool cfl, double dt_max);
} // namespace mhd
