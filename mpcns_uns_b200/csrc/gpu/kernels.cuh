// Host-side launchers of the hot-path kernels, shared between the translation units that
// define the kernels and the fused step.
#pragma once
#include "sources.cuh"

namespace mhd
{
// gmres.cu: the mesh an induction handle was made on
MhdMesh *induction_mesh(const MhdInduction *I);

// fluid.cu
void launch_limited_gradients(const MeshView &m, const FluidParams &p, SField<const double> W, SField<double> G, cudaStream_t s);
void launch_face_flux(const MeshView &m, const FluidParams &p, SField<const double> W, SField<const double> G, double *F, cudaStream_t s);

// induction.cu
// pa (optional): phi_tot / |A| per face for the table-driven edge pass; sw (optional): switch log of a_f
void launch_face_candidate(const MeshView &m, const double *u, const double *Bt, const double *Bi, const double *phi_tot,
                           const double *phi_add, double *Ef, cudaStream_t s, double *pa = nullptr, uint32_t *sw = nullptr);
// E = begin (0) + ideal UCT EMF of the owned edges, then the boundary edge values (wall 0, inflow E_inf . t);
// mres (per edge, optional): plus the explicit resistive EMF m_e (d1^T star2 phi_ind)_e on the owned edges;
// amb.on: minus the ambipolar EMF on the owned free edges; sw (per edge, optional): the switch log of the
// upwind choices (per face of the edge the cell of the largest |u . m| and its sign, the 2x2 solve's branch)
// geo, pa (optional, together): the per-(edge, slot) geometry table of build_edge_face_geo and the faces'
// phi_ind / |A| of launch_face_candidate; with them the UCT value of edges of at most 8 faces and 8 cells
// comes from the table (same bits, fewer registers, operations and gathers)
void launch_edge_emf_assign(const MeshView &m, const double *Ef, const double *u, const double *phi_ind, double cuct, V3 E_inf,
                            double *E, cudaStream_t s, const double *mres = nullptr, const AmbArgs &amb = AmbArgs{},
                            uint32_t *sw = nullptr, const double *geo = nullptr, const double *pa = nullptr);
void build_edge_face_geo(const MeshView &m, double *geo, cudaStream_t s);
} // namespace mhd
