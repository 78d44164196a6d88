// The FP32 operator of the mixed-precision induction solve (the Arnoldi matvecs of
// mhd_gpu_induction_solve with MHD_PREC_MIXED): d1 of the preconditioned Krylov vector, the cell field,
// the Hall EMF and the edge gather, in single precision with multiply-add contraction (no
// reference-exactness to keep: every restart's true residual is recomputed with the FP64 operator).
#include "induction_op.cuh"

namespace mhd
{
// the same Arnoldi matvec with the FP32 operator (mixed precision inner iterations)
void op32(MhdInduction *I, const MatIn &in, double dt, double *y, const Fused &fz)
{
    const MeshView &m = I->mesh->v;
    cudaStream_t s = I->mesh->stream;
    if (m.nf)
        IND_LAUNCH(I, KI_FACE, s, (m.tri_faces ? k_ind_face<float, true> : k_ind_face<float, false>)<<<g1(m.nf), 256, 0, s>>>(
                                      m, fz.gt, in, I->hall, I->resistive, I->phi32.p, I->s2phi32.p));
    if (I->hall && m.nc)
    {
        IND_LAUNCH(I, KI_BCELL, s, (m.faces_per_cell == 4 ? k_ind_bcell<float, true> : k_ind_bcell<float, false>)<<<g1(m.nc), 256, 0, s>>>(
                                       m, fz.gt, I->recon32.p, I->phi32.p, I->b32.p));
        if (m.no_cells)
            IND_LAUNCH(I, KI_HALL, s,
                       (m.faces_per_cell == 4 ? k_ind_hall32<true> : k_ind_hall32<false>)<<<g1(m.no_cells), 256, 0, s>>>(m, fz.gt, I->slot32.p, I->b32.p, I->alpha32.p, I->B0_32.p, I->vinv32.p,
                                                                   I->g32.p));
    }
    EdgeArgs<float> a;
    a.resistive = I->resistive; a.hall = I->hall;
    a.s2phi = I->s2phi32.p; a.g = I->g32.p; a.mcoef = I->m32.p; a.ecw = I->ecw32.p; a.tvec = I->tv32.p;
    a.in = in; a.dt = dt; a.dtp = fz.dtp; a.vout = fz.vout; a.dir = fz.dir; a.v0 = fz.v0; a.dot = fz.dot; a.gt = fz.gt;
    a.part = I->part.p; a.counter = I->counter.p; a.out = y;
    if (m.ne) IND_LAUNCH(I, KI_EDGE, s, (m.max_valence <= 8 && m.max_edge_cells <= 8 ? k_ind_edge<float, 8> : k_ind_edge<float, 0>)<<<I->edge_blocks, 256, 0, s>>>(m, a));
}

} // namespace mhd
