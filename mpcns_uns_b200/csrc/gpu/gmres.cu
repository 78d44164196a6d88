// nvcc-flags: -fmad=false
// Semi-implicit Hall / resistive induction on the device: the operator of mhd::ImplicitInduction
// and its restarted GMRES (Common/induction/ImplicitInduction.cpp).
//
// The operator's scatters become gathers whose summation order equals the reference's: the
// resistive current flux reaches an edge from its faces in ascending face order (e2f rows), the Hall
// EMF from its cells in ascending cell order (ec rows, the reference's ce lists); the FP64 operator
// is therefore reference-exact.  The Krylov part keeps H, g and the Givens rotations on the device;
// the host reads one value per Arnoldi step (the early-exit test) and one per restart (the true
// residual).  Its dot products are deterministic block reductions, whose rounding differs from the
// reference's sequential sums, so GMRES iterates agree to the solver tolerance, not bit for bit.
//
// Fusions of the Arnoldi step (each keeps the reference's arithmetic per element):
//   * the Jacobi preconditioner z = dir ? 0 : V_j / (1 + dt m d2) is applied while gathering z in d1
//     (with the block ILU(0) preconditioner on, z = M^-1 V_j comes from the triangular solves of ilu.cu,
//     which store V_j, and the matvec gathers z itself);
//   * V_j = w / H(j, j-1) is formed lazily in the next matvec (the face pass gathers w / h, the edge
//     pass stores V_j), so w is not re-read to normalise it;
//   * the edge pass zeroes the Dirichlet rows of w and produces H(0, j) = w . V_0;
//   * the orthogonalisation is classical Gram-Schmidt with a conditional second pass (gram_schmidt.cu) for
//     restarts up to 31; beyond, each modified Gram-Schmidt subtraction w -= H(i-1, j) V_{i-1} is fused
//     with the next dot w . V_i, consecutive passes sweeping the edges in opposite directions so that the
//     tail of w and V_{i-1} left in L2 is reused first;
//   * every dot finishes in the kernel that produces it (the last block adds the block partials), and
//     a restart cycle runs as one CUDA graph whose steps test a device-side flag, so the host waits
//     once per restart instead of once per Arnoldi step.
#include <array>
#include <utility>

#include "induction_op.cuh"

namespace mhd
{
namespace
{
// ---------------------------------------------------------------- one-time tables
// cell-field coefficients of the constructor (:34-62): B_c = sum_k recon_k Phi_{f_k}
__global__ void k_ind_recon(MeshView m, double *recon)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int32_t k = m.c2f_ptr[c]; k < m.c2f_ptr[c + 1]; ++k)
    {
        const int32_t f = m.c2f_idx[k];
        const double A = m.face_area_mag[f];
        for (int i = 0; i < 3; ++i) recon[3 * (int64_t)k + i] = 0.0;
        if (A <= 0) continue;
        const V3 n = (1.0 / A) * ld3(m.face_area, f);
        const double nv[3] = {n.x, n.y, n.z};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) M[i][j] += A * nv[i] * nv[j];
    }
    const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                       M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    const double sc = dmax(dmax(dmax(M[0][0], M[1][1]), M[2][2]), 1e-300);
    if (fabs(det) < 1e-12 * sc * sc * sc) return;
    double I[3][3];
    I[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det; I[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
    I[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det; I[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) / det;
    I[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det; I[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
    I[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) / det; I[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) / det;
    I[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
    for (int32_t k = m.c2f_ptr[c]; k < m.c2f_ptr[c + 1]; ++k)
    {
        const int32_t f = m.c2f_idx[k];
        const double A = m.face_area_mag[f];
        if (A <= 0) continue;
        const V3 n = (1.0 / A) * ld3(m.face_area, f);
        for (int i = 0; i < 3; ++i) recon[3 * (int64_t)k + i] = I[i][0] * n.x + I[i][1] * n.y + I[i][2] * n.z;
    }
}

// d2_e = sum of star2 over the faces of e, ascending face order (:87-89)
__global__ void k_ind_d2(MeshView m, double *d2)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    double s = 0.0;
    for (int32_t k = m.e2f_ptr[e]; k < m.e2f_ptr[e + 1]; ++k) s += m.star2[m.e2f_idx[k]];
    d2[e] = s;
}

// set_frozen_state (:105-111)
__global__ void k_ind_alpha(int32_t nc, const double *taper, const double *ne_eff, int hall, double hall_coef, double *alpha)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    alpha[c] = (hall && ne_eff[c] > 0) ? taper[c] * hall_coef / ne_eff[c] : 0.0;
}

// FP32 copies of the operator's tables (mixed precision)
__global__ void k_ind_tables32(MeshView m, const double *recon, const double *mcoef, float *recon32, float *m32, float *ecw32,
                               float *tv32, float *vinv32)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < 3 * (int64_t)m.c2f_ptr[m.nc]) recon32[i] = static_cast<float>(recon[i]);
    if (i < m.ec_ptr[m.ne]) ecw32[i] = static_cast<float>(m.ec_weight[i]);
    if (i < m.ne)
    {
        m32[i] = static_cast<float>(mcoef[i]);
        for (int a = 0; a < 3; ++a) tv32[3 * i + a] = static_cast<float>(m.edge_vec[3 * i + a]);
    }
    if (i < m.nc) vinv32[i] = static_cast<float>(1.0 / m.cell_volume[i]);
}

// Per c2f slot of a cell: the cell across the face (-1 if the face has one cell) and the signed area
// vector s A_f, so that the Hall pass reads its cell's slots contiguously instead of chasing f2c.
__global__ void k_ind_slots(MeshView m, int32_t *slot_nb, double *slot_sa, float4 *slot32)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    for (int32_t k = m.c2f_ptr[c]; k < m.c2f_ptr[c + 1]; ++k)
    {
        const int32_t f = m.c2f_idx[k];
        const int32_t p0 = m.f2c_ptr[f];
        int32_t o = -1;
        if (m.f2c_ptr[f + 1] - p0 == 2) o = m.f2c_idx[p0] == c ? m.f2c_idx[p0 + 1] : m.f2c_idx[p0];
        const V3 sa = double(m.c2f_sgn[k]) * ld3(m.face_area, f);
        slot_nb[k] = o;
        st3(slot_sa, k, sa);
        if (slot32)
            slot32[k] = make_float4(static_cast<float>(sa.x), static_cast<float>(sa.y), static_cast<float>(sa.z), __int_as_float(o));
    }
}

__global__ void k_to_float(const double *a, float *b, int64_t n)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = static_cast<float>(a[i]);
}

__global__ void k_ind_s2phi(MeshView m, const double *__restrict__ phi, double *__restrict__ s2phi)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < m.nf) s2phi[f] = m.star2[f] * phi[f];
}

// Hall EMF per owned cell (:159-178): J_c = (1/V) sum s A x 1/2 (b_c + b_nb), g_c = alpha_c J_c x B0_c.
// g_c = 0 where the reference skips the cell (alpha = 0, or not fluid: its ce list is empty), so that
// the edge gather may add every owned cell: adding the zero product leaves each sum unchanged.
template <bool TET>
__global__ void k_ind_hall(MeshView m, Gate gt, const int32_t *__restrict__ slot_nb, const double *__restrict__ slot_sa,
                           const double *__restrict__ b, const double *__restrict__ alpha, const double *__restrict__ B0,
                           double *__restrict__ g)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.no_cells || gt.off()) return;
    if (alpha[c] == 0.0 || m.material[c] != 0)
    {
        st3(g, c, mk(0, 0, 0));
        return;
    }
    V3 sum = mk(0, 0, 0);
    const V3 bc = ld3(b, c);
    const int32_t kb = TET ? 4 * c : m.c2f_ptr[c], ke = TET ? 4 * c + 4 : m.c2f_ptr[c + 1];
#pragma unroll 4
    for (int32_t k = kb; k < ke; ++k)
    {
        const int32_t o = slot_nb[k];
        V3 bf = bc;
        if (o >= 0) bf = 0.5 * (bc + ld3(b, o));
        sum = sum + cross(ld3(slot_sa, k), bf);
    }
    const V3 J = (1.0 / m.cell_volume[c]) * sum;
    st3(g, c, alpha[c] * cross(J, ld3(B0, c)));
}

// ---------------------------------------------------------------- Krylov vectors (FP64)
// a . b over the owned edges -> op(sum) in *out
__global__ void __launch_bounds__(256) k_dot(const double *__restrict__ a, const double *__restrict__ b, int32_t n, double *part,
                                             unsigned *counter, int op, double *out)
{
    double s = 0.0;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * b[i];
    grid_sum_tail(s, part, counter, op, out);
}

// Modified Gram-Schmidt step fused with the next dot (:340-345): w -= (*h) Vprev on all edges, then
// *out = w . Vi over the owned edges (Vi null: |w|).  `reverse` sweeps from the last edge so that what
// the previous pass left in L2 is read first.
__global__ void __launch_bounds__(256) k_mgs(Gate gt, double *__restrict__ w, const double *__restrict__ Vprev,
                                              const double *__restrict__ h, const double *__restrict__ Vi, int32_t n_all,
                                              int32_t n_owned, int reverse, double *part, unsigned *counter, double *out,
                                              const double *__restrict__ pd, double *__restrict__ zs, float *__restrict__ zs32)
{
    if (gt.off()) return;
    constexpr int U = 4;
    const double hv = *h;
    const int32_t stride = gridDim.x * blockDim.x;
    double s = 0.0;
    for (int32_t t0 = blockIdx.x * blockDim.x + threadIdx.x; t0 < n_all; t0 += U * stride)
    {
        int32_t idx[U];
        double wv[U], pv[U], iv[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int32_t t = t0 + u * stride;
            idx[u] = t < n_all ? (reverse ? n_all - 1 - t : t) : -1;
            if (idx[u] >= 0)
            {
                wv[u] = w[idx[u]];
                pv[u] = Vprev[idx[u]];
                iv[u] = Vi ? Vi[idx[u]] : 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            if (idx[u] < 0) continue;
            const double wi = wv[u] - hv * pv[u];
            w[idx[u]] = wi;
            if (idx[u] < n_owned) s += wi * (Vi ? iv[u] : wi);
            if (zs) zs[idx[u]] = wi * pd[idx[u]];
            if (zs32) zs32[idx[u]] = static_cast<float>(wi * pd[idx[u]]);
        }
    }
    grid_sum_tail(s, part, counter, Vi ? 0 : 1, out);
}


__global__ void k_vec_x0(int32_t n, const double *Ee, const double *corr, const int8_t *dir, double *x0, double *delta)
{
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x0[i] = (corr && !dir[i]) ? Ee[i] + corr[i] : Ee[i];
    delta[i] = 0.0;
}
__global__ void k_vec_add(int32_t n, const double *a, const double *b, double *c)
{
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) c[i] = a[i] + b[i];
}
// r = dir ? 0 : b - Ax
__global__ void k_vec_resid(int32_t n, const double *b, const double *Ax, const int8_t *dir, double *r)
{
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = dir[i] ? 0.0 : b[i] - Ax[i];
}
// pd = dir ? 0 : 1 / (1 + dt m d2), dt_e in place of dt when given (Jacobi, :315-316); dirc = the caller's
// Dirichlet flags, kept for the cycle
__global__ void k_vec_pd(int32_t n, double dt, const double *dte, const double *mc, const double *d2, const int8_t *dir, double *pd,
                         int8_t *dirc)
{
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pd[i] = dir[i] ? 0.0 : 1.0 / (1.0 + (dte ? dte[i] : dt) * mc[i] * d2[i]);
    dirc[i] = dir[i];
}
// V0 = r / beta, and the face pass's input V0 * pd
__global__ void k_vec_v0(int32_t n, const double *r, const double *beta, double *V0, const double *pd, double *zs, float *zs32)
{
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = r[i] / *beta;
    V0[i] = v;
    if (zs) zs[i] = v * pd[i];
    if (zs32) zs32[i] = static_cast<float>(v * pd[i]);
}

// start of a restart cycle: g = (beta, 0, ...), at most `limit` Arnoldi steps, early exit at |g_{j+1}| <= tol
__global__ void k_cycle_init(Ctl *ctl, int limit, double tol, double dt, double *g, int n, const double *beta)
{
    ctl->done = 0;
    ctl->jend = 0;
    ctl->limit = limit;
    ctl->reorth = 0;
    ctl->n_reorth = 0;
    ctl->tol = tol;
    ctl->dt = dt;
    for (int i = 0; i < n; ++i) g[i] = 0.0;
    g[0] = *beta;
}

// Givens rotations of column j and the residual estimate (:337-347); single thread.
// H is (m+1) x m row-major; nrm[j+1] keeps H(j+1, j) before the rotation (the divisor of V_{j+1}).
__global__ void k_givens(Ctl *ctl, double *H, int mcols, int j, double *cs, double *sn, double *g, double *nrm)
{
    if (ctl->done || j >= ctl->limit) return;
    auto h = [&](int r, int c) -> double & { return H[r * mcols + c]; };
    nrm[j + 1] = h(j + 1, j);
    for (int i = 0; i < j; ++i)
    {
        const double t = cs[i] * h(i, j) + sn[i] * h(i + 1, j);
        h(i + 1, j) = -sn[i] * h(i, j) + cs[i] * h(i + 1, j);
        h(i, j) = t;
    }
    const double den = hypot(h(j, j), h(j + 1, j));
    cs[j] = den > 0 ? h(j, j) / den : 1.0;
    sn[j] = den > 0 ? h(j + 1, j) / den : 0.0;
    h(j, j) = den;
    h(j + 1, j) = 0.0;
    g[j + 1] = -sn[j] * g[j];
    g[j] = cs[j] * g[j];
    ctl->jend = j + 1;
    if (fabs(g[j + 1]) <= ctl->tol) ctl->done = 1;
}

// back substitution of the least-squares problem (:349-354) over the jend steps of the cycle; single thread
__global__ void k_backsub(const Ctl *ctl, const double *H, int mcols, const double *g, double *y, double *jend_out)
{
    const int j = ctl->jend;
    for (int i = j - 1; i >= 0; --i)
    {
        double s = g[i];
        for (int k = i + 1; k < j; ++k) s -= H[i * mcols + k] * y[k];
        y[i] = s / H[i * mcols + i];
    }
    jend_out[0] = j;
    jend_out[1] = ctl->n_reorth;
}

// delta += dir ? 0 : (sum_i y_i V_i) / (1 + dt m d2)  (:355-364); z = x0 + delta for the true residual
__global__ void k_vec_update(const Ctl *ctl, int32_t n, const double *V, const double *y, const double *pd, const int8_t *dir,
                             const double *x0, double *delta, double *z)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int j = ctl->jend;
    double s = 0.0;
    for (int i = 0; i < j; ++i) s += y[i] * V[(int64_t)i * n + e];
    const double d = delta[e] + (dir[e] ? 0.0 : s * pd[e]);
    delta[e] = d;
    z[e] = x0[e] + d;
}

// comb = sum_i y_i V_i (:357-362), the input of the ILU(0) correction
__global__ void k_vec_comb(const Ctl *ctl, int32_t n, const double *V, const double *y, double *comb)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int j = ctl->jend;
    double s = 0.0;
    for (int i = 0; i < j; ++i) s += y[i] * V[(int64_t)i * n + e];
    comb[e] = s;
}

// delta += M^-1 comb (:374); z = x0 + delta for the true residual
__global__ void k_vec_addz(int32_t n, const double *pz, const double *x0, double *delta, double *z)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const double d = delta[e] + pz[e];
    delta[e] = d;
    z[e] = x0[e] + d;
}

// E = x0 + delta, corr = dir ? 0 : E - E_expl (:379-381)
__global__ void k_vec_final(int32_t n, const double *x0, const double *delta, const double *Ee, const int8_t *dir, double *E, double *corr)
{
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = x0[i] + delta[i];
    E[i] = v;
    corr[i] = dir[i] ? 0.0 : v - Ee[i];
}
} // namespace
} // namespace mhd

using namespace mhd;

namespace mhd
{
namespace
{
// y = F(phi) (no input in `in`, phi given) or y = A x; optional fused outputs as in EdgeArgs.  only_ideal: the
// ideal part alone (ImplicitInduction::ideal_linear, :118-124).
void op64(MhdInduction *I, const MatIn &in, const double *phi_in, double dt, double *y, const Fused &fz = Fused{}, bool only_ideal = false)
{
    const MeshView &m = I->mesh->v;
    cudaStream_t s = I->mesh->stream;
    const bool resistive = I->resistive && !only_ideal, hall = I->hall && !only_ideal, ideal = I->ideal;
    const double *phi = phi_in;
    if (in.x || in.src)
    {
        if (m.nf)
            IND_LAUNCH(I, KI_FACE, s, (m.tri_faces ? k_ind_face<double, true> : k_ind_face<double, false>)<<<g1(m.nf), 256, 0, s>>>(
                                          m, fz.gt, in, hall || ideal, resistive, I->phi.p, I->s2phi.p));
        phi = I->phi.p;
    }
    else if (resistive && m.nf)
        IND_LAUNCH(I, KI_FACE, s, k_ind_s2phi<<<g1(m.nf), 256, 0, s>>>(m, phi, I->s2phi.p));
    // the cell field from the face fluxes (:138-149), for the Hall and the ideal parts
    if ((hall || ideal) && m.nc)
        IND_LAUNCH(I, KI_BCELL, s, (m.faces_per_cell == 4 ? k_ind_bcell<double, true> : k_ind_bcell<double, false>)<<<g1(m.nc), 256, 0, s>>>(
                                       m, fz.gt, I->recon.p, phi, I->bcell.p));
    // the ideal EMF of the frozen velocities and the cell field of phi (:150-158); masked in the edge pass
    if (ideal && m.ne)
    {
        IND_LAUNCH(I, KI_IDEAL, s, MHD_CUDA(cudaMemsetAsync(I->ide.p, 0, (size_t)m.ne * sizeof(double), s)));
        IND_LAUNCH(I, KI_IDEAL, s,
                   ideal_emf_enqueue(m, I->u_ideal.p, I->bcell.p, I->bcell.p, phi, phi, I->cuct, I->face3.p, I->ide.p, s));
        if (m.no_edges) ++I->launches; // the enqueue is two kernels
    }
    if (hall && m.nc && m.no_cells)
        IND_LAUNCH(I, KI_HALL, s,
                   (m.faces_per_cell == 4 ? k_ind_hall<true> : k_ind_hall<false>)<<<g1(m.no_cells), 256, 0, s>>>(m, fz.gt, I->slot_nb.p, I->slot_sa.p, I->bcell.p, I->alpha.p, I->B0.p,
                                                                 I->g.p));
    EdgeArgs<double> a;
    a.resistive = resistive; a.hall = hall;
    if (ideal)
    {
        a.ide = I->ide.p;
        a.imask = I->imask.p;
    }
    a.s2phi = I->s2phi.p; a.g = I->g.p; a.mcoef = I->mcoef.p; a.ecw = m.ec_weight; a.tvec = m.edge_vec;
    a.in = in; a.dt = dt; a.dtp = fz.dtp; a.vout = fz.vout; a.dir = fz.dir; a.v0 = fz.v0; a.dot = fz.dot; a.gt = fz.gt;
    a.part = I->part.p; a.counter = I->counter.p; a.out = y;
    if (m.ne) IND_LAUNCH(I, KI_EDGE, s, (m.max_valence <= 8 && m.max_edge_cells <= 8 ? k_ind_edge<double, 8> : k_ind_edge<double, 0>)<<<I->edge_blocks, 256, 0, s>>>(m, a));
}

void apply_plain(MhdInduction *I, const double *x, double dt, double *y, const double *dte = nullptr)
{
    MatIn in;
    in.x = x;
    in.dte = dte;
    op64(I, in, nullptr, dt, y);
}

// dot over the owned edges into *out (op as grid_sum_tail)
void dev_dot(MhdInduction *I, const double *a, const double *b, int op, double *out)
{
    cudaStream_t s = I->mesh->stream;
    IND_LAUNCH(I, KI_VECTOR, s, k_dot<<<kRedBlocks, 256, 0, s>>>(a, b, I->mesh->v.no_edges, I->part.p, I->counter.p, op, out));
}

// The mr Arnoldi steps of one restart cycle (:333-348), each gated by the cycle control:
// w = A P^-1 V_j with V_j = w_prev / H(j, j-1) formed on the fly, Dirichlet rows zeroed and H(0, j) = w . V_0;
// modified Gram-Schmidt w -= H(i-1, j) V_{i-1} fused with H(i, j) = w . V_i; Givens and the early-exit test.
void enqueue_cycle(MhdInduction *I)
{
    const MeshView &m = I->mesh->v;
    cudaStream_t s = I->mesh->stream;
    const int32_t ne = m.ne;
    const int mr = I->p.restart;
    double *V = I->V.p, *H = I->H.p;
    for (int j = 0; j < mr; ++j)
    {
        Gate gt;
        gt.ctl = I->ctl.p;
        gt.j = j;
        MatIn in;
        const bool ilu = I->mode == 2;
        in.dte = I->mode == 1 ? I->dte.p : nullptr;
        if (ilu)
        {
            // z = M^-1 V_j (:337) by the two triangular solves, V_j = w / H(j, j-1) stored on the way
            ilu_apply(I, gt, j == 0 ? V : I->w.p, j == 0 ? nullptr : I->nrm.p + j, I->dirc.p, j == 0 ? nullptr : V + (int64_t)j * ne);
            in.x = I->ilu.z.p;
        }
        else
        {
            in.src = j == 0 ? V : I->w.p;
            in.hs = j == 0 ? nullptr : I->nrm.p + j;
            in.pd = I->pd.p;
            if (I->mixed) in.zs32 = I->zs32.p;
            else in.zs = I->zs.p;
        }
        Fused fz;
        fz.vout = j == 0 || ilu ? nullptr : V + (int64_t)j * ne;
        fz.dir = I->dirc.p;
        const bool cgs = mr <= kCgsMax;
        fz.v0 = cgs ? nullptr : V;
        fz.dot = cgs ? nullptr : H + j;
        fz.dtp = &I->ctl.p->dt;
        fz.gt = gt;
        // the FP32 operator has no ideal part: the mixed solve uses the FP64 operator while it is on
        if (I->mixed && !I->ideal) op32(I, in, 0.0, I->w.p, fz);
        else op64(I, in, nullptr, 0.0, I->w.p, fz);
        if (cgs)
        {
            CgsArgs ca{gt, I->ctl.p, I->w.p, V, ne, ne, m.no_edges, I->part.p, I->red.p, H, I->counter.p, mr, I->pd.p,
                       I->mixed ? nullptr : I->zs.p, I->mixed ? I->zs32.p : nullptr};
            for (int pass = 0; pass < 3; ++pass) IND_LAUNCH(I, KI_MGS, s, cgs_launch(j, ca, I->cgs_grid + 2 * j, s, pass));
            IND_LAUNCH(I, KI_SCALAR, s, k_givens<<<1, 1, 0, s>>>(I->ctl.p, H, mr, j, I->cs.p, I->sn.p, I->gv.p, I->nrm.p));
            continue;
        }
        for (int i = 1; i <= j + 1; ++i)
        {
            const bool last = i == j + 1; // the norm of w, and the next face pass's input w * pd
            const double *Vi = last ? nullptr : V + (int64_t)i * ne;
            IND_LAUNCH(I, KI_MGS, s,
                       k_mgs<<<kRedBlocks, 256, 0, s>>>(gt, I->w.p, V + (int64_t)(i - 1) * ne, H + (int64_t)(i - 1) * mr + j, Vi, ne,
                                                        m.no_edges, i & 1, I->part.p, I->counter.p, H + (int64_t)i * mr + j, I->pd.p,
                                                        last && !I->mixed ? I->zs.p : nullptr, last && I->mixed ? I->zs32.p : nullptr));
        }
        IND_LAUNCH(I, KI_SCALAR, s, k_givens<<<1, 1, 0, s>>>(I->ctl.p, H, mr, j, I->cs.p, I->sn.p, I->gv.p, I->nrm.p));
    }
}

// Capture the cycle once as a CUDA graph; a stream that cannot be captured keeps direct launches.
void build_cycle_graph(MhdInduction *I)
{
    const int md = I->mode;
    I->cycle_tried[md] = true;
    cudaStream_t s = I->mesh->stream;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    {
        cudaGetLastError();
        return;
    }
    const int64_t l0 = I->launches;
    I->capturing = true;
    enqueue_cycle(I);
    I->capturing = false;
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    I->cycle_kernels[md] = I->launches - l0;
    I->launches = l0;
    if (ce != cudaSuccess || !graph)
    {
        cudaGetLastError();
        if (graph) cudaGraphDestroy(graph);
        return;
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess)
    {
        cudaGetLastError();
        return;
    }
    I->cycle[md] = exec;
}

void host_read(MhdInduction *I, const double *dev, int n)
{
    cudaStream_t s = I->mesh->stream;
    MHD_CUDA(cudaMemcpyAsync(I->pinned, dev, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    MHD_CUDA(cudaStreamSynchronize(s));
}
// ImplicitInduction::solve (:299-390); dte != null: the per-edge pseudo-time step (A x = x + F(d1 diag(dt_e) x),
// Jacobi 1 / (1 + dt_e m d2), no ILU(0)), dt unused.
int solve_impl(MhdInduction *I, const double *Phi, const double *Ee, const int8_t *dir, double dt, const double *dte_in, int32_t warm,
               double *E, int32_t *iterations, double *rel_res)
{
    int status = MHD_OK;
    int rc = guarded([&] {
        MHD_REQUIRE(I && MHD_ARR(Phi, I->mesh->v.nf) && MHD_ARR(Ee, I->mesh->v.ne) && MHD_ARR(dir, I->mesh->v.ne) &&
                        MHD_ARR(E, I->mesh->v.ne),
                    "null argument");
        const MeshView &m = I->mesh->v;
        cudaStream_t s = I->mesh->stream;
        const int32_t ne = m.ne;
        if (iterations) *iterations = 0;
        if (rel_res) *rel_res = 0.0;
        if (ne == 0) return;
        const int mr = I->p.restart;
        const int ge = g1(ne);
        const double *dte = nullptr;
        if (dte_in)
        {
            I->dte.alloc(ne);
            MHD_CUDA(cudaMemcpyAsync(I->dte.p, dte_in, (size_t)ne * sizeof(double), cudaMemcpyDeviceToDevice, s));
            dte = I->dte.p;
        }
        // the ILU(0) is built for a scalar dt (:317) and only without the ideal part (:102)
        I->mode = dte ? 1 : (I->ilu.on && !I->ideal ? 2 : 0);
        const double dtA = dte ? 1.0 : dt; // A x = x + dtA F(d1 [diag(dt_e)] x): d1 carries dt_e (:196)
        if (!warm) I->have_corr = false;
        I->last_reorth = 0;
        double *sc = I->scal.p; // [0] |b|  [1] beta  [2] steps of the last cycle
        IND_LAUNCH(I, KI_VECTOR, s, k_vec_x0<<<ge, 256, 0, s>>>(ne, Ee, I->have_corr ? I->corr.p : nullptr, dir, I->x0.p, I->delta.p));
        op64(I, MatIn{}, Phi, 0.0, I->Fn.p);                                                      // F(Phi^n)
        IND_LAUNCH(I, KI_VECTOR, s, k_vec_add<<<ge, 256, 0, s>>>(ne, Ee, I->Fn.p, I->b.p));     // b = E_expl + F(Phi^n)
        apply_plain(I, I->x0.p, dtA, I->Ax.p, dte);                                               // A x0
        IND_LAUNCH(I, KI_VECTOR, s, k_vec_resid<<<ge, 256, 0, s>>>(ne, I->b.p, I->Ax.p, dir, I->r.p));
        IND_LAUNCH(I, KI_VECTOR, s, k_vec_pd<<<ge, 256, 0, s>>>(ne, dt, dte, I->mcoef.p, I->d2.p, dir, I->pd.p, I->dirc.p));
        if (I->mode == 2) ilu_factor(I, dt, dir); // (:317-318)
        dev_dot(I, I->b.p, I->b.p, 2, sc + 0);
        dev_dot(I, I->r.p, I->r.p, 1, sc + 1);
        MHD_LAUNCH_CHECK();
        host_read(I, sc + 0, 2);
        const double bnorm = I->pinned[0];
        double beta = I->pinned[1];
        const double tol = I->p.rtol * bnorm;
        int total = 0;
        while (beta > tol && total < I->p.max_it)
        {
            IND_LAUNCH(I, KI_VECTOR, s,
                       k_vec_v0<<<ge, 256, 0, s>>>(ne, I->r.p, sc + 1, I->V.p, I->pd.p, I->mixed ? nullptr : I->zs.p,
                                                   I->mixed ? I->zs32.p : nullptr));
            IND_LAUNCH(I, KI_SCALAR, s,
                       k_cycle_init<<<1, 1, 0, s>>>(I->ctl.p, std::min(mr, I->p.max_it - total), tol, dtA, I->gv.p, mr + 1, sc + 1));
            if (!I->prof.on && !I->cycle_tried[I->mode]) build_cycle_graph(I);
            if (!I->prof.on && I->cycle[I->mode])
            {
                MHD_CUDA(cudaGraphLaunch(I->cycle[I->mode], s));
                I->launches += I->cycle_kernels[I->mode];
            }
            else
                enqueue_cycle(I);
            IND_LAUNCH(I, KI_SCALAR, s, k_backsub<<<1, 1, 0, s>>>(I->ctl.p, I->H.p, mr, I->gv.p, I->yv.p, sc + 2));
            if (I->mode == 2)
            {
                IND_LAUNCH(I, KI_VECTOR, s, k_vec_comb<<<ge, 256, 0, s>>>(I->ctl.p, ne, I->V.p, I->yv.p, I->w.p));
                ilu_apply(I, Gate{}, I->w.p, nullptr, dir, nullptr);
                IND_LAUNCH(I, KI_VECTOR, s, k_vec_addz<<<ge, 256, 0, s>>>(ne, I->ilu.z.p, I->x0.p, I->delta.p, I->z.p));
            }
            else
                IND_LAUNCH(I, KI_VECTOR, s,
                           k_vec_update<<<ge, 256, 0, s>>>(I->ctl.p, ne, I->V.p, I->yv.p, I->pd.p, dir, I->x0.p, I->delta.p, I->z.p));
            // true residual in FP64 (the outer iterative refinement of the mixed-precision solve)
            apply_plain(I, I->z.p, dtA, I->Ax.p, dte);
            IND_LAUNCH(I, KI_VECTOR, s, k_vec_resid<<<ge, 256, 0, s>>>(ne, I->b.p, I->Ax.p, dir, I->r.p));
            dev_dot(I, I->r.p, I->r.p, 1, sc + 1);
            MHD_LAUNCH_CHECK();
            host_read(I, sc + 1, 3);
            beta = I->pinned[0];
            total += static_cast<int>(I->pinned[1]);
            I->last_reorth += static_cast<int32_t>(I->pinned[2]);
        }
        IND_LAUNCH(I, KI_VECTOR, s, k_vec_final<<<ge, 256, 0, s>>>(ne, I->x0.p, I->delta.p, Ee, dir, E, I->corr.p));
        MHD_LAUNCH_CHECK();
        MHD_CUDA(cudaStreamSynchronize(s));
        if (I->mode == 2) ilu_check(I);
        I->have_corr = true;
        if (iterations) *iterations = total;
        if (rel_res) *rel_res = beta / bnorm;
        if (beta > tol) status = MHD_ENOCONV;
    });
    return rc != MHD_OK ? rc : status;
}

} // namespace

MhdMesh *induction_mesh(const MhdInduction *I) { return I->mesh; }

void drop_cycle_graphs(MhdInduction *I)
{
    MHD_CUDA(cudaStreamSynchronize(I->mesh->stream));
    for (int k = 0; k < 3; ++k)
    {
        if (I->cycle[k]) MHD_CUDA(cudaGraphExecDestroy(I->cycle[k]));
        I->cycle[k] = nullptr;
        I->cycle_tried[k] = false;
    }
}
} // namespace mhd

extern "C" {

int mhd_gpu_induction_create(MhdMesh *mesh, const MhdInductionParams *p, const double *m_edge_host, MhdInduction **out)
{
    MhdInduction *I = nullptr;
    int rc = guarded([&] {
        MHD_REQUIRE(mesh && p && out, "null argument");
        MHD_REQUIRE(p->precision == MHD_PREC_FP64 || p->precision == MHD_PREC_MIXED, "unknown precision");
        MHD_REQUIRE(p->restart >= 1 && p->max_it >= 0, "bad restart / max_it");
        const MeshView &m = mesh->v;
        cudaStream_t s = mesh->stream;
        I = new MhdInduction;
        I->mesh = mesh;
        I->p = *p;
        I->p.restart = std::max(2, p->restart); // restart_(std::max(2, cfg.ind_restart)) of the constructor
        I->hall = p->hall && p->hall_coef > 0;
        I->mixed = p->precision == MHD_PREC_MIXED;
        I->edge_blocks = g1(m.ne);
        {
            int dev = 0, sms = 0;
            MHD_CUDA(cudaGetDevice(&dev));
            MHD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            for (int k = 0; k < kCgsMax; ++k) cgs_grids_for(k, sms, I->cgs_grid + 2 * k);
        }
        const size_t ne = m.ne, nf = m.nf, nc = m.nc;
        std::vector<double> mc(ne, 0.0);
        if (m_edge_host)
            for (size_t e = 0; e < ne; ++e)
            {
                mc[e] = m_edge_host[e];
                I->resistive |= mc[e] != 0.0;
            }
        I->mcoef.upload(mc);
        // Hall radial taper with the host's tanh, as the reference computes it (:23-30)
        std::vector<double> xc(3 * nc);
        std::vector<int8_t> mat(nc);
        if (nc)
        {
            MHD_CUDA(cudaMemcpy(xc.data(), m.cell_center, 3 * nc * sizeof(double), cudaMemcpyDeviceToHost));
            MHD_CUDA(cudaMemcpy(mat.data(), m.material, nc, cudaMemcpyDeviceToHost));
        }
        std::vector<double> taper(nc, 0.0);
        const double mid = 0.5 * (p->hall_r_min + p->hall_r_max), width = p->hall_r_max - p->hall_r_min;
        for (size_t c = 0; c < nc; ++c)
        {
            if (mat[c] == 1) continue;
            const double x = xc[3 * c], y = xc[3 * c + 1], z = xc[3 * c + 2];
            const double r = std::sqrt(x * x + y * y + z * z);
            taper[c] = width <= 0 ? (r >= p->hall_r_min ? 1.0 : 0.0) : 0.5 * (1.0 + std::tanh(2.0 * (r - mid) / width));
        }
        I->taper.upload(taper);
        int32_t nnz_c = 0, nnz_ec = 0;
        MHD_CUDA(cudaMemcpy(&nnz_c, m.c2f_ptr + m.nc, sizeof(int32_t), cudaMemcpyDeviceToHost));
        MHD_CUDA(cudaMemcpy(&nnz_ec, m.ec_ptr + m.ne, sizeof(int32_t), cudaMemcpyDeviceToHost));
        I->alpha.alloc(nc); I->B0.alloc(3 * nc); I->recon.alloc(3 * (size_t)nnz_c); I->d2.alloc(ne); I->corr.alloc(ne);
        I->phi.alloc(nf); I->s2phi.alloc(nf); I->bcell.alloc(3 * nc); I->g.alloc(3 * nc);
        const int mr = I->p.restart;
        I->V.alloc((size_t)(mr + 1) * ne); I->w.alloc(ne); I->z.alloc(ne); I->r.alloc(ne); I->b.alloc(ne); I->x0.alloc(ne);
        I->delta.alloc(ne); I->Ax.alloc(ne); I->pd.alloc(ne); I->Fn.alloc(ne); I->dirc.alloc(ne);
        I->part.alloc((size_t)std::max(32 * kRedBlocks, I->edge_blocks));
        I->red.alloc(96);
        I->H.alloc((size_t)(mr + 1) * mr); I->cs.alloc(mr); I->sn.alloc(mr); I->gv.alloc(mr + 1); I->yv.alloc(mr);
        I->nrm.alloc(mr + 1); I->scal.alloc(8); I->counter.alloc(1); I->ctl.alloc(1);
        I->slot_nb.alloc(nnz_c); I->slot_sa.alloc(3 * (size_t)nnz_c);
        if (!I->mixed) I->zs.alloc(ne);
        MHD_CUDA(cudaMallocHost(&I->pinned, 8 * sizeof(double)));
        MHD_CUDA(cudaMemsetAsync(I->counter.p, 0, sizeof(unsigned), s));
        MHD_CUDA(cudaMemsetAsync(I->ctl.p, 0, sizeof(Ctl), s));
        MHD_CUDA(cudaMemsetAsync(I->scal.p, 0, 8 * sizeof(double), s));
        if (nc)
        {
            MHD_CUDA(cudaMemsetAsync(I->alpha.p, 0, nc * sizeof(double), s));
            MHD_CUDA(cudaMemsetAsync(I->B0.p, 0, 3 * nc * sizeof(double), s));
            MHD_CUDA(cudaMemsetAsync(I->g.p, 0, 3 * nc * sizeof(double), s));
            k_ind_recon<<<g1(nc), 256, 0, s>>>(m, I->recon.p);
        }
        if (ne) k_ind_d2<<<g1(ne), 256, 0, s>>>(m, I->d2.p);
        MHD_CUDA(cudaMemsetAsync(I->H.p, 0, (size_t)(mr + 1) * mr * sizeof(double), s));
        MHD_LAUNCH_CHECK();
        if (I->mixed)
        {
            I->recon32.alloc(3 * (size_t)nnz_c); I->m32.alloc(ne); I->ecw32.alloc(nnz_ec); I->tv32.alloc(3 * ne); I->zs32.alloc(ne); I->slot32.alloc(nnz_c);
            I->vinv32.alloc(nc); I->alpha32.alloc(nc); I->B0_32.alloc(3 * nc); I->phi32.alloc(nf); I->s2phi32.alloc(nf);
            I->b32.alloc(3 * nc); I->g32.alloc(3 * nc);
            const int64_t nmax = std::max<int64_t>({3 * (int64_t)nnz_c, (int64_t)nnz_ec, (int64_t)ne, (int64_t)nf, (int64_t)nc});
            if (nmax)
                k_ind_tables32<<<grid_for(nmax, 256), 256, 0, s>>>(m, I->recon.p, I->mcoef.p, I->recon32.p, I->m32.p, I->ecw32.p,
                                                                 I->tv32.p, I->vinv32.p);
            if (nc)
            {
                MHD_CUDA(cudaMemsetAsync(I->alpha32.p, 0, nc * sizeof(float), s));
                MHD_CUDA(cudaMemsetAsync(I->g32.p, 0, 3 * nc * sizeof(float), s));
            }
            MHD_LAUNCH_CHECK();
        }
        if (nc) k_ind_slots<<<g1(nc), 256, 0, s>>>(m, I->slot_nb.p, I->slot_sa.p, I->mixed ? I->slot32.p : nullptr);
        MHD_LAUNCH_CHECK();
        MHD_CUDA(cudaStreamSynchronize(s));
        *out = I;
    });
    if (rc != MHD_OK) delete I;
    return rc;
}

int mhd_gpu_induction_destroy(MhdInduction *I)
{
    return guarded([&] {
        if (!I) return;
        cudaStreamSynchronize(I->mesh->stream);
        delete I;
    });
}

int mhd_gpu_induction_set_frozen(MhdInduction *I, const double *B0, const double *ne_eff)
{
    return guarded([&] {
        MHD_REQUIRE(I && MHD_ARR(B0, I->mesh->v.nc) && MHD_ARR(ne_eff, I->mesh->v.nc), "null argument");
        const MeshView &m = I->mesh->v;
        cudaStream_t s = I->mesh->stream;
        if (!m.nc) return;
        MHD_CUDA(cudaMemcpyAsync(I->B0.p, B0, 3 * (size_t)m.nc * sizeof(double), cudaMemcpyDeviceToDevice, s));
        k_ind_alpha<<<g1(m.nc), 256, 0, s>>>(m.nc, I->taper.p, ne_eff, I->hall ? 1 : 0, I->p.hall_coef, I->alpha.p);
        if (I->mixed)
        {
            k_to_float<<<g1(3 * (int64_t)m.nc), 256, 0, s>>>(I->B0.p, I->B0_32.p, 3 * (int64_t)m.nc);
            k_to_float<<<g1(m.nc), 256, 0, s>>>(I->alpha.p, I->alpha32.p, m.nc);
        }
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_induction_set_frozen_alpha(MhdInduction *I, const double *B0, const double *alpha)
{
    return guarded([&] {
        MHD_REQUIRE(I && MHD_ARR(B0, I->mesh->v.nc) && MHD_ARR(alpha, I->mesh->v.nc), "null argument");
        const MeshView &m = I->mesh->v;
        cudaStream_t s = I->mesh->stream;
        if (!m.nc) return;
        MHD_CUDA(cudaMemcpyAsync(I->B0.p, B0, 3 * (size_t)m.nc * sizeof(double), cudaMemcpyDeviceToDevice, s));
        MHD_CUDA(cudaMemcpyAsync(I->alpha.p, alpha, (size_t)m.nc * sizeof(double), cudaMemcpyDeviceToDevice, s));
        if (I->mixed)
        {
            k_to_float<<<g1(3 * (int64_t)m.nc), 256, 0, s>>>(I->B0.p, I->B0_32.p, 3 * (int64_t)m.nc);
            k_to_float<<<g1(m.nc), 256, 0, s>>>(I->alpha.p, I->alpha32.p, m.nc);
        }
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_induction_apply_F(MhdInduction *I, const double *phi, double *out)
{
    return guarded([&] {
        MHD_REQUIRE(I && MHD_ARR(phi, I->mesh->v.ne) && MHD_ARR(out, I->mesh->v.ne), "null argument");
        op64(I, MatIn{}, phi, 0.0, out);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_induction_apply_A(MhdInduction *I, const double *x, double dt, double *y)
{
    return guarded([&] {
        MHD_REQUIRE(I && MHD_ARR(x, I->mesh->v.ne) && MHD_ARR(y, I->mesh->v.ne), "null argument");
        apply_plain(I, x, dt, y);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_induction_solve(MhdInduction *I, const double *Phi, const double *Ee, const int8_t *dir, double dt, int32_t warm, double *E,
                            int32_t *iterations, double *rel_res)
{
    return solve_impl(I, Phi, Ee, dir, dt, nullptr, warm, E, iterations, rel_res);
}

int mhd_gpu_induction_solve_dt_edge(MhdInduction *I, const double *Phi, const double *Ee, const int8_t *dir, const double *dt_edge,
                                    int32_t warm, double *E, int32_t *iterations, double *rel_res)
{
    if (I && I->mesh && !MHD_ARR(dt_edge, I->mesh->v.ne))
    {
        set_last_error("null dt_edge");
        return MHD_EINVAL;
    }
    return solve_impl(I, Phi, Ee, dir, 0.0, dt_edge, warm, E, iterations, rel_res);
}

int mhd_gpu_induction_set_ideal(MhdInduction *I, const double *u_cell, const int8_t *mask, double cuct)
{
    return guarded([&] {
        MHD_REQUIRE(I, "null induction handle");
        const MeshView &m = I->mesh->v;
        const bool on = u_cell != nullptr;
        MHD_REQUIRE(!on || (MHD_ARR(mask, m.ne) && std::isfinite(cuct)), "null mask or non-finite cuct");
        cudaStream_t s = I->mesh->stream;
        if (on)
        {
            I->u_ideal.alloc(std::max<size_t>(1, 3 * (size_t)m.nc));
            I->imask.alloc(std::max<size_t>(1, (size_t)m.ne));
            I->ide.alloc(std::max<size_t>(1, (size_t)m.ne));
            I->face3.alloc(std::max<size_t>(1, 3 * (size_t)m.nf));
            if (m.nc) MHD_CUDA(cudaMemcpyAsync(I->u_ideal.p, u_cell, 3 * (size_t)m.nc * sizeof(double), cudaMemcpyDeviceToDevice, s));
            if (m.ne) MHD_CUDA(cudaMemcpyAsync(I->imask.p, mask, (size_t)m.ne, cudaMemcpyDeviceToDevice, s));
            I->cuct = cuct;
        }
        // the captured restart cycles hold the other operator (and the mixed solve the other precision)
        if (on != I->ideal) drop_cycle_graphs(I);
        I->ideal = on;
    });
}

int mhd_gpu_induction_ideal_linear(MhdInduction *I, const double *phi, double *out)
{
    return guarded([&] {
        MHD_REQUIRE(I && MHD_ARR(phi, I->mesh->v.nf) && MHD_ARR(out, I->mesh->v.ne), "null argument");
        op64(I, MatIn{}, phi, 0.0, out, Fused{}, true);
        MHD_LAUNCH_CHECK();
    });
}

int mhd_gpu_induction_profile(MhdInduction *I, int32_t enable)
{
    return guarded([&] {
        MHD_REQUIRE(I, "null induction handle");
        MHD_CUDA(cudaStreamSynchronize(I->mesh->stream));
        I->prof.on = enable != 0;
        for (auto &u : I->prof.used) u = 0;
    });
}

int mhd_gpu_induction_profile_read(MhdInduction *I, int32_t max_kernels, char *names, double *ms_total, int64_t *count, int32_t *n_out)
{
    return guarded([&] {
        MHD_REQUIRE(I && names && ms_total && count && n_out, "null argument");
        MHD_CUDA(cudaStreamSynchronize(I->mesh->stream));
        int n = 0;
        for (int k = 0; k < KI_COUNT && n < max_kernels; ++k, ++n)
        {
            std::strncpy(names + 32 * n, kIndKernelNames[k], 31);
            names[32 * n + 31] = 0;
            I->prof.read(k, ms_total[n], count[n]);
        }
        *n_out = n;
    });
}

int mhd_gpu_induction_last_solve_stats(MhdInduction *I, int32_t *reorth_passes)
{
    return guarded([&] {
        MHD_REQUIRE(I && reorth_passes, "null argument");
        *reorth_passes = I->last_reorth;
    });
}

int mhd_gpu_induction_launches(MhdInduction *I, int64_t *out)
{
    return guarded([&] {
        MHD_REQUIRE(I && out, "null argument");
        *out = I->launches;
    });
}

} // extern "C"
