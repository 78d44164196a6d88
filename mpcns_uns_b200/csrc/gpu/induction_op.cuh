// The pieces of the semi-implicit induction operator that its FP64 (gmres.cu) and FP32 (gmres32.cu)
// matvecs share: the cycle control, the grid-wide dot tail, the face / cell-field / edge kernels as
// templates over the arithmetic type, the FP32 Hall pass, and the handle.  gmres.cu compiles the FP64
// instances reference-exact (no multiply-add contraction); gmres32.cu compiles the FP32 operator of the
// mixed-precision solve with contraction on.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace mhd
{
constexpr int kRedBlocks = 8 * 148; // streaming reductions: 8 resident 256-thread blocks per SM

// kernel classes of the solve, timed with CUDA events on the handle's stream when profiling is on
enum IndKernel { KI_FACE = 0, KI_BCELL, KI_HALL, KI_EDGE, KI_MGS, KI_SCALAR, KI_VECTOR, KI_ILU, KI_IDEAL, KI_COUNT };
const char *const kIndKernelNames[KI_COUNT] = {"face_d1",      "cell_field",    "hall_emf",      "edge_gather", "gram_schmidt",
                                               "krylov_scalar", "krylov_vector", "ilu",          "ideal_emf"};

// Device-side control of one restart cycle: the Arnoldi steps of a cycle are enqueued (or replayed as
// one CUDA graph) without host round trips; a step whose predecessor met the tolerance, or that lies
// beyond the iteration limit, returns at once.
struct Ctl
{
    int done, jend, limit, reorth; // reorth: the Gram-Schmidt step of this column needs its second pass
    int n_reorth, pad;             // second passes run in this cycle
    double tol, dt;
};
struct Gate
{
    const Ctl *ctl = nullptr;
    int j = 0;
    __device__ __forceinline__ bool off() const { return ctl && (ctl->done || j >= ctl->limit); }
};

// ---------------------------------------------------------------- classical Gram-Schmidt (gram_schmidt.cu)
constexpr int kCgsMax = 31; // basis vectors one pass handles (restart <= 31); the 32nd partial is |w|^2
struct CgsArgs
{
    Gate gt;
    Ctl *ctl;
    double *w;
    const double *V;
    int64_t ldv;
    int32_t n_all, n_owned;
    double *part, *red, *H;
    unsigned *counter;
    int mcols;
    const double *pd;
    double *zs;
    float *zs32;
};
// pass 0: the dots; 1: the update; 2: the gated second update (column j = number of basis vectors - 1)
void cgs_launch(int j, const CgsArgs &a, const int *grid, cudaStream_t s, int pass);
// the resident grids of column k's passes (2 ints), for an SM count
void cgs_grids_for(int k, int sms, int *grid);

// ---------------------------------------------------------------- block-Jacobi ILU(0) (ilu.cu)
// Control of the row-ordered passes (factorisation, lower and upper solve): rows are claimed in order
// through `ticket`; a finished row raises its flag to the pass's epoch; the last block of a pass resets
// the ticket and advances the epoch.  err != 0: a wait gave up (the pass's results are invalid).
struct IluCtl
{
    unsigned ticket, done, epoch, err;
};
constexpr int kIluMaxRow = 64; // longest row accepted
struct IluState
{
    bool built = false, on = false;
    double shift = 0.3;   // Config::ind_ilu_shift
    int32_t no = 0;       // owned edges (the rows)
    int64_t nnz = 0;
    int32_t depth_l = 0, depth_u = 0; // levels of the lower / upper dependency order
    int32_t npos_l = 0, npos_u = 0;   // positions of the level orders (levels padded to whole warps)
    int grid_l = 0, grid_u = 0;       // blocks of the passes: a few levels of rows in flight
    int64_t resident = 0;             // blocks of a pass resident on the device at once
    int32_t window_levels = 8;        // levels of rows in flight
    unsigned backoff_ns = 128;        // longest pause between two polls
    unsigned spin_polls = 0;          // polls without a pause before the back-off
    uint64_t wait_ns = 2000000000ull; // a wait on another row gives up after this long
    int32_t unpublished = -1;         // test hook: a row that never raises its flag
    DBuf<int32_t> ptr, col, diag, order_l, order_u;
    DBuf<double> coef, val, y, z; // y, z: results of the lower and upper solves (z = M^-1 v)
    DBuf<unsigned> flag;
    DBuf<IluCtl> ctl;
};

// ---------------------------------------------------------------- operator
// Input of a matvec: x_e directly (apply_A), or the preconditioned Krylov vector
// x_e = (src_e / *hs) * pd_e with pd_e = dir_e ? 0 : 1 / (1 + dt m_e d2_e)  (:338)
// The face pass gathers one edge vector: x itself, or zs = w_prev * pd (stored by the last
// Gram-Schmidt pass of the previous step, FP32 for the FP32 operator) whose d1 it divides by *hs.
struct MatIn
{
    const double *x = nullptr;
    const double *src = nullptr, *hs = nullptr, *pd = nullptr;
    const double *zs = nullptr;
    const float *zs32 = nullptr;
    const double *dte = nullptr; // per-edge pseudo-time step: Phi' = d1 diag(dt_e) x (:188)
};

template <class T> struct EdgeArgs
{
    int resistive = 0, hall = 0;
    const T *s2phi = nullptr, *g = nullptr, *mcoef = nullptr, *ecw = nullptr, *tvec = nullptr;
    MatIn in;                    // x of y = x + dt F; no input: y = F (apply_F)
    double dt = 0;
    const double *dtp = nullptr; // dt read from the cycle control instead
    double *vout = nullptr;      // stores src / *hs (the lazily normalised Krylov vector V_j)
    const int8_t *dir = nullptr; // zero y on Dirichlet edges (:339)
    const double *v0 = nullptr;  // y . v0 over the owned edges, stored to *dot
    double *part = nullptr, *dot = nullptr;
    unsigned *counter = nullptr;
    double *out = nullptr;
    const double *ide = nullptr;   // implicit ideal EMF of the owned edges (part2, :151-158) where imask is set
    const int8_t *imask = nullptr;
    Gate gt;
};
} // namespace mhd

namespace mhd
{
namespace
{
__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double sh[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0)
    {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

// Block partials of a grid-wide sum; the last block to finish adds them in block order (deterministic)
// and stores op(sum) to *out (op 0: the sum, 1: its square root, 2: sqrt(max(sum, 1e-300))), then
// re-arms the counter.  No block waits for another.
__device__ __forceinline__ void grid_sum_tail(double v, double *part, unsigned *counter, int op, double *out)
{
    __shared__ bool last;
    v = block_sum(v);
    if (threadIdx.x == 0)
    {
        part[blockIdx.x] = v;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double s = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) s += __ldcg(part + i);
    s = block_sum(s);
    if (threadIdx.x == 0)
    {
        *out = op == 0 ? s : (op == 1 ? sqrt(s) : sqrt(dmax(s, 1e-300)));
        *counter = 0;
    }
}

// Phi' = d1 x on every face (:185-190), with star2 Phi' for the resistive current flux (:131-136).
// FP64 sums in both precisions; the FP32 operator stores the rounded results.
// TRI: every face a triangle (f2e row of face f at 3f): the three gathers unrolled, in the row's order
template <class T, bool TRI = false>
__global__ void k_ind_face(MeshView m, Gate gt, MatIn in, int hall, int resistive, T *__restrict__ phi, T *__restrict__ s2phi)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf || gt.off()) return;
    double s = 0;
    if constexpr (TRI)
    {
        const int64_t k0 = 3 * (int64_t)f;
        const int32_t e0 = m.f2e_idx[k0], e1 = m.f2e_idx[k0 + 1], e2 = m.f2e_idx[k0 + 2];
        const double s0 = m.f2e_sgn[k0], s1 = m.f2e_sgn[k0 + 1], s2 = m.f2e_sgn[k0 + 2];
        double v0, v1, v2;
        if (in.zs32) { v0 = in.zs32[e0]; v1 = in.zs32[e1]; v2 = in.zs32[e2]; }
        else if (in.zs) { v0 = in.zs[e0]; v1 = in.zs[e1]; v2 = in.zs[e2]; }
        else { v0 = in.x[e0]; v1 = in.x[e1]; v2 = in.x[e2]; }
        if (in.dte)
        {
            s += (s0 * in.dte[e0]) * v0;
            s += (s1 * in.dte[e1]) * v1;
            s += (s2 * in.dte[e2]) * v2;
        }
        else
        {
            s += s0 * v0;
            s += s1 * v1;
            s += s2 * v2;
        }
    }
    else
    {
        const int32_t k0 = m.f2e_ptr[f], k1 = m.f2e_ptr[f + 1];
        for (int32_t k = k0; k < k1; ++k)
        {
            const int32_t e = m.f2e_idx[k];
            const double v = in.zs32 ? static_cast<double>(in.zs32[e]) : (in.zs ? in.zs[e] : in.x[e]);
            const double sg = m.f2e_sgn[k];
            s += (in.dte ? sg * in.dte[e] : sg) * v;
        }
    }
    if ((in.zs || in.zs32) && in.hs) s = s / *in.hs;
    if (hall) phi[f] = static_cast<T>(s);
    if (resistive) s2phi[f] = static_cast<T>(m.star2[f] * s);
}

// cell field from the face fluxes (:139-149); TET: every cell a tetrahedron (c2f row of cell c at 4c), the
// four slots unrolled in the row's order
template <class T, bool TET = false>
__global__ void k_ind_bcell(MeshView m, Gate gt, const T *__restrict__ recon, const T *__restrict__ phi, T *__restrict__ b)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc || gt.off()) return;
    T bx = 0, by = 0, bz = 0;
    const int32_t kb = TET ? 4 * c : m.c2f_ptr[c], ke = TET ? 4 * c + 4 : m.c2f_ptr[c + 1];
#pragma unroll 4
    for (int32_t k = kb; k < ke; ++k)
    {
        const T v = phi[m.c2f_idx[k]];
        bx += recon[3 * (int64_t)k] * v;
        by += recon[3 * (int64_t)k + 1] * v;
        bz += recon[3 * (int64_t)k + 2] * v;
    }
    b[3 * (int64_t)c] = bx; b[3 * (int64_t)c + 1] = by; b[3 * (int64_t)c + 2] = bz;
}

template <bool TET = false>
__global__ void k_ind_hall32(MeshView m, Gate gt, const float4 *__restrict__ slot32, const float *__restrict__ b,
                             const float *__restrict__ alpha, const float *__restrict__ B0, const float *__restrict__ vinv,
                             float *__restrict__ g)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.no_cells || gt.off()) return;
    const float a = alpha[c];
    if (a == 0.f || m.material[c] != 0)
    {
        g[3 * (int64_t)c] = g[3 * (int64_t)c + 1] = g[3 * (int64_t)c + 2] = 0.f;
        return;
    }
    float sx = 0.f, sy = 0.f, sz = 0.f;
    const float bcx = b[3 * (int64_t)c], bcy = b[3 * (int64_t)c + 1], bcz = b[3 * (int64_t)c + 2];
    const int32_t kb = TET ? 4 * c : m.c2f_ptr[c], ke = TET ? 4 * c + 4 : m.c2f_ptr[c + 1];
#pragma unroll 4
    for (int32_t k = kb; k < ke; ++k)
    {
        const float4 sl = slot32[k];
        const int32_t o = __float_as_int(sl.w);
        float bx = bcx, by = bcy, bz = bcz;
        if (o >= 0)
        {
            bx = 0.5f * (bcx + b[3 * (int64_t)o]);
            by = 0.5f * (bcy + b[3 * (int64_t)o + 1]);
            bz = 0.5f * (bcz + b[3 * (int64_t)o + 2]);
        }
        const float ax = sl.x, ay = sl.y, az = sl.z;
        sx += ay * bz - az * by;
        sy += az * bx - ax * bz;
        sz += ax * by - ay * bx;
    }
    const float iv = vinv[c];
    const float Jx = iv * sx, Jy = iv * sy, Jz = iv * sz;
    const float Bx = B0[3 * (int64_t)c], By = B0[3 * (int64_t)c + 1], Bz = B0[3 * (int64_t)c + 2];
    g[3 * (int64_t)c] = a * (Jy * Bz - Jz * By);
    g[3 * (int64_t)c + 1] = a * (Jz * Bx - Jx * Bz);
    g[3 * (int64_t)c + 2] = a * (Jx * By - Jy * Bx);
}

// Per edge: part0 = sum_f s star2 Phi' (resistive, ascending faces), part1 = sum_c g_c . (w_ec t_e)
// (Hall, ascending cells), F = m part0 + part1 + part2 (:176-182); y = F, or y = x + dt F (:191-197).
// MAXK > 0: every edge has at most MAXK faces and MAXK cells (tetrahedral meshes: 8); both gathers are
// unrolled over that bound (predicated beyond the row), so that a row's loads are in flight together.  The
// sums run over the rows in their order either way.
template <class T, int MAXK>
__global__ void __launch_bounds__(256) k_ind_edge(MeshView m, EdgeArgs<T> a)
{
    if (a.gt.off()) return;
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    double contrib = 0.0;
    if (e < m.ne)
    {
        T p0 = 0, p1 = 0;
        if (a.resistive)
        {
            const int32_t k0 = m.e2f_ptr[e], k1 = m.e2f_ptr[e + 1];
            if constexpr (MAXK > 0)
            {
#pragma unroll
                for (int i = 0; i < MAXK; ++i)
                    if (k0 + i < k1) p0 += static_cast<T>(m.e2f_sgn[k0 + i]) * a.s2phi[m.e2f_idx[k0 + i]];
            }
            else
                for (int32_t k = k0; k < k1; ++k) p0 += static_cast<T>(m.e2f_sgn[k]) * a.s2phi[m.e2f_idx[k]];
        }
        if (a.hall)
        {
            const T tx = a.tvec[3 * (int64_t)e], ty = a.tvec[3 * (int64_t)e + 1], tz = a.tvec[3 * (int64_t)e + 2];
            const int32_t k0 = m.ec_ptr[e], k1 = m.ec_ptr[e + 1];
            auto term = [&](int32_t k) {
                const int32_t c = m.ec_cell[k];
                if (c >= m.no_cells) return;
                const T w = a.ecw[k];
                const T wx = w * tx, wy = w * ty, wz = w * tz;
                p1 += a.g[3 * (int64_t)c] * wx + a.g[3 * (int64_t)c + 1] * wy + a.g[3 * (int64_t)c + 2] * wz;
            };
            if constexpr (MAXK > 0)
            {
#pragma unroll
                for (int i = 0; i < MAXK; ++i)
                    if (k0 + i < k1) term(k0 + i);
            }
            else
                for (int32_t k = k0; k < k1; ++k) term(k);
        }
        const T p2 = (a.ide && a.imask[e]) ? static_cast<T>(a.ide[e]) : static_cast<T>(0);
        const T F = a.mcoef[e] * p0 + p1 + p2;
        double y = static_cast<double>(F);
        if (a.in.src || a.in.x)
        {
            double xe;
            if (a.in.src)
            {
                double v = a.in.src[e];
                if (a.in.hs) v = v / *a.in.hs;
                if (a.vout) a.vout[e] = v;
                xe = v * a.in.pd[e];
            }
            else
                xe = a.in.x[e];
            y = xe + (a.dtp ? *a.dtp : a.dt) * static_cast<double>(F);
        }
        if (a.dir && a.dir[e]) y = 0.0;
        a.out[e] = y;
        if (a.v0 && e < m.no_edges) contrib = y * a.v0[e];
    }
    if (a.v0) grid_sum_tail(contrib, a.part, a.counter, 0, a.dot);
}

} // namespace
} // namespace mhd

struct MhdInduction
{
    MhdMesh *mesh = nullptr;
    MhdInductionParams p{};
    bool resistive = false, hall = false, mixed = false, have_corr = false;
    int edge_blocks = 0;
    int cgs_grid[64] = {}; // grids of the Gram-Schmidt passes per column size (dots, update): resident blocks on every SM
    mhd::DBuf<double> mcoef, taper, alpha, B0, recon, d2, corr, phi, s2phi, bcell, g;
    mhd::DBuf<double> V, w, z, r, b, x0, delta, Ax, pd, Fn, part, H, cs, sn, gv, yv, nrm, scal, red;
    mhd::DBuf<float> recon32, m32, ecw32, tv32, vinv32, alpha32, B0_32, phi32, s2phi32, b32, g32, zs32;
    mhd::DBuf<double> slot_sa, zs;
    mhd::DBuf<int32_t> slot_nb;
    mhd::DBuf<float4> slot32;
    mhd::DBuf<int8_t> dirc;
    mhd::DBuf<unsigned> counter;
    mhd::DBuf<mhd::Ctl> ctl;
    mhd::IluState ilu;
    double *pinned = nullptr;
    mhd::EventProfiler<mhd::KI_COUNT> prof;
    int64_t launches = 0;
    int32_t last_reorth = 0; // Gram-Schmidt second passes of the last solve
    // the implicit ideal part of F (set_ideal_state): cell velocities, edges that carry it, its UCT strength
    bool ideal = false;
    double cuct = 0.5;
    mhd::DBuf<double> u_ideal, ide, face3, dte;
    mhd::DBuf<int8_t> imask;
    // one restart cycle (mr Arnoldi steps) captured as a CUDA graph on the first unprofiled solve of each
    // kind (mode 0: Jacobi with a scalar dt; 1: Jacobi with the per-edge dt; 2: ILU(0))
    int mode = 0;
    cudaGraphExec_t cycle[3] = {nullptr, nullptr, nullptr};
    bool cycle_tried[3] = {false, false, false};
    int64_t cycle_kernels[3] = {0, 0, 0};
    bool capturing = false;
    ~MhdInduction()
    {
        for (auto &g : cycle)
            if (g) cudaGraphExecDestroy(g);
        if (pinned) cudaFreeHost(pinned);
    }
};

namespace mhd
{
inline int g1(int64_t n) { return grid_for(n, 256); }

// one launch of kernel class k on the handle's stream, counted and (when profiling, outside a graph
// capture) timed
#define IND_LAUNCH(I, k, s, ...)                                                                                         \
    do                                                                                                                   \
    {                                                                                                                    \
        if (!(I)->capturing) (I)->prof.begin(k, s);                                                                      \
        __VA_ARGS__;                                                                                                     \
        if (!(I)->capturing) (I)->prof.end(k, s);                                                                        \
        ++(I)->launches;                                                                                                 \
    } while (0)

struct Fused
{
    double *vout = nullptr;
    const int8_t *dir = nullptr;
    const double *v0 = nullptr;
    double *dot = nullptr;
    const double *dtp = nullptr;
    Gate gt;
};

// the Arnoldi matvec with the FP32 operator (gmres32.cu)
void op32(MhdInduction *I, const MatIn &in, double dt, double *y, const Fused &fz);

// ILU(0) passes on the handle's stream (ilu.cu): factor_precond (:247-275) for dt and the Dirichlet flags;
// apply_precond (:277-297) of v = dir ? 0 : src / *hs (hs may be null) into I->ilu.z, storing src / *hs to
// vout when given (the lazily normalised Krylov vector); gated by gt inside a restart cycle.  The result
// stays valid until the next application.
void ilu_factor(MhdInduction *I, double dt, const int8_t *dir);
void ilu_apply(MhdInduction *I, const Gate &gt, const double *src, const double *hs, const int8_t *dir, double *vout);
// MHD_ECUDA if a wait of an ILU(0) pass gave up since the last check (synchronises the stream)
void ilu_check(MhdInduction *I);
// Drop the captured restart cycles (after a change of preconditioner, launch shape or operator parts);
// synchronises the stream.
void drop_cycle_graphs(MhdInduction *I);
// The ideal UCT EMF added into E (owned edges) from u, B_tot, B_ind (3 per cell) and phi_tot, phi_ind
// (per face), with face3 (3 per face) as the face candidates' scratch (induction.cu).
void ideal_emf_enqueue(const MeshView &m, const double *u, const double *Bt, const double *Bi, const double *phi_tot,
                       const double *phi_ind, double cuct, double *face3, double *E, cudaStream_t s);
} // namespace mhd
