// nvcc-flags: -fmad=false
// Block-Jacobi ILU(0) preconditioner of the semi-implicit induction solve (mhd::ImplicitInduction,
// Common/induction/ImplicitInduction.cpp:209-297): the pattern of I + dt M d1^T S2 d1 on the owned edges,
// its incomplete factorisation for a solve's dt and Dirichlet flags, and the two triangular solves.
//
// The pattern is built once on the host, row by row as the reference builds it, sorted by std::sort with
// the reference's comparator so that duplicate columns (the diagonal gathers one term per face) are
// summed in the same order: the coefficients are bit-identical.  The factorisation (IKJ) and the
// triangular solves are sequential in the row order.  On the device each row is one thread; the rows
// are ordered by dependency level (a row of the lower solve and of the factorisation reads its lower
// columns, a row of the upper solve its upper columns; level = 1 + the largest level it reads), each
// level padded to whole warps, and warps claim 32 positions of that order at a time through an atomic
// ticket.  A row waits for the rows it reads to raise their flags; they lie in lower levels, claimed
// before it by warps already running, and never in its own warp, so every pass completes.  The wait
// still gives up after 2 s (recording the failure) so that no input can hold the GPU.  Within a row the
// reference's arithmetic is kept operation for operation (products, quotients and differences rounded
// separately, the row's terms subtracted in column order), so factors and results are the reference's
// bit for bit.  The dependency depth of the natural edge order of a cubed-sphere shell is about 14 x
// its radial layer count, so every pass is bound by that chain's latency (depth x one row's loads), not
// by bandwidth.
#include <algorithm>
#include <thread>
#include <utility>

#include "induction_op.cuh"

namespace mhd
{
namespace
{
constexpr int kIluThreads = 128; // 4 warps per block; every warp claims 32 positions of a level order
constexpr int kIluChunk = 16;    // entries of a row loaded together (their flags, values and z)

struct IluView
{
    int32_t no;
    const int32_t *ptr, *col, *diag;
    const double *coef;
    double *val;
    unsigned *flag;
    IluCtl *ctl;
    uint64_t wait_ns;    // a wait gives up after this long
    int32_t unpublished; // test hook: this row never raises its flag (-1: none)
    unsigned backoff;    // longest pause between two polls (ns)
    unsigned spin;       // polls without a pause before the back-off starts
};

__device__ __forceinline__ unsigned ld_relaxed(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void st_release(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The flags of columns col[k0 .. k0+n) (n <= kIluChunk): loaded together, the unfinished ones polled
// together until they are raised (every round one round trip for all of them: spin rounds without a
// pause, then 32 ns doubling to P.backoff), then one fence orders the caller's later loads of those rows'
// results after their release.  Gives up after P.wait_ns (raising ctl->err), and at once when another
// wait has given up.
__device__ __forceinline__ void ilu_wait_chunk(const IluView &P, int32_t k0, int n, unsigned ep, int32_t *c)
{
    unsigned f[kIluChunk];
#pragma unroll
    for (int u = 0; u < kIluChunk; ++u) c[u] = u < n ? __ldg(P.col + k0 + u) : 0;
#pragma unroll
    for (int u = 0; u < kIluChunk; ++u) f[u] = u < n ? ld_relaxed(P.flag + c[u]) : ep;
    unsigned pending = 0;
#pragma unroll
    for (int u = 0; u < kIluChunk; ++u)
        if (f[u] != ep) pending |= 1u << u;
    // the unfinished rows polled together, one round trip per round for all of them
    const uint64_t t0 = pending ? global_ns() : 0;
    unsigned ns = 32;
    for (unsigned it = 1; pending; ++it)
    {
        if (it > P.spin)
        {
            __nanosleep(ns);
            ns = ns < P.backoff ? 2 * ns : P.backoff;
        }
#pragma unroll
        for (int u = 0; u < kIluChunk; ++u)
            if (pending & (1u << u)) f[u] = ld_relaxed(P.flag + c[u]);
#pragma unroll
        for (int u = 0; u < kIluChunk; ++u)
            if ((pending & (1u << u)) && f[u] == ep) pending &= ~(1u << u);
        if (pending && (it & 15) == 0)
        {
            if (*(volatile unsigned *)&P.ctl->err) break;
            if (global_ns() - t0 > P.wait_ns)
            {
                atomicOr(&P.ctl->err, 1u);
                break;
            }
        }
    }
    fence_acq_rel();
}

// Claim the next 32 positions of the pass's order for this warp (one ticket per warp).
__device__ __forceinline__ unsigned ilu_claim(const IluView &P)
{
    unsigned base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(&P.ctl->ticket, 32u);
    return __shfl_sync(0xffffffffu, base, 0);
}

// End of a pass: the last block resets the ticket and publishes the epoch the pass wrote.
__device__ __forceinline__ void ilu_finish(const IluView &P, unsigned ep)
{
    __syncthreads();
    if (threadIdx.x != 0) return;
    __threadfence();
    if (atomicAdd(&P.ctl->done, 1u) != gridDim.x - 1) return;
    P.ctl->ticket = 0;
    P.ctl->done = 0;
    __threadfence();
    P.ctl->epoch = ep;
}

// Publish row i of this pass (its stores made visible first).
__device__ __forceinline__ void ilu_publish(const IluView &P, int32_t i, unsigned ep)
{
    if (i != P.unpublished) st_release(P.flag + i, ep);
}

// factor_precond (:247-275), one row per thread, rows in the order of their lower levels (a level's rows
// padded to whole warps, so that no row waits on a row of its own warp): the initial values from the
// pattern, then the IKJ elimination a_ik /= u_kk; a_ij -= l_ik u_kj over the row's lower columns k in
// ascending order and the columns j > k of row k that row i holds, then the breakdown guard.
__global__ void __launch_bounds__(kIluThreads) k_ilu_factor(IluView P, const int32_t *__restrict__ order, int32_t npos, double dt,
                                                           double shift, const int8_t *__restrict__ dir)
{
    const unsigned ep = __ldcg(&P.ctl->epoch) + 1;
    for (;;)
    {
        const unsigned base = ilu_claim(P);
        if (base >= (unsigned)npos) break;
        const int32_t i = __ldg(order + base + (threadIdx.x & 31));
        if (i < 0) continue;
        const int32_t a = __ldg(P.ptr + i), b = __ldg(P.ptr + i + 1), d = __ldg(P.diag + i);
        const bool di = dir && __ldg(dir + i);
        double *v = P.val;
        for (int32_t k = a; k < b; ++k)
        {
            const int32_t c = __ldg(P.col + k);
            const double one = c == i ? 1.0 : 0.0;
            const double cf = __ldg(P.coef + k);
            // Dirichlet unknowns are removed: identity row and no coupling into them
            double x = (di || (dir && __ldg(dir + c))) ? one : __dadd_rn(one, __dmul_rn(dt, cf));
            if (c == i && !di) x = __dadd_rn(x, __dmul_rn(__dmul_rn(shift, dt), cf));
            v[k] = x;
        }
        for (int32_t k0 = a; k0 < d; k0 += kIluChunk)
        {
            // the chunk's rows k: wait for them, then their diagonal positions and row ends together
            const int n = min(kIluChunk, d - k0);
            int32_t kc[kIluChunk], kd[kIluChunk], ke[kIluChunk];
            ilu_wait_chunk(P, k0, n, ep, kc);
#pragma unroll
            for (int u = 0; u < kIluChunk; ++u)
            {
                kd[u] = u < n ? __ldg(P.diag + kc[u]) : 0;
                ke[u] = u < n ? __ldg(P.ptr + kc[u] + 1) : 0;
            }
#pragma unroll
            for (int u = 0; u < kIluChunk; ++u)
            {
                if (u >= n) break;
                const int32_t kk = k0 + u;
                const double pivot = __ldcg(v + kd[u]);
                const double lik = __ddiv_rn(v[kk], pivot);
                v[kk] = lik;
                int32_t p = kk + 1;
                // the columns j > k of row k, a chunk at a time, merged with the rest of row i
                for (int32_t j0 = kd[u] + 1; j0 < ke[u] && p < b; j0 += kIluChunk)
                {
                    const int m = min(kIluChunk, ke[u] - j0);
                    int32_t cj[kIluChunk];
                    double uj[kIluChunk];
#pragma unroll
                    for (int q = 0; q < kIluChunk; ++q)
                    {
                        cj[q] = q < m ? __ldg(P.col + j0 + q) : 0;
                        uj[q] = q < m ? __ldcg(v + j0 + q) : 0.0;
                    }
#pragma unroll
                    for (int q = 0; q < kIluChunk; ++q)
                    {
                        if (q >= m) break;
                        while (p < b && __ldg(P.col + p) < cj[q]) ++p;
                        if (p == b) break;
                        if (__ldg(P.col + p) == cj[q]) v[p] = __dsub_rn(v[p], __dmul_rn(lik, uj[q]));
                    }
                }
            }
        }
        if (!(fabs(v[d]) > 1e-12)) v[d] = 1.0; // breakdown guard
        ilu_publish(P, i, ep);
    }
    ilu_finish(P, ep);
}

// The result of a row of a triangular solve is its own ready flag: the result arrays hold kUnset (all
// bits set, a NaN that no arithmetic result carries here: a result with those bits is stored as the
// canonical NaN instead) until the row stores its value, and the rows that read it poll the value itself.
constexpr long long kUnset = -1ll;
__device__ __forceinline__ double ld_relaxed_f64(const double *p)
{
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_f64(double *p, double v)
{
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ bool unset(double v) { return __double_as_longlong(v) == kUnset; }

// Poll the results of the pending rows c[u] (bits of `pending`) until all are set: every round reloads all
// of them at once, then pauses (spin rounds without a pause, then 32 ns doubling to P.backoff).  Gives up
// as ilu_wait_chunk does (the unset values stay then).
__device__ __forceinline__ void ilu_poll_values(const IluView &P, const double *out, const int32_t *c, double *x, unsigned pending)
{
    const uint64_t t0 = global_ns();
    unsigned ns = 32;
    for (unsigned it = 1; pending; ++it)
    {
        if (it > P.spin)
        {
            __nanosleep(ns);
            ns = ns < P.backoff ? 2 * ns : P.backoff;
        }
#pragma unroll
        for (int u = 0; u < kIluChunk; ++u)
            if (pending & (1u << u)) x[u] = ld_relaxed_f64(out + c[u]);
#pragma unroll
        for (int u = 0; u < kIluChunk; ++u)
            if ((pending & (1u << u)) && !unset(x[u])) pending &= ~(1u << u);
        if (pending && (it & 15) == 0)
        {
            if (*(volatile unsigned *)&P.ctl->err) return;
            if (global_ns() - t0 > P.wait_ns)
            {
                atomicOr(&P.ctl->err, 1u);
                return;
            }
        }
    }
}

// apply_precond (:277-297), one triangle per launch, one row per thread in the order of the triangle's
// levels.  Lower (unit diagonal), into y: y_i = (dir_i ? 0 : v_i) - sum_{k < diag} a_ik y_k with
// v = src / *hs; upper, into z: z_i = dir_i ? 0 : (y_i - sum_{k > diag} a_ik z_k) / a_ii.  The terms are
// subtracted in column order.  Each row re-arms the other triangle's result for the next application
// (the lower pass unsets z_i, the previous application's output, the upper pass y_i after reading it).
template <bool UPPER>
__global__ void __launch_bounds__(kIluThreads) k_ilu_trsv(Gate gt, IluView P, const int32_t *__restrict__ order, int32_t npos,
                                                         const double *__restrict__ src, const double *hs, const int8_t *__restrict__ dir,
                                                         double *vout, double *y, double *z)
{
    if (gt.off()) return;
    const unsigned ep = __ldcg(&P.ctl->epoch) + 1;
    const double h = (!UPPER && hs) ? *hs : 1.0;
    double *out = UPPER ? z : y;
    for (;;)
    {
        const unsigned base = ilu_claim(P);
        if (base >= (unsigned)npos) break;
        const int32_t i = __ldg(order + base + (threadIdx.x & 31));
        if (i < 0) continue;
        const int32_t d = __ldg(P.diag + i);
        const int32_t lo = UPPER ? d + 1 : __ldg(P.ptr + i), hi = UPPER ? __ldg(P.ptr + i + 1) : d;
        const bool di = dir && __ldg(dir + i);
        double acc;
        if (UPPER)
        {
            acc = __ldcg(y + i);
            y[i] = __longlong_as_double(kUnset);
        }
        else
        {
            const double vi = hs ? __ddiv_rn(src[i], h) : src[i];
            if (vout) vout[i] = vi;
            acc = di ? 0.0 : vi;
            z[i] = __longlong_as_double(kUnset);
        }
        for (int32_t k0 = lo; k0 < hi; k0 += kIluChunk)
        {
            const int n = min(kIluChunk, hi - k0);
            int32_t c[kIluChunk];
            double a[kIluChunk], x[kIluChunk];
#pragma unroll
            for (int u = 0; u < kIluChunk; ++u)
            {
                c[u] = u < n ? __ldg(P.col + k0 + u) : 0;
                a[u] = u < n ? __ldg(P.val + k0 + u) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kIluChunk; ++u) x[u] = u < n ? ld_relaxed_f64(out + c[u]) : 0.0;
            // the unfinished rows polled together, one round trip per round for all of them
            unsigned pending = 0;
#pragma unroll
            for (int u = 0; u < kIluChunk; ++u)
                if (u < n && unset(x[u])) pending |= 1u << u;
            if (pending) ilu_poll_values(P, out, c, x, pending);
#pragma unroll
            for (int u = 0; u < kIluChunk; ++u)
                if (u < n) acc = __dsub_rn(acc, __dmul_rn(a[u], x[u]));
        }
        double r = UPPER ? (di ? 0.0 : __ddiv_rn(acc, __ldg(P.val + d))) : acc;
        if (unset(r)) r = __longlong_as_double(0x7ff8000000000000ll);
        if (i != P.unpublished) st_relaxed_f64(out + i, r);
    }
    ilu_finish(P, ep);
}

// z = 0 on the non-owned edges (their values come from the owners' exchange); V_j there as well
__global__ void k_ilu_tail(Gate gt, int32_t no, int32_t ne, const double *src, const double *hs, double *vout, double *z)
{
    if (gt.off()) return;
    const int32_t e = no + blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    z[e] = 0.0;
    if (vout) vout[e] = hs ? src[e] / *hs : src[e];
}

IluView view(MhdInduction *I)
{
    IluState &L = I->ilu;
    return IluView{L.no, L.ptr.p, L.col.p, L.diag.p, L.coef.p, L.val.p, L.flag.p, L.ctl.p, L.wait_ns, L.unpublished, L.backoff_ns, L.spin_polls};
}

// build_precond_pattern (:209-242) for rows [r0, r1): counts per row and the rows' (column, coefficient) runs
template <class P>
void pattern_rows(int32_t r0, int32_t r1, int32_t no, const P *e2f_ptr, const int32_t *e2f_idx, const int8_t *e2f_sgn, const P *f2e_ptr,
                  const int32_t *f2e_idx, const int8_t *f2e_sgn, const double *star2, const double *m, int64_t *cnt,
                  std::vector<int32_t> &col, std::vector<double> &coef)
{
    std::vector<std::pair<int32_t, double>> row;
    for (int32_t e = r0; e < r1; ++e)
    {
        row.clear();
        row.emplace_back(e, 0.0); // the diagonal is always present
        for (P kf = e2f_ptr[e]; kf < e2f_ptr[e + 1]; ++kf)
        {
            const int32_t f = e2f_idx[kf];
            const double se = e2f_sgn[kf];
            for (P k = f2e_ptr[f]; k < f2e_ptr[f + 1]; ++k)
            {
                const int32_t e2 = f2e_idx[k];
                if (e2 >= no) continue; // other ranks: block Jacobi
                row.emplace_back(e2, m[e] * se * f2e_sgn[k] * star2[f]);
            }
        }
        std::sort(row.begin(), row.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
        int64_t n = 0;
        for (size_t i = 0; i < row.size();)
        {
            size_t j = i;
            double sum = 0;
            for (; j < row.size() && row[j].first == row[i].first; ++j) sum += row[j].second;
            col.push_back(row[i].first);
            coef.push_back(sum);
            ++n;
            i = j;
        }
        cnt[e - r0] = n;
    }
}

// The whole pattern over host threads (rows split into contiguous ranges, concatenated in order).
template <class P>
void build_pattern(int32_t no, const P *e2f_ptr, const int32_t *e2f_idx, const int8_t *e2f_sgn, const P *f2e_ptr, const int32_t *f2e_idx,
                   const int8_t *f2e_sgn, const double *star2, const double *m, std::vector<int64_t> &ptr, std::vector<int32_t> &col,
                   std::vector<double> &coef)
{
    const int nt = std::max(1, std::min<int>(32, (int)std::thread::hardware_concurrency()));
    const int parts = std::max(1, std::min<int>(nt, no / 4096 + 1));
    std::vector<std::vector<int32_t>> cols(parts);
    std::vector<std::vector<double>> coefs(parts);
    ptr.assign((size_t)no + 1, 0);
    auto work = [&](int p) {
        const int32_t r0 = (int32_t)((int64_t)no * p / parts), r1 = (int32_t)((int64_t)no * (p + 1) / parts);
        pattern_rows(r0, r1, no, e2f_ptr, e2f_idx, e2f_sgn, f2e_ptr, f2e_idx, f2e_sgn, star2, m, ptr.data() + 1 + r0, cols[p], coefs[p]);
    };
    std::vector<std::thread> th;
    for (int p = 1; p < parts; ++p) th.emplace_back(work, p);
    work(0);
    for (auto &t : th) t.join();
    for (int32_t e = 0; e < no; ++e) ptr[e + 1] += ptr[e];
    col.clear();
    coef.clear();
    col.reserve((size_t)ptr[no]);
    coef.reserve((size_t)ptr[no]);
    for (int p = 0; p < parts; ++p)
    {
        col.insert(col.end(), cols[p].begin(), cols[p].end());
        coef.insert(coef.end(), coefs[p].begin(), coefs[p].end());
    }
}

// The blocks of the passes: about window_levels levels of rows in flight, enough for a level's rows to
// start together and few enough that the rows waiting on later levels do not flood L2 with polls; never
// more than are resident.
void ilu_grids(IluState &L)
{
    auto grid_for_depth = [&](int32_t depth, int32_t npos) {
        const int64_t rows = (int64_t)L.window_levels * (((int64_t)npos + depth - 1) / std::max(depth, 1));
        const int64_t blocks = (rows + kIluThreads - 1) / kIluThreads;
        return (int)std::max<int64_t>(1, std::min<int64_t>({L.resident, blocks, ((int64_t)npos + kIluThreads - 1) / kIluThreads}));
    };
    L.grid_l = grid_for_depth(L.depth_l, L.npos_l);
    L.grid_u = grid_for_depth(L.depth_u, L.npos_u);
}

// every owned row's results unset (the bytes of kUnset are all 0xff)
void ilu_unset(IluState &L, cudaStream_t s)
{
    MHD_CUDA(cudaMemsetAsync(L.y.p, 0xff, (size_t)std::max(L.no, 1) * sizeof(double), s));
    MHD_CUDA(cudaMemsetAsync(L.z.p, 0xff, (size_t)std::max(L.no, 1) * sizeof(double), s));
}

template <class T> std::vector<T> down(const T *p, size_t n)
{
    std::vector<T> h(n);
    if (n) MHD_CUDA(cudaMemcpy(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost));
    return h;
}

// The pattern of the handle's mesh and m_e, uploaded with its diagonal positions; the pass control.
void ilu_build(MhdInduction *I)
{
    IluState &L = I->ilu;
    const MeshView &m = I->mesh->v;
    const int32_t no = m.no_edges, ne = m.ne, nf = m.nf;
    auto e2f_ptr = down(m.e2f_ptr, (size_t)ne + 1);
    auto e2f_idx = down(m.e2f_idx, (size_t)e2f_ptr[ne]);
    auto e2f_sgn = down(m.e2f_sgn, (size_t)e2f_ptr[ne]);
    auto f2e_ptr = down(m.f2e_ptr, (size_t)nf + 1);
    auto f2e_idx = down(m.f2e_idx, (size_t)f2e_ptr[nf]);
    auto f2e_sgn = down(m.f2e_sgn, (size_t)f2e_ptr[nf]);
    auto star2 = down(m.star2, (size_t)nf);
    auto mc = down(I->mcoef.p, (size_t)ne);
    std::vector<int64_t> ptr;
    std::vector<int32_t> col;
    std::vector<double> coef;
    build_pattern(no, e2f_ptr.data(), e2f_idx.data(), e2f_sgn.data(), f2e_ptr.data(), f2e_idx.data(), f2e_sgn.data(), star2.data(),
                  mc.data(), ptr, col, coef);
    MHD_REQUIRE(ptr[no] < INT32_MAX, "ILU(0) pattern has 2^31 entries or more");
    std::vector<int32_t> p32((size_t)no + 1), dg((size_t)no);
    int64_t longest = 0;
    for (int32_t e = 0; e <= no; ++e) p32[e] = (int32_t)ptr[e];
    for (int32_t e = 0; e < no; ++e)
    {
        longest = std::max(longest, ptr[e + 1] - ptr[e]);
        for (int64_t k = ptr[e]; k < ptr[e + 1]; ++k)
            if (col[k] == e) dg[e] = (int32_t)k;
    }
    MHD_REQUIRE(longest <= kIluMaxRow, "ILU(0) rows longer than 64 entries");
    // dependency levels: a row of the lower solve (and of the factorisation) reads its lower columns, a row
    // of the upper solve its upper columns; level = 1 + the largest level it reads
    std::vector<int32_t> lev_l((size_t)no), lev_u((size_t)no);
    int32_t depth_l = 0, depth_u = 0;
    for (int32_t e = 0; e < no; ++e)
    {
        int32_t l = 0;
        for (int64_t k = ptr[e]; k < dg[e]; ++k) l = std::max(l, lev_l[col[k]] + 1);
        lev_l[e] = l;
        depth_l = std::max(depth_l, l + 1);
    }
    for (int32_t e = no - 1; e >= 0; --e)
    {
        int32_t l = 0;
        for (int64_t k = dg[e] + 1; k < ptr[e + 1]; ++k) l = std::max(l, lev_u[col[k]] + 1);
        lev_u[e] = l;
        depth_u = std::max(depth_u, l + 1);
    }
    // rows by level (ascending row index within a level), each level padded to whole warps with -1
    auto level_order = [&](const std::vector<int32_t> &lev, int32_t depth) {
        std::vector<int64_t> start((size_t)depth + 1, 0);
        for (int32_t e = 0; e < no; ++e) ++start[lev[e] + 1];
        for (int32_t l = 0; l < depth; ++l) start[l + 1] = start[l] + (start[l + 1] + 31) / 32 * 32;
        std::vector<int32_t> order((size_t)start[depth], -1);
        std::vector<int64_t> fill(start.begin(), start.end() - 1);
        for (int32_t e = 0; e < no; ++e) order[fill[lev[e]]++] = e;
        return order;
    };
    auto ol = level_order(lev_l, depth_l), ou = level_order(lev_u, depth_u);
    MHD_REQUIRE(ol.size() < INT32_MAX && ou.size() < INT32_MAX, "ILU(0) level order too long");
    L.no = no;
    L.nnz = ptr[no];
    L.depth_l = depth_l;
    L.depth_u = depth_u;
    L.npos_l = (int32_t)ol.size();
    L.npos_u = (int32_t)ou.size();
    L.ptr.upload(p32);
    L.diag.upload(dg);
    L.col.upload(col);
    L.coef.upload(coef);
    L.order_l.upload(ol);
    L.order_u.upload(ou);
    L.val.alloc((size_t)L.nnz);
    L.y.alloc((size_t)std::max(no, 1));
    L.z.alloc((size_t)std::max(ne, 1));
    L.flag.alloc((size_t)std::max(no, 1));
    L.ctl.alloc(1);
    cudaStream_t s = I->mesh->stream;
    MHD_CUDA(cudaMemsetAsync(L.flag.p, 0, (size_t)std::max(no, 1) * sizeof(unsigned), s));
    MHD_CUDA(cudaMemsetAsync(L.ctl.p, 0, sizeof(IluCtl), s));
    if (L.nnz) MHD_CUDA(cudaMemsetAsync(L.val.p, 0, (size_t)L.nnz * sizeof(double), s));
    ilu_unset(L, s);
    int dev = 0, sms = 0;
    MHD_CUDA(cudaGetDevice(&dev));
    MHD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int per_f = 0, per_l = 0, per_u = 0;
    MHD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_f, k_ilu_factor, kIluThreads, 0));
    MHD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_l, k_ilu_trsv<false>, kIluThreads, 0));
    MHD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_u, k_ilu_trsv<true>, kIluThreads, 0));
    L.resident = (int64_t)sms * std::max(1, std::min({per_f, per_l, per_u}));
    ilu_grids(L);
    MHD_CUDA(cudaStreamSynchronize(s));
    L.built = true;
}
} // namespace

void ilu_factor(MhdInduction *I, double dt, const int8_t *dir)
{
    IluState &L = I->ilu;
    if (!L.no) return;
    cudaStream_t s = I->mesh->stream;
    IND_LAUNCH(I, KI_ILU, s, k_ilu_factor<<<L.grid_l, kIluThreads, 0, s>>>(view(I), L.order_l.p, L.npos_l, dt, L.shift, dir));
}

void ilu_apply(MhdInduction *I, const Gate &gt, const double *src, const double *hs, const int8_t *dir, double *vout)
{
    IluState &L = I->ilu;
    const MeshView &m = I->mesh->v;
    cudaStream_t s = I->mesh->stream;
    if (L.no)
    {
        IND_LAUNCH(I, KI_ILU, s,
                   k_ilu_trsv<false><<<L.grid_l, kIluThreads, 0, s>>>(gt, view(I), L.order_l.p, L.npos_l, src, hs, dir, vout, L.y.p, L.z.p));
        IND_LAUNCH(I, KI_ILU, s,
                   k_ilu_trsv<true><<<L.grid_u, kIluThreads, 0, s>>>(gt, view(I), L.order_u.p, L.npos_u, nullptr, nullptr, dir, nullptr, L.y.p,
                                                                     L.z.p));
    }
    if (m.ne > L.no)
        IND_LAUNCH(I, KI_VECTOR, s, k_ilu_tail<<<g1(m.ne - L.no), 256, 0, s>>>(gt, L.no, m.ne, src, hs, vout, L.z.p));
}

// After a solve or an explicit pass: MHD_ECUDA if a wait gave up.
void ilu_check(MhdInduction *I)
{
    IluState &L = I->ilu;
    if (!L.built) return;
    IluCtl c{};
    MHD_CUDA(cudaMemcpyAsync(&c, L.ctl.p, sizeof(IluCtl), cudaMemcpyDeviceToHost, I->mesh->stream));
    MHD_CUDA(cudaStreamSynchronize(I->mesh->stream));
    if (c.err)
    {
        MHD_CUDA(cudaMemsetAsync(L.ctl.p, 0, sizeof(IluCtl), I->mesh->stream));
        MHD_CUDA(cudaMemsetAsync(L.flag.p, 0, (size_t)std::max(L.no, 1) * sizeof(unsigned), I->mesh->stream));
        ilu_unset(L, I->mesh->stream);
        MHD_CUDA(cudaStreamSynchronize(I->mesh->stream));
        throw ApiError(MHD_ECUDA, "ILU(0) pass timed out");
    }
}
} // namespace mhd

using namespace mhd;

extern "C" {

int mhd_gpu_induction_set_ilu(MhdInduction *I, int32_t enable, double shift)
{
    return guarded([&] {
        MHD_REQUIRE(I, "null induction handle");
        MHD_REQUIRE(std::isfinite(shift), "non-finite ILU shift");
        const bool was = I->ilu.on;
        I->ilu.shift = shift;
        I->ilu.on = enable != 0;
        // the reference builds the pattern when the operator is active (:102)
        if (I->ilu.on && !I->ilu.built && (I->resistive || I->hall)) ilu_build(I);
        if (!I->ilu.built) I->ilu.on = false;
        // the captured restart cycles hold the other preconditioner: capture again at the next solve
        if (I->ilu.on != was) drop_cycle_graphs(I);
    });
}

int mhd_gpu_induction_ilu_debug(MhdInduction *I, double wait_s, int32_t unpublished_row)
{
    return guarded([&] {
        MHD_REQUIRE(I, "null induction handle");
        MHD_REQUIRE(wait_s > 0 && wait_s <= 2.0, "wait limit outside (0, 2] s");
        I->ilu.wait_ns = static_cast<uint64_t>(wait_s * 1e9);
        I->ilu.unpublished = unpublished_row;
    });
}

int mhd_gpu_induction_ilu_tune(MhdInduction *I, int32_t window_levels, int32_t max_backoff_ns, int32_t spin_polls)
{
    return guarded([&] {
        MHD_REQUIRE(I, "null induction handle");
        MHD_REQUIRE(window_levels >= 1 && window_levels <= 1024, "window_levels outside [1, 1024]");
        MHD_REQUIRE(max_backoff_ns >= 32 && max_backoff_ns <= 100000, "max_backoff_ns outside [32, 100000]");
        MHD_REQUIRE(spin_polls >= 0 && spin_polls <= 100000, "spin_polls outside [0, 100000]");
        MHD_CUDA(cudaStreamSynchronize(I->mesh->stream));
        I->ilu.window_levels = window_levels;
        I->ilu.backoff_ns = (unsigned)max_backoff_ns;
        I->ilu.spin_polls = (unsigned)spin_polls;
        if (I->ilu.built) ilu_grids(I->ilu);
        // the captured restart cycles hold the old grids
        drop_cycle_graphs(I);
    });
}

int mhd_gpu_induction_ilu_factor(MhdInduction *I, double dt, const int8_t *dir)
{
    return guarded([&] {
        MHD_REQUIRE(I, "null induction handle");
        MHD_REQUIRE(I->ilu.built, "ILU(0) pattern not built (mhd_gpu_induction_set_ilu)");
        ilu_factor(I, dt, dir);
        MHD_LAUNCH_CHECK();
        ilu_check(I);
    });
}

int mhd_gpu_induction_ilu_apply(MhdInduction *I, const int8_t *dir, const double *v, double *z)
{
    return guarded([&] {
        MHD_REQUIRE(I, "null induction handle");
        MHD_REQUIRE(I->ilu.built, "ILU(0) pattern not built (mhd_gpu_induction_set_ilu)");
        MHD_REQUIRE(MHD_ARR(v, I->mesh->v.ne) && MHD_ARR(z, I->mesh->v.ne), "null argument");
        ilu_apply(I, Gate{}, v, nullptr, dir, nullptr);
        if (I->mesh->v.ne)
            MHD_CUDA(cudaMemcpyAsync(z, I->ilu.z.p, (size_t)I->mesh->v.ne * sizeof(double), cudaMemcpyDeviceToDevice, I->mesh->stream));
        MHD_LAUNCH_CHECK();
        ilu_check(I);
    });
}

int mhd_gpu_induction_ilu_arrays(MhdInduction *I, int32_t *n_owned, int64_t *nnz, int64_t *ptr, int32_t *col, double *coef, double *val,
                                 int64_t *diag)
{
    return guarded([&] {
        MHD_REQUIRE(I, "null induction handle");
        IluState &L = I->ilu;
        MHD_CUDA(cudaStreamSynchronize(I->mesh->stream));
        if (n_owned) *n_owned = L.built ? L.no : 0;
        if (nnz) *nnz = L.built ? L.nnz : 0;
        if (!L.built) return;
        if (ptr)
        {
            auto p = down(L.ptr.p, (size_t)L.no + 1);
            for (size_t i = 0; i < p.size(); ++i) ptr[i] = p[i];
        }
        if (diag)
        {
            auto p = down(L.diag.p, (size_t)L.no);
            for (size_t i = 0; i < p.size(); ++i) diag[i] = p[i];
        }
        if (col && L.nnz) MHD_CUDA(cudaMemcpy(col, L.col.p, (size_t)L.nnz * sizeof(int32_t), cudaMemcpyDeviceToHost));
        if (coef && L.nnz) MHD_CUDA(cudaMemcpy(coef, L.coef.p, (size_t)L.nnz * sizeof(double), cudaMemcpyDeviceToHost));
        if (val && L.nnz) MHD_CUDA(cudaMemcpy(val, L.val.p, (size_t)L.nnz * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int mhd_ilu_pattern(int32_t n_edges, int32_t n_owned, int32_t n_faces, const int64_t *e2f_ptr, const int32_t *e2f_idx, const int8_t *e2f_sgn,
                    const int64_t *f2e_ptr, const int32_t *f2e_idx, const int8_t *f2e_sgn, const double *star2, const double *m_edge,
                    int64_t *ptr, int32_t *col, double *coef)
{
    return guarded([&] {
        MHD_REQUIRE(n_edges >= 0 && n_owned >= 0 && n_owned <= n_edges && n_faces >= 0, "bad sizes");
        MHD_REQUIRE(ptr && e2f_ptr && f2e_ptr, "null argument");
        MHD_REQUIRE(MHD_ARR(m_edge, n_edges) && MHD_ARR(star2, n_faces), "null argument");
        std::vector<int64_t> p;
        std::vector<int32_t> c;
        std::vector<double> cf;
        build_pattern(n_owned, e2f_ptr, e2f_idx, e2f_sgn, f2e_ptr, f2e_idx, f2e_sgn, star2, m_edge, p, c, cf);
        std::copy(p.begin(), p.end(), ptr);
        if (col) std::copy(c.begin(), c.end(), col);
        if (coef) std::copy(cf.begin(), cf.end(), coef);
    });
}

} // extern "C"
