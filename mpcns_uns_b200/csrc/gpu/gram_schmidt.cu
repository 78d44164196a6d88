// Classical Gram-Schmidt of the GMRES Arnoldi step (gmres.cu enqueues it): the Krylov basis orthogonalisation
// in FP64, in its own translation unit so that its dot products and updates contract into fused
// multiply-adds.  Its rounding is not the reference's in any case (the reference runs modified Gram-Schmidt
// with sequential sums); GMRES holds it to the solver's tolerance.
#include <array>
#include <utility>

#include "induction_op.cuh"

namespace mhd
{
namespace
{
// ---------------------------------------------------------------- classical Gram-Schmidt, twice if needed
// The Arnoldi step orthogonalises w against V_0..V_j with classical Gram-Schmidt and one conditional
// re-orthogonalisation (the "twice is enough" criterion: again only if |w'| < |w| / sqrt(2), Giraud,
// Langou, Rozloznik, "The loss of orthogonality in the Gram-Schmidt orthogonalization process", Comput.
// Math. Appl. 50, 2005), skipped when the dots of the first result against the basis, which the update
// pass forms anyway, are already at round-off (|V^T w'| <= 1e-12 |w'|: the new vector is orthogonal to
// working accuracy).  It spans the same space and produces the same Hessenberg column as the
// reference's modified Gram-Schmidt (ImplicitInduction.cpp:340-345) up to rounding, in two or three
// passes over the basis instead of j + 1: every pass reads w and V_0..V_j once and forms all its dot
// products together.

// Warp reduce-scatter of 32 partial sums: afterwards lane l holds the warp's sum of acc[l] in acc[0].
__device__ __forceinline__ double warp_reduce_scatter32(double (&acc)[32])
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1)
    {
        const bool up = lane & o;
#pragma unroll
        for (int k = 0; k < o; ++k)
        {
            const double send = up ? acc[k] : acc[k + o];
            const double keep = up ? acc[k + o] : acc[k];
            acc[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return acc[0];
}

// The 32 grid-wide sums whose warp sums lane l of every warp holds for index l: block partials, then the
// last block to finish adds them (in a fixed order: deterministic) into out[0..31] and re-arms the counter.
// Returns true in that last block (all of its threads), after out is written and visible to them.
__device__ __forceinline__ bool grid_sum32(double v, double *part, unsigned *counter, double *out)
{
    __shared__ double sh[8][32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    sh[wid][lane] = v;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w][threadIdx.x];
        part[(int64_t)blockIdx.x * 32 + threadIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // every thread of the last block: value v = t % 32 over the blocks b = t / 32 (mod warps), four
    // accumulators so that the loads overlap; then the warps' sums in warp order
    {
        const int k = threadIdx.x >> 5, nk = blockDim.x >> 5;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        unsigned b = k;
        for (; b + 3u * nk < gridDim.x; b += 4u * nk)
        {
            a0 += __ldcg(part + (int64_t)b * 32 + lane);
            a1 += __ldcg(part + (int64_t)(b + nk) * 32 + lane);
            a2 += __ldcg(part + (int64_t)(b + 2 * nk) * 32 + lane);
            a3 += __ldcg(part + (int64_t)(b + 3 * nk) * 32 + lane);
        }
        for (; b < gridDim.x; b += nk) a0 += __ldcg(part + (int64_t)b * 32 + lane);
        sh[k][lane] = (a0 + a1) + (a2 + a3);
    }
    __syncthreads();
    if (threadIdx.x < 32)
    {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w][threadIdx.x];
        out[threadIdx.x] = s;
    }
    if (threadIdx.x == 0) *counter = 0;
    __syncthreads();
    return true;
}

// The passes are instantiated for every number NV = j + 1 of basis vectors (1..31), so that a thread
// holds exactly NV + 1 running sums and NV basis values, all loads are unconditional and the registers
// (and so the resident warps) follow the column.  A thread adds its edges' products into its running
// sums; the sums meet once, at the end, in the warp reduce-scatter and the grid tail.

// Both passes stream NV (+2) vectors tile by tile: a block of kGsThreads threads takes tiles of kGsThreads
// consecutive edges, and while it works on one tile the next tiles' values are already on their way into
// shared memory (cp.async, kGsStages stages, each thread copying and reading only its own column: no block
// barrier), so that a thread keeps many loads in flight without holding them in registers.  8-byte copies:
// the basis vectors start at i * ldv, which need not be 16-byte aligned.
constexpr int kGsThreads = 128;
constexpr int kGsStages = 3; // tiles in flight per block: the one being read and kGsStages - 1 ahead
__device__ __forceinline__ void cp_async8(double *smem, const double *gmem)
{
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Pass 1: h_i = V_i . w (i < NV) into H(i, j), and |w|^2 into red[32], over the owned edges.  red holds 96
// doubles: [0, 31) the re-orthogonalisation dots, [32] |w|^2 before the update, [64, 96) the last pass's sums.
// Dynamic shared memory: kGsStages stages x (NV + 1) vectors x kGsThreads doubles.
template <int NV>
__global__ void __launch_bounds__(kGsThreads) k_cgs_dots(Gate gt, const double *__restrict__ w, const double *__restrict__ V, int64_t ldv,
                                                          int32_t n_owned, double *part, unsigned *counter, double *red, double *H, int mcols)
{
    if (gt.off()) return;
    constexpr int j = NV - 1, NVEC = NV + 1;
    extern __shared__ double sm[];
    const int tid = threadIdx.x;
    const int64_t ntiles = (n_owned + kGsThreads - 1) / kGsThreads;
    auto issue = [&](int64_t tile, int stage) {
        const int64_t e = tile * kGsThreads + tid;
        if (e < n_owned)
        {
            double *col = sm + (int64_t)stage * NVEC * kGsThreads + tid;
#pragma unroll
            for (int i = 0; i < NV; ++i) cp_async8(col + i * kGsThreads, V + i * ldv + e);
            cp_async8(col + NV * kGsThreads, w + e);
        }
        cp_async_commit();
    };
    double acc[NV + 1];
#pragma unroll
    for (int i = 0; i <= NV; ++i) acc[i] = 0.0;
    int64_t tile = blockIdx.x;
#pragma unroll
    for (int q = 0; q < kGsStages - 1; ++q) issue(tile + q * gridDim.x, q);
    for (int k = 0; tile < ntiles; ++k, tile += gridDim.x)
    {
        issue(tile + (kGsStages - 1) * (int64_t)gridDim.x, (k + kGsStages - 1) % kGsStages); // past the end: an empty group
        cp_async_wait<kGsStages - 1>();
        const int64_t e = tile * kGsThreads + tid;
        if (e < n_owned)
        {
            const double *col = sm + (int64_t)(k % kGsStages) * NVEC * kGsThreads + tid;
            const double we = col[NV * kGsThreads];
#pragma unroll
            for (int i = 0; i < NV; ++i) acc[i] += col[i * kGsThreads] * we;
            acc[NV] += we * we;
        }
    }
    cp_async_wait<0>();
    double p[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) p[i] = i < NV ? acc[i] : (i == 31 ? acc[NV] : 0.0);
    if (!grid_sum32(warp_reduce_scatter32(p), part, counter, red + 64)) return;
    if (threadIdx.x <= j) H[threadIdx.x * mcols + j] = red[64 + threadIdx.x];
    if (threadIdx.x == 31) red[32] = red[64 + 31];
}

// Pass 2 (and 3): w -= sum_i c_i V_i on every edge, with c = H(:, j) (pass 2) or the re-orthogonalisation
// dots red[0..j] (pass 3); the next face pass's input zs = w * pd; and over the owned edges the dots
// s_i = V_i . w and |w|^2 of the result.  Pass 2 (reorth == 0) then decides: if the subtraction cancelled
// (|w|^2 < |w_before|^2 / 2, red[32] holds |w_before|^2 from pass 1) and the remaining components along
// the basis are above round-off (|s| > 1e-12 |w|), it leaves s in red[0..j] and raises ctl->reorth; else it
// stores H(j+1, j) = |w|.  Pass 3 (reorth == 1) runs only when raised: it adds c to H(:, j), stores
// H(j+1, j) = |w| and lowers the flag.  reverse: the tiles in descending order (the previous pass's tail is
// in L2).  Dynamic shared memory: kGsStages stages x (NV + 2) vectors (the basis, w, pd) x kGsThreads doubles.
template <int NV, bool F32>
__global__ void __launch_bounds__(kGsThreads) k_cgs_update(Gate gt, Ctl *ctl, int reorth, double *__restrict__ w, const double *__restrict__ V,
                                                            int64_t ldv, int32_t n_all, int32_t n_owned, int reverse, double *part,
                                                            unsigned *counter, double *red, double *H, int mcols,
                                                            const double *__restrict__ pd, double *__restrict__ zs, float *__restrict__ zs32)
{
    if (gt.off() || (reorth && !ctl->reorth)) return;
    constexpr int j = NV - 1, NVEC = NV + 2;
    extern __shared__ double sm[];
    __shared__ double csh[NV];
    const int tid = threadIdx.x;
    if (tid < NV) csh[tid] = reorth ? red[tid] : H[tid * mcols + j];
    __syncthreads();
    const int64_t ntiles = (n_all + kGsThreads - 1) / kGsThreads;
    auto tile_of = [&](int64_t t) { return reverse ? ntiles - 1 - t : t; };
    auto issue = [&](int64_t t, int stage) {
        const int64_t e = t < ntiles ? tile_of(t) * kGsThreads + tid : n_all;
        if (e < n_all)
        {
            double *col = sm + (int64_t)stage * NVEC * kGsThreads + tid;
#pragma unroll
            for (int i = 0; i < NV; ++i) cp_async8(col + i * kGsThreads, V + i * ldv + e);
            cp_async8(col + NV * kGsThreads, w + e);
            cp_async8(col + (NV + 1) * kGsThreads, pd + e);
        }
        cp_async_commit();
    };
    double acc[NV + 1];
#pragma unroll
    for (int i = 0; i <= NV; ++i) acc[i] = 0.0;
    int64_t t = blockIdx.x;
#pragma unroll
    for (int q = 0; q < kGsStages - 1; ++q) issue(t + q * gridDim.x, q);
    for (int k = 0; t < ntiles; ++k, t += gridDim.x)
    {
        issue(t + (kGsStages - 1) * (int64_t)gridDim.x, (k + kGsStages - 1) % kGsStages);
        cp_async_wait<kGsStages - 1>();
        const int64_t e = tile_of(t) * kGsThreads + tid;
        if (e < n_all)
        {
            const double *col = sm + (int64_t)(k % kGsStages) * NVEC * kGsThreads + tid;
            double we = col[NV * kGsThreads];
#pragma unroll
            for (int i = 0; i < NV; ++i) we -= csh[i] * col[i * kGsThreads];
            w[e] = we;
            const double z = we * col[(NV + 1) * kGsThreads];
            if (F32) zs32[e] = static_cast<float>(z);
            else zs[e] = z;
            if (e < n_owned)
            {
#pragma unroll
                for (int i = 0; i < NV; ++i) acc[i] += col[i * kGsThreads] * we;
                acc[NV] += we * we;
            }
        }
    }
    cp_async_wait<0>();
    double p[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) p[i] = i < NV ? acc[i] : (i == 31 ? acc[NV] : 0.0);
    // the sums of s and |w|^2 go to red[64..95]; red[32] keeps |w_before|^2 of pass 1
    const bool last = grid_sum32(warp_reduce_scatter32(p), part, counter, red + 64);
    if (!last || threadIdx.x != 0) return;
    const double nn = red[64 + 31];
    double ss = 0.0;
    for (int i = 0; i < NV; ++i) ss += red[64 + i] * red[64 + i];
    if (!reorth && nn < 0.5 * red[32] && ss > 1e-24 * nn)
    {
        for (int i = 0; i < NV; ++i) red[i] = red[64 + i];
        ctl->reorth = 1;
        ++ctl->n_reorth;
        return;
    }
    if (reorth)
        for (int i = 0; i < NV; ++i) H[i * mcols + j] += csh[i];
    H[(j + 1) * mcols + j] = sqrt(nn);
    ctl->reorth = 0;
}

// Launchers of the instances for NV = 1..31, and their grids (resident blocks on every SM)
constexpr size_t gs_smem(int nvec) { return size_t(kGsStages) * nvec * kGsThreads * sizeof(double); }
template <int NV> void cgs_step(const CgsArgs &a, const int *grid, cudaStream_t s, int pass)
{
    if (pass == 0)
        k_cgs_dots<NV><<<grid[0], kGsThreads, gs_smem(NV + 1), s>>>(a.gt, a.w, a.V, a.ldv, a.n_owned, a.part, a.counter, a.red, a.H,
                                                                    a.mcols);
    else if (a.zs32)
        k_cgs_update<NV, true><<<grid[1], kGsThreads, gs_smem(NV + 2), s>>>(a.gt, a.ctl, pass - 1, a.w, a.V, a.ldv, a.n_all, a.n_owned,
                                                                            pass == 1, a.part, a.counter, a.red, a.H, a.mcols, a.pd,
                                                                            nullptr, a.zs32);
    else
        k_cgs_update<NV, false><<<grid[1], kGsThreads, gs_smem(NV + 2), s>>>(a.gt, a.ctl, pass - 1, a.w, a.V, a.ldv, a.n_all, a.n_owned,
                                                                             pass == 1, a.part, a.counter, a.red, a.H, a.mcols, a.pd,
                                                                             a.zs, nullptr);
}
// the instances' shared memory opted in, and their resident grids (the partials buffer holds kRedBlocks)
template <int NV> void cgs_grids(int sms, int *grid)
{
    const int sd = static_cast<int>(gs_smem(NV + 1)), su = static_cast<int>(gs_smem(NV + 2));
    MHD_CUDA(cudaFuncSetAttribute(k_cgs_dots<NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, sd));
    MHD_CUDA(cudaFuncSetAttribute(k_cgs_update<NV, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, su));
    MHD_CUDA(cudaFuncSetAttribute(k_cgs_update<NV, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, su));
    int per = 0;
    MHD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cgs_dots<NV>, kGsThreads, sd));
    grid[0] = std::max(1, std::min(kRedBlocks, sms * std::max(per, 1)));
    MHD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cgs_update<NV, false>, kGsThreads, su));
    int per32 = 0;
    MHD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per32, k_cgs_update<NV, true>, kGsThreads, su));
    grid[1] = std::max(1, std::min(kRedBlocks, sms * std::max(std::min(per, per32), 1)));
}
using CgsStepFn = void (*)(const CgsArgs &, const int *, cudaStream_t, int);
using CgsGridFn = void (*)(int, int *);
template <int... N> constexpr std::array<CgsStepFn, sizeof...(N)> cgs_step_table(std::integer_sequence<int, N...>)
{
    return {cgs_step<N + 1>...};
}
template <int... N> constexpr std::array<CgsGridFn, sizeof...(N)> cgs_grid_table(std::integer_sequence<int, N...>)
{
    return {cgs_grids<N + 1>...};
}
const std::array<CgsStepFn, kCgsMax> kCgsStep = cgs_step_table(std::make_integer_sequence<int, kCgsMax>{});
const std::array<CgsGridFn, kCgsMax> kCgsGrid = cgs_grid_table(std::make_integer_sequence<int, kCgsMax>{});

} // namespace

void cgs_launch(int j, const CgsArgs &a, const int *grid, cudaStream_t s, int pass) { kCgsStep[j](a, grid, s, pass); }
void cgs_grids_for(int k, int sms, int *grid) { kCgsGrid[k](sms, grid); }
} // namespace mhd
