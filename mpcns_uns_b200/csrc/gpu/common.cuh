// Shared device-side definitions of the B200 hot path: small-vector arithmetic, strided
// field views, the device mesh, error plumbing of the C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "mhd_gpu.h"

namespace mhd
{
// ---------------------------------------------------------------- errors
struct ApiError : std::runtime_error
{
    int code;
    ApiError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};
void set_last_error(const std::string &msg);

#define MHD_CUDA(call)                                                                                         \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess)                                                                                 \
            throw ::mhd::ApiError(MHD_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));              \
    } while (0)
#define MHD_REQUIRE(cond, msg)                                                                                 \
    do {                                                                                                       \
        if (!(cond)) throw ::mhd::ApiError(MHD_EINVAL, msg);                                                   \
    } while (0)
// an array argument: required unless it holds no entries (an empty rank's vectors may have no storage)
#define MHD_ARR(p, n) ((p) != nullptr || (n) == 0)
#define MHD_LAUNCH_CHECK() MHD_CUDA(cudaGetLastError())

template <class F> int guarded(F &&f)
{
    try
    {
        f();
        return MHD_OK;
    }
    catch (const ApiError &e)
    {
        set_last_error(e.what());
        return e.code;
    }
    catch (const std::exception &e)
    {
        set_last_error(e.what());
        return MHD_EINVAL;
    }
}

// ---------------------------------------------------------------- device buffers
// Every device allocation of the library goes through DBuf; this counts its cudaMalloc and cudaFree
// calls since the library was loaded (mhd_gpu_alloc_calls).
inline std::atomic<int64_t> g_alloc_calls{0};

template <class T> struct DBuf
{
    T *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release()
    {
        if (p)
        {
            cudaFree(p);
            g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
        }
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count)
    {
        if (count == n && p) return;
        release();
        if (count)
        {
            g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
            MHD_CUDA(cudaMalloc(&p, count * sizeof(T)));
        }
        n = count;
    }
    void upload(const T *h, size_t count)
    {
        alloc(count);
        if (count) MHD_CUDA(cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice));
    }
    void upload(const std::vector<T> &v) { upload(v.data(), v.size()); }
    T *get() const { return p; }
};

// ---------------------------------------------------------------- small vectors
struct V3
{
    double x, y, z;
};
__host__ __device__ __forceinline__ V3 mk(double x, double y, double z) { return {x, y, z}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__host__ __device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// std::max / std::min of the reference (first argument wins ties, NaN propagation as in C++):
// keeps signed zeros and ties bit-identical where fmax / fmin may not.
__host__ __device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }

__device__ __forceinline__ V3 ld3(const double *__restrict__ a, int64_t i)
{
    return {__ldg(a + 3 * i), __ldg(a + 3 * i + 1), __ldg(a + 3 * i + 2)};
}
__device__ __forceinline__ void st3(double *a, int64_t i, V3 v)
{
    a[3 * i] = v.x;
    a[3 * i + 1] = v.y;
    a[3 * i + 2] = v.z;
}

// A field of `ncomp` values per entity: value(i, m) = p[i * si + m * sm].  The reference's
// layout (AoS) is si = ncomp, sm = 1; the species-major state of the fused step is si = 1,
// sm = n.
template <class T> struct Field
{
    T *p;
    int64_t si, sm;
    __device__ __forceinline__ T &operator()(int64_t i, int m) const { return p[i * si + m * sm]; }
};
template <class T> inline Field<T> aos(T *p, int ncomp) { return {p, ncomp, 1}; }
template <class T> inline Field<T> soa(T *p, int64_t n) { return {p, 1, n}; }

struct Prim5
{
    double rho, u, v, w, p;
};

// ---------------------------------------------------------------- device mesh
// Plain-pointer view of the device mesh passed to kernels by value.
struct MeshView
{
    int32_t nn, ne, nf, nc, no_cells, no_edges;
    int32_t max_valence; // largest number of faces at an edge
    int32_t max_edge_cells; // largest number of cells at an edge (ec rows)
    int32_t tri_faces;      // 1 when every face is a triangle
    int32_t faces_per_cell; // 4 when every cell is a tetrahedron (c2f row k of cell c at 4c), else 0
    const double *st_dx; // face_center - cell_center per c2f entry (3 each)
    // tetrahedral meshes only: the stencil as structure of arrays over cells, slot j of cell c at
    // [j*nc + c] (coalesced warp loads): neighbour code, c2f sign, w*d (3 per slot), dx (3 per slot), inverse (6)
    const int32_t *t_nb;
    const int8_t *t_sg;
    const double *t_wd, *t_dx, *t_inv;
    const int32_t *c2f_ptr, *c2f_idx;
    const int8_t *c2f_sgn;
    const int32_t *f2e_ptr, *f2e_idx;
    const int8_t *f2e_sgn;
    const int32_t *e2f_ptr, *e2f_idx;
    const int8_t *e2f_sgn;
    const int32_t *f2c_ptr, *f2c_idx;
    const int8_t *f2c_sgn;
    const int32_t *face_L, *face_R; // cell with c2f sign +1 / -1 (canonical normal from L to R), -1 if none
    const int32_t *cfa_idx;         // c2f rows re-ordered by ascending face id (the reference's scatter order)
    const int8_t *cfa_sgn;
    const int8_t *material, *face_kind, *edge_mode;
    const double *edge_vec, *edge_mid, *edge_len;
    const double *face_area, *face_center, *face_area_mag;
    const double *cell_center, *cell_volume;
    const int32_t *ec_ptr, *ec_cell;
    const double *ec_weight, *ef_weight, *star1, *star2;
    // least-squares stencil of mhd::Stencil (per c2f entry / per cell)
    const int32_t *st_nb;    // neighbour cell, -(f+1) for a virtual boundary neighbour, INT32_MIN for a skipped face
    const double *st_wd;     // w * d (3 per c2f entry)
    const double *st_inv;    // 6 per cell: I00 I01 I02 I11 I12 I22 of the symmetric inverse
    const int8_t *st_valid;  // per cell
    // optional (the mesh descriptor's edge_nodes): start and end node per edge, and per node its fluid
    // cells in ascending order (mercury::AmbipolarEMF's node lists); null without edge_nodes
    const int32_t *e_nodes;
    const int32_t *n2c_ptr, *n2c_cell;
};

constexpr int kMaxValence = 32; // faces per edge handled by the UCT edge kernel (checked at mesh creation)

inline int grid_for(int64_t n, int block) { return static_cast<int>((n + block - 1) / block); }

// Per-kernel-class device time: CUDA event pairs recorded on the launching stream while `on`;
// events are created on first use and reused after each read.
template <int N> struct EventProfiler
{
    bool on = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[N];
    size_t used[N] = {};
    ~EventProfiler()
    {
        for (auto &v : ev)
            for (auto &p : v)
            {
                cudaEventDestroy(p.first);
                cudaEventDestroy(p.second);
            }
    }
    void begin(int k, cudaStream_t s)
    {
        if (!on) return;
        if (used[k] == ev[k].size())
        {
            cudaEvent_t a, b;
            MHD_CUDA(cudaEventCreate(&a));
            MHD_CUDA(cudaEventCreate(&b));
            ev[k].emplace_back(a, b);
        }
        MHD_CUDA(cudaEventRecord(ev[k][used[k]].first, s));
    }
    void end(int k, cudaStream_t s)
    {
        if (!on) return;
        MHD_CUDA(cudaEventRecord(ev[k][used[k]].second, s));
        ++used[k];
    }
    // summed milliseconds and launch count of class k since the last read (the stream must be idle)
    void read(int k, double &ms_total, int64_t &count)
    {
        double tot = 0;
        for (size_t i = 0; i < used[k]; ++i)
        {
            float ms = 0;
            MHD_CUDA(cudaEventElapsedTime(&ms, ev[k][i].first, ev[k][i].second));
            tot += ms;
        }
        ms_total = tot;
        count = static_cast<int64_t>(used[k]);
        used[k] = 0;
    }
};
} // namespace mhd

struct MhdMesh
{
    mhd::MeshView v{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    mhd::DBuf<int32_t> c2f_ptr, c2f_idx, f2e_ptr, f2e_idx, e2f_ptr, e2f_idx, f2c_ptr, f2c_idx, face_L, face_R, ec_ptr, ec_cell, st_nb,
        cfa_idx;
    mhd::DBuf<int8_t> c2f_sgn, f2e_sgn, e2f_sgn, f2c_sgn, material, face_kind, edge_mode, st_valid, cfa_sgn;
    mhd::DBuf<double> edge_vec, edge_mid, edge_len, face_area, face_center, face_area_mag, cell_center, cell_volume, ec_weight,
        ef_weight, star1, star2, st_wd, st_inv, st_dx, t_wd, t_dx, t_inv;
    mhd::DBuf<int32_t> t_nb, e_nodes, n2c_ptr, n2c_cell;
    mhd::DBuf<int8_t> t_sg;
    // scratch reused across calls (stream ordered): face fluxes, face EMF candidates, reductions
    mhd::DBuf<double> scratch_face, scratch_face3, scratch_red;
    mhd::DBuf<double> host_red_dummy;
    double *pinned = nullptr; // small pinned buffer for reduction results
    ~MhdMesh();
};
