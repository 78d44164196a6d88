// nvcc-flags: -fmad=false
// uns::compute_geometry (src/uns/geometry/Geometry.cpp:17-169) on the device: edge, face and cell metric,
// the edge -> cell lists, the dual measures star0..star3 and the UCT weights, bit-identical to the host
// computation.  Every sum the reference accumulates by scattering from the cell loop is gathered here
// per entity in the same order (cells ascending, then the cell's faces, then the face loop), and every
// expression keeps the reference's operation order (no multiply-add contraction).
#include <algorithm>
#include <cfloat>
#include <vector>

#include "common.cuh"

namespace mhd
{
namespace
{
constexpr int kLoop = 16;   // nodes per face loop
constexpr int kCellN = 64;  // distinct nodes per cell
constexpr int kEdgeC = 64;  // cells around an edge
constexpr int kNodeC = 256; // cells around a node

struct GeoView
{
    int32_t nn, ne, nf, nc;
    const double *x;
    const int32_t *en; // start, end per edge
    const int32_t *f2e_ptr, *f2e_idx, *c2f_ptr, *c2f_idx, *e2f_ptr, *e2f_idx, *f2c_ptr, *f2c_idx;
    const int8_t *f2e_sgn, *c2f_sgn;
};

__device__ __forceinline__ V3 X(const GeoView &g, int32_t v) { return ld3(g.x, v); }
__device__ __forceinline__ double norm3(V3 a) { return sqrt(dot(a, a)); }

// uns::CellComplex::face_loop: the node at which each edge of the face is entered
__device__ __forceinline__ int face_loop(const GeoView &g, int32_t f, int32_t *loop, int *err)
{
    const int32_t q0 = g.f2e_ptr[f], k = g.f2e_ptr[f + 1] - q0;
    if (k > kLoop)
    {
        atomicOr(err, 1);
        return 0;
    }
    for (int i = 0; i < k; ++i)
    {
        const int32_t e = g.f2e_idx[q0 + i];
        loop[i] = g.f2e_sgn[q0 + i] > 0 ? g.en[2 * (int64_t)e] : g.en[2 * (int64_t)e + 1];
    }
    return k;
}

__device__ __forceinline__ void sort_small(int32_t *a, int n)
{
    for (int i = 1; i < n; ++i)
        for (int j = i; j > 0 && a[j - 1] > a[j]; --j)
        {
            const int32_t t = a[j - 1];
            a[j - 1] = a[j];
            a[j] = t;
        }
}

// insert v into the ascending distinct list a[0..n) (capacity cap); returns the new length, -1 if full
__device__ __forceinline__ int insert_unique(int32_t *a, int n, int cap, int32_t v)
{
    int i = n;
    while (i > 0 && a[i - 1] > v) --i;
    if (i > 0 && a[i - 1] == v) return n;
    if (n == cap) return -1;
    for (int j = n; j > i; --j) a[j] = a[j - 1];
    a[i] = v;
    return n + 1;
}

__device__ __forceinline__ int unique_sorted(int32_t *a, int n)
{
    int m = 0;
    for (int i = 0; i < n; ++i)
        if (m == 0 || a[m - 1] != a[i]) a[m++] = a[i];
    return m;
}

__global__ void k_geo_edges(GeoView g, double *__restrict__ vec, double *__restrict__ mid, double *__restrict__ len)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= g.ne) return;
    const V3 a = X(g, g.en[2 * (int64_t)e]), b = X(g, g.en[2 * (int64_t)e + 1]);
    const V3 v = b - a;
    st3(vec, e, v);
    st3(mid, e, 0.5 * (a + b));
    len[e] = norm3(v);
}

__global__ void k_geo_faces(GeoView g, double *__restrict__ area, double *__restrict__ center, double *__restrict__ mag, int *err)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= g.nf) return;
    int32_t loop[kLoop];
    const int k = face_loop(g, f, loop, err);
    if (k == 0) return;
    V3 p0 = mk(0, 0, 0);
    for (int i = 0; i < k; ++i) p0 = p0 + X(g, loop[i]);
    p0 = (1.0 / static_cast<double>(k)) * p0;
    V3 cw = mk(0, 0, 0);
    double wsum = 0;
    for (int i = 0; i < k; ++i)
    {
        const V3 a = X(g, loop[i]), b = X(g, loop[(i + 1) % k]);
        const double w = 0.5 * norm3(cross(a - p0, b - p0));
        cw = cw + w * ((1.0 / 3.0) * (p0 + a + b));
        wsum += w;
    }
    const V3 c = wsum > 0 ? (1.0 / wsum) * cw : p0;
    V3 A = mk(0, 0, 0);
    for (int i = 0; i < k; ++i) A = A + 0.5 * cross(X(g, loop[i]) - c, X(g, loop[(i + 1) % k]) - c);
    st3(center, f, c);
    st3(area, f, A);
    mag[f] = norm3(A);
}

// the cells around each edge (those of its faces), ascending: count (fill == null) or fill
__global__ void k_geo_ec(GeoView g, const int64_t *__restrict__ ptr, int32_t *__restrict__ count, int32_t *__restrict__ fill, int *err)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= g.ne) return;
    int32_t t[kEdgeC];
    int n = 0;
    for (int32_t k = g.e2f_ptr[e]; k < g.e2f_ptr[e + 1]; ++k)
    {
        const int32_t f = g.e2f_idx[k];
        for (int32_t q = g.f2c_ptr[f]; q < g.f2c_ptr[f + 1]; ++q)
        {
            if (n == kEdgeC)
            {
                atomicOr(err, 2);
                return;
            }
            t[n++] = g.f2c_idx[q];
        }
    }
    sort_small(t, n);
    n = unique_sorted(t, n);
    if (!fill) count[e] = n;
    else
        for (int i = 0; i < n; ++i) fill[ptr[e] + i] = t[i];
}

// cell centre (volume-weighted centroid of the tetrahedra on the faces about the node mean), volume,
// smallest sub-tetrahedron, star3
__global__ void k_geo_cells(GeoView g, const double *__restrict__ fc, double *__restrict__ cc, double *__restrict__ vol,
                            double *__restrict__ mintet, double *__restrict__ star3, int *err)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nc) return;
    int32_t cn[kCellN], loop[kLoop];
    int n = 0;
    for (int32_t kf = g.c2f_ptr[c]; kf < g.c2f_ptr[c + 1]; ++kf)
    {
        const int k = face_loop(g, g.c2f_idx[kf], loop, err);
        for (int i = 0; i < k; ++i)
        {
            n = insert_unique(cn, n, kCellN, loop[i]);
            if (n < 0)
            {
                atomicOr(err, 4);
                return;
            }
        }
    }
    V3 xc0 = mk(0, 0, 0);
    for (int i = 0; i < n; ++i) xc0 = xc0 + X(g, cn[i]);
    xc0 = (1.0 / static_cast<double>(n)) * xc0;
    double vsum = 0;
    V3 vc = mk(0, 0, 0);
    for (int32_t kf = g.c2f_ptr[c]; kf < g.c2f_ptr[c + 1]; ++kf)
    {
        const int32_t f = g.c2f_idx[kf];
        const int s = g.c2f_sgn[kf];
        const int k = face_loop(g, f, loop, err);
        const V3 cf = ld3(fc, f);
        for (int i = 0; i < k; ++i)
        {
            const V3 a = X(g, loop[i]), b = X(g, loop[(i + 1) % k]);
            const V3 at = (0.5 * s) * cross(a - cf, b - cf);
            const double vt = dot(at, cf - xc0) / 3.0;
            vc = vc + vt * (0.25 * (xc0 + cf + a + b));
            vsum += vt;
        }
    }
    const V3 xc = vsum > 0 ? (1.0 / vsum) * vc : xc0;
    st3(cc, c, xc);
    double v = 0, mt = DBL_MAX;
    for (int32_t kf = g.c2f_ptr[c]; kf < g.c2f_ptr[c + 1]; ++kf)
    {
        const int32_t f = g.c2f_idx[kf];
        const int s = g.c2f_sgn[kf];
        const int k = face_loop(g, f, loop, err);
        const V3 cf = ld3(fc, f);
        for (int i = 0; i < k; ++i)
        {
            const V3 a = X(g, loop[i]), b = X(g, loop[(i + 1) % k]);
            const V3 at = (0.5 * s) * cross(a - cf, b - cf);
            const double vt = dot(at, cf - xc) / 3.0;
            v += vt;
            mt = dmin(mt, vt);
        }
    }
    vol[c] = v;
    mintet[c] = mt;
    star3[c] = v > 0 ? 1.0 / v : 0.0;
}

// star2 = (sum over the face's cells of |x_f - x_c|) / |A_f|
__global__ void k_geo_face_dual(GeoView g, const double *__restrict__ fc, const double *__restrict__ mag, const double *__restrict__ cc,
                                double *__restrict__ star2)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= g.nf) return;
    double d = 0;
    const V3 cf = ld3(fc, f);
    for (int32_t q = g.f2c_ptr[f]; q < g.f2c_ptr[f + 1]; ++q) d += norm3(cf - ld3(cc, g.f2c_idx[q]));
    star2[f] = mag[f] > 0 ? d / mag[f] : 0.0;
}

// per edge: the dual area pieces 1/2 s (x_c - m_e) x (x_f - m_e) of its cells' faces, in the reference's
// scatter order; the misoriented count, the per-cell and per-face UCT weights (normalised), star1
__global__ void k_geo_edge_dual(GeoView g, const double *__restrict__ fc, const double *__restrict__ cc, const double *__restrict__ mid,
                                const double *__restrict__ evec, const double *__restrict__ len, const int64_t *__restrict__ ecp,
                                const int32_t *__restrict__ ecc, double *__restrict__ ecw, double *__restrict__ efw,
                                double *__restrict__ dual, int32_t *__restrict__ mis, double *__restrict__ star1, int *err)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= g.ne) return;
    const int32_t j0 = g.e2f_ptr[e], nfe = g.e2f_ptr[e + 1] - j0;
    if (nfe > kMaxValence)
    {
        atomicOr(err, 8);
        return;
    }
    double wf[kMaxValence];
    for (int j = 0; j < nfe; ++j) wf[j] = 0.0;
    const V3 me = ld3(mid, e), ev = ld3(evec, e);
    V3 da = mk(0, 0, 0);
    int32_t nmis = 0;
    for (int64_t kc = ecp[e]; kc < ecp[e + 1]; ++kc)
    {
        const int32_t c = ecc[kc];
        const V3 xc = ld3(cc, c);
        double wc = 0.0;
        for (int32_t kf = g.c2f_ptr[c]; kf < g.c2f_ptr[c + 1]; ++kf)
        {
            const int32_t f = g.c2f_idx[kf];
            const int s = g.c2f_sgn[kf];
            const V3 cf = ld3(fc, f);
            for (int32_t q = g.f2e_ptr[f]; q < g.f2e_ptr[f + 1]; ++q)
            {
                if (g.f2e_idx[q] != e) continue;
                const int se = s * g.f2e_sgn[q];
                const V3 piece = (0.5 * se) * cross(xc - me, cf - me);
                da = da + piece;
                if (dot(piece, ev) <= 0) ++nmis;
                const double pn = norm3(piece);
                wc += pn;
                for (int j = 0; j < nfe; ++j)
                    if (g.e2f_idx[j0 + j] == f) wf[j] += pn;
            }
        }
        ecw[kc] = wc;
    }
    double s = 0;
    for (int64_t kc = ecp[e]; kc < ecp[e + 1]; ++kc) s += ecw[kc];
    if (s > 0)
    {
        for (int64_t kc = ecp[e]; kc < ecp[e + 1]; ++kc) ecw[kc] /= s;
        for (int j = 0; j < nfe; ++j) wf[j] /= s;
    }
    for (int j = 0; j < nfe; ++j) efw[j0 + j] = wf[j];
    st3(dual, e, da);
    mis[e] = nmis;
    star1[e] = len[e] > 0 ? norm3(da) / len[e] : 0.0;
}

// node -> cells containing it: count (fill == null) or fill (unordered; k_geo_node_sort orders each row)
__global__ void k_geo_n2c(GeoView g, const int64_t *__restrict__ ptr, int32_t *__restrict__ count, int32_t *__restrict__ cursor,
                          int32_t *__restrict__ fill, int *err)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nc) return;
    int32_t cn[kCellN], loop[kLoop];
    int n = 0;
    for (int32_t kf = g.c2f_ptr[c]; kf < g.c2f_ptr[c + 1]; ++kf)
    {
        const int k = face_loop(g, g.c2f_idx[kf], loop, err);
        for (int i = 0; i < k; ++i)
        {
            n = insert_unique(cn, n, kCellN, loop[i]);
            if (n < 0)
            {
                atomicOr(err, 4);
                return;
            }
        }
    }
    for (int i = 0; i < n; ++i)
    {
        if (!fill) atomicAdd(count + cn[i], 1);
        else fill[ptr[cn[i]] + atomicAdd(cursor + cn[i], 1)] = c;
    }
}

__global__ void k_geo_node_sort(int32_t nn, const int64_t *__restrict__ ptr, int32_t *__restrict__ cells, int *err)
{
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    const int64_t a = ptr[v], n = ptr[v + 1] - a;
    if (n > kNodeC)
    {
        atomicOr(err, 16);
        return;
    }
    sort_small(cells + a, static_cast<int>(n));
}

// star0: half of every sub-tetrahedron volume to each of its two loop nodes, gathered per node over its
// cells ascending, then the cell's faces and loop positions (the reference's scatter order)
__global__ void k_geo_star0(GeoView g, const int64_t *__restrict__ ptr, const int32_t *__restrict__ cells, const double *__restrict__ fc,
                            const double *__restrict__ cc, double *__restrict__ star0, int *err)
{
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= g.nn) return;
    int32_t loop[kLoop];
    double s0 = 0.0;
    for (int64_t q = ptr[v]; q < ptr[v + 1]; ++q)
    {
        const int32_t c = cells[q];
        const V3 xc = ld3(cc, c);
        for (int32_t kf = g.c2f_ptr[c]; kf < g.c2f_ptr[c + 1]; ++kf)
        {
            const int32_t f = g.c2f_idx[kf];
            const int s = g.c2f_sgn[kf];
            const int k = face_loop(g, f, loop, err);
            const V3 cf = ld3(fc, f);
            for (int i = 0; i < k; ++i)
            {
                const int32_t va = loop[i], vb = loop[(i + 1) % k];
                if (va != v && vb != v) continue;
                const V3 at = (0.5 * s) * cross(X(g, va) - cf, X(g, vb) - cf);
                const double vt = dot(at, cf - xc) / 3.0;
                if (va == v) s0 += 0.5 * vt;
                if (vb == v) s0 += 0.5 * vt;
            }
        }
    }
    star0[v] = s0;
}

template <class T> void down(T *host, const DBuf<T> &d, size_t n)
{
    if (host && n) MHD_CUDA(cudaMemcpy(host, d.p, n * sizeof(T), cudaMemcpyDeviceToHost));
}

// mhd::BoundaryInfo::build (Common/boundary/BoundaryInfo.cpp:9-49), face loop: the kind of every face from its
// cells' materials, its tag's boundary type (type_of[tag] for 0 < tag < n_tags, else type_none: 1 wall,
// 2 inflow, 3 outflow, 5 farfield, 0 unknown, which raises *err) and, on farfield faces, the side of u_inf.
__global__ void k_bc_faces(int32_t nf, const int32_t *__restrict__ f2c_ptr, const int32_t *__restrict__ f2c_idx,
                           const int8_t *__restrict__ f2c_sgn, const int32_t *__restrict__ material, const int32_t *__restrict__ face_tag,
                           const double *__restrict__ face_area, const double *__restrict__ face_area_mag, int32_t n_tags,
                           const int8_t *__restrict__ type_of, int8_t type_none, V3 u_inf, int8_t *__restrict__ kind, int *err)
{
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int32_t b = f2c_ptr[f];
    if (f2c_ptr[f + 1] - b == 2)
    {
        const bool s0 = material[f2c_idx[b]] == 1, s1 = material[f2c_idx[b + 1]] == 1;
        kind[f] = (s0 && s1) ? 4 : (s0 || s1) ? 1 : 0;
        return;
    }
    if (material[f2c_idx[b]] == 1)
    {
        kind[f] = 4;
        return;
    }
    const int32_t tag = face_tag[f];
    const int8_t type = tag > 0 && tag < n_tags ? type_of[tag] : type_none;
    if (type == 1 || type == 2 || type == 3) kind[f] = type;
    else if (type == 5)
    {
        const double sc = f2c_sgn[b] / face_area_mag[f];
        const V3 n = sc * ld3(face_area, f);
        kind[f] = dot(u_inf, n) < 0 ? 2 : 3;
    }
    else
    {
        kind[f] = 0;
        atomicOr(err, 1);
    }
}

// its edge loop: an edge of a wall face is a wall edge (1), else an edge of an inflow face an inflow edge (2)
__global__ void k_bc_edges(int32_t ne, const int32_t *__restrict__ e2f_ptr, const int32_t *__restrict__ e2f_idx,
                           const int8_t *__restrict__ kind, int8_t *__restrict__ mode)
{
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    bool wall = false, inflow = false;
    for (int32_t k = e2f_ptr[e]; k < e2f_ptr[e + 1]; ++k)
    {
        const int8_t fk = kind[e2f_idx[k]];
        wall |= fk == 1;
        inflow |= fk == 2;
    }
    mode[e] = wall ? 1 : inflow ? 2 : 0;
}

std::vector<int32_t> to32(const int64_t *p, int64_t n, const char *what)
{
    MHD_REQUIRE(p, std::string("missing ") + what);
    std::vector<int32_t> o(static_cast<size_t>(n) + 1);
    for (int64_t i = 0; i <= n; ++i)
    {
        MHD_REQUIRE(p[i] >= 0 && p[i] <= INT32_MAX, std::string(what) + " out of range");
        o[static_cast<size_t>(i)] = static_cast<int32_t>(p[i]);
    }
    return o;
}
} // namespace
} // namespace mhd

using namespace mhd;

extern "C" {

int mhd_gpu_compute_geometry(const MhdGeometryArgs *a)
{
    return guarded([&] {
        MHD_REQUIRE(a && a->x && a->edge_nodes, "null argument");
        MHD_REQUIRE(a->n_nodes >= 0 && a->n_edges >= 0 && a->n_faces >= 0 && a->n_cells >= 0, "negative count");
        const int64_t nn = a->n_nodes, ne = a->n_edges, nf = a->n_faces, nc = a->n_cells;
        DBuf<int32_t> f2ep, f2ei, c2fp, c2fi, e2fp, e2fi, f2cp, f2ci, en;
        DBuf<int8_t> f2es, c2fs;
        DBuf<double> x;
        const auto f2e = to32(a->f2e_ptr, nf, "f2e_ptr"), c2f = to32(a->c2f_ptr, nc, "c2f_ptr"), e2f = to32(a->e2f_ptr, ne, "e2f_ptr"),
                   f2c = to32(a->f2c_ptr, nf, "f2c_ptr");
        f2ep.upload(f2e); c2fp.upload(c2f); e2fp.upload(e2f); f2cp.upload(f2c);
        f2ei.upload(a->f2e_idx, f2e[nf]); f2es.upload(a->f2e_sgn, f2e[nf]);
        c2fi.upload(a->c2f_idx, c2f[nc]); c2fs.upload(a->c2f_sgn, c2f[nc]);
        e2fi.upload(a->e2f_idx, e2f[ne]); f2ci.upload(a->f2c_idx, f2c[nf]);
        en.upload(a->edge_nodes, 2 * ne);
        x.upload(a->x, 3 * nn);
        GeoView g{a->n_nodes, a->n_edges, a->n_faces, a->n_cells, x.p, en.p, f2ep.p, f2ei.p, c2fp.p, c2fi.p, e2fp.p, e2fi.p, f2cp.p, f2ci.p,
                  f2es.p, c2fs.p};
        DBuf<int> err;
        err.alloc(1);
        MHD_CUDA(cudaMemset(err.p, 0, sizeof(int)));
        DBuf<double> evec, emid, elen, farea, fcen, fmag, ccen, cvol, cmin, star0, star1, star2, star3, edual, ecw, efw;
        DBuf<int32_t> mis, eccount, ecc, ncount, ncursor, ncells;
        DBuf<int64_t> ecp, np;
        evec.alloc(3 * ne); emid.alloc(3 * ne); elen.alloc(ne); farea.alloc(3 * nf); fcen.alloc(3 * nf); fmag.alloc(nf);
        ccen.alloc(3 * nc); cvol.alloc(nc); cmin.alloc(nc); star0.alloc(nn); star1.alloc(ne); star2.alloc(nf); star3.alloc(nc);
        edual.alloc(3 * ne); mis.alloc(ne); efw.alloc(e2f[ne]); eccount.alloc(ne);
        if (ne) k_geo_edges<<<grid_for(ne, 128), 128>>>(g, evec.p, emid.p, elen.p);
        if (nf) k_geo_faces<<<grid_for(nf, 128), 128>>>(g, farea.p, fcen.p, fmag.p, err.p);
        if (ne) k_geo_ec<<<grid_for(ne, 128), 128>>>(g, nullptr, eccount.p, nullptr, err.p);
        MHD_LAUNCH_CHECK();
        // edge -> cell row pointers on the host (a prefix sum over the counts)
        std::vector<int32_t> cnt(ne);
        down(cnt.data(), eccount, ne);
        std::vector<int64_t> ptr(ne + 1, 0);
        for (int64_t e = 0; e < ne; ++e) ptr[e + 1] = ptr[e] + cnt[e];
        ecp.upload(ptr);
        ecc.alloc(ptr[ne] ? ptr[ne] : 1);
        ecw.alloc(ptr[ne] ? ptr[ne] : 1);
        if (ne) k_geo_ec<<<grid_for(ne, 128), 128>>>(g, ecp.p, nullptr, ecc.p, err.p);
        if (nc) k_geo_cells<<<grid_for(nc, 128), 128>>>(g, fcen.p, ccen.p, cvol.p, cmin.p, star3.p, err.p);
        if (nf) k_geo_face_dual<<<grid_for(nf, 128), 128>>>(g, fcen.p, fmag.p, ccen.p, star2.p);
        if (ne)
            k_geo_edge_dual<<<grid_for(ne, 128), 128>>>(g, fcen.p, ccen.p, emid.p, evec.p, elen.p, ecp.p, ecc.p, ecw.p, efw.p, edual.p, mis.p,
                                                         star1.p, err.p);
        MHD_LAUNCH_CHECK();
        // node -> cells, then star0
        ncount.alloc(nn ? nn : 1);
        ncursor.alloc(nn ? nn : 1);
        MHD_CUDA(cudaMemset(ncount.p, 0, (nn ? nn : 1) * sizeof(int32_t)));
        MHD_CUDA(cudaMemset(ncursor.p, 0, (nn ? nn : 1) * sizeof(int32_t)));
        if (nc) k_geo_n2c<<<grid_for(nc, 128), 128>>>(g, nullptr, ncount.p, nullptr, nullptr, err.p);
        MHD_LAUNCH_CHECK();
        std::vector<int32_t> ncnt(nn);
        down(ncnt.data(), ncount, nn);
        std::vector<int64_t> nptr(nn + 1, 0);
        for (int64_t v = 0; v < nn; ++v) nptr[v + 1] = nptr[v] + ncnt[v];
        np.upload(nptr);
        ncells.alloc(nptr[nn] ? nptr[nn] : 1);
        if (nc) k_geo_n2c<<<grid_for(nc, 128), 128>>>(g, np.p, nullptr, ncursor.p, ncells.p, err.p);
        if (nn)
        {
            k_geo_node_sort<<<grid_for(nn, 128), 128>>>(a->n_nodes, np.p, ncells.p, err.p);
            k_geo_star0<<<grid_for(nn, 128), 128>>>(g, np.p, ncells.p, fcen.p, ccen.p, star0.p, err.p);
        }
        MHD_LAUNCH_CHECK();
        int e = 0;
        MHD_CUDA(cudaMemcpy(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost));
        MHD_REQUIRE(e == 0, "mesh beyond the device geometry's limits (face loop > 16 nodes, cell > 64 nodes, edge > 64 cells, "
                            "node > 256 cells or edge valence > 32), code " + std::to_string(e));
        down(a->edge_vec, evec, 3 * ne); down(a->edge_mid, emid, 3 * ne); down(a->edge_len, elen, ne);
        down(a->face_area, farea, 3 * nf); down(a->face_center, fcen, 3 * nf); down(a->face_area_mag, fmag, nf);
        down(a->cell_center, ccen, 3 * nc); down(a->cell_volume, cvol, nc); down(a->cell_min_tet_volume, cmin, nc);
        down(a->star0, star0, nn); down(a->star1, star1, ne); down(a->star2, star2, nf); down(a->star3, star3, nc);
        down(a->edge_dual_area, edual, 3 * ne); down(a->ec_misoriented, mis, ne); down(a->ef_weight, efw, e2f[ne]);
        if (a->ec_ptr) std::copy(ptr.begin(), ptr.end(), a->ec_ptr);
        MHD_REQUIRE(!a->ec_cell || a->ec_capacity >= ptr[ne], "ec_capacity below the edge -> cell entries (" + std::to_string(ptr[ne]) + ")");
        down(a->ec_cell, ecc, ptr[ne]);
        down(a->ec_weight, ecw, ptr[ne]);
    });
}

int mhd_gpu_boundary(const MhdBoundaryArgs *a)
{
    return guarded([&] {
        MHD_REQUIRE(a && a->face_kind && a->edge_mode, "null argument");
        MHD_REQUIRE(a->n_edges >= 0 && a->n_faces >= 0 && a->n_cells >= 0 && a->n_tags >= 0, "negative count");
        MHD_REQUIRE(a->cell_material && a->face_tag && a->f2c_idx && a->f2c_sgn && a->e2f_idx && a->face_area && a->face_area_mag,
                    "missing array");
        MHD_REQUIRE(!a->n_tags || a->tag_type, "missing tag types");
        const int64_t ne = a->n_edges, nf = a->n_faces, nc = a->n_cells;
        const auto f2c = to32(a->f2c_ptr, nf, "f2c_ptr"), e2f = to32(a->e2f_ptr, ne, "e2f_ptr");
        for (int64_t f = 0; f < nf; ++f)
            MHD_REQUIRE(f2c[f + 1] - f2c[f] == 1 || f2c[f + 1] - f2c[f] == 2, "every face needs one or two cells");
        for (int64_t k = 0; k < f2c[nf]; ++k) MHD_REQUIRE(a->f2c_idx[k] >= 0 && a->f2c_idx[k] < nc, "f2c_idx out of range");
        for (int64_t k = 0; k < e2f[ne]; ++k) MHD_REQUIRE(a->e2f_idx[k] >= 0 && a->e2f_idx[k] < nf, "e2f_idx out of range");
        DBuf<int32_t> f2cp, f2ci, e2fp, e2fi, mat, tag;
        DBuf<int8_t> f2cs, types, kind, mode;
        DBuf<double> area, mag;
        DBuf<int> err;
        f2cp.upload(f2c); e2fp.upload(e2f);
        f2ci.upload(a->f2c_idx, f2c[nf]); f2cs.upload(a->f2c_sgn, f2c[nf]); e2fi.upload(a->e2f_idx, e2f[ne]);
        mat.upload(a->cell_material, nc); tag.upload(a->face_tag, nf);
        area.upload(a->face_area, 3 * nf); mag.upload(a->face_area_mag, nf);
        types.upload(a->tag_type, a->n_tags);
        kind.alloc(nf); mode.alloc(ne); err.alloc(1);
        MHD_CUDA(cudaMemset(err.p, 0, sizeof(int)));
        const V3 u = mk(a->u_inf[0], a->u_inf[1], a->u_inf[2]);
        if (nf)
            k_bc_faces<<<grid_for(nf, 256), 256>>>(a->n_faces, f2cp.p, f2ci.p, f2cs.p, mat.p, tag.p, area.p, mag.p, a->n_tags, types.p,
                                                   a->type_none, u, kind.p, err.p);
        if (ne) k_bc_edges<<<grid_for(ne, 256), 256>>>(a->n_edges, e2fp.p, e2fi.p, kind.p, mode.p);
        MHD_LAUNCH_CHECK();
        int e = 0;
        MHD_CUDA(cudaMemcpy(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost));
        MHD_REQUIRE(e == 0, "unknown boundary type for a face tag (wall|farfield|inflow|outflow)");
        down(a->face_kind, kind, nf);
        down(a->edge_mode, mode, ne);
    });
}
} // extern "C"
