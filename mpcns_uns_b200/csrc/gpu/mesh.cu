// nvcc-flags: -fmad=false
// Device mesh: upload of one rank's complex, metric and boundary classification, and the
// one-time derived tables (face -> L/R cells, least-squares stencil of mhd::Stencil).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

#include "common.cuh"

namespace mhd
{
namespace
{
thread_local std::string g_last_error;

// mhd::Stencil::Stencil (Common/fluid/Reconstruction.cpp:26-78), one thread per owned cell:
// per face a neighbour (interior fluid|fluid face) or a virtual neighbour at the mirrored cell
// centre (boundary / interface face), weight w = 1/|d|^2; the symmetric inverse of
// sum w d d^T, kept only if |det| >= 1e-9 sc^3.
__global__ void k_stencil(MeshView m, int32_t *nb_out, double *wd_out, double *inv_out, int8_t *valid_out)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.no_cells) return;
    const int32_t k0 = m.c2f_ptr[c], k1 = m.c2f_ptr[c + 1];
    valid_out[c] = 0;
    for (int q = 0; q < 6; ++q) inv_out[6 * (int64_t)c + q] = 0.0;
    if (m.material[c] != 0)
    {
        for (int32_t k = k0; k < k1; ++k) nb_out[k] = INT32_MIN;
        return;
    }
    const V3 xc = ld3(m.cell_center, c);
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int32_t k = k0; k < k1; ++k)
    {
        const int32_t f = m.c2f_idx[k];
        const int kind = m.face_kind[f];
        if (kind == 4) { nb_out[k] = INT32_MIN; continue; }
        V3 d;
        int32_t nb;
        const int32_t p0 = m.f2c_ptr[f], cnt = m.f2c_ptr[f + 1] - p0;
        if (cnt == 2 && kind == 0)
        {
            nb = m.f2c_idx[p0] == c ? m.f2c_idx[p0 + 1] : m.f2c_idx[p0];
            d = ld3(m.cell_center, nb) - xc;
        }
        else
        {
            const double A = m.face_area_mag[f];
            const V3 n = (double(m.c2f_sgn[k]) / A) * ld3(m.face_area, f);
            d = (2.0 * dot(ld3(m.face_center, f) - xc, n)) * n;
            nb = -(f + 1);
        }
        const double w = 1.0 / dot(d, d);
        nb_out[k] = nb;
        const double dv[3] = {d.x, d.y, d.z};
        wd_out[3 * (int64_t)k] = w * d.x;
        wd_out[3 * (int64_t)k + 1] = w * d.y;
        wd_out[3 * (int64_t)k + 2] = w * d.z;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) M[a][b] += w * dv[a] * dv[b];
    }
    const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                       M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    const double sc = dmax(dmax(dmax(M[0][0], M[1][1]), M[2][2]), 1e-300);
    if (fabs(det) < 1e-9 * sc * sc * sc) return;
    double *I = inv_out + 6 * (int64_t)c;
    I[0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det;
    I[1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
    I[2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det;
    I[3] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det;
    I[4] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
    I[5] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
    valid_out[c] = 1;
}

// face_center - cell_center per c2f entry: the offset the limiter and the face reconstruction use
// (Reconstruction.cpp:121, FluxRHS.cpp:54), one exact subtraction precomputed.
__global__ void k_slot_dx(MeshView m, double *dx)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const V3 xc = ld3(m.cell_center, c);
    for (int32_t k = m.c2f_ptr[c]; k < m.c2f_ptr[c + 1]; ++k) st3(dx, k, ld3(m.face_center, m.c2f_idx[k]) - xc);
}

// structure-of-arrays copy of the stencil of a tetrahedral mesh (4 slots per cell)
__global__ void k_tet_tables(MeshView m, int32_t *nb, int8_t *sg, double *wd, double *dx, double *inv)
{
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int64_t n = m.nc;
    for (int j = 0; j < 4; ++j)
    {
        const int64_t k = 4 * (int64_t)c + j;
        nb[j * n + c] = c < m.no_cells ? m.st_nb[k] : INT32_MIN;
        sg[j * n + c] = m.c2f_sgn[k];
        for (int a = 0; a < 3; ++a)
        {
            wd[(3 * j + a) * n + c] = m.st_wd[3 * k + a];
            dx[(3 * j + a) * n + c] = m.st_dx[3 * k + a];
        }
    }
    for (int q = 0; q < 6; ++q) inv[q * n + c] = m.st_inv[6 * (int64_t)c + q];
}

std::vector<int32_t> ptr32(const int64_t *p, int64_t rows, const char *what)
{
    MHD_REQUIRE(p != nullptr, std::string("missing ") + what);
    MHD_REQUIRE(p[0] == 0, std::string(what) + "[0] != 0");
    MHD_REQUIRE(p[rows] < INT32_MAX, std::string(what) + ": more than 2^31-1 entries");
    std::vector<int32_t> o(rows + 1);
    for (int64_t i = 0; i <= rows; ++i)
    {
        MHD_REQUIRE(i == 0 || p[i] >= p[i - 1], std::string(what) + " not monotone");
        o[i] = static_cast<int32_t>(p[i]);
    }
    return o;
}

template <class T> void check_range(const T *idx, int64_t n, int64_t lim, const char *what)
{
    MHD_REQUIRE(idx != nullptr || n == 0, std::string("missing ") + what);
    for (int64_t i = 0; i < n; ++i) MHD_REQUIRE(idx[i] >= 0 && idx[i] < lim, std::string(what) + ": index out of range");
}
} // namespace

void set_last_error(const std::string &msg) { g_last_error = msg; }
const char *last_error() { return g_last_error.c_str(); }
} // namespace mhd

MhdMesh::~MhdMesh()
{
    if (pinned) cudaFreeHost(pinned);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

using namespace mhd;

extern "C" {

const char *mhd_gpu_last_error(void) { return mhd::last_error(); }

int mhd_gpu_device_info(char *name, size_t name_len, int *sm_count)
{
    return guarded([&] {
        int dev = 0;
        MHD_CUDA(cudaGetDevice(&dev));
        cudaDeviceProp p;
        MHD_CUDA(cudaGetDeviceProperties(&p, dev));
        if (name && name_len)
        {
            std::strncpy(name, p.name, name_len - 1);
            name[name_len - 1] = 0;
        }
        if (sm_count) *sm_count = p.multiProcessorCount;
    });
}

int mhd_gpu_mesh_create(const MhdMeshDesc *d, MhdMesh **out)
{
    MhdMesh *m = nullptr;
    int rc = guarded([&] {
        MHD_REQUIRE(d && out, "null argument");
        MHD_REQUIRE(d->n_nodes >= 0 && d->n_edges >= 0 && d->n_faces >= 0 && d->n_cells >= 0, "negative count");
        MHD_REQUIRE(d->n_owned_cells >= 0 && d->n_owned_cells <= d->n_cells, "bad n_owned_cells");
        MHD_REQUIRE(d->n_owned_edges >= 0 && d->n_owned_edges <= d->n_edges, "bad n_owned_edges");
        const int64_t ne = d->n_edges, nf = d->n_faces, nc = d->n_cells;
        const auto c2fp = ptr32(d->c2f_ptr, nc, "c2f_ptr");
        const auto f2ep = ptr32(d->f2e_ptr, nf, "f2e_ptr");
        const auto e2fp = ptr32(d->e2f_ptr, ne, "e2f_ptr");
        const auto f2cp = ptr32(d->f2c_ptr, nf, "f2c_ptr");
        const auto ecp = ptr32(d->ec_ptr, ne, "ec_ptr");
        check_range(d->c2f_idx, c2fp[nc], nf, "c2f_idx");
        check_range(d->f2e_idx, f2ep[nf], ne, "f2e_idx");
        check_range(d->e2f_idx, e2fp[ne], nf, "e2f_idx");
        check_range(d->f2c_idx, f2cp[nf], nc, "f2c_idx");
        check_range(d->ec_cell, ecp[ne], nc, "ec_cell");
        int32_t max_valence = 0, max_edge_cells = 0;
        for (int64_t e = 0; e < ne; ++e)
        {
            MHD_REQUIRE(e2fp[e + 1] - e2fp[e] <= kMaxValence, "edge valence above " + std::to_string(kMaxValence) + " is not supported");
            max_valence = std::max(max_valence, e2fp[e + 1] - e2fp[e]);
            max_edge_cells = std::max(max_edge_cells, ecp[e + 1] - ecp[e]);
        }
        MHD_REQUIRE(d->cell_material && d->face_kind && d->edge_mode, "missing material / boundary classification");
        MHD_REQUIRE(d->edge_vec && d->edge_mid && d->edge_len && d->face_area && d->face_center && d->face_area_mag &&
                        d->cell_center && d->cell_volume && d->ec_weight && d->ef_weight && d->star1 && d->star2,
                    "missing geometry array");
        // canonical L / R cells of every face (reference FluxRHS.cpp:50-53, IdealEMF.cpp:62-64)
        std::vector<int32_t> L(nf, -1), R(nf, -1);
        std::vector<int8_t> mat(nc);
        for (int64_t c = 0; c < nc; ++c)
        {
            MHD_REQUIRE(d->cell_material[c] == 0 || d->cell_material[c] == 1, "cell_material must be 0 or 1");
            mat[c] = static_cast<int8_t>(d->cell_material[c]);
        }
        for (int64_t f = 0; f < nf; ++f)
        {
            const int32_t cnt = f2cp[f + 1] - f2cp[f];
            MHD_REQUIRE(cnt == 1 || cnt == 2, "every face needs one or two cells");
            MHD_REQUIRE(d->face_kind[f] >= 0 && d->face_kind[f] <= 4, "face_kind out of range");
            for (int32_t k = f2cp[f]; k < f2cp[f + 1]; ++k) (d->f2c_sgn[k] > 0 ? L[f] : R[f]) = d->f2c_idx[k];
        }
        // c2f rows in ascending face order: the order in which the reference's face loops scatter into a cell
        std::vector<int32_t> cfa_idx(d->c2f_idx, d->c2f_idx + c2fp[nc]);
        std::vector<int8_t> cfa_sgn(d->c2f_sgn, d->c2f_sgn + c2fp[nc]);
        for (int64_t c = 0; c < nc; ++c)
            for (int32_t a = c2fp[c] + 1; a < c2fp[c + 1]; ++a)
                for (int32_t b = a; b > c2fp[c] && cfa_idx[b - 1] > cfa_idx[b]; --b)
                {
                    std::swap(cfa_idx[b - 1], cfa_idx[b]);
                    std::swap(cfa_sgn[b - 1], cfa_sgn[b]);
                }
        m = new MhdMesh;
        MeshView &v = m->v;
        m->cfa_idx.upload(cfa_idx);
        m->cfa_sgn.upload(cfa_sgn);
        v.cfa_idx = m->cfa_idx.p;
        v.cfa_sgn = m->cfa_sgn.p;
        v.nn = d->n_nodes; v.ne = d->n_edges; v.nf = d->n_faces; v.nc = d->n_cells;
        v.no_cells = d->n_owned_cells; v.no_edges = d->n_owned_edges;
        v.max_valence = max_valence;
        v.max_edge_cells = max_edge_cells;
        v.tri_faces = 1;
        for (int64_t f = 0; f < nf && v.tri_faces; ++f) v.tri_faces = f2ep[f + 1] - f2ep[f] == 3;
        m->c2f_ptr.upload(c2fp); m->c2f_idx.upload(d->c2f_idx, c2fp[nc]); m->c2f_sgn.upload(d->c2f_sgn, c2fp[nc]);
        m->f2e_ptr.upload(f2ep); m->f2e_idx.upload(d->f2e_idx, f2ep[nf]); m->f2e_sgn.upload(d->f2e_sgn, f2ep[nf]);
        m->e2f_ptr.upload(e2fp); m->e2f_idx.upload(d->e2f_idx, e2fp[ne]); m->e2f_sgn.upload(d->e2f_sgn, e2fp[ne]);
        m->f2c_ptr.upload(f2cp); m->f2c_idx.upload(d->f2c_idx, f2cp[nf]); m->f2c_sgn.upload(d->f2c_sgn, f2cp[nf]);
        m->face_L.upload(L); m->face_R.upload(R);
        m->material.upload(mat);
        m->face_kind.upload(d->face_kind, nf);
        m->edge_mode.upload(d->edge_mode, ne);
        m->edge_vec.upload(d->edge_vec, 3 * ne); m->edge_mid.upload(d->edge_mid, 3 * ne); m->edge_len.upload(d->edge_len, ne);
        m->face_area.upload(d->face_area, 3 * nf); m->face_center.upload(d->face_center, 3 * nf);
        m->face_area_mag.upload(d->face_area_mag, nf);
        m->cell_center.upload(d->cell_center, 3 * nc); m->cell_volume.upload(d->cell_volume, nc);
        m->ec_ptr.upload(ecp); m->ec_cell.upload(d->ec_cell, ecp[ne]); m->ec_weight.upload(d->ec_weight, ecp[ne]);
        m->ef_weight.upload(d->ef_weight, e2fp[ne]);
        m->star1.upload(d->star1, ne); m->star2.upload(d->star2, nf);
        v.c2f_ptr = m->c2f_ptr.p; v.c2f_idx = m->c2f_idx.p; v.c2f_sgn = m->c2f_sgn.p;
        v.f2e_ptr = m->f2e_ptr.p; v.f2e_idx = m->f2e_idx.p; v.f2e_sgn = m->f2e_sgn.p;
        v.e2f_ptr = m->e2f_ptr.p; v.e2f_idx = m->e2f_idx.p; v.e2f_sgn = m->e2f_sgn.p;
        v.f2c_ptr = m->f2c_ptr.p; v.f2c_idx = m->f2c_idx.p; v.f2c_sgn = m->f2c_sgn.p;
        v.face_L = m->face_L.p; v.face_R = m->face_R.p;
        v.material = m->material.p; v.face_kind = m->face_kind.p; v.edge_mode = m->edge_mode.p;
        v.edge_vec = m->edge_vec.p; v.edge_mid = m->edge_mid.p; v.edge_len = m->edge_len.p;
        v.face_area = m->face_area.p; v.face_center = m->face_center.p; v.face_area_mag = m->face_area_mag.p;
        v.cell_center = m->cell_center.p; v.cell_volume = m->cell_volume.p;
        v.ec_ptr = m->ec_ptr.p; v.ec_cell = m->ec_cell.p; v.ec_weight = m->ec_weight.p; v.ef_weight = m->ef_weight.p;
        v.star1 = m->star1.p; v.star2 = m->star2.p;
        if (d->edge_nodes)
        {
            // AmbipolarEMF::AmbipolarEMF (MercuryUns/physics/Ambipolar.cpp:35-50): per node its fluid cells, a
            // cell's nodes being the sorted end points of its faces' edges (uns::CellComplex::cell_nodes)
            check_range(d->edge_nodes, 2 * ne, d->n_nodes, "edge_nodes");
            const int64_t nn = d->n_nodes;
            std::vector<int32_t> cnt(nn + 1, 0), cn;
            std::vector<std::pair<int32_t, int32_t>> pr;
            for (int64_t c = 0; c < nc; ++c)
            {
                if (mat[c] == 1) continue;
                cn.clear();
                for (int32_t k = c2fp[c]; k < c2fp[c + 1]; ++k)
                {
                    const int32_t f = d->c2f_idx[k];
                    for (int32_t q = f2ep[f]; q < f2ep[f + 1]; ++q)
                    {
                        const int32_t e = d->f2e_idx[q];
                        cn.push_back(d->edge_nodes[2 * (int64_t)e]);
                        cn.push_back(d->edge_nodes[2 * (int64_t)e + 1]);
                    }
                }
                std::sort(cn.begin(), cn.end());
                cn.erase(std::unique(cn.begin(), cn.end()), cn.end());
                for (int32_t nd : cn) pr.emplace_back(nd, static_cast<int32_t>(c));
            }
            for (auto &q : pr) ++cnt[q.first + 1];
            for (int64_t nd = 0; nd < nn; ++nd) cnt[nd + 1] += cnt[nd];
            std::vector<int32_t> cells(pr.size()), fill(cnt.begin(), cnt.end() - 1);
            for (auto &q : pr) cells[fill[q.first]++] = q.second;
            m->e_nodes.upload(d->edge_nodes, 2 * ne);
            m->n2c_ptr.upload(cnt);
            m->n2c_cell.upload(cells);
            v.e_nodes = m->e_nodes.p;
            v.n2c_ptr = m->n2c_ptr.p;
            v.n2c_cell = m->n2c_cell.p;
        }
        MHD_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
        m->own_stream = true;
        MHD_CUDA(cudaMallocHost(&m->pinned, 64 * sizeof(double)));
        // stencil tables
        m->st_nb.alloc(c2fp[nc]);
        m->st_wd.alloc(3 * static_cast<size_t>(c2fp[nc]));
        m->st_inv.alloc(6 * static_cast<size_t>(nc));
        m->st_valid.alloc(nc);
        if (nc)
        {
            MHD_CUDA(cudaMemsetAsync(m->st_valid.p, 0, nc, m->stream));
            MHD_CUDA(cudaMemsetAsync(m->st_inv.p, 0, 6 * nc * sizeof(double), m->stream));
        }
        if (c2fp[nc]) MHD_CUDA(cudaMemsetAsync(m->st_wd.p, 0, 3 * (size_t)c2fp[nc] * sizeof(double), m->stream));
        if (v.no_cells)
        {
            k_stencil<<<grid_for(v.no_cells, 128), 128, 0, m->stream>>>(v, m->st_nb.p, m->st_wd.p, m->st_inv.p, m->st_valid.p);
            MHD_LAUNCH_CHECK();
        }
        v.st_nb = m->st_nb.p; v.st_wd = m->st_wd.p; v.st_inv = m->st_inv.p; v.st_valid = m->st_valid.p;
        bool tets = nc > 0;
        for (int64_t c = 0; c < nc && tets; ++c) tets = c2fp[c + 1] - c2fp[c] == 4;
        v.faces_per_cell = tets ? 4 : 0;
        m->st_dx.alloc(3 * static_cast<size_t>(c2fp[nc]));
        if (nc)
        {
            k_slot_dx<<<grid_for(nc, 256), 256, 0, m->stream>>>(v, m->st_dx.p);
            MHD_LAUNCH_CHECK();
        }
        v.st_dx = m->st_dx.p;
        if (tets)
        {
            m->t_nb.alloc(4 * static_cast<size_t>(nc));
            m->t_sg.alloc(4 * static_cast<size_t>(nc));
            m->t_wd.alloc(12 * static_cast<size_t>(nc));
            m->t_dx.alloc(12 * static_cast<size_t>(nc));
            m->t_inv.alloc(6 * static_cast<size_t>(nc));
            k_tet_tables<<<grid_for(nc, 256), 256, 0, m->stream>>>(v, m->t_nb.p, m->t_sg.p, m->t_wd.p, m->t_dx.p, m->t_inv.p);
            MHD_LAUNCH_CHECK();
            v.t_nb = m->t_nb.p; v.t_sg = m->t_sg.p; v.t_wd = m->t_wd.p; v.t_dx = m->t_dx.p; v.t_inv = m->t_inv.p;
        }
        MHD_CUDA(cudaStreamSynchronize(m->stream));
        *out = m;
    });
    if (rc != MHD_OK) delete m;
    return rc;
}

int mhd_gpu_mesh_destroy(MhdMesh *mesh)
{
    return guarded([&] {
        if (!mesh) return;
        if (mesh->stream) cudaStreamSynchronize(mesh->stream);
        delete mesh;
    });
}

void *mhd_gpu_mesh_stream(MhdMesh *mesh) { return mesh ? static_cast<void *>(mesh->stream) : nullptr; }

int mhd_gpu_mesh_set_stream(MhdMesh *mesh, void *stream)
{
    return guarded([&] {
        MHD_REQUIRE(mesh, "null mesh");
        if (mesh->own_stream && mesh->stream)
        {
            MHD_CUDA(cudaStreamSynchronize(mesh->stream));
            MHD_CUDA(cudaStreamDestroy(mesh->stream));
        }
        mesh->stream = static_cast<cudaStream_t>(stream);
        mesh->own_stream = false;
    });
}

int mhd_gpu_synchronize(MhdMesh *mesh)
{
    return guarded([&] {
        MHD_REQUIRE(mesh, "null mesh");
        MHD_CUDA(cudaStreamSynchronize(mesh->stream));
    });
}

} // extern "C"
