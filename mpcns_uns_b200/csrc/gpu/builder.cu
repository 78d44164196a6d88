// Tetrahedral cell complex of a hexahedral list, numbered on the device exactly as the reference's
// uns::ComplexBuilder numbers it when the hexahedra's 6 Kuhn tetrahedra are added one by one
// (src/uns/complex/ComplexBuilder.cpp:45-134): faces in the order of their first loop, edges in the order
// of their first (face, loop position), canonical face loops (smallest node first, second node smaller
// than the last), c2f signs -1 where a cell's loop is the reverse of the canonical one, edges from the
// smaller to the larger node, later tags of the same face winning.
//
// The builder's sequential hash-table walk becomes sorts: every (tetrahedron, local face) entry carries
// its sorted node triple; a stable sort groups equal triples with the earliest entry first, which is the
// one that created the face, and an exclusive scan over the entries numbers the creators in creation
// order.  Edges follow from the faces the same way, and the upward incidences (n2e, e2f, f2c) are stable
// sorts by column, which lists every row in ascending order of the rows it comes from, as the
// reference's transpose does (src/uns/complex/Incidence.cpp:8-26).  Sorts and scans are CUB's.
#include <cub/cub.cuh>

#include <string>
#include <vector>

#include "common.cuh"

namespace mhd
{
namespace
{
// Kuhn paths 0 -> a -> a|b -> 7 over the 6 orders of the local axis bits (corner i of a hexahedron at
// (i&1, (i>>1)&1, (i>>2)&1)); PAR is the parity of the order (a negative one swaps the middle corners, so
// that every tetrahedron is positively oriented).  The same table as the host library's split.
__constant__ int kKuhnP[6][3] = {{1, 2, 4}, {1, 4, 2}, {2, 1, 4}, {2, 4, 1}, {4, 1, 2}, {4, 2, 1}};
__constant__ int kKuhnPar[6] = {+1, -1, -1, +1, +1, -1};

// per tetrahedron t (6 per hexahedron, cell t): its 4 outward loops, canonicalised; entry 4t + l holds the
// sorted node triple (which is the canonical loop of a triangle) and whether the loop was reversed
__global__ void k_kuhn_faces(int64_t n_tets, const int32_t *__restrict__ hex8, const int32_t *__restrict__ hex_mat, uint32_t *ka, uint32_t *kb,
                             uint32_t *kc, int8_t *flip, int32_t *cell_mat)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tets) return;
    const int64_t h = t / 6;
    const int k = static_cast<int>(t - 6 * h);
    int32_t v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = hex8[8 * h + q];
    const int a = kKuhnP[k][0], ab = kKuhnP[k][0] | kKuhnP[k][1];
    int32_t p[4] = {v[0], v[a], v[ab], v[7]};
    if (kKuhnPar[k] < 0)
    {
        const int32_t s = p[1];
        p[1] = p[2];
        p[2] = s;
    }
    const int32_t F[4][3] = {{p[0], p[2], p[1]}, {p[0], p[1], p[3]}, {p[1], p[2], p[3]}, {p[0], p[3], p[2]}};
#pragma unroll
    for (int l = 0; l < 4; ++l)
    {
        // ComplexBuilder::canonicalize (:20-31): rotate the smallest node first, reverse if loop[1] > loop[2]
        int s = 0;
        if (F[l][1] < F[l][s]) s = 1;
        if (F[l][2] < F[l][s]) s = 2;
        const int32_t x0 = F[l][s], x1 = F[l][(s + 1) % 3], x2 = F[l][(s + 2) % 3];
        const bool rev = x1 > x2;
        const int64_t e = 4 * t + l;
        ka[e] = static_cast<uint32_t>(x0);
        kb[e] = static_cast<uint32_t>(rev ? x2 : x1);
        kc[e] = static_cast<uint32_t>(rev ? x1 : x2);
        flip[e] = rev ? 1 : 0;
    }
    cell_mat[t] = hex_mat ? hex_mat[h] : 0;
}

__global__ void k_pack_ab(int64_t n, const uint32_t *__restrict__ ka, const uint32_t *__restrict__ kb, const uint32_t *__restrict__ idx,
                          uint64_t *key)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t e = idx[i];
    key[i] = (static_cast<uint64_t>(ka[e]) << 32) | kb[e];
}

// Groups of equal keys in sorted order: the first entry of a group created it.  new_flag[entry] = 1 for
// creators; creator[entry] = the group's first entry.  Groups larger than `max_group` (a face shared by
// more than two cells) raise err.
__global__ void k_groups(int64_t n, const uint64_t *__restrict__ key_hi, const uint32_t *__restrict__ key_lo_src,
                         const uint32_t *__restrict__ sorted_idx, uint32_t *new_flag, uint32_t *creator, int max_group, int *err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t e = sorted_idx[i];
    auto same = [&](int64_t x, int64_t y) {
        return key_hi[x] == key_hi[y] && (!key_lo_src || key_lo_src[sorted_idx[x]] == key_lo_src[sorted_idx[y]]);
    };
    int64_t head = i;
    while (head > 0 && same(head - 1, i) && i - head < max_group) --head;
    if (i - head >= max_group) atomicOr(err, 1);
    new_flag[e] = head == i ? 1u : 0u;
    creator[e] = sorted_idx[head];
}

// number of every entry's object: the creator's place in the creation-ordered scan
__global__ void k_ids(int64_t n, const uint32_t *__restrict__ creator, const uint32_t *__restrict__ scan, int32_t *id)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) id[e] = static_cast<int32_t>(scan[creator[e]]);
}

// the faces' edges: face f (created by entry e with canonical loop a < b < c) has the edges (a,b), (b,c),
// (c,a) in loop order, signed +1, +1, -1 (ComplexBuilder::add_cell :56-62)
__global__ void k_face_edges(int64_t n_entries, const uint32_t *__restrict__ new_flag, const int32_t *__restrict__ fid,
                             const uint32_t *__restrict__ ka, const uint32_t *__restrict__ kb, const uint32_t *__restrict__ kc,
                             uint64_t *ekey, int8_t *esgn)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_entries || !new_flag[e]) return;
    const int64_t f = fid[e];
    const uint64_t a = ka[e], b = kb[e], c = kc[e];
    ekey[3 * f] = (a << 32) | b;
    ekey[3 * f + 1] = (b << 32) | c;
    ekey[3 * f + 2] = (a << 32) | c;
    esgn[3 * f] = 1;
    esgn[3 * f + 1] = 1;
    esgn[3 * f + 2] = -1;
}

__global__ void k_edge_nodes(int64_t n, const uint32_t *__restrict__ new_flag, const int32_t *__restrict__ eid, const uint64_t *__restrict__ ekey,
                             int32_t *e2n_idx, int8_t *e2n_sgn)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || !new_flag[j]) return;
    const int64_t e = eid[j];
    e2n_idx[2 * e] = static_cast<int32_t>(ekey[j] >> 32);
    e2n_idx[2 * e + 1] = static_cast<int32_t>(ekey[j] & 0xffffffffULL);
    e2n_sgn[2 * e] = -1;
    e2n_sgn[2 * e + 1] = 1;
}

__global__ void k_c2f_sgn(int64_t n, const int8_t *__restrict__ flip, int8_t *sgn)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) sgn[e] = flip[e] ? -1 : 1;
}

// tags: the face of each tagged triangle by binary search in the sorted face keys; later tags win
// (ComplexBuilder::tag_face keeps the last tag of a node set, :87-92)
__global__ void k_tags(int32_t n_tags, const int32_t *__restrict__ tri, int64_t n, const uint64_t *__restrict__ key_ab,
                       const uint32_t *__restrict__ kc, const uint32_t *__restrict__ sorted_idx, const int32_t *__restrict__ fid, int32_t *last)
{
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tags) return;
    int32_t x[3] = {tri[3 * t], tri[3 * t + 1], tri[3 * t + 2]};
    if (x[0] > x[1]) { const int32_t s = x[0]; x[0] = x[1]; x[1] = s; }
    if (x[1] > x[2]) { const int32_t s = x[1]; x[1] = x[2]; x[2] = s; }
    if (x[0] > x[1]) { const int32_t s = x[0]; x[0] = x[1]; x[1] = s; }
    const uint64_t kab = (static_cast<uint64_t>(static_cast<uint32_t>(x[0])) << 32) | static_cast<uint32_t>(x[1]);
    const uint32_t kcc = static_cast<uint32_t>(x[2]);
    int64_t lo = 0, hi = n;
    while (lo < hi)
    {
        const int64_t mid = (lo + hi) / 2;
        const uint64_t m1 = key_ab[mid];
        const uint32_t m2 = kc[sorted_idx[mid]];
        if (m1 < kab || (m1 == kab && m2 < kcc)) lo = mid + 1;
        else hi = mid;
    }
    if (lo < n && key_ab[lo] == kab && kc[sorted_idx[lo]] == kcc) atomicMax(&last[fid[sorted_idx[lo]]], t);
}

__global__ void k_tag_ids(int64_t nf, const int32_t *__restrict__ last, const int32_t *__restrict__ tag_id, int32_t *face_tag)
{
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f < nf) face_tag[f] = last[f] >= 0 ? tag_id[last[f]] : 0;
}

// transpose of a CSR with `per_row` entries per row (rows r, columns col[k]): entries sorted stably by column
__global__ void k_count_cols(int64_t n, const int32_t *__restrict__ col, int64_t *count)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) atomicAdd(reinterpret_cast<unsigned long long *>(&count[col[k] + 1]), 1ull);
}
__global__ void k_transpose_fill(int64_t n, int per_row, const uint32_t *__restrict__ sorted_entry, const int8_t *__restrict__ sgn,
                                 int32_t *t_idx, int8_t *t_sgn)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = sorted_entry[i];
    t_idx[i] = static_cast<int32_t>(k / per_row);
    t_sgn[i] = sgn[k];
}
__global__ void k_iota(int64_t n, uint32_t *v)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = static_cast<uint32_t>(i);
}
__global__ void k_fill_ptr(int64_t rows, int per_row, int64_t *ptr)
{
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r <= rows) ptr[r] = r * per_row;
}

int bits_for(uint64_t v)
{
    int b = 1;
    while (b < 64 && (v >> b)) ++b;
    return b;
}
inline int g256(int64_t n) { return static_cast<int>((n + 255) / 256); }
} // namespace
} // namespace mhd

using namespace mhd;

// one incidence table on the device: ptr (rows + 1), idx, sgn
struct DevCsr
{
    DBuf<int64_t> ptr;
    DBuf<int32_t> idx;
    DBuf<int8_t> sgn;
};

struct MhdTetBuild
{
    int64_t n_nodes = 0, ne = 0, nf = 0, nc = 0;
    DevCsr e2n, f2e, c2f, n2e, e2f, f2c;
    DBuf<int32_t> cell_material, face_tag;
};

namespace
{
// temp storage of CUB calls, grown on demand
struct CubTemp
{
    DBuf<unsigned char> buf;
    void *get(size_t bytes)
    {
        if (bytes > buf.n) buf.alloc(bytes);
        return buf.p;
    }
};

// stable sort of (key, value) pairs over the low `bits` bits of the key
template <class K>
void sort_pairs(CubTemp &tmp, const K *kin, K *kout, const uint32_t *vin, uint32_t *vout, int64_t n, int bits, cudaStream_t s)
{
    size_t bytes = 0;
    MHD_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, 0, bits, s));
    MHD_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(bytes), bytes, kin, kout, vin, vout, n, 0, bits, s));
}

void exclusive_scan(CubTemp &tmp, const uint32_t *in, uint32_t *out, int64_t n, cudaStream_t s)
{
    size_t bytes = 0;
    MHD_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
    MHD_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(bytes), bytes, in, out, n, s));
}

// the transpose of (rows, per_row entries each, columns col, signs sgn) into t (ncols rows)
void transpose(CubTemp &tmp, int64_t rows, int per_row, const int32_t *col, const int8_t *sgn, int64_t ncols, DevCsr &t, cudaStream_t s)
{
    const int64_t n = rows * per_row;
    t.ptr.alloc(ncols + 1);
    t.idx.alloc(n);
    t.sgn.alloc(n);
    MHD_CUDA(cudaMemsetAsync(t.ptr.p, 0, (ncols + 1) * sizeof(int64_t), s));
    if (!n) return;
    k_count_cols<<<g256(n), 256, 0, s>>>(n, col, t.ptr.p);
    {
        size_t bytes = 0;
        MHD_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, t.ptr.p, t.ptr.p, ncols + 1, s));
        MHD_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(bytes), bytes, t.ptr.p, t.ptr.p, ncols + 1, s));
    }
    DBuf<uint32_t> kin, kout, vin, vout;
    kin.alloc(n); kout.alloc(n); vin.alloc(n); vout.alloc(n);
    MHD_CUDA(cudaMemcpyAsync(kin.p, col, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    k_iota<<<g256(n), 256, 0, s>>>(n, vin.p);
    sort_pairs(tmp, kin.p, kout.p, vin.p, vout.p, n, bits_for(static_cast<uint64_t>(ncols)), s);
    k_transpose_fill<<<g256(n), 256, 0, s>>>(n, per_row, vout.p, sgn, t.idx.p, t.sgn.p);
    MHD_LAUNCH_CHECK();
    MHD_CUDA(cudaStreamSynchronize(s)); // the temporaries above are freed on return
}
} // namespace

extern "C" {

int mhd_gpu_tet_build(int32_t n_nodes, int64_t n_hex, const int32_t *hex8, const int32_t *hex_material, int32_t n_tags,
                      const int32_t *tag_tri, const int32_t *tag_id, MhdTetBuild **out)
{
    MhdTetBuild *b = nullptr;
    const int rc = guarded([&] {
        MHD_REQUIRE(out && (n_hex == 0 || hex8) && n_nodes >= 0 && n_hex >= 0 && n_tags >= 0 && (n_tags == 0 || (tag_tri && tag_id)),
                    "bad argument");
        MHD_REQUIRE(6 * n_hex <= INT32_MAX / 4, "too many cells for 32-bit entry numbers");
        for (int64_t i = 0; i < 8 * n_hex; ++i) MHD_REQUIRE(hex8[i] >= 0 && hex8[i] < n_nodes, "hexahedron node out of range");
        for (int64_t i = 0; i < 3 * (int64_t)n_tags; ++i) MHD_REQUIRE(tag_tri[i] >= 0 && tag_tri[i] < n_nodes, "tag node out of range");
        cudaStream_t s = nullptr;
        MHD_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        struct StreamGuard
        {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamDestroy(s); }
        } sg{s};
        b = new MhdTetBuild;
        b->n_nodes = n_nodes;
        const int64_t nc = 6 * n_hex, nent = 4 * nc;
        b->nc = nc;
        CubTemp tmp;
        DBuf<int32_t> dhex, dmat;
        dhex.upload(hex8, 8 * n_hex);
        if (hex_material) dmat.upload(hex_material, n_hex);
        DBuf<uint32_t> ka, kb, kc;
        DBuf<int8_t> flip;
        ka.alloc(nent); kb.alloc(nent); kc.alloc(nent); flip.alloc(nent);
        b->cell_material.alloc(nc);
        if (nc)
            k_kuhn_faces<<<g256(nc), 256, 0, s>>>(nc, dhex.p, dmat.p, ka.p, kb.p, kc.p, flip.p, b->cell_material.p);
        MHD_LAUNCH_CHECK();
        dhex.release();
        const int nbits = bits_for(static_cast<uint64_t>(n_nodes));
        // faces: stable sort of the entries by their node triples (c first, then (a, b): least significant first)
        DBuf<uint32_t> idx0, idx1, kc_s;
        DBuf<uint64_t> kab, kab_s;
        idx0.alloc(nent); idx1.alloc(nent); kc_s.alloc(nent); kab.alloc(nent); kab_s.alloc(nent);
        DBuf<int32_t> fid;
        DBuf<uint32_t> fnew, fcre, fscan;
        fid.alloc(nent); fnew.alloc(nent); fcre.alloc(nent); fscan.alloc(nent);
        DBuf<int> err;
        err.alloc(1);
        MHD_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
        if (nent)
        {
            k_iota<<<g256(nent), 256, 0, s>>>(nent, idx0.p);
            sort_pairs(tmp, kc.p, kc_s.p, idx0.p, idx1.p, nent, nbits, s);
            kc_s.release();
            k_pack_ab<<<g256(nent), 256, 0, s>>>(nent, ka.p, kb.p, idx1.p, kab.p);
            sort_pairs(tmp, kab.p, kab_s.p, idx1.p, idx0.p, nent, 32 + nbits, s);
            kab.release();
            // sorted order: kab_s with entries idx0
            k_groups<<<g256(nent), 256, 0, s>>>(nent, kab_s.p, kc.p, idx0.p, fnew.p, fcre.p, 2, err.p);
            exclusive_scan(tmp, fnew.p, fscan.p, nent, s);
            k_ids<<<g256(nent), 256, 0, s>>>(nent, fcre.p, fscan.p, fid.p);
            MHD_LAUNCH_CHECK();
        }
        uint32_t last_scan = 0, last_new = 0;
        if (nent)
        {
            MHD_CUDA(cudaMemcpyAsync(&last_scan, fscan.p + nent - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            MHD_CUDA(cudaMemcpyAsync(&last_new, fnew.p + nent - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        }
        int herr = 0;
        MHD_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        MHD_CUDA(cudaStreamSynchronize(s));
        MHD_REQUIRE(!herr, "a face is shared by more than two cells");
        const int64_t nf = static_cast<int64_t>(last_scan) + last_new;
        b->nf = nf;
        // c2f
        b->c2f.ptr.alloc(nc + 1);
        b->c2f.sgn.alloc(nent);
        k_fill_ptr<<<g256(nc + 1), 256, 0, s>>>(nc, 4, b->c2f.ptr.p);
        if (nent) k_c2f_sgn<<<g256(nent), 256, 0, s>>>(nent, flip.p, b->c2f.sgn.p);
        // tags
        b->face_tag.alloc(nf);
        {
            DBuf<int32_t> last, dtri, dtid;
            last.alloc(nf);
            MHD_CUDA(cudaMemsetAsync(last.p, 0xff, nf * sizeof(int32_t), s));
            if (n_tags && nent)
            {
                dtri.upload(tag_tri, 3 * (size_t)n_tags);
                dtid.upload(tag_id, n_tags);
                k_tags<<<g256(n_tags), 256, 0, s>>>(n_tags, dtri.p, nent, kab_s.p, kc.p, idx0.p, fid.p, last.p);
            }
            else
                dtid.alloc(1);
            if (nf) k_tag_ids<<<g256(nf), 256, 0, s>>>(nf, last.p, dtid.p, b->face_tag.p);
            MHD_LAUNCH_CHECK();
            MHD_CUDA(cudaStreamSynchronize(s));
        }
        kab_s.release();
        // edges of the faces in creation order, then numbered like the faces
        const int64_t nfe = 3 * nf;
        DBuf<uint64_t> ekey, ekey_s;
        DBuf<int8_t> esgn;
        ekey.alloc(nfe); esgn.alloc(nfe);
        if (nent) k_face_edges<<<g256(nent), 256, 0, s>>>(nent, fnew.p, fid.p, ka.p, kb.p, kc.p, ekey.p, esgn.p);
        MHD_LAUNCH_CHECK();
        ka.release(); kb.release(); kc.release(); flip.release(); fnew.release(); fcre.release(); fscan.release(); idx1.release();
        b->c2f.idx.alloc(nent);
        if (nent) MHD_CUDA(cudaMemcpyAsync(b->c2f.idx.p, fid.p, nent * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
        fid.release();
        idx0.release();
        DBuf<uint32_t> j0, j1, enew, ecre, escan;
        DBuf<int32_t> eid;
        j0.alloc(nfe); j1.alloc(nfe); ekey_s.alloc(nfe); enew.alloc(nfe); ecre.alloc(nfe); escan.alloc(nfe); eid.alloc(nfe);
        int64_t ne = 0;
        if (nfe)
        {
            k_iota<<<g256(nfe), 256, 0, s>>>(nfe, j0.p);
            sort_pairs(tmp, ekey.p, ekey_s.p, j0.p, j1.p, nfe, 32 + nbits, s);
            k_groups<<<g256(nfe), 256, 0, s>>>(nfe, ekey_s.p, nullptr, j1.p, enew.p, ecre.p, INT32_MAX, err.p);
            exclusive_scan(tmp, enew.p, escan.p, nfe, s);
            k_ids<<<g256(nfe), 256, 0, s>>>(nfe, ecre.p, escan.p, eid.p);
            MHD_LAUNCH_CHECK();
            uint32_t ls = 0, ln = 0;
            MHD_CUDA(cudaMemcpyAsync(&ls, escan.p + nfe - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            MHD_CUDA(cudaMemcpyAsync(&ln, enew.p + nfe - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            MHD_CUDA(cudaStreamSynchronize(s));
            ne = static_cast<int64_t>(ls) + ln;
        }
        b->ne = ne;
        ekey_s.release(); j0.release(); j1.release(); ecre.release(); escan.release();
        // f2e, e2n
        b->f2e.ptr.alloc(nf + 1);
        k_fill_ptr<<<g256(nf + 1), 256, 0, s>>>(nf, 3, b->f2e.ptr.p);
        b->f2e.idx.alloc(nfe);
        if (nfe) MHD_CUDA(cudaMemcpyAsync(b->f2e.idx.p, eid.p, nfe * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
        b->e2n.ptr.alloc(ne + 1);
        b->e2n.idx.alloc(2 * ne);
        b->e2n.sgn.alloc(2 * ne);
        k_fill_ptr<<<g256(ne + 1), 256, 0, s>>>(ne, 2, b->e2n.ptr.p);
        if (nfe) k_edge_nodes<<<g256(nfe), 256, 0, s>>>(nfe, enew.p, eid.p, ekey.p, b->e2n.idx.p, b->e2n.sgn.p);
        MHD_LAUNCH_CHECK();
        MHD_CUDA(cudaStreamSynchronize(s));
        b->f2e.sgn.alloc(nfe);
        if (nfe) MHD_CUDA(cudaMemcpyAsync(b->f2e.sgn.p, esgn.p, nfe * sizeof(int8_t), cudaMemcpyDeviceToDevice, s));
        MHD_CUDA(cudaStreamSynchronize(s));
        ekey.release(); esgn.release(); enew.release(); eid.release();
        // upward incidences
        transpose(tmp, nc, 4, b->c2f.idx.p, b->c2f.sgn.p, nf, b->f2c, s);
        transpose(tmp, nf, 3, b->f2e.idx.p, b->f2e.sgn.p, ne, b->e2f, s);
        transpose(tmp, ne, 2, b->e2n.idx.p, b->e2n.sgn.p, n_nodes, b->n2e, s);
        MHD_CUDA(cudaStreamSynchronize(s));
        *out = b;
    });
    if (rc != MHD_OK) delete b;
    return rc;
}

int mhd_gpu_tet_build_counts(const MhdTetBuild *b, int64_t *counts)
{
    return guarded([&] {
        MHD_REQUIRE(b && counts, "bad argument");
        counts[0] = b->n_nodes; counts[1] = b->ne; counts[2] = b->nf; counts[3] = b->nc;
    });
}

int mhd_gpu_tet_build_copy(const MhdTetBuild *b, const MhdComplexOut *o)
{
    return guarded([&] {
        MHD_REQUIRE(b && o, "bad argument");
        auto cp = [](void *dst, const void *src, size_t bytes) {
            if (dst && bytes) MHD_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
        };
        const DevCsr *t[6] = {&b->e2n, &b->f2e, &b->c2f, &b->n2e, &b->e2f, &b->f2c};
        const int64_t rows[6] = {b->ne, b->nf, b->nc, b->n_nodes, b->ne, b->nf};
        for (int k = 0; k < 6; ++k)
        {
            cp(o->ptr[k], t[k]->ptr.p, (rows[k] + 1) * sizeof(int64_t));
            cp(o->idx[k], t[k]->idx.p, t[k]->idx.n * sizeof(int32_t));
            cp(o->sgn[k], t[k]->sgn.p, t[k]->sgn.n * sizeof(int8_t));
        }
        cp(o->cell_material, b->cell_material.p, b->nc * sizeof(int32_t));
        cp(o->face_tag, b->face_tag.p, b->nf * sizeof(int32_t));
    });
}

int mhd_gpu_tet_build_free(MhdTetBuild *b)
{
    return guarded([&] { delete b; });
}

} // extern "C"
