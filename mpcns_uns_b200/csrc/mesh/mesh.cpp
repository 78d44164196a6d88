// Host-side mesh services: builder, generators, metric and boundary classification.
//
// These produce the reference's own data model (uns::CellComplex, uns::Geometry,
// mhd::BoundaryInfo) so that a mesh built here and a mesh built by the reference from the
// same cells hash to the same uns::topology_hash and carry bit-identical geometry (the
// arithmetic below keeps the reference's operation order; build with -ffp-contract=off).
// The hash tables are flat open-addressing tables sized for 10^8 entities, replacing the
// reference's node-based std::unordered_map, which does not scale to 40M-cell meshes.
#include "mhd_mesh.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace
{
thread_local std::string g_err;

struct V3
{
    double x = 0, y = 0, z = 0;
};
inline V3 operator+(V3 a, const V3 &b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
inline V3 operator-(V3 a, const V3 &b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
inline V3 operator*(double s, V3 a) { a.x *= s; a.y *= s; a.z *= s; return a; }
inline V3 operator*(V3 a, double s) { a.x *= s; a.y *= s; a.z *= s; return a; }
inline V3 &operator+=(V3 &a, const V3 &b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
inline double dot(const V3 &a, const V3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(const V3 &a, const V3 &b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm(const V3 &a) { return std::sqrt(dot(a, a)); }

struct Csr
{
    std::vector<int64_t> ptr{0};
    std::vector<int32_t> idx;
    std::vector<int8_t> sgn;
    int32_t rows() const { return static_cast<int32_t>(ptr.size()) - 1; }
    void push(int32_t c, int s) { idx.push_back(c); sgn.push_back(static_cast<int8_t>(s)); }
    void close() { ptr.push_back(static_cast<int64_t>(idx.size())); }
    // rows visited in ascending order, so every transposed row is sorted by column
    // (reference: src/uns/complex/Incidence.cpp:8-26)
    Csr transpose(int32_t ncols) const
    {
        Csr t;
        t.ptr.assign(static_cast<size_t>(ncols) + 1, 0);
        for (int32_t c : idx) ++t.ptr[static_cast<size_t>(c) + 1];
        for (int32_t c = 0; c < ncols; ++c) t.ptr[c + 1] += t.ptr[c];
        t.idx.resize(idx.size());
        t.sgn.resize(sgn.size());
        std::vector<int64_t> fill(t.ptr.begin(), t.ptr.end() - 1);
        for (int32_t r = 0; r < rows(); ++r)
            for (int64_t k = ptr[r]; k < ptr[r + 1]; ++k)
            {
                const int64_t p = fill[idx[k]]++;
                t.idx[p] = r;
                t.sgn[p] = sgn[k];
            }
        return t;
    }
};

inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// splitmix64 stream: the documented generator of every seeded input of this library
struct SplitMix
{
    uint64_t s;
    explicit SplitMix(uint64_t seed) : s(seed) {}
    uint64_t next() { return mix64(s += 0x9e3779b97f4a7c15ULL); }
    double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; } // [0,1)
};

// open addressing uint64 -> int32
class U64Map
{
public:
    explicit U64Map(size_t expect = 1024) { rehash(cap_for(expect)); }
    int32_t find_or_insert(uint64_t key, int32_t value_if_new, bool &inserted)
    {
        if (2 * (n_ + 1) > keys_.size()) rehash(keys_.size() * 2);
        size_t i = mix64(key) & mask_;
        while (true)
        {
            if (vals_[i] < 0) { keys_[i] = key; vals_[i] = value_if_new; ++n_; inserted = true; return value_if_new; }
            if (keys_[i] == key) { inserted = false; return vals_[i]; }
            i = (i + 1) & mask_;
        }
    }
private:
    static size_t cap_for(size_t n) { size_t c = 1024; while (c < 2 * n) c *= 2; return c; }
    void rehash(size_t cap)
    {
        std::vector<uint64_t> ok = std::move(keys_);
        std::vector<int32_t> ov = std::move(vals_);
        keys_.assign(cap, 0);
        vals_.assign(cap, -1);
        mask_ = cap - 1;
        n_ = 0;
        for (size_t j = 0; j < ov.size(); ++j)
            if (ov[j] >= 0)
            {
                size_t i = mix64(ok[j]) & mask_;
                while (vals_[i] >= 0) i = (i + 1) & mask_;
                keys_[i] = ok[j]; vals_[i] = ov[j]; ++n_;
            }
    }
    std::vector<uint64_t> keys_;
    std::vector<int32_t> vals_;
    size_t mask_ = 0, n_ = 0;
};

// Builder with the numbering and orientation rules of the reference's uns::ComplexBuilder
// (src/uns/complex/ComplexBuilder.cpp): faces and edges are numbered in creation order, a
// face keeps the canonical form of the first loop that created it (start at the smallest
// node, second node smaller than the last), edges run from the smaller to the larger node.
class Builder
{
public:
    explicit Builder(int32_t n_nodes, size_t expect_faces = 1024) : n_nodes_(n_nodes), edge_map_(expect_faces)
    {
        size_t cap = 1024;
        while (cap < 2 * expect_faces) cap *= 2;
        face_tab_.assign(cap, -1);
    }

    // ComplexBuilder::canonicalize (:20-31)
    static bool canonicalize(int32_t *loop, int m)
    {
        int s = 0;
        for (int i = 1; i < m; ++i)
            if (loop[i] < loop[s]) s = i;
        std::rotate(loop, loop + s, loop + m);
        if (loop[1] > loop[m - 1]) { std::reverse(loop + 1, loop + m); return true; }
        return false;
    }

    // ComplexBuilder::add_cell (:45-76)
    void add_cell(const int32_t *const *loops, const int *sizes, int nloops, int material)
    {
        if (nloops < 4) throw std::runtime_error("ComplexBuilder: cell with fewer than 4 faces");
        int32_t loop[64], key[64];
        for (int l = 0; l < nloops; ++l)
        {
            const int m = sizes[l];
            if (m < 3) throw std::runtime_error("ComplexBuilder: face with fewer than 3 nodes");
            if (m > 64) throw std::runtime_error("face with more than 64 nodes");
            std::memcpy(loop, loops[l], m * sizeof(int32_t));
            std::memcpy(key, loops[l], m * sizeof(int32_t));
            std::sort(key, key + m);
            const bool flipped = canonicalize(loop, m);
            bool inserted = false;
            const int32_t fid = face_lookup(key, m, true, inserted);
            if (inserted)
            {
                for (int i = 0; i < m; ++i)
                {
                    const int32_t a = loop[i], b = loop[(i + 1) % m];
                    f2e_.push(edge_id(a, b), a < b ? +1 : -1);
                }
                f2e_.close();
            }
            c2f_.push(fid, flipped ? -1 : +1);
        }
        c2f_.close();
        material_.push_back(material);
    }

    // ComplexBuilder::tag_face (:87-92): later tags of the same node set win
    void tag_face(const int32_t *nodes, int m, int tag)
    {
        std::vector<int32_t> key(nodes, nodes + m);
        std::sort(key.begin(), key.end());
        tags_.emplace_back(std::move(key), tag);
    }

    // ComplexBuilder::finish (:102-134) without the per-rank bookkeeping (one rank owns everything)
    void finish(Csr &e2n, Csr &f2e, Csr &c2f, std::vector<int32_t> &material, std::vector<int32_t> &face_tag)
    {
        e2n = Csr();
        e2n.idx.reserve(2 * edges_.size());
        e2n.sgn.reserve(2 * edges_.size());
        e2n.ptr.reserve(edges_.size() + 1);
        for (const auto &e : edges_)
        {
            e2n.push(e.first, -1);
            e2n.push(e.second, +1);
            e2n.close();
        }
        f2e = std::move(f2e_);
        c2f = std::move(c2f_);
        material = std::move(material_);
        face_tag.assign(f2e.rows(), 0);
        for (const auto &t : tags_)
        {
            bool ins = false;
            const int32_t fid = face_lookup(t.first.data(), static_cast<int>(t.first.size()), false, ins);
            if (fid >= 0) face_tag[fid] = t.second;
        }
    }

private:
    int32_t edge_id(int32_t a, int32_t b)
    {
        const int32_t lo = std::min(a, b), hi = std::max(a, b);
        const uint64_t key = (static_cast<uint64_t>(static_cast<uint32_t>(lo)) << 32) | static_cast<uint32_t>(hi);
        bool ins = false;
        const int32_t id = edge_map_.find_or_insert(key, static_cast<int32_t>(edges_.size()), ins);
        if (ins) edges_.emplace_back(lo, hi);
        return id;
    }

    static uint64_t key_hash(const int32_t *key, int m)
    {
        uint64_t h = 0x243f6a8885a308d3ULL ^ static_cast<uint64_t>(m);
        for (int i = 0; i < m; ++i) h = mix64(h + static_cast<uint32_t>(key[i]) + 0x9e3779b97f4a7c15ULL);
        return h;
    }
    void grow_faces(size_t want)
    {
        size_t cap = face_tab_.size();
        while (cap < 2 * want) cap *= 2;
        if (cap == face_tab_.size()) return;
        std::vector<int32_t> tab(cap, -1);
        const size_t mask = cap - 1;
        for (int32_t f = 0; f < static_cast<int32_t>(key_ptr_.size()) - 1; ++f)
        {
            size_t i = key_hash(&key_pool_[key_ptr_[f]], static_cast<int>(key_ptr_[f + 1] - key_ptr_[f])) & mask;
            while (tab[i] >= 0) i = (i + 1) & mask;
            tab[i] = f;
        }
        face_tab_ = std::move(tab);
    }
    int32_t face_lookup(const int32_t *key, int m, bool insert, bool &inserted)
    {
        inserted = false;
        const int32_t nf = static_cast<int32_t>(key_ptr_.size()) - 1;
        if (insert && 2 * static_cast<size_t>(nf + 1) > face_tab_.size()) grow_faces(2 * static_cast<size_t>(nf + 1));
        const size_t mask = face_tab_.size() - 1;
        size_t i = key_hash(key, m) & mask;
        while (true)
        {
            const int32_t f = face_tab_[i];
            if (f < 0)
            {
                if (!insert) return -1;
                face_tab_[i] = nf;
                key_pool_.insert(key_pool_.end(), key, key + m);
                key_ptr_.push_back(static_cast<int64_t>(key_pool_.size()));
                inserted = true;
                return nf;
            }
            const int64_t b = key_ptr_[f], e = key_ptr_[f + 1];
            if (e - b == m && std::equal(key, key + m, key_pool_.begin() + b)) return f;
            i = (i + 1) & mask;
        }
    }

    int32_t n_nodes_;
    U64Map edge_map_;
    std::vector<std::pair<int32_t, int32_t>> edges_;
    std::vector<int32_t> face_tab_;
    std::vector<int32_t> key_pool_;
    std::vector<int64_t> key_ptr_{0};
    Csr f2e_, c2f_;
    std::vector<int32_t> material_;
    std::vector<std::pair<std::vector<int32_t>, int>> tags_;
};

// A hexahedral mesh before building: reference uns::HexMesh (include/uns/generate/HexMesh.h:13-21)
struct HexList
{
    std::vector<V3> x;
    std::vector<std::array<int32_t, 8>> hex;
    std::vector<int> material;
    struct Tagged { std::array<int32_t, 4> nodes; std::array<int, 4> local; int tag; int32_t cell; };
    std::vector<Tagged> tagged;
    std::vector<std::string> tag_names;
};

// uns::make_box (src/uns/generate/BoxMesh.cpp:5-33)
HexList make_box(int nx, int ny, int nz, V3 lo, V3 hi)
{
    HexList h;
    auto nid = [&](int i, int j, int k) { return static_cast<int32_t>((k * (ny + 1) + j) * (nx + 1) + i); };
    h.x.resize(static_cast<size_t>(nx + 1) * (ny + 1) * (nz + 1));
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i <= nx; ++i)
                h.x[nid(i, j, k)] = {lo.x + (hi.x - lo.x) * i / nx, lo.y + (hi.y - lo.y) * j / ny, lo.z + (hi.z - lo.z) * k / nz};
    h.tag_names = {"", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax"};
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
            {
                std::array<int32_t, 8> v;
                for (int q = 0; q < 8; ++q) v[q] = nid(i + (q & 1), j + ((q >> 1) & 1), k + ((q >> 2) & 1));
                const int32_t c = static_cast<int32_t>(h.hex.size());
                h.hex.push_back(v);
                h.material.push_back(0);
                auto tag = [&](int a, int b, int cc, int d, int t) { h.tagged.push_back({{v[a], v[b], v[cc], v[d]}, {a, b, cc, d}, t, c}); };
                if (i == 0) tag(0, 2, 4, 6, 1);
                if (i == nx - 1) tag(1, 3, 5, 7, 2);
                if (j == 0) tag(0, 1, 4, 5, 3);
                if (j == ny - 1) tag(2, 3, 6, 7, 4);
                if (k == 0) tag(0, 1, 2, 3, 5);
                if (k == nz - 1) tag(4, 5, 6, 7, 6);
            }
    return h;
}

// uns::make_cubed_sphere_shell (src/uns/generate/CubedSphereMesh.cpp:12-83), spherical outer surface
HexList make_shell(int M, int nr, int n_solid, double r_in, double r_out, double r_stretch)
{
    HexList h;
    h.tag_names = {"", "inner", "outer"};
    std::vector<double> frac(nr + 1);
    {
        double sum = 0, dr = 1;
        std::vector<double> w(nr);
        for (int k = 0; k < nr; ++k) { w[k] = dr; sum += dr; dr *= r_stretch; }
        frac[0] = 0;
        for (int k = 0; k < nr; ++k) frac[k + 1] = frac[k] + w[k] / sum;
    }
    const double pi4 = std::atan(1.0);
    U64Map ids(static_cast<size_t>(6) * (M + 1) * (M + 1) * (nr + 1));
    auto node = [&](const int q[3], int k) -> int32_t {
        const uint64_t key = (static_cast<uint64_t>(q[0]) << 48) | (static_cast<uint64_t>(q[1]) << 32) | (static_cast<uint64_t>(q[2]) << 16) |
                             static_cast<uint64_t>(k);
        bool ins = false;
        const int32_t id = ids.find_or_insert(key, static_cast<int32_t>(h.x.size()), ins);
        if (!ins) return id;
        auto ang = [&](int i) { return std::tan(pi4 * (2.0 * i / M - 1.0)); };
        V3 d{ang(q[0]), ang(q[1]), ang(q[2])};
        d = d * (1.0 / norm(d));
        const double r = r_in + (r_out - r_in) * frac[k];
        h.x.push_back(r * d);
        return id;
    };
    for (int axis = 0; axis < 3; ++axis)
        for (int side = 0; side <= 1; ++side)
            for (int iu = 0; iu < M; ++iu)
                for (int iv = 0; iv < M; ++iv)
                    for (int k = 0; k < nr; ++k)
                    {
                        std::array<int32_t, 8> v;
                        for (int q = 0; q < 8; ++q)
                        {
                            int lat[3];
                            lat[axis] = side ? M : 0;
                            lat[(axis + 1) % 3] = iu + (q & 1);
                            lat[(axis + 2) % 3] = iv + ((q >> 1) & 1);
                            v[q] = node(lat, k + ((q >> 2) & 1));
                        }
                        const V3 e1 = h.x[v[1]] - h.x[v[0]], e2 = h.x[v[2]] - h.x[v[0]], e3 = h.x[v[4]] - h.x[v[0]];
                        if (dot(cross(e1, e2), e3) < 0) { std::swap(v[1], v[2]); std::swap(v[5], v[6]); }
                        const int32_t c = static_cast<int32_t>(h.hex.size());
                        h.hex.push_back(v);
                        h.material.push_back(k < n_solid ? 1 : 0);
                        if (k == 0) h.tagged.push_back({{v[0], v[1], v[2], v[3]}, {0, 1, 2, 3}, 1, c});
                        if (k == nr - 1) h.tagged.push_back({{v[4], v[5], v[6], v[7]}, {4, 5, 6, 7}, 2, c});
                    }
    return h;
}

struct HostMesh
{
    int32_t n_nodes = 0;
    std::vector<double> x;
    Csr e2n, f2e, c2f, e2f, f2c, n2e;
    std::vector<int32_t> cell_material, face_tag;
    std::vector<std::string> tag_names;

    bool have_geo = false;
    std::vector<double> edge_vec, edge_mid, edge_len, face_area, face_center, face_area_mag, cell_center, cell_volume, cell_min_tet_volume,
        edge_dual_area, ec_weight, ef_weight, star0, star1, star2, star3;
    std::vector<int64_t> ec_ptr;
    std::vector<int32_t> ec_cell, ec_misoriented;

    bool have_bc = false;
    std::vector<int8_t> face_kind, edge_mode;

    // a hexahedral list before its complex is built elsewhere (mhdm_shell_hexes): 8 nodes per hexahedron,
    // its material, and the tagged triangles of the tetrahedral split (3 nodes each) with their tag ids
    std::vector<int32_t> hex8, hex_material, tag_tri, tag_tri_id;

    int32_t ne() const { return e2n.rows(); }
    int32_t nf() const { return f2e.rows(); }
    int32_t nc() const { return c2f.rows(); }
    V3 X(int32_t v) const { return {x[3 * static_cast<size_t>(v)], x[3 * static_cast<size_t>(v) + 1], x[3 * static_cast<size_t>(v) + 2]}; }
};

void finish_mesh(HostMesh &m, Builder &b)
{
    b.finish(m.e2n, m.f2e, m.c2f, m.cell_material, m.face_tag);
    m.n2e = m.e2n.transpose(m.n_nodes);
    m.e2f = m.f2e.transpose(m.ne());
    m.f2c = m.c2f.transpose(m.nf());
}

// The two triangles of a tagged quad of the tetrahedral split: the quad is cut along its lattice diagonal,
// from the AND to the OR of its 4 local corner indices; fn(tri nodes, tag) in the builder's tag order.
template <class F> void split_tags(const HexList &h, F &&fn)
{
    for (const auto &t : h.tagged)
    {
        int lo = 7, hi = 0;
        for (int q : t.local) { lo &= q; hi |= q; }
        const auto &v = h.hex[t.cell];
        for (int q : t.local)
        {
            if (q == lo || q == hi) continue;
            const int32_t tri[3] = {v[lo], v[q], v[hi]};
            fn(tri, t.tag);
        }
    }
}

// Cells of a hexahedral list: the hexahedron itself (reference ComplexBuilder::add_hex,
// ComplexBuilder.cpp:78-85) or its 6 Kuhn tetrahedra.
HostMesh build_hexes(HexList &&h, bool as_tets)
{
    HostMesh m;
    m.n_nodes = static_cast<int32_t>(h.x.size());
    m.x.resize(3 * h.x.size());
    for (size_t i = 0; i < h.x.size(); ++i) { m.x[3 * i] = h.x[i].x; m.x[3 * i + 1] = h.x[i].y; m.x[3 * i + 2] = h.x[i].z; }
    m.tag_names = h.tag_names;
    const size_t expect = h.hex.size() * (as_tets ? 13 : 4) + 1024;
    Builder b(m.n_nodes, expect);
    static const int L[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
    // Kuhn paths 0 -> a -> a|b -> 7 over the 6 orders of the local axis bits; sign = parity of the order
    static const int P[6][3] = {{1, 2, 4}, {1, 4, 2}, {2, 1, 4}, {2, 4, 1}, {4, 1, 2}, {4, 2, 1}};
    static const int PAR[6] = {+1, -1, -1, +1, +1, -1};
    int32_t buf[6][4];
    const int32_t *lp[6];
    int sz[6];
    for (size_t c = 0; c < h.hex.size(); ++c)
    {
        const auto &v = h.hex[c];
        if (!as_tets)
        {
            for (int f = 0; f < 6; ++f)
            {
                for (int k = 0; k < 4; ++k) buf[f][k] = v[L[f][k]];
                lp[f] = buf[f];
                sz[f] = 4;
            }
            b.add_cell(lp, sz, 6, h.material[c]);
            continue;
        }
        for (int t = 0; t < 6; ++t)
        {
            const int a = P[t][0], ab = P[t][0] | P[t][1];
            int32_t p[4] = {v[0], v[a], v[ab], v[7]};
            if (PAR[t] < 0) std::swap(p[1], p[2]); // positively oriented (right-handed local frame)
            // outward loops of a positive tetrahedron (p0,p1,p2,p3)
            const int32_t F[4][3] = {{p[0], p[2], p[1]}, {p[0], p[1], p[3]}, {p[1], p[2], p[3]}, {p[0], p[3], p[2]}};
            for (int f = 0; f < 4; ++f)
            {
                std::memcpy(buf[f], F[f], 3 * sizeof(int32_t));
                lp[f] = buf[f];
                sz[f] = 3;
            }
            b.add_cell(lp, sz, 4, h.material[c]);
        }
    }
    if (as_tets)
        split_tags(h, [&](const int32_t *tri, int tag) { b.tag_face(tri, 3, tag); });
    else
        for (const auto &t : h.tagged) b.tag_face(t.nodes.data(), 4, t.tag);
    finish_mesh(m, b);
    return m;
}

// uns::compute_geometry (src/uns/geometry/Geometry.cpp:17-169), same operation order.
void compute_geometry(HostMesh &m)
{
    const int32_t ne = m.ne(), nf = m.nf(), nc = m.nc(), nn = m.n_nodes;
    auto put3 = [](std::vector<double> &a, size_t i, const V3 &v) { a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z; };
    auto get3 = [](const std::vector<double> &a, size_t i) { return V3{a[3 * i], a[3 * i + 1], a[3 * i + 2]}; };
    auto edge_nodes = [&](int32_t e, int32_t &s, int32_t &t) {
        s = t = -1;
        for (int64_t k = m.e2n.ptr[e]; k < m.e2n.ptr[e + 1]; ++k) (m.e2n.sgn[k] < 0 ? s : t) = m.e2n.idx[k];
    };
    auto face_loop = [&](int32_t f, std::vector<int32_t> &nodes) {
        nodes.clear();
        for (int64_t k = m.f2e.ptr[f]; k < m.f2e.ptr[f + 1]; ++k)
        {
            int32_t a, b;
            edge_nodes(m.f2e.idx[k], a, b);
            nodes.push_back(m.f2e.sgn[k] > 0 ? a : b);
        }
    };
    m.edge_vec.assign(3 * static_cast<size_t>(ne), 0);
    m.edge_mid.assign(3 * static_cast<size_t>(ne), 0);
    m.edge_len.assign(ne, 0);
    for (int32_t e = 0; e < ne; ++e)
    {
        int32_t a, b;
        edge_nodes(e, a, b);
        const V3 v = m.X(b) - m.X(a);
        put3(m.edge_vec, e, v);
        put3(m.edge_mid, e, 0.5 * (m.X(a) + m.X(b)));
        m.edge_len[e] = norm(v);
    }
    m.face_area.assign(3 * static_cast<size_t>(nf), 0);
    m.face_center.assign(3 * static_cast<size_t>(nf), 0);
    m.face_area_mag.assign(nf, 0);
    std::vector<int32_t> loop;
    for (int32_t f = 0; f < nf; ++f)
    {
        face_loop(f, loop);
        const size_t k = loop.size();
        V3 p0;
        for (int32_t v : loop) p0 += m.X(v);
        p0 = p0 * (1.0 / static_cast<double>(k));
        V3 cw;
        double wsum = 0;
        for (size_t i = 0; i < k; ++i)
        {
            const V3 a = m.X(loop[i]), b = m.X(loop[(i + 1) % k]);
            const double w = 0.5 * norm(cross(a - p0, b - p0));
            cw += w * ((p0 + a + b) * (1.0 / 3.0));
            wsum += w;
        }
        const V3 c = wsum > 0 ? cw * (1.0 / wsum) : p0;
        V3 A;
        for (size_t i = 0; i < k; ++i) A += 0.5 * cross(m.X(loop[i]) - c, m.X(loop[(i + 1) % k]) - c);
        put3(m.face_center, f, c);
        put3(m.face_area, f, A);
        m.face_area_mag[f] = norm(A);
    }
    m.cell_center.assign(3 * static_cast<size_t>(nc), 0);
    m.cell_volume.assign(nc, 0);
    m.cell_min_tet_volume.assign(nc, 0);
    m.star0.assign(nn, 0);
    m.star1.assign(ne, 0);
    m.star2.assign(nf, 0);
    m.star3.assign(nc, 0);
    m.edge_dual_area.assign(3 * static_cast<size_t>(ne), 0);
    m.ec_misoriented.assign(ne, 0);
    m.ec_ptr.assign(static_cast<size_t>(ne) + 1, 0);
    m.ec_cell.clear();
    std::vector<int32_t> tmp;
    for (int32_t e = 0; e < ne; ++e)
    {
        tmp.clear();
        for (int64_t k = m.e2f.ptr[e]; k < m.e2f.ptr[e + 1]; ++k)
        {
            const int32_t f = m.e2f.idx[k];
            for (int64_t q = m.f2c.ptr[f]; q < m.f2c.ptr[f + 1]; ++q) tmp.push_back(m.f2c.idx[q]);
        }
        std::sort(tmp.begin(), tmp.end());
        tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
        m.ec_cell.insert(m.ec_cell.end(), tmp.begin(), tmp.end());
        m.ec_ptr[e + 1] = static_cast<int64_t>(m.ec_cell.size());
    }
    m.ec_weight.assign(m.ec_cell.size(), 0.0);
    m.ef_weight.assign(m.e2f.idx.size(), 0.0);
    std::vector<double> dual_len_face(nf, 0.0);
    std::vector<int32_t> cn;
    for (int32_t c = 0; c < nc; ++c)
    {
        cn.clear();
        for (int64_t k = m.c2f.ptr[c]; k < m.c2f.ptr[c + 1]; ++k)
        {
            face_loop(m.c2f.idx[k], loop);
            cn.insert(cn.end(), loop.begin(), loop.end());
        }
        std::sort(cn.begin(), cn.end());
        cn.erase(std::unique(cn.begin(), cn.end()), cn.end());
        V3 xc0;
        for (int32_t v : cn) xc0 += m.X(v);
        xc0 = xc0 * (1.0 / static_cast<double>(cn.size()));
        double vsum = 0;
        V3 vc;
        for (int64_t kf = m.c2f.ptr[c]; kf < m.c2f.ptr[c + 1]; ++kf)
        {
            const int32_t f = m.c2f.idx[kf];
            const int s = m.c2f.sgn[kf];
            face_loop(f, loop);
            const size_t k = loop.size();
            const V3 cf = get3(m.face_center, f);
            for (size_t i = 0; i < k; ++i)
            {
                const V3 a = m.X(loop[i]), b = m.X(loop[(i + 1) % k]);
                const V3 at = (0.5 * s) * cross(a - cf, b - cf);
                const double vt = dot(at, cf - xc0) / 3.0;
                vc += vt * ((xc0 + cf + a + b) * 0.25);
                vsum += vt;
            }
        }
        const V3 xc = vsum > 0 ? vc * (1.0 / vsum) : xc0;
        put3(m.cell_center, c, xc);
        double vol = 0, mintet = std::numeric_limits<double>::max();
        for (int64_t kf = m.c2f.ptr[c]; kf < m.c2f.ptr[c + 1]; ++kf)
        {
            const int32_t f = m.c2f.idx[kf];
            const int s = m.c2f.sgn[kf];
            face_loop(f, loop);
            const size_t k = loop.size();
            const V3 cf = get3(m.face_center, f);
            dual_len_face[f] += norm(cf - xc);
            for (size_t i = 0; i < k; ++i)
            {
                const int32_t va = loop[i], vb = loop[(i + 1) % k];
                const V3 a = m.X(va), b = m.X(vb);
                const V3 at = (0.5 * s) * cross(a - cf, b - cf);
                const double vt = dot(at, cf - xc) / 3.0;
                vol += vt;
                mintet = std::min(mintet, vt);
                m.star0[va] += 0.5 * vt;
                m.star0[vb] += 0.5 * vt;
                const int64_t ke = m.f2e.ptr[f] + static_cast<int64_t>(i);
                const int32_t e = m.f2e.idx[ke];
                const int se = s * m.f2e.sgn[ke];
                const V3 mid = get3(m.edge_mid, e);
                const V3 piece = (0.5 * se) * cross(xc - mid, cf - mid);
                V3 da = get3(m.edge_dual_area, e);
                da += piece;
                put3(m.edge_dual_area, e, da);
                if (dot(piece, get3(m.edge_vec, e)) <= 0) ++m.ec_misoriented[e];
                const auto lo = m.ec_cell.begin() + m.ec_ptr[e], hi = m.ec_cell.begin() + m.ec_ptr[e + 1];
                m.ec_weight[std::lower_bound(lo, hi, c) - m.ec_cell.begin()] += norm(piece);
                const auto flo = m.e2f.idx.begin() + m.e2f.ptr[e], fhi = m.e2f.idx.begin() + m.e2f.ptr[e + 1];
                m.ef_weight[std::lower_bound(flo, fhi, f) - m.e2f.idx.begin()] += norm(piece);
            }
        }
        m.cell_volume[c] = vol;
        m.cell_min_tet_volume[c] = mintet;
        m.star3[c] = vol > 0 ? 1.0 / vol : 0.0;
    }
    for (int32_t e = 0; e < ne; ++e)
    {
        double s = 0;
        for (int64_t k = m.ec_ptr[e]; k < m.ec_ptr[e + 1]; ++k) s += m.ec_weight[k];
        if (s > 0)
        {
            for (int64_t k = m.ec_ptr[e]; k < m.ec_ptr[e + 1]; ++k) m.ec_weight[k] /= s;
            for (int64_t k = m.e2f.ptr[e]; k < m.e2f.ptr[e + 1]; ++k) m.ef_weight[k] /= s;
        }
        m.star1[e] = m.edge_len[e] > 0 ? norm(get3(m.edge_dual_area, e)) / m.edge_len[e] : 0.0;
    }
    for (int32_t f = 0; f < nf; ++f) m.star2[f] = m.face_area_mag[f] > 0 ? dual_len_face[f] / m.face_area_mag[f] : 0.0;
    m.have_geo = true;
}

// mhd::BoundaryInfo::build (Common/boundary/BoundaryInfo.cpp:9-49)
// face kinds: 0 Interior, 1 Wall, 2 Inflow, 3 Outflow, 4 Skip; edge modes: 0 free, 1 wall (E = 0), 2 inflow
void boundary(HostMesh &m, const std::string &bc_default, const std::map<std::string, std::string> &by_tag, const double *u_inf)
{
    if (!m.have_geo) compute_geometry(m);
    const int32_t nf = m.nf();
    m.face_kind.assign(nf, 0);
    m.edge_mode.assign(m.ne(), 0);
    for (int32_t f = 0; f < nf; ++f)
    {
        const int64_t b = m.f2c.ptr[f];
        const int n = static_cast<int>(m.f2c.ptr[f + 1] - b);
        if (n == 2)
        {
            const bool s0 = m.cell_material[m.f2c.idx[b]] == 1, s1 = m.cell_material[m.f2c.idx[b + 1]] == 1;
            m.face_kind[f] = (s0 && s1) ? 4 : (s0 || s1) ? 1 : 0;
            continue;
        }
        const int32_t c = m.f2c.idx[b];
        if (m.cell_material[c] == 1) { m.face_kind[f] = 4; continue; }
        const int tag = m.face_tag[f];
        const std::string name = tag > 0 && tag < static_cast<int>(m.tag_names.size()) ? m.tag_names[tag] : "";
        const auto it = by_tag.find(name);
        const std::string type = it != by_tag.end() ? it->second : bc_default;
        if (type == "wall") m.face_kind[f] = 1;
        else if (type == "inflow") m.face_kind[f] = 2;
        else if (type == "outflow") m.face_kind[f] = 3;
        else if (type == "farfield")
        {
            const double s = m.f2c.sgn[b] / m.face_area_mag[f];
            const V3 A{m.face_area[3 * static_cast<size_t>(f)], m.face_area[3 * static_cast<size_t>(f) + 1], m.face_area[3 * static_cast<size_t>(f) + 2]};
            const V3 n = s * A;
            const V3 u{u_inf[0], u_inf[1], u_inf[2]};
            m.face_kind[f] = dot(u, n) < 0 ? 2 : 3;
        }
        else
            throw std::runtime_error("unknown boundary type '" + type + "' for face tag '" + name + "' (wall|farfield|inflow|outflow)");
    }
    for (int32_t f = 0; f < nf; ++f)
        if (m.face_kind[f] == 2)
            for (int64_t k = m.f2e.ptr[f]; k < m.f2e.ptr[f + 1]; ++k) m.edge_mode[m.f2e.idx[k]] = 2;
    for (int32_t f = 0; f < nf; ++f)
        if (m.face_kind[f] == 1)
            for (int64_t k = m.f2e.ptr[f]; k < m.f2e.ptr[f + 1]; ++k) m.edge_mode[m.f2e.idx[k]] = 1;
    m.have_bc = true;
}

template <class F> int guarded(F &&f)
{
    try { f(); return 0; }
    catch (const std::exception &e) { g_err = e.what(); return -1; }
}
} // namespace

struct MhdHostMesh : HostMesh
{
};

extern "C" {

const char *mhdm_last_error(void) { return g_err.c_str(); }

int mhdm_from_cells(int32_t n_nodes, const double *x, int32_t n_cells, const int64_t *cell_ptr, const int64_t *loop_ptr,
                    const int32_t *loop_nodes, const int32_t *material, int32_t n_tagged, const int64_t *tag_ptr, const int32_t *tag_nodes,
                    const int32_t *tag_id, int32_t n_names, const char *const *tag_names, MhdHostMesh **out)
{
    return guarded([&] {
        if (!out) throw std::runtime_error("null output handle");
        auto *m = new MhdHostMesh;
        try
        {
            m->n_nodes = n_nodes;
            m->x.assign(x, x + 3 * static_cast<size_t>(n_nodes));
            for (int32_t i = 0; i < n_names; ++i) m->tag_names.emplace_back(tag_names[i]);
            Builder b(n_nodes, static_cast<size_t>(n_cells) * 4 + 1024);
            std::vector<const int32_t *> lp;
            std::vector<int> sz;
            for (int32_t c = 0; c < n_cells; ++c)
            {
                lp.clear();
                sz.clear();
                for (int64_t l = cell_ptr[c]; l < cell_ptr[c + 1]; ++l)
                {
                    lp.push_back(loop_nodes + loop_ptr[l]);
                    sz.push_back(static_cast<int>(loop_ptr[l + 1] - loop_ptr[l]));
                }
                for (int64_t l = cell_ptr[c]; l < cell_ptr[c + 1]; ++l)
                    for (int64_t q = loop_ptr[l]; q < loop_ptr[l + 1]; ++q)
                        if (loop_nodes[q] < 0 || loop_nodes[q] >= n_nodes) throw std::runtime_error("node id out of range");
                b.add_cell(lp.data(), sz.data(), static_cast<int>(lp.size()), material ? material[c] : 0);
            }
            for (int32_t t = 0; t < n_tagged; ++t) b.tag_face(tag_nodes + tag_ptr[t], static_cast<int>(tag_ptr[t + 1] - tag_ptr[t]), tag_id[t]);
            finish_mesh(*m, b);
        }
        catch (...) { delete m; throw; }
        *out = m;
    });
}

int mhdm_reorder_cells(const MhdHostMesh *src, const int32_t *order, MhdHostMesh **out)
{
    return guarded([&] {
        if (!src || !order || !out) throw std::runtime_error("null argument");
        const HostMesh &m = *src;
        const int32_t nc = m.nc();
        std::vector<char> seen(nc, 0);
        for (int32_t i = 0; i < nc; ++i)
        {
            if (order[i] < 0 || order[i] >= nc || seen[order[i]]) throw std::runtime_error("order is not a permutation of the cells");
            seen[order[i]] = 1;
        }
        // the loop of face f as the builder stored it: the node at which each edge is entered
        auto face_loop = [&](int32_t f, std::vector<int32_t> &loop) {
            loop.clear();
            for (int64_t k = m.f2e.ptr[f]; k < m.f2e.ptr[f + 1]; ++k)
            {
                const int32_t e = m.f2e.idx[k];
                int32_t a = -1, b = -1;
                for (int64_t q = m.e2n.ptr[e]; q < m.e2n.ptr[e + 1]; ++q) (m.e2n.sgn[q] < 0 ? a : b) = m.e2n.idx[q];
                loop.push_back(m.f2e.sgn[k] > 0 ? a : b);
            }
        };
        auto *r = new MhdHostMesh;
        try
        {
            r->n_nodes = m.n_nodes;
            r->x = m.x;
            r->tag_names = m.tag_names;
            Builder b(m.n_nodes, static_cast<size_t>(nc) * 4 + 1024);
            std::vector<std::vector<int32_t>> loops;
            std::vector<const int32_t *> lp;
            std::vector<int> sz;
            for (int32_t i = 0; i < nc; ++i)
            {
                const int32_t c = order[i];
                const int64_t k0 = m.c2f.ptr[c], k1 = m.c2f.ptr[c + 1];
                loops.resize(static_cast<size_t>(k1 - k0));
                lp.clear();
                sz.clear();
                for (int64_t k = k0; k < k1; ++k)
                {
                    auto &l = loops[static_cast<size_t>(k - k0)];
                    face_loop(m.c2f.idx[k], l);
                    if (m.c2f.sgn[k] < 0) std::reverse(l.begin(), l.end()); // outward
                    lp.push_back(l.data());
                    sz.push_back(static_cast<int>(l.size()));
                }
                b.add_cell(lp.data(), sz.data(), static_cast<int>(lp.size()), m.cell_material[c]);
            }
            std::vector<int32_t> l;
            for (int32_t f = 0; f < m.nf(); ++f)
                if (m.face_tag[f] > 0)
                {
                    face_loop(f, l);
                    b.tag_face(l.data(), static_cast<int>(l.size()), m.face_tag[f]);
                }
            finish_mesh(*r, b);
        }
        catch (...) { delete r; throw; }
        *out = r;
    });
}

int mhdm_box(int32_t nx, int32_t ny, int32_t nz, const double *lo, const double *hi, int32_t as_tets, double jitter, uint64_t seed,
             MhdHostMesh **out)
{
    return guarded([&] {
        if (nx < 1 || ny < 1 || nz < 1) throw std::runtime_error("box: cell counts must be positive");
        HexList h = make_box(nx, ny, nz, {lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]});
        if (jitter > 0)
        {
            SplitMix rng(seed);
            const double hx = (hi[0] - lo[0]) / nx, hy = (hi[1] - lo[1]) / ny, hz = (hi[2] - lo[2]) / nz;
            for (int k = 1; k < nz; ++k)
                for (int j = 1; j < ny; ++j)
                    for (int i = 1; i < nx; ++i)
                    {
                        V3 &p = h.x[static_cast<size_t>((k * (ny + 1) + j) * (nx + 1) + i)];
                        p.x += jitter * hx * (2.0 * rng.uniform() - 1.0);
                        p.y += jitter * hy * (2.0 * rng.uniform() - 1.0);
                        p.z += jitter * hz * (2.0 * rng.uniform() - 1.0);
                    }
        }
        auto *m = new MhdHostMesh;
        static_cast<HostMesh &>(*m) = build_hexes(std::move(h), as_tets != 0);
        *out = m;
    });
}

int mhdm_shell(int32_t ncube, int32_t nr, int32_t n_solid, double r_in, double r_out, double r_stretch, int32_t as_tets, MhdHostMesh **out)
{
    return guarded([&] {
        if (ncube < 1 || nr < 1 || ncube > 4096 || nr > 65534) throw std::runtime_error("shell: bad resolution");
        auto *m = new MhdHostMesh;
        static_cast<HostMesh &>(*m) = build_hexes(make_shell(ncube, nr, n_solid, r_in, r_out, r_stretch), as_tets != 0);
        *out = m;
    });
}

int mhdm_shell_hexes(int32_t ncube, int32_t nr, int32_t n_solid, double r_in, double r_out, double r_stretch, MhdHostMesh **out)
{
    return guarded([&] {
        if (ncube < 1 || nr < 1 || ncube > 4096 || nr > 65534) throw std::runtime_error("shell: bad resolution");
        HexList h = make_shell(ncube, nr, n_solid, r_in, r_out, r_stretch);
        auto *m = new MhdHostMesh;
        m->n_nodes = static_cast<int32_t>(h.x.size());
        m->x.resize(3 * h.x.size());
        for (size_t i = 0; i < h.x.size(); ++i) { m->x[3 * i] = h.x[i].x; m->x[3 * i + 1] = h.x[i].y; m->x[3 * i + 2] = h.x[i].z; }
        m->tag_names = h.tag_names;
        m->hex8.resize(8 * h.hex.size());
        for (size_t c = 0; c < h.hex.size(); ++c) std::copy(h.hex[c].begin(), h.hex[c].end(), m->hex8.begin() + 8 * c);
        m->hex_material.assign(h.material.begin(), h.material.end());
        split_tags(h, [&](const int32_t *tri, int tag) {
            m->tag_tri.insert(m->tag_tri.end(), tri, tri + 3);
            m->tag_tri_id.push_back(tag);
        });
        *out = m;
    });
}

int mhdm_reserve_complex(MhdHostMesh *m, int64_t n_edges, int64_t n_faces, int64_t n_cells, int32_t faces_per_cell,
                         int32_t edges_per_face)
{
    return guarded([&] {
        if (!m || n_edges < 0 || n_faces < 0 || n_cells < 0 || n_edges > INT32_MAX || n_faces > INT32_MAX || n_cells > INT32_MAX)
            throw std::runtime_error("bad argument");
        auto size = [](Csr &t, int64_t rows, int64_t nnz) {
            t.ptr.assign(static_cast<size_t>(rows) + 1, 0);
            t.idx.assign(static_cast<size_t>(nnz), 0);
            t.sgn.assign(static_cast<size_t>(nnz), 0);
        };
        const int64_t n_c2f = n_cells * faces_per_cell, n_f2e = n_faces * edges_per_face;
        size(m->e2n, n_edges, 2 * n_edges); size(m->f2e, n_faces, n_f2e); size(m->c2f, n_cells, n_c2f);
        size(m->n2e, m->n_nodes, 2 * n_edges); size(m->e2f, n_edges, n_f2e); size(m->f2c, n_faces, n_c2f);
        m->cell_material.assign(static_cast<size_t>(n_cells), 0);
        m->face_tag.assign(static_cast<size_t>(n_faces), 0);
        std::vector<int32_t>().swap(m->hex8);
        std::vector<int32_t>().swap(m->hex_material);
        std::vector<int32_t>().swap(m->tag_tri);
        std::vector<int32_t>().swap(m->tag_tri_id);
        m->have_geo = m->have_bc = false;
    });
}

void *mhdm_array_mut(MhdHostMesh *m, const char *name, int64_t *count)
{
    return const_cast<void *>(mhdm_array(m, name, count));
}

void mhdm_free(MhdHostMesh *m) { delete m; }

void mhdm_counts(const MhdHostMesh *m, int32_t *counts)
{
    counts[0] = m->n_nodes; counts[1] = m->ne(); counts[2] = m->nf(); counts[3] = m->nc();
}

// uns::topology_hash (src/uns/complex/CellComplex.cpp:56-70): FNV-1a over e2n, f2e, c2f
uint64_t mhdm_topology_hash(const MhdHostMesh *m)
{
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](const void *p, size_t n) {
        const unsigned char *b = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ull; }
    };
    for (const Csr *t : {&m->e2n, &m->f2e, &m->c2f})
    {
        mix(t->ptr.data(), t->ptr.size() * sizeof(int64_t));
        mix(t->idx.data(), t->idx.size() * sizeof(int32_t));
        mix(t->sgn.data(), t->sgn.size());
    }
    return h;
}

int mhdm_set_geometry(MhdHostMesh *m, const MhdGeometryArrays *g)
{
    return guarded([&] {
        if (!m || !g || !g->ec_ptr) throw std::runtime_error("null argument");
        const size_t ne = m->ne(), nf = m->nf(), nc = m->nc(), nn = m->n_nodes;
        auto cp = [](std::vector<double> &v, const double *p, size_t n) {
            if (!p) throw std::runtime_error("missing geometry array");
            v.assign(p, p + n);
        };
        cp(m->edge_vec, g->edge_vec, 3 * ne); cp(m->edge_mid, g->edge_mid, 3 * ne); cp(m->edge_len, g->edge_len, ne);
        cp(m->face_area, g->face_area, 3 * nf); cp(m->face_center, g->face_center, 3 * nf); cp(m->face_area_mag, g->face_area_mag, nf);
        cp(m->cell_center, g->cell_center, 3 * nc); cp(m->cell_volume, g->cell_volume, nc);
        cp(m->cell_min_tet_volume, g->cell_min_tet_volume, nc); cp(m->edge_dual_area, g->edge_dual_area, 3 * ne);
        cp(m->star0, g->star0, nn); cp(m->star1, g->star1, ne); cp(m->star2, g->star2, nf); cp(m->star3, g->star3, nc);
        m->ec_ptr.assign(g->ec_ptr, g->ec_ptr + ne + 1);
        const size_t nec = static_cast<size_t>(m->ec_ptr[ne]);
        if (!g->ec_cell || !g->ec_misoriented) throw std::runtime_error("missing geometry array");
        m->ec_cell.assign(g->ec_cell, g->ec_cell + nec);
        cp(m->ec_weight, g->ec_weight, nec);
        cp(m->ef_weight, g->ef_weight, m->e2f.idx.size());
        m->ec_misoriented.assign(g->ec_misoriented, g->ec_misoriented + ne);
        m->have_geo = true;
    });
}

int mhdm_compute_geometry(MhdHostMesh *m)
{
    return guarded([&] { if (!m->have_geo) compute_geometry(*m); });
}

int mhdm_boundary(MhdHostMesh *m, const char *bc_default, int32_t n_pairs, const char *const *tag_names, const char *const *types,
                  const double *u_inf)
{
    return guarded([&] {
        std::map<std::string, std::string> by;
        for (int32_t i = 0; i < n_pairs; ++i) by[tag_names[i]] = types[i];
        const double zero[3] = {0, 0, 0};
        boundary(*m, bc_default ? bc_default : "outflow", by, u_inf ? u_inf : zero);
    });
}

int mhdm_tag_types(const MhdHostMesh *m, const char *bc_default, int32_t n_pairs, const char *const *tag_names, const char *const *types,
                   int32_t cap, int8_t *tag_type, int8_t *type_none, int32_t *n_tags)
{
    return guarded([&] {
        std::map<std::string, std::string> by;
        for (int32_t i = 0; i < n_pairs; ++i) by[tag_names[i]] = types[i];
        const std::string def = bc_default ? bc_default : "outflow";
        // the type a face of tag name `name` takes in boundary(): its pair, else the default
        auto code = [&](const std::string &name) -> int8_t {
            const auto it = by.find(name);
            const std::string t = it != by.end() ? it->second : def;
            return t == "wall" ? 1 : t == "inflow" ? 2 : t == "outflow" ? 3 : t == "farfield" ? 5 : 0;
        };
        const int32_t nt = static_cast<int32_t>(m->tag_names.size());
        if (cap < nt) throw std::runtime_error("tag_type holds fewer entries than the mesh has tag names");
        for (int32_t t = 0; t < nt; ++t) tag_type[t] = t > 0 ? code(m->tag_names[t]) : code("");
        *type_none = code("");
        *n_tags = nt;
    });
}

int mhdm_set_boundary(MhdHostMesh *m, const int8_t *face_kind, const int8_t *edge_mode)
{
    return guarded([&] {
        if (!face_kind || !edge_mode) throw std::runtime_error("null argument");
        m->face_kind.assign(face_kind, face_kind + m->nf());
        m->edge_mode.assign(edge_mode, edge_mode + m->ne());
        m->have_bc = true;
    });
}

const void *mhdm_array(const MhdHostMesh *m, const char *cname, int64_t *count)
{
    const std::string n(cname);
    auto ret = [&](const auto &v) -> const void * { *count = static_cast<int64_t>(v.size()); return v.data(); };
    const auto us = n.find('_');
    if (us != std::string::npos)
    {
        const std::string tab = n.substr(0, us), part = n.substr(us + 1);
        const Csr *t = tab == "e2n" ? &m->e2n : tab == "f2e" ? &m->f2e : tab == "c2f" ? &m->c2f : tab == "e2f" ? &m->e2f
                     : tab == "f2c" ? &m->f2c : tab == "n2e" ? &m->n2e : nullptr;
        if (t)
        {
            if (part == "ptr") return ret(t->ptr);
            if (part == "idx") return ret(t->idx);
            if (part == "sgn") return ret(t->sgn);
        }
    }
    if (n == "x") return ret(m->x);
    if (n == "hex") return ret(m->hex8);
    if (n == "hex_material") return ret(m->hex_material);
    if (n == "tag_tri") return ret(m->tag_tri);
    if (n == "tag_tri_id") return ret(m->tag_tri_id);
    if (n == "cell_material") return ret(m->cell_material);
    if (n == "face_tag") return ret(m->face_tag);
    if (m->have_bc)
    {
        if (n == "face_kind") return ret(m->face_kind);
        if (n == "edge_mode") return ret(m->edge_mode);
    }
    if (m->have_geo)
    {
        if (n == "edge_vec") return ret(m->edge_vec);
        if (n == "edge_mid") return ret(m->edge_mid);
        if (n == "edge_len") return ret(m->edge_len);
        if (n == "face_area") return ret(m->face_area);
        if (n == "face_center") return ret(m->face_center);
        if (n == "face_area_mag") return ret(m->face_area_mag);
        if (n == "cell_center") return ret(m->cell_center);
        if (n == "cell_volume") return ret(m->cell_volume);
        if (n == "cell_min_tet_volume") return ret(m->cell_min_tet_volume);
        if (n == "edge_dual_area") return ret(m->edge_dual_area);
        if (n == "ec_ptr") return ret(m->ec_ptr);
        if (n == "ec_cell") return ret(m->ec_cell);
        if (n == "ec_weight") return ret(m->ec_weight);
        if (n == "ef_weight") return ret(m->ef_weight);
        if (n == "ec_misoriented") return ret(m->ec_misoriented);
        if (n == "star0") return ret(m->star0);
        if (n == "star1") return ret(m->star1);
        if (n == "star2") return ret(m->star2);
        if (n == "star3") return ret(m->star3);
    }
    *count = -1;
    return nullptr;
}


} // extern "C"

// ------------------------------------------------------------------ UNSBIN field files
namespace
{
// dtype codes of uns::io::DType (include/uns/io/BinContainer.h): I8 0, I32 1, I64 2, F32 3, F64 4
struct BinRec
{
    uint8_t type;
    uint32_t cols;
    uint64_t rows;
    std::vector<char> bytes;
};
size_t bin_elem(uint8_t t) { return t == 0 ? 1 : (t == 1 || t == 3) ? 4 : 8; }
const char kBinMagic[8] = {'U', 'N', 'S', 'B', 'I', 'N', 0, 1};

struct BinOut
{
    std::vector<std::pair<std::string, BinRec>> recs;
    template <class T> void put(const std::string &name, uint8_t type, const T *p, size_t n, uint32_t cols)
    {
        BinRec r;
        r.type = type;
        r.cols = cols;
        r.rows = cols ? n / cols : 0;
        r.bytes.assign(reinterpret_cast<const char *>(p), reinterpret_cast<const char *>(p) + n * sizeof(T));
        recs.emplace_back(name, std::move(r));
    }
    void write(const std::string &path) const
    {
        std::FILE *f = std::fopen(path.c_str(), "wb");
        if (!f) throw std::runtime_error("cannot open '" + path + "' (wb)");
        auto wr = [&](const void *p, size_t n) {
            if (n && std::fwrite(p, 1, n, f) != n)
            {
                std::fclose(f);
                throw std::runtime_error("write failed");
            }
        };
        wr(kBinMagic, 8);
        const uint64_t n = recs.size();
        wr(&n, 8);
        static const char zeros[8] = {0};
        for (const auto &kv : recs)
        {
            const uint32_t nl = static_cast<uint32_t>(kv.first.size());
            wr(&nl, 4);
            wr(kv.first.data(), nl);
            const uint8_t t[4] = {kv.second.type, 0, 0, 0};
            wr(t, 4);
            wr(&kv.second.cols, 4);
            wr(&kv.second.rows, 8);
            wr(kv.second.bytes.data(), kv.second.bytes.size());
            wr(zeros, (8 - kv.second.bytes.size() % 8) % 8);
        }
        if (std::fclose(f) != 0) throw std::runtime_error("write failed");
    }
};

// records by name; a repeated name keeps the first, as the reference's std::map::emplace does
std::map<std::string, BinRec> bin_read(const std::string &path)
{
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open '" + path + "' (rb)");
    std::map<std::string, BinRec> recs;
    auto rd = [&](void *p, size_t n) {
        if (n && std::fread(p, 1, n, f) != n)
        {
            std::fclose(f);
            throw std::runtime_error("read failed / truncated file");
        }
    };
    char magic[8];
    rd(magic, 8);
    if (std::memcmp(magic, kBinMagic, 8) != 0)
    {
        std::fclose(f);
        throw std::runtime_error("'" + path + "' is not an UNSBIN file");
    }
    uint64_t n;
    rd(&n, 8);
    for (uint64_t i = 0; i < n; ++i)
    {
        uint32_t nl;
        rd(&nl, 4);
        std::string name(nl, '\0');
        rd(name.data(), nl);
        uint8_t t[4];
        rd(t, 4);
        BinRec r;
        r.type = t[0];
        rd(&r.cols, 4);
        rd(&r.rows, 8);
        r.bytes.resize(r.rows * r.cols * bin_elem(r.type));
        rd(r.bytes.data(), r.bytes.size());
        char pad[8];
        rd(pad, (8 - r.bytes.size() % 8) % 8);
        recs.emplace(std::move(name), std::move(r));
    }
    std::fclose(f);
    return recs;
}

const BinRec &bin_find(const std::map<std::string, BinRec> &recs, const std::string &name, uint8_t type)
{
    auto it = recs.find(name);
    if (it == recs.end()) throw std::runtime_error("UNSBIN: missing record '" + name + "'");
    if (it->second.type != type) throw std::runtime_error("UNSBIN: record '" + name + "' has a different data type");
    return it->second;
}

struct FieldRec
{
    std::string name;
    int32_t dim, ncomp;
    std::vector<double> values;
};
} // namespace

struct MhdFieldFile
{
    uint64_t hash = 0;
    std::vector<FieldRec> fields;
};

extern "C" {
int mhdm_write_fields(const char *path, uint64_t topology_hash, int32_t n, const char *const *names, const int32_t *dims,
                      const int32_t *ncomps, const int64_t *counts, const double *const *values)
{
    return guarded([&] {
        if (!path || (n > 0 && (!names || !dims || !ncomps || !counts || !values))) throw std::runtime_error("null argument");
        BinOut w;
        const int64_t h = static_cast<int64_t>(topology_hash);
        w.put("hash", 2, &h, 1, 1);
        std::string index;
        for (int32_t i = 0; i < n; ++i)
        {
            if (ncomps[i] < 1 || counts[i] < 0 || counts[i] % ncomps[i] != 0)
                throw std::runtime_error(std::string("field '") + names[i] + "': count must be a multiple of ncomp");
            const std::string name = names[i];
            index += name + "\n";
            const int32_t info[2] = {dims[i], ncomps[i]};
            w.put("f." + name + ".info", 1, info, 2, 1);
            w.put("f." + name, 4, values[i], static_cast<size_t>(counts[i]), static_cast<uint32_t>(ncomps[i]));
        }
        w.put("index", 0, reinterpret_cast<const int8_t *>(index.data()), index.size(), 1);
        w.write(path);
    });
}

int mhdm_read_fields(const char *path, MhdFieldFile **out)
{
    MhdFieldFile *ff = nullptr;
    int rc = guarded([&] {
        if (!path || !out) throw std::runtime_error("null argument");
        const auto recs = bin_read(path);
        ff = new MhdFieldFile;
        const BinRec &h = bin_find(recs, "hash", 2);
        if (h.bytes.size() < 8) throw std::runtime_error("UNSBIN: empty hash record");
        int64_t hv;
        std::memcpy(&hv, h.bytes.data(), 8);
        ff->hash = static_cast<uint64_t>(hv);
        const BinRec &ix = bin_find(recs, "index", 0);
        const std::string index(ix.bytes.begin(), ix.bytes.end());
        size_t a = 0;
        while (a < index.size())
        {
            size_t b = index.find('\n', a);
            if (b == std::string::npos) b = index.size();
            FieldRec f;
            f.name = index.substr(a, b - a);
            a = b + 1;
            const BinRec &inf = bin_find(recs, "f." + f.name + ".info", 1);
            if (inf.bytes.size() < 8) throw std::runtime_error("UNSBIN: short info record of '" + f.name + "'");
            int32_t info[2];
            std::memcpy(info, inf.bytes.data(), 8);
            f.dim = info[0];
            f.ncomp = info[1];
            const BinRec &v = bin_find(recs, "f." + f.name, 4);
            f.values.resize(v.bytes.size() / 8);
            std::memcpy(f.values.data(), v.bytes.data(), f.values.size() * 8);
            ff->fields.push_back(std::move(f));
        }
        *out = ff;
    });
    if (rc != 0) delete ff;
    return rc;
}

void mhdm_fields_free(MhdFieldFile *f) { delete f; }

int32_t mhdm_fields_count(const MhdFieldFile *f, uint64_t *topology_hash)
{
    if (!f) return -1;
    if (topology_hash) *topology_hash = f->hash;
    return static_cast<int32_t>(f->fields.size());
}

int mhdm_field(const MhdFieldFile *f, int32_t i, char *name, int32_t len, int32_t *dim, int32_t *ncomp, int64_t *count, double *out)
{
    return guarded([&] {
        if (!f || i < 0 || i >= static_cast<int32_t>(f->fields.size())) throw std::runtime_error("no such record");
        const FieldRec &r = f->fields[static_cast<size_t>(i)];
        if (name && len > 0)
        {
            std::strncpy(name, r.name.c_str(), static_cast<size_t>(len - 1));
            name[len - 1] = 0;
        }
        if (dim) *dim = r.dim;
        if (ncomp) *ncomp = r.ncomp;
        if (count) *count = static_cast<int64_t>(r.values.size());
        if (out) std::memcpy(out, r.values.data(), r.values.size() * sizeof(double));
    });
}
} // extern "C"
