// C entry points over the reference's own C++ code (compiled in place from the
// reference tree by oracle/Makefile into oracle/_ref/libmhdref.so).
//
// Test infrastructure only: the parity tests, the golden-vector generator and
// bench.py's CPU-baseline leg call these through ctypes.  Every function here
// forwards to the reference implementation named in its comment; the only
// code of this file's own is argument marshalling and the composition of the
// hot-path sequence of one SSP-RK2 step (ref_rk2_step), which follows
// MercuryUns/driver/Solver.cpp:94-125 (prepare), :132-169 (rhs),
// :194-206 (advance), :481-516 (step) with the model sources left out.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "boundary/BoundaryInfo.h"
#include "diagnostics/DivB.h"
#include "fluid/FluxRHS.h"
#include "fluid/MercurySources.h"
#include "fluid/Reconstruction.h"
#include "physics/Ambipolar.h"
#include "physics/Gyration.h"
#include "induction/Current.h"
#include "induction/EdgeEMF.h"
#include "induction/Faraday.h"
#include "induction/IdealEMF.h"
#include "uns/complex/ComplexBuilder.h"
#include "uns/complex/Validate.h"
#include "uns/generate/HexMesh.h"
#include "uns/io/MeshIO.h"
#include "uns/geometry/Geometry.h"
#include "uns/geometry/Reconstruct.h"
#include "uns/refine/Refine.h"
// The per-edge resistivity of ImplicitInduction (m_) is only filled from its
// built-in tanh window; the checker sets arbitrary per-edge profiles, so the
// class is opened here (the layout is unchanged: GCC lays members out in
// declaration order whatever their access).
#define private public
#include "induction/ImplicitInduction.h"
#undef private

using namespace uns;
using namespace mhd;

namespace
{
struct RefMesh
{
    LocalMesh lm;
    Geometry geo;
    bool have_geo = false;
    BoundaryInfo bc;
    bool have_bc = false;
    Config cfg;
    std::unique_ptr<Stencil> stencil;
    std::vector<char> active;
    // resistive operator of the explicit resistive EMF (declared after res_ex: destroyed first)
    std::unique_ptr<comm::Exchanger> res_ex;
    std::unique_ptr<ImplicitInduction> res_op;
    std::unique_ptr<mercury::AmbipolarEMF> amb;
};

thread_local std::string g_err;

template <class F> int guarded(F &&f)
{
    try { f(); return 0; }
    catch (const std::exception &e) { g_err = e.what(); return -1; }
}

RefMesh *wrap(Mesh &&m)
{
    auto *r = new RefMesh;
    r->lm.mesh = std::move(m);
    r->active = active_faces(r->lm.mesh.cx);
    return r;
}

void ensure_geo(RefMesh *r)
{
    if (!r->have_geo) { r->geo = compute_geometry(r->lm.mesh); r->have_geo = true; }
}

template <class T> int64_t put(const std::vector<T> &v, void *out)
{
    if (out) std::memcpy(out, v.data(), v.size() * sizeof(T));
    return static_cast<int64_t>(v.size());
}
int64_t put3(const std::vector<Vec3> &v, void *out)
{
    if (out)
    {
        double *o = static_cast<double *>(out);
        for (size_t i = 0; i < v.size(); ++i) { o[3 * i] = v[i].x; o[3 * i + 1] = v[i].y; o[3 * i + 2] = v[i].z; }
    }
    return static_cast<int64_t>(3 * v.size());
}
int64_t put_inc(const Incidence &t, const std::string &part, void *out)
{
    if (part == "ptr") return put(t.ptr, out);
    if (part == "idx") return put(t.idx, out);
    if (part == "sgn") return put(t.sgn, out);
    return -1;
}
} // namespace

extern "C" {

const char *ref_last_error() { return g_err.c_str(); }

// ---------------------------------------------------------------- meshes
// Generic polyhedral cells through ComplexBuilder::add_cell / tag_face / finish
// (src/uns/complex/ComplexBuilder.cpp:45-76, :87-92, :102-134).  Cell c owns the
// outward loops cell_ptr[c]..cell_ptr[c+1]; loop l has nodes loop_nodes[loop_ptr[l]..loop_ptr[l+1]].
void *ref_mesh_from_cells(int32_t n_nodes, const double *x, int32_t n_cells, const int64_t *cell_ptr, const int64_t *loop_ptr,
                          const int32_t *loop_nodes, const int32_t *material, int32_t n_tagged, const int64_t *tag_ptr,
                          const int32_t *tag_nodes, const int32_t *tag_id, int32_t n_names, const char *const *names)
{
    RefMesh *out = nullptr;
    guarded([&] {
        ComplexBuilder b(n_nodes);
        std::vector<std::vector<Id>> loops;
        for (int32_t c = 0; c < n_cells; ++c)
        {
            loops.clear();
            for (int64_t l = cell_ptr[c]; l < cell_ptr[c + 1]; ++l)
                loops.emplace_back(loop_nodes + loop_ptr[l], loop_nodes + loop_ptr[l + 1]);
            b.add_cell(loops, material ? material[c] : kFluid);
        }
        for (int32_t t = 0; t < n_tagged; ++t)
            b.tag_face(std::vector<Id>(tag_nodes + tag_ptr[t], tag_nodes + tag_ptr[t + 1]), tag_id[t]);
        Mesh m;
        m.cx = b.finish();
        m.x.resize(n_nodes);
        for (int32_t i = 0; i < n_nodes; ++i) m.x[i] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
        m.tag_names.assign(names, names + n_names);
        out = wrap(std::move(m));
    });
    return out;
}

// uns::make_box + build_mesh (src/uns/generate/BoxMesh.cpp:5-33, HexMesh.cpp:7-18)
void *ref_mesh_box(int32_t nx, int32_t ny, int32_t nz, const double *lo, const double *hi)
{
    RefMesh *out = nullptr;
    guarded([&] {
        BoxSpec s;
        s.nx = nx; s.ny = ny; s.nz = nz;
        s.lo = {lo[0], lo[1], lo[2]}; s.hi = {hi[0], hi[1], hi[2]};
        out = wrap(build_mesh(make_box(s)));
    });
    return out;
}

// uns::make_cubed_sphere_shell (src/uns/generate/CubedSphereMesh.cpp:12-83)
void *ref_mesh_shell(int32_t ncube, int32_t nr, int32_t n_solid, double r_in, double r_out, double r_stretch)
{
    RefMesh *out = nullptr;
    guarded([&] {
        CubedSphereSpec s;
        s.ncube = ncube; s.nr = nr; s.n_solid = n_solid; s.r_in = r_in; s.r_out = r_out; s.r_stretch = r_stretch;
        out = wrap(build_mesh(make_cubed_sphere_shell(s)));
    });
    return out;
}

// The cubed-sphere shell of uns::make_cubed_sphere_shell (src/uns/generate/CubedSphereMesh.cpp:12-83) with
// every hexahedron cut into 6 tetrahedra, built by the reference's ComplexBuilder (add_cell, tag_face,
// finish: src/uns/complex/ComplexBuilder.cpp:45-134).  The reference generates hexahedra only; the split
// is the one of the benchmark workloads: the Kuhn paths 0 -> a -> a|b -> 7 of the hexahedron's local
// corner bits (corner i at (i&1, (i>>1)&1, (i>>2)&1)), one tetrahedron per order of the three axis bits,
// each given its four outward loops; a tagged quad becomes the two triangles on either side of the
// diagonal joining its lowest and highest local corners.  Cells, faces and edges come out in the
// creation order of the split hexahedra, so this mesh is the benchmark's shell, entity for entity.
void *ref_mesh_shell_tets(int32_t ncube, int32_t nr, int32_t n_solid, double r_in, double r_out, double r_stretch)
{
    RefMesh *out = nullptr;
    guarded([&] {
        CubedSphereSpec s;
        s.ncube = ncube; s.nr = nr; s.n_solid = n_solid; s.r_in = r_in; s.r_out = r_out; s.r_stretch = r_stretch;
        HexMesh h = make_cubed_sphere_shell(s);
        ComplexBuilder b(static_cast<Id>(h.x.size()));
        static const int P[6][3] = {{1, 2, 4}, {1, 4, 2}, {2, 1, 4}, {2, 4, 1}, {4, 1, 2}, {4, 2, 1}};
        static const int PAR[6] = {+1, -1, -1, +1, +1, -1};
        static const int L[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
        std::vector<std::vector<Id>> loops(4, std::vector<Id>(3));
        for (size_t c = 0; c < h.hex.size(); ++c)
        {
            const auto &v = h.hex[c];
            for (int t = 0; t < 6; ++t)
            {
                Id p[4] = {v[0], v[P[t][0]], v[P[t][0] | P[t][1]], v[7]};
                if (PAR[t] < 0) std::swap(p[1], p[2]);
                loops[0] = {p[0], p[2], p[1]};
                loops[1] = {p[0], p[1], p[3]};
                loops[2] = {p[1], p[2], p[3]};
                loops[3] = {p[0], p[3], p[2]};
                b.add_cell(loops, h.material.empty() ? kFluid : h.material[c]);
            }
        }
        // tagged quads: find each one's hexahedron face to know its local corners
        std::map<std::array<Id, 4>, int> tag_of;
        for (const auto &t : h.tagged)
        {
            std::array<Id, 4> k = t.nodes;
            std::sort(k.begin(), k.end());
            tag_of[k] = t.tag;
        }
        for (size_t c = 0; c < h.hex.size() && !tag_of.empty(); ++c)
        {
            const auto &v = h.hex[c];
            for (int f = 0; f < 6; ++f)
            {
                std::array<Id, 4> k = {v[L[f][0]], v[L[f][1]], v[L[f][2]], v[L[f][3]]};
                std::sort(k.begin(), k.end());
                auto it = tag_of.find(k);
                if (it == tag_of.end()) continue;
                int lo = 7, hi = 0;
                for (int q = 0; q < 4; ++q) { lo &= L[f][q]; hi |= L[f][q]; }
                for (int q = 0; q < 4; ++q)
                {
                    const int lq = L[f][q];
                    if (lq == lo || lq == hi) continue;
                    b.tag_face({v[lo], v[lq], v[hi]}, it->second);
                }
            }
        }
        Mesh m;
        m.cx = b.finish();
        m.x = h.x;
        m.tag_names = h.tag_names;
        out = wrap(std::move(m));
    });
    return out;
}

// Hanging-node polyhedra: a box refined inside a sphere, as in tests/test_ideal_emf.cpp:357-364
// (uns::build_refined_mesh, src/uns/refine/RefineMesh.cpp).
void *ref_mesh_hanging_box(int32_t nx, int32_t ny, int32_t nz, const double *hi, const double *sphere, int32_t level)
{
    RefMesh *out = nullptr;
    guarded([&] {
        BoxSpec bs;
        bs.nx = nx; bs.ny = ny; bs.nz = nz; bs.hi = {hi[0], hi[1], hi[2]};
        Mesh box = build_mesh(make_box(bs));
        RefineSpec rs;
        rs.max_level = level;
        Region reg;
        reg.kind = Region::Kind::Sphere;
        reg.a = {sphere[0], sphere[1], sphere[2], sphere[3]};
        reg.level = level;
        rs.regions.push_back(reg);
        out = wrap(build_refined_mesh(box, rs, std::vector<int>(box.cx.n_cells(), 0)).fine);
    });
    return out;
}

void ref_mesh_free(void *h) { delete static_cast<RefMesh *>(h); }

void ref_mesh_counts(void *h, int32_t *out)
{
    const CellComplex &cx = static_cast<RefMesh *>(h)->lm.mesh.cx;
    out[0] = cx.n_nodes(); out[1] = cx.n_edges(); out[2] = cx.n_faces(); out[3] = cx.n_cells();
}

uint64_t ref_topology_hash(void *h) { return topology_hash(static_cast<RefMesh *>(h)->lm.mesh.cx); }

// uns::validate_topology (src/uns/complex/Validate.cpp:18-69): ok, euler, d1d0, d2d1, boundary faces
void ref_validate(void *h, int64_t *out)
{
    const TopologyReport r = validate_topology(static_cast<RefMesh *>(h)->lm.mesh.cx);
    out[0] = r.ok; out[1] = r.euler; out[2] = r.d1d0_violations; out[3] = r.d2d1_violations; out[4] = r.boundary_faces;
}

// uns::check_geometry (src/uns/geometry/Geometry.cpp:171-205)
void ref_check_geometry(void *h, double *out)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    ensure_geo(r);
    const GeometryReport g = check_geometry(r->lm.mesh, r->geo);
    out[0] = g.ok; out[1] = g.min_volume; out[2] = g.max_volume; out[3] = g.min_tet; out[4] = g.max_closure;
    out[5] = static_cast<double>(g.nonpositive_volume); out[6] = static_cast<double>(g.nonpositive_star);
    out[7] = static_cast<double>(g.misoriented_dual);
}

// Copies the named array (topology, geometry or boundary classification) into out (if non-null); returns its
// element count, or -1 for an unknown name.  Vec3 arrays are flattened x,y,z per entity.
int64_t ref_array(void *h, const char *cname, void *out)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    const CellComplex &cx = r->lm.mesh.cx;
    const std::string name(cname);
    const auto us = name.find('_');
    if (us != std::string::npos)
    {
        const std::string tab = name.substr(0, us), part = name.substr(us + 1);
        if (tab == "e2n") return put_inc(cx.e2n, part, out);
        if (tab == "f2e") return put_inc(cx.f2e, part, out);
        if (tab == "c2f") return put_inc(cx.c2f, part, out);
        if (tab == "e2f") return put_inc(cx.e2f, part, out);
        if (tab == "f2c") return put_inc(cx.f2c, part, out);
        if (tab == "n2e") return put_inc(cx.n2e, part, out);
    }
    if (name == "x") return put3(r->lm.mesh.x, out);
    if (name == "cell_material") return put(cx.cell_material, out);
    if (name == "face_tag") return put(cx.face_tag, out);
    if (name == "face_kind" || name == "edge_mode")
    {
        if (!r->have_bc) return -1;
        if (name == "edge_mode") return put(r->bc.edge_mode, out);
        std::vector<int8_t> k(r->bc.face_kind.size());
        for (size_t i = 0; i < k.size(); ++i) k[i] = static_cast<int8_t>(r->bc.face_kind[i]);
        return put(k, out);
    }
    ensure_geo(r);
    const Geometry &g = r->geo;
    if (name == "edge_vec") return put3(g.edge_vec, out);
    if (name == "edge_mid") return put3(g.edge_mid, out);
    if (name == "edge_len") return put(g.edge_len, out);
    if (name == "face_area") return put3(g.face_area, out);
    if (name == "face_center") return put3(g.face_center, out);
    if (name == "face_area_mag") return put(g.face_area_mag, out);
    if (name == "cell_center") return put3(g.cell_center, out);
    if (name == "cell_volume") return put(g.cell_volume, out);
    if (name == "cell_min_tet_volume") return put(g.cell_min_tet_volume, out);
    if (name == "edge_dual_area") return put3(g.edge_dual_area, out);
    if (name == "ec_ptr") return put(g.ec_ptr, out);
    if (name == "ec_cell") return put(g.ec_cell, out);
    if (name == "ec_weight") return put(g.ec_weight, out);
    if (name == "ef_weight") return put(g.ef_weight, out);
    if (name == "ec_misoriented") return put(g.ec_misoriented, out);
    if (name == "star0") return put(g.star0, out);
    if (name == "star1") return put(g.star1, out);
    if (name == "star2") return put(g.star2, out);
    if (name == "star3") return put(g.star3, out);
    return -1;
}

// mhd::BoundaryInfo::build (Common/boundary/BoundaryInfo.cpp:9-49) for a bc_default and per-tag types.
int ref_boundary_build(void *h, const char *bc_default, int32_t n_pairs, const char *const *tags, const char *const *types,
                       const double *u_inf)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    return guarded([&] {
        ensure_geo(r);
        r->cfg.bc_default = bc_default;
        r->cfg.bc_by_tag.clear();
        for (int32_t i = 0; i < n_pairs; ++i) r->cfg.bc_by_tag[tags[i]] = types[i];
        r->cfg.u_inf = {u_inf[0], u_inf[1], u_inf[2]};
        r->bc = BoundaryInfo::build(r->lm, r->geo, r->cfg);
        r->have_bc = true;
        r->stencil.reset();
    });
}

// ---------------------------------------------------------------- fluid
// mhd::to_prim (Common/physics/Euler.h:13-21) on n cells of a 5-per-cell array.
void ref_to_prim(const double *U, int64_t n, double gamma, double rho_floor, double p_floor, double *W)
{
    for (int64_t c = 0; c < n; ++c)
    {
        const Prim w = to_prim(U + 5 * c, gamma, rho_floor, p_floor);
        W[5 * c] = w.rho; W[5 * c + 1] = w.u; W[5 * c + 2] = w.v; W[5 * c + 3] = w.w; W[5 * c + 4] = w.p;
    }
}

static void ensure_stencil(RefMesh *r)
{
    if (!r->have_bc) throw std::runtime_error("boundary classification missing");
    if (!r->stencil) r->stencil = std::make_unique<Stencil>(r->lm, r->geo, r->bc);
}

// mhd::Stencil::Stencil + limited_gradients (Common/fluid/Reconstruction.cpp:26-78, :80-142)
int ref_limited_gradients(void *h, const double *W, int32_t species, const double *fs, int32_t limit, double rel_limit, double *grad)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    return guarded([&] {
        ensure_stencil(r);
        r->stencil->set_rel_limit(rel_limit);
        const Prim p{fs[0], fs[1], fs[2], fs[3], fs[4]};
        r->stencil->limited_gradients(r->lm, r->geo, r->bc, W, species, p, limit != 0, grad);
    });
}

// A GhostFn (Common/fluid/Reconstruction.h:21) over a per-face table, bound as the ten-ion solver binds
// its ghost_ (MarsUns/driver/MarsSolver.cpp:124-128): listed wall faces return the table's state of the
// species, every other face ghost_state.  prims: [species][i][5] with species_stride entries per species.
static GhostFn table_ghost(const RefMesh *r, int32_t n_wall, const int32_t *faces, const double *prims, int64_t species_stride,
                    std::unordered_map<Id, int32_t> &slot, const Prim *fs_all, bool species_relative)
{
    slot.clear();
    for (int32_t i = 0; i < n_wall; ++i) slot.emplace(faces[i], i);
    const BoundaryInfo *bc = &r->bc;
    return [bc, &slot, prims, species_stride, fs_all, species_relative](Id f, int s, const Prim &in, const Vec3 &n) -> Prim {
        const FaceKind k = bc->face_kind[f];
        if (k == FaceKind::Wall)
        {
            auto it = slot.find(f);
            if (it != slot.end())
            {
                const double *w = prims + 5 * (species_stride * (species_relative ? 0 : s) + it->second);
                return Prim{w[0], w[1], w[2], w[3], w[4]};
            }
        }
        return ghost_state(k, s, in, n, fs_all[species_relative ? 0 : s]);
    };
}

// limited_gradients with the table GhostFn; prims [n_wall][5] of this species
int ref_limited_gradients_wall(void *h, const double *W, int32_t species, const double *fs, int32_t limit, double rel_limit,
                               int32_t n_wall, const int32_t *faces, const double *prims, double *grad)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    return guarded([&] {
        if (!r->have_bc) throw std::runtime_error("boundary classification missing");
        ensure_stencil(r);
        r->stencil->set_rel_limit(rel_limit);
        const Prim p{fs[0], fs[1], fs[2], fs[3], fs[4]};
        std::unordered_map<Id, int32_t> slot;
        const GhostFn g = table_ghost(r, n_wall, faces, prims, n_wall, slot, &p, true);
        r->stencil->limited_gradients(r->lm, r->geo, r->bc, W, species, p, limit != 0, grad, &g);
    });
}

// fluid_flux_rhs with the table GhostFn; prims [n_wall][5] of this species
int ref_flux_rhs_wall(void *h, double gamma, int32_t species, const double *fs, const double *W, const double *grad, int32_t n_wall,
                      const int32_t *faces, const double *prims, double *rhs)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    return guarded([&] {
        if (!r->have_bc) throw std::runtime_error("boundary classification missing");
        r->cfg.sc.gamma = gamma;
        const Prim p{fs[0], fs[1], fs[2], fs[3], fs[4]};
        std::unordered_map<Id, int32_t> slot;
        const GhostFn g = table_ghost(r, n_wall, faces, prims, n_wall, slot, &p, true);
        fluid_flux_rhs(r->lm, r->geo, r->bc, r->cfg, species, p, W, grad, rhs, &g);
    });
}

// mhd::fluid_flux_rhs (Common/fluid/FluxRHS.cpp:30-74)
int ref_flux_rhs(void *h, double gamma, int32_t species, const double *fs, const double *W, const double *grad, double *rhs)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    return guarded([&] {
        if (!r->have_bc) throw std::runtime_error("boundary classification missing");
        r->cfg.sc.gamma = gamma;
        const Prim p{fs[0], fs[1], fs[2], fs[3], fs[4]};
        fluid_flux_rhs(r->lm, r->geo, r->bc, r->cfg, species, p, W, grad, rhs);
    });
}

// ---------------------------------------------------------------- induction
// uns::reconstruct_cell_vector (src/uns/geometry/Reconstruct.cpp:8-46)
void ref_cell_vector(void *h, const double *phi, double *out)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    ensure_geo(r);
    const CellComplex &cx = r->lm.mesh.cx;
    const auto b = reconstruct_cell_vector(cx, r->geo, phi, cx.n_cells());
    for (Id c = 0; c < cx.n_cells(); ++c) { out[3 * c] = b[c].x; out[3 * c + 1] = b[c].y; out[3 * c + 2] = b[c].z; }
}

// mhd::add_ideal_emf (Common/induction/IdealEMF.cpp:25-129); adds into E.
void ref_ideal_emf(void *h, const double *u, const double *Btot, const double *Bind, const double *phitot, const double *phiind,
                   double cuct, double *E)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    ensure_geo(r);
    IdealInputs in;
    in.u_cell = u; in.B_cell_tot = Btot; in.B_cell_ind = Bind; in.phi_tot = phitot; in.phi_ind = phiind;
    IdealParams p;
    p.cuct = cuct;
    add_ideal_emf(r->lm, r->geo, in, p, E);
}

// mhd::faraday_update (Common/induction/Faraday.cpp:15-24) over active_faces (:7-13)
void ref_faraday(void *h, const double *E, double *B, double dt)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    faraday_update(r->lm.mesh.cx, r->active, E, B, dt);
}

// mhd::faraday_update_edge_dt (Common/induction/Faraday.cpp:27-36)
void ref_faraday_edge_dt(void *h, const double *E, const double *dt_edge, double *B)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    faraday_update_edge_dt(r->lm.mesh.cx, r->active, E, dt_edge, B);
}

// mhd::div_b (Common/diagnostics/DivB.cpp:8-24): max_abs, max_rel, worst gid
void ref_div_b(void *h, const double *B, const double *extra, double *out)
{
    const DivBReport d = div_b(static_cast<RefMesh *>(h)->lm.mesh.cx, B, extra);
    out[0] = d.max_abs; out[1] = d.max_rel; out[2] = static_cast<double>(d.worst_cell_gid);
}

// mhd::cell_current (Common/induction/Current.cpp:9-31)
void ref_cell_current(void *h, const double *B, double *J)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    ensure_geo(r);
    cell_current(r->lm, r->geo, B, J);
}

// mercury::local_time_step (MercuryUns/fluid/MercurySources.cpp:65-116), two species.
double ref_local_time_step(void *h, double gamma, double cfl, double inver_MA2, double rho_floor_dt, const double *WH,
                           const double *WNa, const double *B)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    ensure_geo(r);
    Config c = r->cfg;
    c.sc.gamma = gamma; c.cfl = cfl; c.sc.inver_MA2 = inver_MA2; c.rho_floor_dt = rho_floor_dt;
    return mercury::local_time_step(r->lm, r->geo, c, WH, WNa, B);
}

struct RefIndParams
{
    int32_t resistive, hall, max_it, restart, ilu, implicit_ideal;
    double inver_Rem, eta_r_inner, eta_r_outer, eta_width, hall_coef, hall_r_min, hall_r_max, rtol, ilu_shift, cuct;
};

struct RefInd
{
    RefMesh *mesh;
    comm::Exchanger ex;
    std::unique_ptr<ImplicitInduction> ind;
    std::vector<double> u_ideal; // the cell velocities set_ideal_state points to
    RefInd(RefMesh *m) : mesh(m), ex(MPI_COMM_SELF, m->lm) {}
};

// The reference objects behind a RefMesh handle (LocalMesh, Geometry, BoundaryInfo, Config, Stencil), for
// the drop-in test driver, which calls the reference's signatures on them: out[0..4].
int ref_mesh_objects(void *h, void **out)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    return guarded([&] {
        if (!r->have_bc) throw std::runtime_error("boundary classification not built");
        ensure_stencil(r);
        out[0] = &r->lm; out[1] = &r->geo; out[2] = &r->bc; out[3] = &r->cfg; out[4] = r->stencil.get();
    });
}

// mhd::ImplicitInduction::ImplicitInduction (Common/induction/ImplicitInduction.cpp:10-103)
void *ref_ind_create(void *h, const RefIndParams *p)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    RefInd *out = nullptr;
    guarded([&] {
        ensure_geo(r);
        Config c;
        c.resistive = p->resistive != 0; c.sc.inver_Rem = p->inver_Rem;
        c.eta_r_inner = p->eta_r_inner; c.eta_r_outer = p->eta_r_outer; c.eta_width = p->eta_width;
        c.hall = p->hall != 0; c.sc.hall_coef = p->hall_coef; c.hall_r_min = p->hall_r_min; c.hall_r_max = p->hall_r_max;
        c.ind_rtol = p->rtol; c.ind_max_it = p->max_it; c.ind_restart = p->restart; c.ind_ilu = p->ilu != 0;
        c.ind_ilu_shift = p->ilu_shift;
        c.implicit_ideal = p->implicit_ideal != 0;
        c.ideal.cuct = p->cuct;
        auto *ri = new RefInd(r);
        ri->ind = std::make_unique<ImplicitInduction>(r->lm, r->geo, ri->ex, c);
        out = ri;
    });
    return out;
}

void ref_ind_free(void *h) { delete static_cast<RefInd *>(h); }
void *ref_ind_object(void *h) { return static_cast<RefInd *>(h)->ind.get(); }

// Per-edge resistive coefficient m_e (eta_e / star1_e) in place of the constructor's tanh window.
void ref_ind_set_m(void *h, const double *m)
{
    RefInd *ri = static_cast<RefInd *>(h);
    std::copy(m, m + ri->ind->m_.size(), ri->ind->m_.begin());
    ri->ind->resistive_ = true;
    // the constructor built the ILU(0) pattern from its own m_ (:102): build it again from these
    if (ri->ind->use_ilu_ && !ri->ind->ideal_) ri->ind->build_precond_pattern();
}

// ImplicitInduction::factor_precond (:247-275) for dt and dir, then apply_precond (:277-297) of v into z
// (both n_edges); the pattern must exist (ilu on).
int ref_ind_precond(void *h, double dt, const int8_t *dir, const double *v, double *z)
{
    return guarded([&] {
        ImplicitInduction &I = *static_cast<RefInd *>(h)->ind;
        if (I.pc_ptr_.empty()) throw std::runtime_error("no ILU(0) pattern");
        const size_t ne = I.m_.size();
        std::vector<char> d(ne);
        for (size_t e = 0; e < ne; ++e) d[e] = dir ? dir[e] : 0;
        I.factor_precond(dt, d);
        std::vector<double> vv(v, v + ne), zz(ne, 0.0);
        I.apply_precond(vv, zz, d);
        std::copy(zz.begin(), zz.end(), z);
    });
}

int64_t ref_ind_array(void *h, const char *cname, void *out)
{
    ImplicitInduction &I = *static_cast<RefInd *>(h)->ind;
    const std::string n(cname);
    if (n == "m") return put(I.m_, out);
    if (n == "d2") return put(I.d2_, out);
    if (n == "recon") return put(I.recon_, out);
    if (n == "taper") return put(I.taper_, out);
    if (n == "alpha") return put(I.alpha_, out);
    if (n == "ce_ptr") return put(I.ce_ptr_, out);
    if (n == "ce_edge") return put(I.ce_edge_, out);
    if (n == "ce_wt") return put3(I.ce_wt_, out);
    if (n == "corr") return put(I.corr_, out);
    if (n == "pc_ptr") return put(I.pc_ptr_, out);
    if (n == "pc_col") return put(I.pc_col_, out);
    if (n == "pc_coef") return put(I.pc_coef_, out);
    if (n == "pc_val") return put(I.pc_val_, out);
    if (n == "pc_diag") return put(I.pc_diag_, out);
    return -1;
}

// ImplicitInduction::set_frozen_state (:105-111)
void ref_ind_set_frozen(void *h, const double *B0, const double *ne) { static_cast<RefInd *>(h)->ind->set_frozen_state(B0, ne); }

// ImplicitInduction::apply_F (:127-183)
void ref_ind_apply_F(void *h, const double *phi, double *out) { static_cast<RefInd *>(h)->ind->apply_F(phi, out); }

// ImplicitInduction::apply_A (:185-198): y = x + dt F(d1 x)
void ref_ind_apply_A(void *h, const double *x, double dt, double *y)
{
    ImplicitInduction &I = *static_cast<RefInd *>(h)->ind;
    const size_t ne = I.m_.size();
    std::vector<double> xv(x, x + ne), yv(ne);
    I.apply_A(xv, yv, dt);
    std::copy(yv.begin(), yv.end(), y);
}

// ImplicitInduction::set_ideal_state (:112-116): u 3 per cell (kept in the handle, the object holds a
// pointer), mask 1 per edge
void ref_ind_set_ideal(void *h, const double *u, const int8_t *mask)
{
    RefInd *ri = static_cast<RefInd *>(h);
    ImplicitInduction &I = *ri->ind;
    const size_t nc = I.alpha_.size(), ne = I.m_.size();
    ri->u_ideal.assign(u, u + 3 * nc);
    std::vector<char> mk(ne);
    for (size_t e = 0; e < ne; ++e) mk[e] = mask[e];
    I.set_ideal_state(ri->u_ideal.data(), mk);
}

// ImplicitInduction::ideal_linear (:118-124)
void ref_ind_ideal_linear(void *h, const double *phi, double *out) { static_cast<RefInd *>(h)->ind->ideal_linear(phi, out); }

// ImplicitInduction::solve with the per-edge pseudo-time step dt_edge (:299-390, system (I + F d1 diag(dt_e)) E)
int32_t ref_ind_solve_dte(void *h, const double *Phi, const double *Eexpl, const int8_t *dir, const double *dt_edge, int32_t use_guess,
                          double *E, double *rel_res)
{
    ImplicitInduction &I = *static_cast<RefInd *>(h)->ind;
    if (!use_guess) I.corr_.clear();
    std::vector<char> d(I.m_.size());
    for (size_t e = 0; e < d.size(); ++e) d[e] = dir[e];
    return I.solve(Phi, Eexpl, d, 0.0, E, rel_res, dt_edge);
}

// ImplicitInduction::solve (:299-390).  use_guess = 0 clears the warm start first.
int32_t ref_ind_solve(void *h, const double *Phi, const double *Eexpl, const int8_t *dir, double dt, int32_t use_guess, double *E,
                      double *rel_res)
{
    ImplicitInduction &I = *static_cast<RefInd *>(h)->ind;
    if (!use_guess) I.corr_.clear();
    std::vector<char> d(I.m_.size());
    for (size_t e = 0; e < d.size(); ++e) d[e] = dir[e];
    return I.solve(Phi, Eexpl, d, dt, E, rel_res);
}

// ---------------------------------------------------------------- one SSP-RK2 step of the hot path
struct RefStepParams
{
    int32_t n_species, second_order;
    double gamma, rho_floor, p_floor, cuct, M_ref, ne_floor, rel_limit;
    double u_inf[3], B_imf[3];
    double mass[16];
    double fs[16][5];
    // model sources of the two-ion step: J x B force (add_sources_n) and the exact gyration (gyrate)
    int32_t lorentz, pad;
    double induce_coeff, inver_MA2;
    // explicit resistive EMF: E += ImplicitInduction::apply_F(Phi) with only the resistive part on and the
    // per-edge m_e = eta_e / star1_e given here (null: off), added to the owned edges
    const double *m_res;
    // the rest of add_sources_n and the ambipolar EMF (Config::ambipolar / chemistry, Scales constants),
    // with the chemistry's source fields photo and vst (one per cell, null: absent)
    int32_t ambipolar, chemistry;
    double pressure_coef, a1_Na, a4, a5, a6, state_coeff_H, state_coeff_Na, T_ref, Tn0;
    const double *photo, *vst;
    // Dirichlet wall table (the ten-ion solver's GhostFn): faces[n_wall], prims[species][n_wall][5]
    int32_t n_wall, pad2;
    const int32_t *wall_faces;
    const double *wall_prims;
    // time_order = 1 (Solver::step_first_order, Solver.cpp:228-277): forward Euler of the fluid and the
    // semi-implicit induction solve of `ind` (a RefInd handle) for the EMF; iterations and rel_res out
    int32_t first_order, ind_iterations;
    void *ind;
    double ind_rel_res;
};

namespace
{
// Config / Scales of the two-ion source terms (MercurySources.cpp:20-63, Gyration.cpp)
Config source_config(const RefMesh *r, const RefStepParams &p)
{
    Config c = r->cfg;
    c.sc.gamma = p.gamma; c.sc.M_ref = p.M_ref; c.sc.M_H = p.mass[0]; c.sc.M_Na = p.mass[1];
    c.sc.ne_floor = p.ne_floor; c.sc.inver_MA2 = p.inver_MA2; c.sc.induce_coeff = p.induce_coeff;
    c.rho_floor = p.rho_floor; c.p_floor = p.p_floor;
    c.lorentz_force = p.lorentz != 0; c.ambipolar = p.ambipolar != 0; c.chemistry = p.chemistry != 0;
    c.sc.pressure_coef = p.pressure_coef; c.sc.a1_Na = p.a1_Na; c.sc.a4 = p.a4; c.sc.a5 = p.a5; c.sc.a6 = p.a6;
    c.sc.state_coeff_H = p.state_coeff_H; c.sc.state_coeff_Na = p.state_coeff_Na; c.sc.T_ref = p.T_ref; c.chem.Tn0 = p.Tn0;
    return c;
}
} // namespace

// mercury::add_sources (MercuryUns/fluid/MercurySources.cpp:13-63) for species s; dpe, photo, vst: the
// SourceFields (null: absent)
void ref_add_sources(void *h, const RefStepParams *p, int32_t s, const double *WH, const double *WNa, const double *up,
                     const double *B, const double *J, const double *dpe, const double *photo, const double *vst, double dt, double *rhs)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    const Config c = source_config(r, *p);
    mercury::SourceFields sf;
    sf.dpe = dpe; sf.photo = photo; sf.vst = vst;
    mercury::add_sources(r->lm, c, s, WH, WNa, up, B, J, sf, dt, rhs, nullptr);
}

// mercury::electron_pressure_gradient (MercuryUns/physics/Ambipolar.cpp:10-31)
void ref_electron_pressure_gradient(void *h, const double *WH, const double *WNa, double *dpe)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    ensure_geo(r);
    mercury::electron_pressure_gradient(r->lm, r->geo, WH, WNa, dpe);
}

// mercury::AmbipolarEMF::add (Ambipolar.cpp:52-88), E in place
void ref_ambipolar_emf(void *h, const RefStepParams *p, const double *WH, const double *WNa, double *E)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    ensure_geo(r);
    if (!r->amb) r->amb = std::make_unique<mercury::AmbipolarEMF>(r->lm, r->geo);
    r->amb->add(source_config(r, *p), WH, WNa, E);
}

// mercury::gyrate (MercuryUns/physics/Gyration.cpp), in place on UH, UNa
void ref_gyrate(void *h, const RefStepParams *p, const double *B, double dt, double *UH, double *UNa)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    const Config c = source_config(r, *p);
    mercury::gyrate(r->lm, c, B, dt, UH, UNa);
}

namespace
{
struct StepWork
{
    std::vector<std::vector<double>> W, grad, rhs, U1, U2;
    std::vector<double> Bind, Btot, uplus, PhiTot, E, Phi1, Phi2, J, Eres, dpe;
};

// charge-weighted ion velocity of Solver::prepare (Solver.cpp:108-118) with mhd::Scales::numinfo (Scales.cpp:50-62)
void uplus_of(const RefStepParams &p, const CellComplex &cx, const std::vector<std::vector<double>> &W, std::vector<double> &up)
{
    const Id nc = cx.n_cells();
    up.assign(3 * static_cast<size_t>(nc), 0.0);
    for (Id c = 0; c < nc; ++c)
    {
        if (cx.cell_material[c] != kFluid) continue;
        if (p.n_species == 2)
        {
            Scales sc;
            sc.M_ref = p.M_ref; sc.M_H = p.mass[0]; sc.M_Na = p.mass[1]; sc.ne_floor = p.ne_floor;
            const NumInfo ni = sc.numinfo(W[0][5 * c], W[1][5 * c]);
            for (int a = 0; a < 3; ++a) up[3 * c + a] = ni.chiH * W[0][5 * c + 1 + a] + ni.chiNa * W[1][5 * c + 1 + a];
            continue;
        }
        double n[16], ne = 0;
        for (int s = 0; s < p.n_species; ++s) { n[s] = std::max(W[s][5 * c], 0.0) / p.mass[s] * p.M_ref; ne += n[s]; }
        for (int s = 0; s < p.n_species; ++s)
        {
            const double chi = ne > 1e-300 ? n[s] / ne : (s == 0 ? 1.0 : 0.0);
            for (int a = 0; a < 3; ++a) up[3 * c + a] += chi * W[s][5 * c + 1 + a];
        }
    }
}

// Solver::enforce_floors (Solver.cpp:171-191) over all species
void floors(const RefStepParams &p, const CellComplex &cx, std::vector<double *> &U)
{
    for (int k = 0; k < p.n_species; ++k)
        for (Id c = 0; c < cx.ent[3].n_owned; ++c)
        {
            if (cx.cell_material[c] == kSolid) continue;
            double *u = U[k] + 5 * static_cast<size_t>(c);
            const double ke = u[0] > 0 ? 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0] : 0.0;
            if (!(u[0] >= p.rho_floor)) to_cons(Prim{p.rho_floor, 0, 0, 0, p.p_floor}, p.gamma, u);
            else if ((p.gamma - 1.0) * (u[4] - ke) < p.p_floor) to_cons(to_prim(u, p.gamma, p.rho_floor, p.p_floor), p.gamma, u);
        }
}
} // namespace

// U[s]: 5 per cell (AoS) per species, updated in place; Phi: induced face flux, updated in place.
int ref_rk2_step(void *h, RefStepParams *pp, double *const *U, double *Phi, const double *PhiAdd, const double *BaddCell, double dt)
{
    RefMesh *r = static_cast<RefMesh *>(h);
    return guarded([&] {
        const RefStepParams &p = *pp;
        ensure_stencil(r);
        r->cfg.sc.gamma = p.gamma;
        const CellComplex &cx = r->lm.mesh.cx;
        const Id nc = cx.n_cells(), ne = cx.n_edges(), nf = cx.n_faces();
        const int ns = p.n_species;
        static thread_local StepWork w;
        w.W.assign(ns, std::vector<double>(5 * static_cast<size_t>(nc)));
        w.grad.assign(ns, std::vector<double>(15 * static_cast<size_t>(nc)));
        w.rhs.assign(ns, std::vector<double>(5 * static_cast<size_t>(nc)));
        w.U1.assign(ns, std::vector<double>());
        w.U2.assign(ns, std::vector<double>());
        w.E.assign(ne, 0.0);
        w.PhiTot.assign(nf, 0.0);
        r->stencil->set_rel_limit(p.rel_limit);
        const Vec3 uinf(p.u_inf[0], p.u_inf[1], p.u_inf[2]), bimf(p.B_imf[0], p.B_imf[1], p.B_imf[2]);
        const Vec3 E_inf = -1.0 * cross(uinf, bimf);
        const bool lorentz = p.lorentz != 0, ambipolar = p.ambipolar != 0, chemistry = p.chemistry != 0;
        if ((lorentz || ambipolar || chemistry) && ns != 2) throw std::runtime_error("the source terms are those of the two-ion model");
        const Config scfg = source_config(r, p);
        const bool split = lorentz && p.induce_coeff > 0; // Strang splitting of the gyration (Solver.cpp:492-498)
        // the resistive operator of ImplicitInduction (Hall and ideal parts off) with the given per-edge m_e
        ImplicitInduction *res = nullptr;
        if (p.m_res)
        {
            if (!r->res_op)
            {
                ensure_geo(r);
                r->res_ex = std::make_unique<comm::Exchanger>(MPI_COMM_SELF, r->lm);
                Config c;
                c.resistive = true; c.sc.inver_Rem = 1.0; c.hall = false;
                r->res_op = std::make_unique<ImplicitInduction>(r->lm, r->geo, *r->res_ex, c);
            }
            res = r->res_op.get();
            std::copy(p.m_res, p.m_res + res->m_.size(), res->m_.begin());
            res->resistive_ = true; res->hall_ = false; res->ideal_ = false;
            w.Eres.assign(ne, 0.0);
        }

        // prepare + rhs of one stage on (Us, phis); the stage result goes to (Uo, phio)
        auto stage = [&](std::vector<double *> &Us, const double *phis, std::vector<double *> &Uo, double *phio) {
            for (int k = 0; k < ns; ++k) ref_to_prim(Us[k], nc, p.gamma, p.rho_floor, p.p_floor, w.W[k].data());
            const auto bi = reconstruct_cell_vector(cx, r->geo, phis, nc);
            w.Bind.assign(3 * static_cast<size_t>(nc), 0.0);
            w.Btot.assign(3 * static_cast<size_t>(nc), 0.0);
            for (Id c = 0; c < nc; ++c)
            {
                const double b[3] = {bi[c].x, bi[c].y, bi[c].z};
                for (int a = 0; a < 3; ++a) { w.Bind[3 * c + a] = b[a]; w.Btot[3 * c + a] = b[a] + BaddCell[3 * c + a]; }
            }
            uplus_of(p, cx, w.W, w.uplus);
            for (Id f = 0; f < nf; ++f) w.PhiTot[f] = phis[f] + PhiAdd[f];
            if (lorentz)
            {
                w.J.assign(3 * static_cast<size_t>(nc), 0.0);
                cell_current(r->lm, r->geo, w.Bind.data(), w.J.data());
            }
            if (ambipolar) // Solver::prepare (Solver.cpp:124)
            {
                w.dpe.assign(3 * static_cast<size_t>(nc), 0.0);
                mercury::electron_pressure_gradient(r->lm, r->geo, w.W[0].data(), w.W[1].data(), w.dpe.data());
            }
            Prim fs_all[16];
            for (int k = 0; k < ns; ++k) fs_all[k] = Prim{p.fs[k][0], p.fs[k][1], p.fs[k][2], p.fs[k][3], p.fs[k][4]};
            std::unordered_map<Id, int32_t> wslot;
            const GhostFn wg = p.n_wall > 0 ? table_ghost(r, p.n_wall, p.wall_faces, p.wall_prims, p.n_wall, wslot, fs_all, false) : GhostFn{};
            const GhostFn *gp = p.n_wall > 0 ? &wg : nullptr;
            for (int k = 0; k < ns; ++k)
            {
                const Prim &fs = fs_all[k];
                if (p.second_order) r->stencil->limited_gradients(r->lm, r->geo, r->bc, w.W[k].data(), k, fs, true, w.grad[k].data(), gp);
                else std::fill(w.grad[k].begin(), w.grad[k].end(), 0.0);
                fluid_flux_rhs(r->lm, r->geo, r->bc, r->cfg, k, fs, w.W[k].data(), w.grad[k].data(), w.rhs[k].data(), gp);
            }
            if (lorentz || ambipolar || chemistry) // Solver::rhs (Solver.cpp:146-149): sources of both species after both flux passes
            {
                mercury::SourceFields sf;
                sf.photo = p.photo; sf.vst = p.vst; sf.dpe = ambipolar ? w.dpe.data() : nullptr;
                for (int k = 0; k < ns; ++k)
                    mercury::add_sources(r->lm, scfg, k, w.W[0].data(), w.W[1].data(), w.uplus.data(), w.Btot.data(),
                                         lorentz ? w.J.data() : nullptr, sf, dt, w.rhs[k].data(), nullptr);
            }
            std::fill(w.E.begin(), w.E.end(), 0.0);
            IdealInputs in;
            in.u_cell = w.uplus.data(); in.B_cell_tot = w.Btot.data(); in.B_cell_ind = w.Bind.data();
            in.phi_tot = w.PhiTot.data(); in.phi_ind = phis;
            IdealParams ip;
            ip.cuct = p.cuct;
            add_ideal_emf(r->lm, r->geo, in, ip, w.E.data());
            if (ambipolar) // Solver::rhs (Solver.cpp:158), before the boundary edge values
            {
                if (!r->amb) r->amb = std::make_unique<mercury::AmbipolarEMF>(r->lm, r->geo);
                r->amb->add(scfg, w.W[0].data(), w.W[1].data(), w.E.data());
            }
            for (Id e = 0; e < cx.ent[1].n_owned; ++e)
            {
                if (r->bc.edge_mode[e] == 1) w.E[e] = 0.0;
                else if (r->bc.edge_mode[e] == 2) w.E[e] = dot(E_inf, r->geo.edge_vec[e]);
            }
            if (res)
            {
                res->apply_F(phis, w.Eres.data());
                for (Id e = 0; e < cx.ent[1].n_owned; ++e) w.E[e] += w.Eres[e];
            }
            // advance: out = base + dt * rhs on the owned fluid cells, CT on the active faces, floors
            for (int k = 0; k < ns; ++k)
            {
                std::copy(Us[k], Us[k] + 5 * static_cast<size_t>(nc), Uo[k]);
                for (Id c = 0; c < cx.ent[3].n_owned; ++c)
                {
                    if (cx.cell_material[c] == kSolid) continue;
                    for (int m = 0; m < 5; ++m) Uo[k][5 * static_cast<size_t>(c) + m] += dt * w.rhs[k][5 * static_cast<size_t>(c) + m];
                }
            }
            std::copy(phis, phis + nf, phio);
            if (p.first_order)
            {
                // the implicit linear terms with the total EMF as the unknown (Solver.cpp:252-265): frozen total
                // field and n_e,eff of the fluid cells, inflow edges Dirichlet, E_expl the rhs's EMF
                ImplicitInduction &ind = *static_cast<RefInd *>(p.ind)->ind;
                std::vector<double> ne(nc, 0.0);
                for (Id c = 0; c < nc; ++c)
                    if (cx.cell_material[c] == kFluid) ne[c] = scfg.sc.numinfo(w.W[0][5 * static_cast<size_t>(c)], w.W[1][5 * static_cast<size_t>(c)]).ne_eff;
                ind.set_frozen_state(w.Btot.data(), ne.data());
                std::vector<char> dir(cx.n_edges(), 0);
                for (Id e = 0; e < cx.n_edges(); ++e) dir[e] = r->bc.edge_mode[e] == 2;
                std::vector<double> Eimp(cx.n_edges());
                double res = 0;
                pp->ind_iterations = ind.solve(phis, w.E.data(), dir, dt, Eimp.data(), &res);
                pp->ind_rel_res = res;
                w.E = Eimp;
            }
            faraday_update(cx, r->active, w.E.data(), phio, dt);
            floors(p, cx, Uo);
        };
        std::vector<double *> U0(U, U + ns), U1(ns), U2(ns);
        for (int k = 0; k < ns; ++k)
        {
            w.U1[k].resize(5 * static_cast<size_t>(nc));
            w.U2[k].resize(5 * static_cast<size_t>(nc));
            U1[k] = w.U1[k].data();
            U2[k] = w.U2[k].data();
        }
        w.Phi1.resize(nf);
        w.Phi2.resize(nf);
        if (split)
        {
            // Btot of prepare(s_) (Solver.cpp:487): the cell fit of Phi plus the background
            const auto bi = reconstruct_cell_vector(cx, r->geo, Phi, nc);
            std::vector<double> bt(3 * static_cast<size_t>(nc));
            for (Id c = 0; c < nc; ++c)
            {
                bt[3 * c] = bi[c].x + BaddCell[3 * c]; bt[3 * c + 1] = bi[c].y + BaddCell[3 * c + 1]; bt[3 * c + 2] = bi[c].z + BaddCell[3 * c + 2];
            }
            mercury::gyrate(r->lm, scfg, bt.data(), 0.5 * dt, U0[0], U0[1]);
        }
        if (p.first_order)
        {
            // one forward Euler stage in place; the closing half step with the Btot of its prepare (Solver.cpp:274)
            stage(U0, Phi, U1, w.Phi1.data());
            for (int k = 0; k < ns; ++k) std::copy(U1[k], U1[k] + 5 * static_cast<size_t>(nc), U0[k]);
            std::copy(w.Phi1.begin(), w.Phi1.end(), Phi);
            if (split) mercury::gyrate(r->lm, scfg, w.Btot.data(), 0.5 * dt, U0[0], U0[1]);
            return;
        }
        stage(U0, Phi, U1, w.Phi1.data());
        stage(U1, w.Phi1.data(), U2, w.Phi2.data());
        for (int k = 0; k < ns; ++k)
            for (size_t i = 0; i < 5 * static_cast<size_t>(nc); ++i) U0[k][i] = 0.5 * (U0[k][i] + U2[k][i]);
        for (Id f = 0; f < nf; ++f) Phi[f] = 0.5 * (Phi[f] + w.Phi2[f]);
        // the closing half step uses Btot of the last prepare, that of the stage-2 input (Solver.cpp:510)
        if (split) mercury::gyrate(r->lm, scfg, w.Btot.data(), 0.5 * dt, U0[0], U0[1]);
    });
}

// uns::io::write_fields (src/uns/io/MeshIO.cpp:117-130): n records, values[i] holding counts[i] doubles
int ref_write_fields(const char *path, uint64_t hash, int32_t n, const char *const *names, const int32_t *dims, const int32_t *ncomps,
                     const int64_t *counts, const double *const *values)
{
    return guarded([&] {
        std::vector<io::FieldRecord> fs;
        for (int32_t i = 0; i < n; ++i)
        {
            io::FieldRecord f;
            f.name = names[i];
            f.dim = static_cast<Dim>(dims[i]);
            f.ncomp = ncomps[i];
            f.values.assign(values[i], values[i] + counts[i]);
            fs.push_back(std::move(f));
        }
        io::write_fields(path, hash, fs);
    });
}

// uns::io::read_fields (MeshIO.cpp:132-150): the records in file order; query with ref_fields_get
namespace
{
thread_local std::vector<io::FieldRecord> g_fields;
thread_local uint64_t g_hash = 0;
} // namespace
int32_t ref_read_fields(const char *path, uint64_t *hash)
{
    int32_t n = -1;
    guarded([&] {
        g_fields = io::read_fields(path, &g_hash);
        n = static_cast<int32_t>(g_fields.size());
    });
    if (hash) *hash = g_hash;
    return n;
}
// the i-th record of the last ref_read_fields: name (into a buffer of len chars), dim, ncomp, count;
// values copied when out is given
void ref_fields_get(int32_t i, char *name, int32_t len, int32_t *dim, int32_t *ncomp, int64_t *count, double *out)
{
    const io::FieldRecord &f = g_fields.at(static_cast<size_t>(i));
    std::strncpy(name, f.name.c_str(), static_cast<size_t>(len - 1));
    name[len - 1] = 0;
    *dim = static_cast<int32_t>(f.dim);
    *ncomp = f.ncomp;
    *count = static_cast<int64_t>(f.values.size());
    if (out) std::copy(f.values.begin(), f.values.end(), out);
}

} // extern "C"

// ---------------------------------------------------------------- the ten-ion solver
// mars::MarsSolver (MarsUns/driver/MarsSolver.cpp) built on a checker mesh, with its private members opened
// to this file only (the class layout is unchanged), so that each phase of MarsSolver::step runs alone and
// its arrays can be read and set.  Ion arrays cross this boundary species-major, 5 values per cell.
#include <array>
#include <complex>
#include <istream>
#include <string_view>

#include "induction/IdealEMF.h"
#include "induction/ImplicitInduction.h"
#include "physics/MarsAtmosphereModel.h"
#include "physics/MarsChemistry.h"
#include "physics/MarsDipoles.h"
#include "physics/MarsSpecies.h"
#include "uns/comm/Exchanger.h"
#include "uns/core/Params.h"
#define private public
#include "driver/MarsSolver.h"
#undef private

struct RefMars
{
    int last_it = 0;     // the Hall solve of the last step: GMRES iterations and relative residual
    double last_res = 0;
    mars::MarsParams prm;
    std::unique_ptr<mars::MarsSolver> s;
    std::vector<double> rhs_sum; // scratch
};

extern "C" {

// MarsParams::from_params of the given "name=value" overrides, the solver on the mesh, initialize()
void *ref_mars_create(void *mesh, int32_t n_overrides, const char *const *overrides)
{
    RefMars *out = nullptr;
    guarded([&] {
        RefMesh *r = static_cast<RefMesh *>(mesh);
        Params p;
        for (int32_t i = 0; i < n_overrides; ++i) p.set_override(overrides[i]);
        auto *m = new RefMars;
        m->prm = mars::MarsParams::from_params(p);
        m->s = std::make_unique<mars::MarsSolver>(MPI_COMM_SELF, r->lm, m->prm);
        m->s->initialize();
        out = m;
    });
    return out;
}

void ref_mars_free(void *h) { delete static_cast<RefMars *>(h); }

// the scales in the order of MhdMarsParams: rho_ref n_ref p_ref time_ref kB L U q B mag_scale pressure_scale
// ne_floor rho_floor p_floor gamma, then cfl sw_u(3) sw_B(3) ambipolar hall second_order cuct rel_limit hall_scale
void ref_mars_params(void *h, double *out)
{
    const mars::MarsParams &q = static_cast<RefMars *>(h)->prm;
    const double v[] = {q.rho_ref, q.n, q.p_ref, q.time_ref, q.kB, q.L, q.U, q.q, q.B, q.mag_scale, q.pressure_scale, q.ne_floor,
                        q.rho_floor, q.p_floor, q.cfg.sc.gamma, q.cfg.cfl, q.sw_u.x, q.sw_u.y, q.sw_u.z, q.sw_B.x, q.sw_B.y, q.sw_B.z,
                        q.ambipolar ? 1.0 : 0.0, q.hall ? 1.0 : 0.0, q.cfg.second_order ? 1.0 : 0.0, q.cfg.ideal.cuct,
                        q.cfg.recon_rel_limit, q.hall_scale};
    std::memcpy(out, v, sizeof(v));
}

// the free streams fs_ of the ions (the inflow ghosts), 5 per species
void ref_mars_freestream(void *h, double *out)
{
    const mars::MarsSolver &s = *static_cast<RefMars *>(h)->s;
    for (int k = 0; k < mars::NS; ++k)
    {
        const Prim &f = s.fs_[k];
        out[5 * k] = f.rho; out[5 * k + 1] = f.u; out[5 * k + 2] = f.v; out[5 * k + 3] = f.w; out[5 * k + 4] = f.p;
    }
}

namespace
{
std::vector<double> *mars_array(mars::MarsSolver &s, const std::string &n)
{
    if (n == "Phi") return &s.Phi_;
    if (n == "PhiAdd") return &s.PhiAdd_;
    if (n == "PhiTot") return &s.PhiTot_;
    if (n == "BaddCell") return &s.BaddCell_;
    if (n == "Bind") return &s.Bind_;
    if (n == "Btot") return &s.Btot_;
    if (n == "J") return &s.J_;
    if (n == "uplus") return &s.uplus_;
    if (n == "ne") return &s.ne_;
    if (n == "ne_eff") return &s.ne_eff_;
    if (n == "pe") return &s.pe_;
    if (n == "dpe") return &s.dpe_;
    if (n == "neutral") return &s.neutral_;
    if (n == "photo") return &s.photo_;
    return nullptr;
}
std::vector<double> *mars_species(mars::MarsSolver &s, const std::string &n)
{
    if (n == "U") return s.U_;
    if (n == "W") return s.W_;
    if (n == "grad") return s.grad_;
    if (n == "rhs") return s.rhs_;
    return nullptr;
}
} // namespace

// size of a named array (species arrays: all species)
int64_t ref_mars_size(void *h, const char *name)
{
    mars::MarsSolver &s = *static_cast<RefMars *>(h)->s;
    if (auto *a = mars_array(s, name)) return static_cast<int64_t>(a->size());
    if (auto *a = mars_species(s, name)) return static_cast<int64_t>(a[0].size()) * mars::NS;
    return -1;
}

int ref_mars_get(void *h, const char *name, double *out)
{
    return guarded([&] {
        mars::MarsSolver &s = *static_cast<RefMars *>(h)->s;
        if (auto *a = mars_array(s, name)) { std::copy(a->begin(), a->end(), out); return; }
        auto *sp = mars_species(s, name);
        if (!sp) throw std::runtime_error(std::string("unknown array ") + name);
        for (int k = 0; k < mars::NS; ++k) std::copy(sp[k].begin(), sp[k].end(), out + k * sp[0].size());
    });
}

int ref_mars_set(void *h, const char *name, const double *in)
{
    return guarded([&] {
        mars::MarsSolver &s = *static_cast<RefMars *>(h)->s;
        if (auto *a = mars_array(s, name)) { std::copy(in, in + a->size(), a->begin()); return; }
        auto *sp = mars_species(s, name);
        if (!sp) throw std::runtime_error(std::string("unknown array ") + name);
        for (int k = 0; k < mars::NS; ++k) std::copy(in + k * sp[0].size(), in + (k + 1) * sp[0].size(), sp[k].begin());
    });
}

int ref_mars_prepare(void *h) { return guarded([&] { static_cast<RefMars *>(h)->s->prepare(); }); }
int ref_mars_local_dt(void *h, double *dt) { return guarded([&] { *dt = static_cast<RefMars *>(h)->s->local_dt_(); }); }
int ref_mars_fluid_and_sources(void *h, double dt) { return guarded([&] { static_cast<RefMars *>(h)->s->fluid_and_sources_(dt); }); }
int ref_mars_ambipolar_emf(void *h, double *E) { return guarded([&] { static_cast<RefMars *>(h)->s->ambipolar_emf_(E); }); }
int ref_mars_implicit_sources(void *h, double dt) { return guarded([&] { static_cast<RefMars *>(h)->s->implicit_sources_(dt); }); }
int ref_mars_floors(void *h) { return guarded([&] { static_cast<RefMars *>(h)->s->floors_(); }); }

// emf_ (ideal + ambipolar + the boundary edge values) into E (n_edges)
int ref_mars_emf(void *h, double *E)
{
    return guarded([&] {
        mars::MarsSolver &s = *static_cast<RefMars *>(h)->s;
        std::vector<double> e;
        s.emf_(e);
        std::copy(e.begin(), e.end(), E);
    });
}

// The Hall solve's GMRES settings (the reference's Config defaults otherwise: rtol 1e-4, 100 iterations,
// restart 20), for comparisons at the solver's tolerance
int ref_mars_set_induction(void *h, double rtol, int32_t max_it, int32_t restart)
{
    return guarded([&] {
        mars::MarsSolver &s = *static_cast<RefMars *>(h)->s;
        s.ind_.rtol_ = rtol;
        s.ind_.max_it_ = max_it;
        s.ind_.restart_ = std::max(2, static_cast<int>(restart));
    });
}

void ref_mars_last_solve(void *h, int32_t *it, double *res)
{
    *it = static_cast<RefMars *>(h)->last_it;
    *res = static_cast<RefMars *>(h)->last_res;
}

// MarsSolver::step (:705-744) without the photochemistry (chemistry_), with the Hall solve when the solver
// has it on: prepare, dt, fluxes and explicit sources, EMF, forward Euler, Hall solve, Faraday, implicit
// sources, floors
int ref_mars_step_nochem(void *h, double dt_max, double *dt_used)
{
    return guarded([&] {
        mars::MarsSolver &s = *static_cast<RefMars *>(h)->s;
        const CellComplex &cx = s.lm_.mesh.cx;
        s.prepare();
        double dt = std::min(s.local_dt_(), dt_max);
        if (!std::isfinite(dt) || dt <= 0) throw std::runtime_error("invalid time step");
        s.fluid_and_sources_(dt);
        std::vector<double> E;
        s.emf_(E);
        for (int k = 0; k < mars::NS; ++k)
            for (Id c = 0; c < cx.ent[3].n_owned; ++c)
            {
                if (cx.cell_material[c] == kSolid) continue;
                for (int m = 0; m < 5; ++m) s.U_[k][5 * static_cast<std::size_t>(c) + m] += dt * s.rhs_[k][5 * static_cast<std::size_t>(c) + m];
            }
        if (s.ind_.active()) // the Hall branch of MarsSolver::step (:723-735) as the reference runs it
        {
            std::vector<double> ne(cx.n_cells(), 0.0);
            for (Id c = 0; c < cx.n_cells(); ++c)
                if (cx.cell_material[c] == kFluid) ne[c] = s.ne_eff_[c];
            s.ind_.set_frozen_state(s.Btot_.data(), ne.data());
            std::vector<char> dir(cx.n_edges(), 0);
            for (Id e = 0; e < cx.n_edges(); ++e) dir[e] = s.bc_.edge_mode[e] != 0;
            std::vector<double> Eimp = E;
            double res = 0;
            static_cast<RefMars *>(h)->last_it = s.ind_.solve(s.Phi_.data(), E.data(), dir, dt, Eimp.data(), &res);
            static_cast<RefMars *>(h)->last_res = res;
            E.swap(Eimp);
        }
        faraday_update(cx, s.active_, E.data(), s.Phi_.data(), dt);
        s.implicit_sources_(dt);
        s.floors_();
        *dt_used = dt;
    });
}

// the wall ghost of every wall face (wall_state_, :147-165): faces[n], prims[species][n][5]; returns n
int32_t ref_mars_wall_table(void *h, int32_t *faces, double *prims)
{
    int32_t n = 0;
    guarded([&] {
        mars::MarsSolver &s = *static_cast<RefMars *>(h)->s;
        const CellComplex &cx = s.lm_.mesh.cx;
        std::vector<Id> wf;
        for (Id f = 0; f < cx.n_faces(); ++f)
            if (s.bc_.face_kind[f] == FaceKind::Wall) wf.push_back(f);
        n = static_cast<int32_t>(wf.size());
        if (!faces) return;
        for (int32_t i = 0; i < n; ++i) faces[i] = static_cast<int32_t>(wf[i]);
        for (int k = 0; k < mars::NS; ++k)
            for (int32_t i = 0; i < n; ++i)
            {
                const Prim w = s.wall_state_(wf[i], k);
                double *o = prims + (static_cast<std::size_t>(k) * n + i) * 5;
                o[0] = w.rho; o[1] = w.u; o[2] = w.v; o[3] = w.w; o[4] = w.p;
            }
    });
    return n;
}

// the solver's boundary classification (face_kind, edge_mode), for the device mesh
void ref_mars_boundary(void *h, int8_t *face_kind, int8_t *edge_mode)
{
    mars::MarsSolver &s = *static_cast<RefMars *>(h)->s;
    const CellComplex &cx = s.lm_.mesh.cx;
    for (Id f = 0; f < cx.n_faces(); ++f) face_kind[f] = static_cast<int8_t>(s.bc_.face_kind[f]);
    for (Id e = 0; e < cx.n_edges(); ++e) edge_mode[e] = static_cast<int8_t>(s.bc_.edge_mode[e]);
}

} // extern "C"
