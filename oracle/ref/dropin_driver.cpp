// Test driver of the drop-in library (mpcns_uns_b200/lib/libmhd_dropin.so): C entry points that call the
// reference's own C++ signatures (mhd::fluid_flux_rhs, mhd::Stencil::limited_gradients, ...) on reference
// objects built by the compiled reference (oracle/_ref/libmhdref.so, which hands their addresses over).
// This library links the drop-in and not the reference, so every call below resolves to the drop-in's
// GPU body; the parity test compares its results with the reference's CPU bodies on the same objects.
// Test infrastructure only.
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "diagnostics/DivB.h"
#include "fluid/FluxRHS.h"
#include "fluid/Reconstruction.h"
#include "induction/Faraday.h"
#include "induction/IdealEMF.h"
#include "induction/ImplicitInduction.h"
#include "uns/geometry/Reconstruct.h"

namespace mhd_dropin
{
void attach(const uns::LocalMesh &lm, const uns::Geometry &geo, const mhd::BoundaryInfo &bc);
void detach(const uns::LocalMesh &lm);
} // namespace mhd_dropin

namespace
{
thread_local std::string g_err;
template <class F> int guarded(F &&f)
{
    try { f(); return 0; }
    catch (const std::exception &e) { g_err = e.what(); return -1; }
}
const uns::LocalMesh &LM(void *p) { return *static_cast<const uns::LocalMesh *>(p); }
const uns::Geometry &GEO(void *p) { return *static_cast<const uns::Geometry *>(p); }
const mhd::BoundaryInfo &BC(void *p) { return *static_cast<const mhd::BoundaryInfo *>(p); }
mhd::Prim prim(const double *f) { return mhd::Prim{f[0], f[1], f[2], f[3], f[4]}; }
// mhd::active_faces (Common/induction/Faraday.cpp:7-13): the faces of the owned cells (restated here: this
// driver links the drop-in alone, not the reference's Faraday.cpp)
std::vector<char> active(const uns::CellComplex &cx)
{
    std::vector<char> a(cx.n_faces(), 0);
    for (uns::Id c = 0; c < cx.ent[3].n_owned; ++c)
        for (int64_t k = cx.c2f.begin(c); k < cx.c2f.end(c); ++k) a[cx.c2f.idx[k]] = 1;
    return a;
}
} // namespace

extern "C" {
const char *drv_last_error() { return g_err.c_str(); }

int drv_attach(void *lm, void *geo, void *bc) { return guarded([&] { mhd_dropin::attach(LM(lm), GEO(geo), BC(bc)); }); }
int drv_detach(void *lm) { return guarded([&] { mhd_dropin::detach(LM(lm)); }); }

int drv_flux_rhs(void *lm, void *geo, void *bc, void *cfg, int species, const double *fs, const double *W, const double *grad, double *rhs)
{
    return guarded([&] {
        mhd::fluid_flux_rhs(LM(lm), GEO(geo), BC(bc), *static_cast<const mhd::Config *>(cfg), species, prim(fs), W, grad, rhs);
    });
}

int drv_limited_gradients(void *stencil, void *lm, void *geo, void *bc, const double *W, int species, const double *fs, int limit,
                          double rel_limit, double *grad)
{
    return guarded([&] {
        auto *st = static_cast<mhd::Stencil *>(stencil);
        st->set_rel_limit(rel_limit);
        st->limited_gradients(LM(lm), GEO(geo), BC(bc), W, species, prim(fs), limit != 0, grad);
    });
}

int drv_cell_vector(void *lm, void *geo, const double *flux, int32_t ncells, double *out)
{
    return guarded([&] {
        const std::vector<uns::Vec3> b = uns::reconstruct_cell_vector(LM(lm).mesh.cx, GEO(geo), flux, ncells);
        for (size_t i = 0; i < b.size(); ++i) { out[3 * i] = b[i].x; out[3 * i + 1] = b[i].y; out[3 * i + 2] = b[i].z; }
    });
}

int drv_ideal_emf(void *lm, void *geo, const double *u, const double *Bt, const double *Bi, const double *phit, const double *phii,
                  double cuct, double *E)
{
    return guarded([&] {
        mhd::IdealInputs in;
        in.u_cell = u; in.B_cell_tot = Bt; in.B_cell_ind = Bi; in.phi_tot = phit; in.phi_ind = phii;
        mhd::IdealParams prm;
        prm.cuct = cuct;
        mhd::add_ideal_emf(LM(lm), GEO(geo), in, prm, E);
    });
}

int drv_faraday(void *lm, const double *E, double *B, double dt)
{
    return guarded([&] { mhd::faraday_update(LM(lm).mesh.cx, active(LM(lm).mesh.cx), E, B, dt); });
}

int drv_faraday_edge_dt(void *lm, const double *E, const double *dt_edge, double *B)
{
    return guarded([&] { mhd::faraday_update_edge_dt(LM(lm).mesh.cx, active(LM(lm).mesh.cx), E, dt_edge, B); });
}

int drv_div_b(void *lm, const double *B, const double *extra, double *out)
{
    return guarded([&] {
        const mhd::DivBReport r = mhd::div_b(LM(lm).mesh.cx, B, extra);
        out[0] = r.max_abs; out[1] = r.max_rel; out[2] = static_cast<double>(r.worst_cell_gid);
    });
}

int drv_ind_solve(void *ind, const double *Phi, const double *Ee, const int8_t *dir, int64_t n_edges, double dt, double *E, int32_t *it,
                  double *rr)
{
    return guarded([&] {
        std::vector<char> d(dir, dir + n_edges);
        *it = static_cast<mhd::ImplicitInduction *>(ind)->solve(Phi, Ee, d, dt, E, rr);
    });
}

// the per-edge pseudo-time form of the same call
int drv_ind_solve_dte(void *ind, const double *Phi, const double *Ee, const int8_t *dir, int64_t n_edges, const double *dt_edge, double *E,
                      int32_t *it, double *rr)
{
    return guarded([&] {
        std::vector<char> d(dir, dir + n_edges);
        *it = static_cast<mhd::ImplicitInduction *>(ind)->solve(Phi, Ee, d, 0.0, E, rr, dt_edge);
    });
}
} // extern "C"
