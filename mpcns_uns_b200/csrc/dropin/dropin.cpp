// The reference's own hot-path signatures, dispatching to the B200 C-ABI (include/mhd_gpu.h).
//
// This translation unit is compiled against the MPCNS_Uns headers: it defines, with the reference's exact
// declarations, the functions a GPU build of the reference links instead of its CPU bodies:
//   mhd::fluid_flux_rhs             Common/fluid/FluxRHS.h:10-12
//   mhd::Stencil::limited_gradients Common/fluid/Reconstruction.h:28-29
//   uns::reconstruct_cell_vector    include/uns/geometry/Reconstruct.h:14 (raw-pointer form)
//   mhd::add_ideal_emf              Common/induction/IdealEMF.h:40
//   mhd::faraday_update, faraday_update_edge_dt   Common/induction/Faraday.h:17-19
//   mhd::div_b                      Common/diagnostics/DivB.h:15
//   mhd::ImplicitInduction::solve   Common/induction/ImplicitInduction.h:51-52
// Every call takes the reference's host arrays, copies them to device buffers, runs the entry point on
// the mesh handle of its complex and copies the outputs back (the reference keeps its state on the host
// between calls; a solver that keeps the state on the device uses the fused step instead).
//
// Mesh handles.  The first call with a (LocalMesh, Geometry, BoundaryInfo) creates the device mesh of
// that complex; calls that pass only the CellComplex (faraday_update, div_b, reconstruct_cell_vector)
// and add_ideal_emf find it by the complex's address, so one of the calls with a BoundaryInfo (or
// mhd_dropin::attach) must come first.  A complex that changes after its handle was made (refinement,
// repartitioning) must be detached (mhd_dropin::detach) before its next call; a complex destroyed and
// another made at the same address is recognised by its counts and storage and gets a new handle.
//
// Not covered by the C-ABI, and reported as std::runtime_error (the reference's error convention): a
// non-empty GhostFn (the ten-ion solver's wall table has its own entry points).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "diagnostics/DivB.h"
#include "fluid/FluxRHS.h"
#include "fluid/Reconstruction.h"
#include "induction/Faraday.h"
#include "induction/IdealEMF.h"
#include "induction/ImplicitInduction.h"
#include "mhd_gpu.h"
#include "uns/geometry/Reconstruct.h"

namespace mhd_dropin
{
namespace
{
void ok(int rc)
{
    if (rc != MHD_OK) throw std::runtime_error(std::string("mhd_gpu: ") + mhd_gpu_last_error());
}
void cuda_ok(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// a device buffer that grows on demand
struct Buf
{
    void *p = nullptr;
    size_t bytes = 0;
    ~Buf()
    {
        if (p) cudaFree(p);
    }
    template <class T> T *get(size_t n)
    {
        const size_t want = n * sizeof(T);
        if (want > bytes)
        {
            if (p) cudaFree(p);
            p = nullptr;
            bytes = 0;
            cuda_ok(cudaMalloc(&p, want ? want : 1), "cudaMalloc");
            bytes = want;
        }
        return static_cast<T *>(p);
    }
};

struct Entry
{
    MhdMesh *mesh = nullptr;
    cudaStream_t stream = nullptr;
    const uns::CellComplex *cx = nullptr;
    // what the handle was made from: a complex made later at the same address (the first one destroyed
    // without detach) shows up as different counts or storage and gets a new handle
    std::array<int64_t, 4> counts{};
    const void *storage[3] = {};
    Buf b[10];
    std::vector<int32_t> e2n; // start and end node of every edge (the descriptor's edge_nodes)
    ~Entry()
    {
        if (mesh) mhd_gpu_mesh_destroy(mesh);
    }
    template <class T> T *up(int slot, const T *host, size_t n)
    {
        T *d = b[slot].get<T>(n);
        if (n) cuda_ok(cudaMemcpyAsync(d, host, n * sizeof(T), cudaMemcpyHostToDevice, stream), "cudaMemcpyAsync");
        return d;
    }
    template <class T> void down(T *host, const T *dev, size_t n)
    {
        if (n) cuda_ok(cudaMemcpyAsync(host, dev, n * sizeof(T), cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync");
        cuda_ok(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    }
};

std::mutex g_mu;
std::unordered_map<const uns::CellComplex *, std::unique_ptr<Entry>> g_entries;

const double *v3(const std::vector<uns::Vec3> &v) { return v.empty() ? nullptr : &v[0].x; }

Entry &make(const uns::LocalMesh &lm, const uns::Geometry &geo, const mhd::BoundaryInfo &bc)
{
    std::lock_guard<std::mutex> lock(g_mu);
    const uns::CellComplex &cx = lm.mesh.cx;
    const std::array<int64_t, 4> counts{cx.n_nodes(), cx.n_edges(), cx.n_faces(), cx.n_cells()};
    const void *storage[3] = {cx.c2f.idx.data(), cx.f2e.idx.data(), geo.cell_volume.data()};
    auto it = g_entries.find(&cx);
    if (it != g_entries.end())
    {
        const Entry &o = *it->second;
        if (o.counts == counts && std::equal(storage, storage + 3, o.storage)) return *it->second;
        g_entries.erase(it);
    }
    auto e = std::make_unique<Entry>();
    e->cx = &cx;
    e->counts = counts;
    std::copy(storage, storage + 3, e->storage);
    e->e2n.resize(2 * static_cast<size_t>(cx.n_edges()));
    for (uns::Id k = 0; k < cx.n_edges(); ++k)
        for (int64_t q = cx.e2n.begin(k); q < cx.e2n.end(k); ++q) e->e2n[2 * k + (cx.e2n.sgn[q] > 0 ? 1 : 0)] = cx.e2n.idx[q];
    MhdMeshDesc d{};
    d.n_nodes = cx.n_nodes(); d.n_edges = cx.n_edges(); d.n_faces = cx.n_faces(); d.n_cells = cx.n_cells();
    d.n_owned_cells = cx.ent[3].n_owned; d.n_owned_edges = cx.ent[1].n_owned;
    d.c2f_ptr = cx.c2f.ptr.data(); d.c2f_idx = cx.c2f.idx.data(); d.c2f_sgn = cx.c2f.sgn.data();
    d.f2e_ptr = cx.f2e.ptr.data(); d.f2e_idx = cx.f2e.idx.data(); d.f2e_sgn = cx.f2e.sgn.data();
    d.e2f_ptr = cx.e2f.ptr.data(); d.e2f_idx = cx.e2f.idx.data(); d.e2f_sgn = cx.e2f.sgn.data();
    d.f2c_ptr = cx.f2c.ptr.data(); d.f2c_idx = cx.f2c.idx.data(); d.f2c_sgn = cx.f2c.sgn.data();
    d.cell_material = cx.cell_material.data();
    d.edge_vec = v3(geo.edge_vec); d.edge_mid = v3(geo.edge_mid); d.edge_len = geo.edge_len.data();
    d.face_area = v3(geo.face_area); d.face_center = v3(geo.face_center); d.face_area_mag = geo.face_area_mag.data();
    d.cell_center = v3(geo.cell_center); d.cell_volume = geo.cell_volume.data();
    d.ec_ptr = geo.ec_ptr.data(); d.ec_cell = geo.ec_cell.data(); d.ec_weight = geo.ec_weight.data();
    d.ef_weight = geo.ef_weight.data();
    d.star1 = geo.star1.data(); d.star2 = geo.star2.data();
    static_assert(sizeof(mhd::FaceKind) == 1, "FaceKind is one byte");
    d.face_kind = reinterpret_cast<const int8_t *>(bc.face_kind.data());
    d.edge_mode = reinterpret_cast<const int8_t *>(bc.edge_mode.data());
    d.edge_nodes = e->e2n.data();
    ok(mhd_gpu_mesh_create(&d, &e->mesh));
    e->stream = static_cast<cudaStream_t>(mhd_gpu_mesh_stream(e->mesh));
    Entry &ref = *e;
    g_entries.emplace(&cx, std::move(e));
    return ref;
}

Entry &find(const uns::CellComplex &cx)
{
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_entries.find(&cx);
    if (it == g_entries.end())
        throw std::runtime_error("mhd_gpu drop-in: no device mesh for this complex; attach it (mhd_dropin::attach) or call a "
                                 "function that takes its BoundaryInfo first");
    return *it->second;
}

void no_ghost(const mhd::GhostFn *ghost)
{
    if (ghost && *ghost)
        throw std::runtime_error("mhd_gpu drop-in: a GhostFn has no device form; a Dirichlet wall table maps to "
                                 "mhd_gpu_limited_gradients_wall / mhd_gpu_flux_rhs_wall");
}
} // namespace

// Device mesh of a complex, created from its metric and boundary classification; detach drops it.
void attach(const uns::LocalMesh &lm, const uns::Geometry &geo, const mhd::BoundaryInfo &bc) { make(lm, geo, bc); }
void detach(const uns::LocalMesh &lm)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_entries.erase(&lm.mesh.cx);
}
} // namespace mhd_dropin

using mhd_dropin::Entry;

namespace mhd
{
void fluid_flux_rhs(const uns::LocalMesh &lm, const uns::Geometry &geo, const BoundaryInfo &bc, const Config &cfg, int species,
                    const Prim &freestream, const double *W, const double *grad, double *rhs, const GhostFn *ghost)
{
    mhd_dropin::no_ghost(ghost);
    Entry &e = mhd_dropin::make(lm, geo, bc);
    const size_t nc = lm.mesh.cx.n_cells();
    const double *dW = e.up(0, W, 5 * nc), *dg = e.up(1, grad, 15 * nc);
    double *dr = e.b[2].get<double>(5 * nc);
    const MhdPrim fs{freestream.rho, freestream.u, freestream.v, freestream.w, freestream.p};
    mhd_dropin::ok(mhd_gpu_flux_rhs(e.mesh, cfg.sc.gamma, species, &fs, dW, dg, dr));
    e.down(rhs, dr, 5 * nc);
}

void Stencil::limited_gradients(const uns::LocalMesh &lm, const uns::Geometry &geo, const BoundaryInfo &bc, const double *W, int species,
                                const Prim &freestream, bool limit, double *grad, const GhostFn *ghost) const
{
    mhd_dropin::no_ghost(ghost);
    Entry &e = mhd_dropin::make(lm, geo, bc);
    const size_t nc = lm.mesh.cx.n_cells();
    const double *dW = e.up(0, W, 5 * nc);
    double *dg = e.b[1].get<double>(15 * nc);
    const MhdPrim fs{freestream.rho, freestream.u, freestream.v, freestream.w, freestream.p};
    mhd_dropin::ok(mhd_gpu_limited_gradients(e.mesh, dW, species, &fs, limit ? 1 : 0, rel_limit_, dg));
    e.down(grad, dg, 15 * nc);
}

void add_ideal_emf(const uns::LocalMesh &lm, const uns::Geometry &, const IdealInputs &in, const IdealParams &prm, double *E)
{
    Entry &e = mhd_dropin::find(lm.mesh.cx);
    const uns::CellComplex &cx = lm.mesh.cx;
    const size_t nc = cx.n_cells(), nf = cx.n_faces(), ne = cx.n_edges();
    const double *du = e.up(0, in.u_cell, 3 * nc), *dbt = e.up(1, in.B_cell_tot, 3 * nc), *dbi = e.up(2, in.B_cell_ind, 3 * nc);
    const double *dpt = e.up(3, in.phi_tot, nf), *dpi = e.up(4, in.phi_ind, nf);
    double *dE = e.up(5, static_cast<const double *>(E), ne);
    mhd_dropin::ok(mhd_gpu_ideal_emf(e.mesh, du, dbt, dbi, dpt, dpi, prm.cuct, dE));
    e.down(E, dE, ne);
}

void faraday_update(const uns::CellComplex &cx, const std::vector<char> &, const double *E, double *B, double dt)
{
    Entry &e = mhd_dropin::find(cx);
    const double *dE = e.up(0, E, (size_t)cx.n_edges());
    double *dB = e.up(1, static_cast<const double *>(B), (size_t)cx.n_faces());
    mhd_dropin::ok(mhd_gpu_faraday(e.mesh, dE, dB, dt));
    e.down(B, dB, (size_t)cx.n_faces());
}

void faraday_update_edge_dt(const uns::CellComplex &cx, const std::vector<char> &, const double *E, const double *dt_edge, double *B)
{
    Entry &e = mhd_dropin::find(cx);
    const double *dE = e.up(0, E, (size_t)cx.n_edges()), *ddt = e.up(2, dt_edge, (size_t)cx.n_edges());
    double *dB = e.up(1, static_cast<const double *>(B), (size_t)cx.n_faces());
    mhd_dropin::ok(mhd_gpu_faraday_edge_dt(e.mesh, dE, ddt, dB));
    e.down(B, dB, (size_t)cx.n_faces());
}

DivBReport div_b(const uns::CellComplex &cx, const double *B, const double *scale_extra)
{
    Entry &e = mhd_dropin::find(cx);
    const double *dB = e.up(0, B, (size_t)cx.n_faces());
    const double *dx = scale_extra ? e.up(1, scale_extra, (size_t)cx.n_faces()) : nullptr;
    double out[3];
    mhd_dropin::ok(mhd_gpu_div_b(e.mesh, dB, dx, out));
    DivBReport r;
    r.max_abs = out[0];
    r.max_rel = out[1];
    const long c = static_cast<long>(out[2]);
    r.worst_cell_gid = c >= 0 ? static_cast<long>(cx.ent[3].gid[c]) : -1;
    return r;
}

// ImplicitInduction::solve (ImplicitInduction.cpp:299-390) on the device: the handle is made on the first solve
// from the object's resistivity m_, Hall switch and GMRES settings; every solve hands over the frozen state
// the object holds (B0_ and alpha_ = taper * hall_coef / n_e,eff of set_frozen_state), and its implicit ideal
// part (u_ideal_, ideal_mask_ of set_ideal_state) where it has one.  use_guess_ maps to the warm start; dt_edge
// to the per-edge form of the solve.
namespace
{
// The device handle of an ImplicitInduction object, with the settings it was made from: an object made
// later at the same address (the first one destroyed) or with other settings gets a new handle.
struct IndEntry
{
    MhdInduction *ind = nullptr;
    MhdMesh *mesh = nullptr;
    bool hall = false, resistive = false, ilu = false;
    double hall_coef = 0, rtol = 0, shift = 0;
    int max_it = 0, restart = 0;
    std::vector<double> m;
    ~IndEntry()
    {
        if (ind) mhd_gpu_induction_destroy(ind);
    }
};
std::mutex g_ind_mu;
std::unordered_map<const ImplicitInduction *, std::unique_ptr<IndEntry>> g_ind;
} // namespace

int ImplicitInduction::solve(const double *Phi_n, const double *E_expl, const std::vector<char> &dirichlet, double dt, double *E,
                             double *rel_res, const double *dt_edge)
{
    // the block-ILU(0) preconditioner where the object built its pattern (:102, :317)
    const bool ilu = use_ilu_ && !pc_ptr_.empty();
    Entry &e = mhd_dropin::find(lm_.mesh.cx);
    IndEntry *ie = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_ind_mu);
        auto &slot = g_ind[this];
        if (slot && !(slot->mesh == e.mesh && slot->hall == hall_ && slot->resistive == resistive_ && slot->hall_coef == hall_coef_ &&
                      slot->rtol == rtol_ && slot->max_it == max_it_ && slot->restart == restart_ && slot->ilu == ilu &&
                      (!ilu || slot->shift == shift_) && (!resistive_ || slot->m == m_)))
            slot.reset();
        if (!slot)
        {
            slot = std::make_unique<IndEntry>();
            slot->mesh = e.mesh;
            slot->hall = hall_;
            slot->resistive = resistive_;
            slot->hall_coef = hall_coef_;
            slot->rtol = rtol_;
            slot->max_it = max_it_;
            slot->restart = restart_;
            slot->ilu = ilu;
            slot->shift = shift_;
            if (resistive_) slot->m = m_;
            MhdInductionParams p{};
            p.hall = hall_ ? 1 : 0;
            p.max_it = max_it_;
            p.restart = restart_;
            p.precision = MHD_PREC_FP64;
            p.hall_coef = hall_coef_;
            p.rtol = rtol_;
            // the object's own taper is in alpha_, handed over with the frozen state: the handle's taper stays 1
            p.hall_r_min = -1.0;
            p.hall_r_max = -1.0;
            mhd_dropin::ok(mhd_gpu_induction_create(e.mesh, &p, resistive_ ? m_.data() : nullptr, &slot->ind));
            if (ilu) mhd_dropin::ok(mhd_gpu_induction_set_ilu(slot->ind, 1, shift_));
        }
        ie = slot.get();
    }
    const uns::CellComplex &cx = lm_.mesh.cx;
    const size_t nc = cx.n_cells(), nf = cx.n_faces(), ne = cx.n_edges();
    const double *dB0 = e.up(0, B0_.data(), 3 * nc), *dal = e.up(1, alpha_.data(), nc);
    mhd_dropin::ok(mhd_gpu_induction_set_frozen_alpha(ie->ind, dB0, dal));
    // the implicit ideal part where the object has its frozen velocities (set_ideal_state, :112-116)
    if (ideal_ && u_ideal_)
    {
        const double *du = e.up(6, u_ideal_, 3 * nc);
        const int8_t *dm = e.up(7, reinterpret_cast<const int8_t *>(ideal_mask_.data()), ne);
        mhd_dropin::ok(mhd_gpu_induction_set_ideal(ie->ind, du, dm, ideal_prm_.cuct));
    }
    else
        mhd_dropin::ok(mhd_gpu_induction_set_ideal(ie->ind, nullptr, nullptr, ideal_prm_.cuct));
    const double *dPhi = e.up(2, Phi_n, nf), *dEe = e.up(3, E_expl, ne);
    static_assert(sizeof(char) == sizeof(int8_t), "char is one byte");
    const int8_t *ddir = e.up(4, reinterpret_cast<const int8_t *>(dirichlet.data()), ne);
    double *dE = e.b[5].get<double>(ne);
    int32_t it = 0;
    double rr = 0;
    const int rc = dt_edge ? mhd_gpu_induction_solve_dt_edge(ie->ind, dPhi, dEe, ddir, e.up(8, dt_edge, ne), use_guess_ ? 1 : 0, dE, &it, &rr)
                           : mhd_gpu_induction_solve(ie->ind, dPhi, dEe, ddir, dt, use_guess_ ? 1 : 0, dE, &it, &rr);
    if (rc != MHD_OK && rc != MHD_ENOCONV) mhd_dropin::ok(rc);
    e.down(E, dE, ne);
    if (rel_res) *rel_res = rr;
    return it;
}
} // namespace mhd

namespace uns
{
std::vector<Vec3> reconstruct_cell_vector(const CellComplex &cx, const Geometry &, const double *flux, Id ncells)
{
    Entry &e = mhd_dropin::find(cx);
    const double *df = e.up(0, flux, (size_t)cx.n_faces());
    double *dout = e.b[1].get<double>(3 * (size_t)(ncells > 0 ? ncells : 0));
    mhd_dropin::ok(mhd_gpu_cell_vector(e.mesh, df, ncells, dout));
    std::vector<Vec3> out(ncells > 0 ? ncells : 0);
    double *host = out.empty() ? nullptr : &out[0].x;
    e.down(host, dout, 3 * out.size());
    return out;
}
} // namespace uns
