/* C-ABI of the B200 hot path of the MPCNS_Uns Hall-MHD step.
 *
 * One opaque handle (MhdMesh) holds a device copy of one rank's signed cell complex, its
 * metric and boundary classification, plus the tables derived from them once (least-squares
 * stencil inverses, cell-field reconstruction coefficients, face -> (L, R) cells).  Every
 * entry point below replaces one function of the reference and keeps its meaning: same
 * inputs, same outputs, same layout of the arrays (the reference's AoS order: value(i, comp)
 * = a[i*ncomp + comp]).  Array arguments are DEVICE pointers unless the name says `host`;
 * all work is ordered on the handle's CUDA stream (mhd_gpu_mesh_stream) and calls return
 * when it is enqueued, except calls with host outputs, which synchronise.
 *
 * An array argument may be NULL where it holds no entries (an empty rank: no cells, faces or edges); the
 * call then does nothing for it, as the reference's loops run zero times.
 *
 * Status: 0 ok, MHD_EINVAL bad argument, MHD_ECUDA CUDA error, MHD_ESTATE non-finite or
 * invalid state detected, MHD_ENOCONV GMRES stopped at max_it above rtol (the solution and
 * its relative residual are still returned).  mhd_gpu_last_error() gives the message of the
 * calling thread's last failure.  No C++ exception crosses this boundary.  A handle is used
 * by one host thread at a time (the reference's one-rank-one-thread model).
 */
#ifndef MHD_GPU_H
#define MHD_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MHD_OK 0
#define MHD_EINVAL (-1)
#define MHD_ECUDA (-2)
#define MHD_ESTATE (-3)
#define MHD_ENOCONV (-4)

typedef struct MhdMesh MhdMesh;
typedef struct MhdInduction MhdInduction;
typedef struct MhdState MhdState;

/* Host arrays of one rank's mesh, in the layout of the reference's uns::CellComplex
 * (include/uns/complex/CellComplex.h:29-53: signed CSR, int64 ptr / int32 idx / int8 sgn),
 * uns::Geometry (include/uns/geometry/Geometry.h:25-43; Vec3 = 3 doubles) and
 * mhd::BoundaryInfo (Common/boundary/BoundaryInfo.h:21-29).  Copied at creation. */
typedef struct MhdMeshDesc {
    int32_t n_nodes, n_edges, n_faces, n_cells;
    int32_t n_owned_cells, n_owned_edges; /* reference LocalMesh ent[3].n_owned / ent[1].n_owned */
    const int64_t *c2f_ptr; const int32_t *c2f_idx; const int8_t *c2f_sgn;
    const int64_t *f2e_ptr; const int32_t *f2e_idx; const int8_t *f2e_sgn;
    const int64_t *e2f_ptr; const int32_t *e2f_idx; const int8_t *e2f_sgn;
    const int64_t *f2c_ptr; const int32_t *f2c_idx; const int8_t *f2c_sgn;
    const int32_t *cell_material;          /* 0 fluid, 1 solid */
    const double *edge_vec, *edge_mid, *edge_len;
    const double *face_area, *face_center, *face_area_mag;
    const double *cell_center, *cell_volume;
    const int64_t *ec_ptr; const int32_t *ec_cell; const double *ec_weight;
    const double *ef_weight;               /* aligned with e2f */
    const double *star1, *star2;
    const int8_t *face_kind;               /* 0 Interior 1 Wall 2 Inflow 3 Outflow 4 Skip */
    const int8_t *edge_mode;               /* 0 free 1 wall (E = 0) 2 inflow */
    /* optional: start and end node of every edge (2 per edge, uns::CellComplex::edge_nodes); with it the
     * handle builds the node -> fluid-cell lists of mercury::AmbipolarEMF (MercuryUns/physics/Ambipolar.cpp:35-50) */
    const int32_t *edge_nodes;
} MhdMeshDesc;

/* Primitive state W = (rho, u, v, w, p) of mhd::Prim (Common/physics/Euler.h:7-10). */
typedef struct MhdPrim { double rho, u, v, w, p; } MhdPrim;

const char *mhd_gpu_last_error(void);
int mhd_gpu_device_info(char *name, size_t name_len, int *sm_count);

/* uns::compute_geometry (src/uns/geometry/Geometry.cpp:17-169) on the device, bit-identical to the
 * reference's host computation: topology (reference CSR layouts) and node coordinates in, every uns::Geometry
 * array out into the caller's host arrays (any output may be NULL: skipped).  ec_cell / ec_weight hold
 * ec_capacity entries; 2 * e2f_ptr[n_edges] always suffices, the count used is ec_ptr[n_edges].
 * Limits: face loops of at most 16 nodes, cells of at most 64 nodes, edges of at most 32 faces. */
typedef struct MhdGeometryArgs {
    int32_t n_nodes, n_edges, n_faces, n_cells;
    const double *x;              /* 3 per node */
    const int32_t *edge_nodes;    /* start, end per edge (uns::CellComplex::edge_nodes) */
    const int64_t *f2e_ptr; const int32_t *f2e_idx; const int8_t *f2e_sgn;
    const int64_t *c2f_ptr; const int32_t *c2f_idx; const int8_t *c2f_sgn;
    const int64_t *e2f_ptr; const int32_t *e2f_idx;   /* rows in ascending face order */
    const int64_t *f2c_ptr; const int32_t *f2c_idx;
    double *edge_vec, *edge_mid, *edge_len;           /* 3, 3, 1 per edge */
    double *face_area, *face_center, *face_area_mag;  /* 3, 3, 1 per face */
    double *cell_center, *cell_volume, *cell_min_tet_volume;
    double *star0, *star1, *star2, *star3;            /* per node, edge, face, cell */
    double *edge_dual_area;                           /* 3 per edge */
    int32_t *ec_misoriented;                          /* per edge */
    double *ef_weight;                                /* aligned with e2f */
    int64_t *ec_ptr;                                  /* n_edges + 1 */
    int32_t *ec_cell; double *ec_weight; int64_t ec_capacity;
} MhdGeometryArgs;
int mhd_gpu_compute_geometry(const MhdGeometryArgs *args);

/* mhd::BoundaryInfo::build (Common/boundary/BoundaryInfo.cpp:9-49) on the device: face kinds (0 Interior,
 * 1 Wall, 2 Inflow, 3 Outflow, 4 Skip) and edge modes (0 free, 1 wall, 2 inflow) into the caller's host arrays,
 * equal to the reference's.  The caller resolves its tag-name -> type map: tag_type[t] for the tag ids
 * 0 < t < n_tags, type_none for tag 0 and ids out of range (the reference's empty name), each 1 wall,
 * 2 inflow, 3 outflow, 5 farfield or 0 unknown (MHD_EINVAL if a boundary face has it, as the reference
 * throws).  Every face has one or two cells. */
typedef struct MhdBoundaryArgs {
    int32_t n_edges, n_faces, n_cells, n_tags;
    const int64_t *f2c_ptr; const int32_t *f2c_idx; const int8_t *f2c_sgn;
    const int64_t *e2f_ptr; const int32_t *e2f_idx;
    const int32_t *cell_material, *face_tag;
    const double *face_area, *face_area_mag;
    const int8_t *tag_type;
    int8_t type_none, pad[7];
    double u_inf[3];
    int8_t *face_kind, *edge_mode;
} MhdBoundaryArgs;
int mhd_gpu_boundary(const MhdBoundaryArgs *args);

/* The tetrahedral cell complex of a hexahedral list on the device: every hexahedron (8 node ids in the
 * reference's local corner order, corner i at (i&1, (i>>1)&1, (i>>2)&1)) cut into the 6 Kuhn tetrahedra of
 * its body diagonal, numbered exactly as uns::ComplexBuilder numbers them when the tetrahedra are added in
 * that order (src/uns/complex/ComplexBuilder.cpp:45-134: add_cell, tag_face, finish; the same complex and
 * uns::topology_hash as the host library's mhdm_shell / mhdm_box with as_tets), with the upward
 * incidences of CellComplex::build_up (n2e, e2f, f2c: rows in ascending order of their entries).
 * tag_tri: 3 nodes per tagged triangle (any order), tag_id its tag; later tags of a face win.  Host
 * inputs; the complex stays on the device until copied out.  Faces shared by more than two cells are
 * rejected with MHD_EINVAL. */
typedef struct MhdTetBuild MhdTetBuild;
int mhd_gpu_tet_build(int32_t n_nodes, int64_t n_hex, const int32_t *hex8, const int32_t *hex_material, int32_t n_tags,
                      const int32_t *tag_tri, const int32_t *tag_id, MhdTetBuild **out);
/* counts[0..3] = nodes, edges, faces, cells */
int mhd_gpu_tet_build_counts(const MhdTetBuild *b, int64_t *counts);
/* Host outputs (any may be NULL: skipped), tables in the order e2n, f2e, c2f, n2e, e2f, f2c: ptr rows + 1
 * entries, idx and sgn one per incidence; cell_material per cell, face_tag per face. */
typedef struct MhdComplexOut {
    int64_t *ptr[6];
    int32_t *idx[6];
    int8_t *sgn[6];
    int32_t *cell_material, *face_tag;
} MhdComplexOut;
int mhd_gpu_tet_build_copy(const MhdTetBuild *b, const MhdComplexOut *out);
int mhd_gpu_tet_build_free(MhdTetBuild *b);

/* Upload a mesh; replaces the reference's per-call use of LocalMesh + Geometry + BoundaryInfo
 * and the one-time setup of mhd::Stencil::Stencil (Common/fluid/Reconstruction.cpp:26-78). */
int mhd_gpu_mesh_create(const MhdMeshDesc *desc, MhdMesh **out);
int mhd_gpu_mesh_destroy(MhdMesh *mesh);
/* The CUDA stream (cudaStream_t) the handle's work is ordered on; may be replaced by the caller's. */
void *mhd_gpu_mesh_stream(MhdMesh *mesh);
int mhd_gpu_mesh_set_stream(MhdMesh *mesh, void *stream);
int mhd_gpu_synchronize(MhdMesh *mesh);

/* mhd::to_prim over n cells (Common/physics/Euler.h:13-21): U, W 5 per cell. */
int mhd_gpu_to_prim(MhdMesh *mesh, const double *U, int32_t n, double gamma, double rho_floor, double p_floor, double *W);

/* mhd::Stencil::limited_gradients (Common/fluid/Reconstruction.h:28-29, .cpp:80-142):
 * W 5 per cell -> grad 15 per cell (3*m + axis), zero outside the valid owned fluid cells.
 * species 1 is the absorbing wall species of ghost_state (Reconstruction.cpp:9-24). */
int mhd_gpu_limited_gradients(MhdMesh *mesh, const double *W, int32_t species, const MhdPrim *freestream, int32_t limit,
                              double rel_limit, double *grad);

/* mhd::fluid_flux_rhs (Common/fluid/FluxRHS.h:10-12, .cpp:30-74): rhs 5 per cell, overwritten
 * on the owned fluid cells, zero elsewhere. */
int mhd_gpu_flux_rhs(MhdMesh *mesh, double gamma, int32_t species, const MhdPrim *freestream, const double *W,
                     const double *grad, double *rhs);

/* The same two passes with a Dirichlet wall table: the GhostFn argument of limited_gradients and
 * fluid_flux_rhs (Common/fluid/Reconstruction.h:21, FluxRHS.h:10-12) as the ten-ion solver binds it
 * (MarsUns/driver/MarsSolver.cpp:124-128): on each listed face (kind wall) the ghost state is
 * wall_prims[5*i .. 5*i+4] (rho u v w p of this species), whatever the inside state; every other face
 * keeps ghost_state.  Device pointers; the faces must be distinct faces of kind wall (MHD_EINVAL
 * otherwise).  n_wall = 0 is the plain pass. */
int mhd_gpu_limited_gradients_wall(MhdMesh *mesh, const double *W, int32_t species, const MhdPrim *freestream, int32_t limit,
                                   double rel_limit, int32_t n_wall, const int32_t *wall_faces, const double *wall_prims,
                                   double *grad);
int mhd_gpu_flux_rhs_wall(MhdMesh *mesh, double gamma, int32_t species, const MhdPrim *freestream, const double *W,
                          const double *grad, int32_t n_wall, const int32_t *wall_faces, const double *wall_prims, double *rhs);

/* uns::reconstruct_cell_vector (include/uns/geometry/Reconstruct.h:14, src/uns/geometry/Reconstruct.cpp:8-46):
 * face flux (canonical orientation) -> 3 per cell for the cells [0, ncells). */
int mhd_gpu_cell_vector(MhdMesh *mesh, const double *flux, int32_t ncells, double *out);

/* mhd::add_ideal_emf (Common/induction/IdealEMF.h:40, .cpp:25-129): adds the ideal UCT EMF of
 * every owned edge to E.  u, B_tot, B_ind: 3 per cell; phi_tot, phi_ind: 1 per face. */
int mhd_gpu_ideal_emf(MhdMesh *mesh, const double *u_cell, const double *B_cell_tot, const double *B_cell_ind,
                      const double *phi_tot, const double *phi_ind, double cuct, double *E);

/* Boundary edge values of mercury::Solver::rhs (MercuryUns/driver/Solver.cpp:162-167):
 * edge_mode 1 -> E = 0, edge_mode 2 -> E = (-u_inf x B_imf) . edge_vec, owned edges. */
int mhd_gpu_edge_modes(MhdMesh *mesh, const double *u_inf, const double *B_imf, double *E);

/* mhd::faraday_update / faraday_update_edge_dt (Common/induction/Faraday.h:17-19, .cpp:15-36)
 * over mhd::active_faces (:7-13): B[f] -= dt * sum f2e.sgn * E, in FP64. */
int mhd_gpu_faraday(MhdMesh *mesh, const double *E, double *B, double dt);
int mhd_gpu_faraday_edge_dt(MhdMesh *mesh, const double *E, const double *dt_edge, double *B);

/* mhd::div_b (Common/diagnostics/DivB.h:15, .cpp:8-24) over the owned cells, FP64.
 * host_out[0] = max |d2 B|, host_out[1] = max relative, host_out[2] = the handle's local index of the
 * worst cell (-1 if d2 B vanishes everywhere).  The reference reports the cell's global id
 * (cx.ent[3].gid[c], DivB.cpp:20); a caller with a per-rank mesh maps the index through its gid table
 * (on one rank built by ComplexBuilder, gid[c] = c).  The call synchronises the handle's stream. */
int mhd_gpu_div_b(MhdMesh *mesh, const double *B, const double *extra, double *host_out);

/* The div B diagnostic of mhd_gpu_div_b for callers that must not allocate device memory once
 * they run: a host application that hands all GPU memory to its own pool or arena at start-up (a
 * cudaMalloc behind its back would fail or break its accounting), or a process under a fixed memory
 * budget whose footprint must not grow after set-up.  This entry point has no counterpart in the
 * reference.  It calls no cudaMalloc / cudaFree and no allocating library routine: its block
 * partials and result live in one static device array of MHD_NOALLOC_DIVB_MAX_BLOCKS partials
 * (1.5 MiB), which every GPU that loads this library holds until the process exits.  One block
 * reduces 1024 cells, so a mesh may have at most MHD_NOALLOC_DIVB_MAX_BLOCKS * 1024 = 67,108,864
 * owned cells; larger meshes are rejected with MHD_EINVAL (mhd_gpu_div_b_noalloc_blocks gives the
 * block count of a mesh size, or that error, without touching the GPU).  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) with that device current; make that
 * first call before any stream capture starts on the device.  Like
 * mhd_gpu_div_b it copies the three results to host_out and synchronises the handle's stream before
 * returning.  Every call overwrites the partials it reads, so nothing has to start at zero; calls
 * that overlap on the GPU (other streams, other threads) share the array and race.  Results equal
 * mhd_gpu_div_b's. */
#define MHD_NOALLOC_DIVB_MAX_BLOCKS 65536
int mhd_gpu_div_b_noalloc(MhdMesh *mesh, const double *B, const double *extra, double *host_out);
int mhd_gpu_div_b_noalloc_blocks(int64_t n_owned_cells, int64_t *blocks);
/* Number of cudaMalloc and cudaFree calls this library has made since it was loaded (every device
 * buffer of every handle); no GPU work. */
int mhd_gpu_alloc_calls(int64_t *out);

/* mhd::cell_current (Common/induction/Current.cpp:9-31): B 3 per cell -> J 3 per cell. */
int mhd_gpu_cell_current(MhdMesh *mesh, const double *B, double *J);

/* ------------------------------------------------------------------ semi-implicit induction
 * mhd::ImplicitInduction (Common/induction/ImplicitInduction.h:27-94): the operator
 *   F(Phi) = M d1^T S2 Phi + H(Phi),  A x = x + dt F(d1 x)
 * and the restarted GMRES(m) with Givens rotations, Jacobi right preconditioner (or block ILU(0):
 * mhd_gpu_induction_set_ilu), true residual at every restart and warm start (.cpp:299-390).  The reference orthogonalises with modified
 * Gram-Schmidt; here (restart <= 31) classical Gram-Schmidt with a second pass where the first
 * cancelled and left components above round-off: the same Krylov space and Hessenberg matrix to
 * rounding, two or three passes over the basis per Arnoldi step (restart > 31: modified Gram-Schmidt).  The resistive
 * coefficient m_e = eta_e / star1_e is given per edge (host array, may be NULL), which covers the
 * reference's tanh window and any other profile.  Mixed precision: the operator and the
 * preconditioner inside the Arnoldi cycles in FP32; Krylov basis, Gram-Schmidt, Hessenberg,
 * least squares and the true residual of every restart (an FP64 iterative refinement) in FP64. */
typedef struct MhdInductionParams {
    int32_t hall;                  /* Config::hall (Hall term on) */
    int32_t max_it, restart;       /* Config::ind_max_it, ind_restart */
    int32_t precision;             /* MHD_PREC_FP64 or MHD_PREC_MIXED */
    double hall_coef, hall_r_min, hall_r_max, rtol; /* Scales::hall_coef, Config::hall_r_min/max, ind_rtol */
} MhdInductionParams;

int mhd_gpu_induction_create(MhdMesh *mesh, const MhdInductionParams *params, const double *m_edge_host, MhdInduction **out);
int mhd_gpu_induction_destroy(MhdInduction *ind);
/* ImplicitInduction::set_frozen_state (:105-111): B0 3 per cell, n_e,eff 1 per cell (device). */
int mhd_gpu_induction_set_frozen(MhdInduction *ind, const double *B0, const double *ne_eff);
/* The same frozen state with the Hall coefficient given per cell, alpha_c = taper_c hall_coef / n_e,eff,c
 * (ImplicitInduction::alpha_, :110), for a caller that keeps its own taper (device arrays). */
int mhd_gpu_induction_set_frozen_alpha(MhdInduction *ind, const double *B0, const double *alpha);
/* ImplicitInduction::apply_F (:127-183) and apply_A (:185-198) in FP64 (device arrays). */
int mhd_gpu_induction_apply_F(MhdInduction *ind, const double *phi, double *out);
int mhd_gpu_induction_apply_A(MhdInduction *ind, const double *x, double dt, double *y);
/* ImplicitInduction::solve (:299-390).  dirichlet[e] != 0 imposes E = E_expl (device int8 array);
 * warm = 0 drops the previous step's correction.  Returns MHD_ENOCONV (with E, iterations and
 * rel_res set) when max_it is reached above rtol, which the reference reports without throwing. */
int mhd_gpu_induction_solve(MhdInduction *ind, const double *Phi, const double *E_expl, const int8_t *dirichlet, double dt,
                            int32_t warm, double *E, int32_t *iterations, double *rel_res);
/* ImplicitInduction::solve with the per-edge pseudo-time step dt_edge (device, one per edge; the steady mode's
 * local time stepping, .h:48-50): the system (I + F d1 diag(dt_e)) E = E_expl + F(Phi^n), the Jacobi scaling
 * 1 / (1 + dt_e m_e d2_e), no ILU(0) (:317).  Otherwise as mhd_gpu_induction_solve. */
int mhd_gpu_induction_solve_dt_edge(MhdInduction *ind, const double *Phi, const double *E_expl, const int8_t *dirichlet,
                                    const double *dt_edge, int32_t warm, double *E, int32_t *iterations, double *rel_res);
/* Implicit ideal induction (Config::implicit_ideal, ImplicitInduction::set_ideal_state, :112-116): the part
 * of the ideal UCT EMF that is linear in the induced flux for frozen cell velocities u (3 per cell) joins
 * F on the edges with mask != 0 (:150-158), with UCT strength cuct (IdealParams::cuct).  u and mask are
 * copied (device arrays); u = NULL switches the part off.  While it is on, solves use the Jacobi
 * preconditioner (the reference builds no ILU(0) pattern then, :102) and the mixed-precision solve runs
 * its Arnoldi matvecs with the FP64 operator.  ideal_linear (:118-124): that part alone, L(phi) on
 * every owned edge (0 on the others). */
int mhd_gpu_induction_set_ideal(MhdInduction *ind, const double *u_cell, const int8_t *mask, double cuct);
int mhd_gpu_induction_ideal_linear(MhdInduction *ind, const double *phi, double *out);
/* Per-kernel-class device time of the solve (CUDA events on the mesh stream while enabled; classes:
 * face_d1, cell_field, hall_emf, edge_gather, gram_schmidt, krylov_scalar, krylov_vector, ilu, ideal_emf; a profiled solve
 * launches its kernels one by one instead of replaying the restart-cycle graph), read as
 * in mhd_gpu_state_profile_read; and the number of kernels the handle has launched. */
int mhd_gpu_induction_profile(MhdInduction *ind, int32_t enable);
int mhd_gpu_induction_profile_read(MhdInduction *ind, int32_t max_kernels, char *names, double *ms_total, int64_t *count,
                                   int32_t *n_out);
int mhd_gpu_induction_launches(MhdInduction *ind, int64_t *out);
/* Gram-Schmidt second passes (re-orthogonalisations) the last solve ran; no GPU work. */
int mhd_gpu_induction_last_solve_stats(MhdInduction *ind, int32_t *reorth_passes);

/* Block-Jacobi ILU(0) preconditioner of I + dt M d1^T S2 d1 on the owned edges (couplings to other ranks
 * and the Hall part dropped): Config::ind_ilu / ind_ilu_shift (Common/config/Config.h:38-39).  enable != 0
 * builds the pattern (ImplicitInduction::build_precond_pattern, .cpp:209-242, on the host from the mesh's
 * e2f / f2e rows, star2 and the handle's m_e) and makes every later solve factor it for its dt and
 * Dirichlet flags (factor_precond, :247-275) and precondition with it (apply_precond, :277-297) in place of
 * the Jacobi diagonal, as solve() does with use_ilu_ (:317-318, 337, 374).  The factorisation and the two
 * triangular solves run on the device with the reference's arithmetic per row (bit-identical factors
 * and results), one thread per row, rows taken in the order of their dependency levels; a wait on
 * another row gives up after 2 s (MHD_ECUDA, "ILU(0) pass timed out"), which no valid input reaches.
 * Rows longer than 64 entries are rejected (MHD_EINVAL).  Both precisions use the FP64 factors. */
int mhd_gpu_induction_set_ilu(MhdInduction *ind, int32_t enable, double shift);
/* factor_precond(dt, dir) alone (dirichlet: device int8 array, NULL: none); then apply_precond of a device
 * vector v into z (n_edges each; z = 0 on the non-owned edges).  The pattern must have been built. */
int mhd_gpu_induction_ilu_factor(MhdInduction *ind, double dt, const int8_t *dirichlet);
int mhd_gpu_induction_ilu_apply(MhdInduction *ind, const int8_t *dirichlet, const double *v, double *z);
/* Test hook of the bounded waits: the wait limit (0 < wait_s <= 2; 2 by default) and one row whose warp
 * never raises its flag (-1: none), so that the rows reading it give up and the call returns MHD_ECUDA
 * ("ILU(0) pass timed out") with the handle usable again. */
int mhd_gpu_induction_ilu_debug(MhdInduction *ind, double wait_s, int32_t unpublished_row);
/* Launch shape of the ILU(0) passes: about window_levels dependency levels of rows in flight (default 8),
 * spin_polls polls of unfinished rows without a pause (default 0), then pauses doubling from 32 ns to
 * max_backoff_ns (default 128). */
int mhd_gpu_induction_ilu_tune(MhdInduction *ind, int32_t window_levels, int32_t max_backoff_ns, int32_t spin_polls);
/* Host copies of the pattern and the current factors (pc_ptr_ n_owned+1, pc_col_ / pc_coef_ / pc_val_
 * nnz, pc_diag_ n_owned); any output may be NULL; *n_owned and *nnz receive the sizes. */
int mhd_gpu_induction_ilu_arrays(MhdInduction *ind, int32_t *n_owned, int64_t *nnz, int64_t *ptr, int32_t *col, double *coef,
                                 double *val, int64_t *diag);
/* build_precond_pattern on host arrays (no GPU work): rows of the n_owned first edges of the signed CSR
 * e2f (edge -> faces) and f2e (face -> edges) with star2 per face and m_e per edge.  Call with col and
 * coef NULL to get ptr (n_owned + 1 entries), then again with both sized ptr[n_owned]. */
int mhd_ilu_pattern(int32_t n_edges, int32_t n_owned, int32_t n_faces, const int64_t *e2f_ptr, const int32_t *e2f_idx,
                    const int8_t *e2f_sgn, const int64_t *f2e_ptr, const int32_t *f2e_idx, const int8_t *f2e_sgn,
                    const double *star2, const double *m_edge, int64_t *ptr, int32_t *col, double *coef);

/* ------------------------------------------------------------------ resident state, fused step
 * The explicit step of mercury::Solver::step (MercuryUns/driver/Solver.cpp:481-516) restricted to
 * the hot path (prepare :94-125 without the current, rhs :132-169 without model sources, advance
 * :194-206 with enforce_floors :171-191, the SSP-RK2 average :505-508), for n_species ion fluids.
 * The state stays on the device between steps, species-major:
 *   U[(s*5 + m)*n_cells + c]  (FP64 conservative variables), Phi[f] induced face flux (FP64). */
typedef struct MhdStepParams {
    int32_t n_species;                 /* 1 .. 16 */
    int32_t second_order;              /* Config::second_order */
    double gamma, rho_floor, p_floor;  /* Scales::gamma, Config::rho_floor / p_floor */
    double cuct;                       /* IdealParams::cuct */
    double M_ref, ne_floor;            /* Scales::M_ref / ne_floor (charge-weighted ion velocity) */
    double rel_limit;                  /* Config::recon_rel_limit */
    double cfl, inver_MA2, rho_floor_dt; /* CFL step of mercury::cell_time_steps (MercurySources.cpp:65-106) */
    double u_inf[3], B_imf[3];         /* free stream (inflow edge EMF) */
    double mass[16];                   /* molar mass per species (Scales::M_H, M_Na, ...) */
    MhdPrim fs[16];                    /* free-stream (inflow ghost) state per species */
    int8_t absorb[16];                 /* wall ghost absorbs the species (reference: species 1) */
    int32_t precision;                 /* MHD_PREC_FP64 or MHD_PREC_MIXED */
    /* Sources of the two-ion model (n_species == 2: species 0 = H+, 1 = Na+; Config::lorentz_force,
     * Scales::induce_coeff): with lorentz != 0 every stage adds the J x B force of
     * mercury::add_sources_n (MercurySources.cpp:20-63), and with induce_coeff > 0 the step is
     * wrapped in two half-step exact gyrations (mercury::gyrate, Strang splitting as in
     * mercury::Solver::step, Solver.cpp:492-510).  Zero-initialised parameters leave them off. */
    int32_t lorentz;
    double induce_coeff;
    /* The rest of add_sources_n (MercurySources.cpp:44-60) and the ambipolar EMF of Solver::rhs
     * (Solver.cpp:158): ambipolar != 0 adds the electron-pressure force -w_s grad p_e (grad p_e by
     * mercury::electron_pressure_gradient, Ambipolar.cpp:10-31) and -pressure_coef d0 p_e / n_e,eff to the
     * edge EMF (AmbipolarEMF::add, :52-88; needs the mesh's edge_nodes); chemistry != 0 adds the drag,
     * temperature relaxation, thermal drift and Na+ production of the source fields set by
     * mhd_gpu_state_set_source_fields.  The constants are those of mhd::Scales / Config::chem. */
    int32_t ambipolar, chemistry;
    double pressure_coef, a1_Na, a4, a5, a6, state_coeff_H, state_coeff_Na, T_ref, Tn0;
} MhdStepParams;

/* FP64 reference-exact: every operation rounds as in the reference's host code.
 * Mixed: reconstruction, limiters, Rusanov fluxes, CFL step and ideal EMF in FP32; the state U,
 * the face fluxes Phi, the CT update and div B in FP64 (tetrahedral meshes). */
#define MHD_PREC_FP64 0
#define MHD_PREC_MIXED 1

#define MHD_FIELD_U 0      /* conservative state of one species, 5 per cell */
#define MHD_FIELD_PHI 1    /* induced face flux */
#define MHD_FIELD_PHIADD 2 /* static background face flux; uploading it also sets the background cell field */
#define MHD_FIELD_BADD 3   /* background cell field (3 per cell), download only */

int mhd_gpu_state_create(MhdMesh *mesh, const MhdStepParams *params, MhdState **out);
int mhd_gpu_state_destroy(MhdState *state);
/* Host transfers in the reference layout (AoS); `species` selects the fluid for MHD_FIELD_U. */
int mhd_gpu_state_upload(MhdState *state, int32_t field, int32_t species, const double *host);
int mhd_gpu_state_download(MhdState *state, int32_t field, int32_t species, double *host);
/* Device pointer of a resident array (U: all species, species-major as above). */
int mhd_gpu_state_device_ptr(MhdState *state, int32_t field, double **out);
/* mercury::local_time_step (MercurySources.cpp:108-116) of the current state, min with dt_max. */
int mhd_gpu_cfl_dt(MhdState *state, double dt_max, double *host_dt);
/* One SSP-RK2 step.  dt_fixed > 0 is used as the step, otherwise the CFL step of the state
 * capped by dt_max is computed on the device.  dt_used (host, may be NULL) receives the step
 * and makes the call synchronous; with NULL the step is only enqueued (no host round trip). */
int mhd_gpu_step_rk2(MhdState *state, double dt_fixed, double dt_max, double *dt_used);
/* One semi-implicit step, mercury::Solver::step_first_order (MercuryUns/driver/Solver.cpp:228-277,
 * Config::time_order = 1): prepare and the CFL step (or dt_fixed), with the J x B force the opening half-step
 * gyration, the rhs and forward Euler of the fluid with floors, then the edge EMF from
 * ImplicitInduction::solve on `ind` (made on the same mesh: its resistivity, Hall coefficient and GMRES
 * settings) with the step's total cell field and n_e,eff of the fluid cells frozen, the inflow edges
 * Dirichlet, the rhs's explicit EMF (ideal, ambipolar, boundary values) as E_expl and the warm start of
 * the previous step, faraday_update with that EMF, and the closing half-step gyration.  FP64 two-ion state.
 * Synchronous; dt_used, iterations and rel_res (host, may be NULL) receive the step and the solve's
 * figures; MHD_ENOCONV when the solve stopped at max_it above rtol (the step is still taken, as the
 * reference takes it). */
int mhd_gpu_step_semi_implicit(MhdState *state, MhdInduction *ind, double dt_fixed, double dt_max, double *dt_used,
                               int32_t *iterations, double *rel_res);

/* mercury::add_sources (MercuryUns/fluid/MercurySources.cpp:13-63) for species 0 or 1 of the two-ion
 * model (params: n_species 2, mass[0..1], M_ref, ne_floor, inver_MA2, lorentz, ambipolar, chemistry and
 * their constants): rhs += the source on the owned fluid cells.  WH, WNa: primitives (5 per cell); B total
 * field, J current (3 per cell); the SourceFields dpe (grad p_e, 3 per cell), photo and vst (1 per cell)
 * may be NULL, as in the reference; FP64 in the reference's operation order. */
int mhd_gpu_add_sources(MhdMesh *mesh, const MhdStepParams *params, int32_t species, const double *WH, const double *WNa,
                        const double *B, const double *J, const double *dpe, const double *photo, const double *vst, double dt,
                        double *rhs);
/* mercury::electron_pressure_gradient (MercuryUns/physics/Ambipolar.cpp:10-31): grad p_e of the owned
 * fluid cells by Gauss' theorem with face-averaged p_e = p_H + p_Na (3 per cell, zero elsewhere). */
int mhd_gpu_electron_pressure_gradient(MhdMesh *mesh, const double *WH, const double *WNa, double *dpe);
/* mercury::AmbipolarEMF::add (Ambipolar.cpp:52-88): E -= pressure_coef (p_b - p_a) / n_e,eff on the owned
 * edges touching fluid cells (nodal p_e volume-averaged over the node's fluid cells, n_e,eff from the
 * edge-averaged densities); needs the mesh's edge_nodes. */
int mhd_gpu_ambipolar_emf(MhdMesh *mesh, const MhdStepParams *params, const double *WH, const double *WNa, double *E);
/* The external source fields of the chemistry terms (mercury::SourceFields photo and vst, host arrays of
 * one value per cell; NULL clears a field, which then contributes nothing, as in the reference). */
/* ---------------------------------------------------------------- the ten-ion (Mars) source pieces
 * mars::MarsSolver (MarsUns/driver/MarsSolver.cpp) as device passes.  Ion arrays are species-major with 5
 * values per cell: U[(s * n_cells + c) * 5 + m] (W likewise, primitives); cell vectors 3 per cell.  The
 * scales are those of MarsParams::from_params (:40-110). */
typedef struct MhdMarsParams {
    int32_t n_species;        /* MARS::NumSpecies (ten ions) */
    int32_t n_neutral;        /* reactive neutrals of the drag (MARS::NumReactiveNeutral): neutral n has mass[n] */
    int32_t neutral_stride;   /* values per cell of the neutral array (MARS::NumNeutral) */
    int32_t ambipolar;        /* is_Ambipolar_Efield */
    double mass[16];          /* MARS::ParticleMass [kg] */
    double rho_ref, n_ref, p_ref, time_ref, kB, L, U, q, B;
    double mag_scale, pressure_scale, ne_floor, rho_floor, p_floor, gamma;
} MhdMarsParams;

/* MarsSolver::prepare (:287-303): n_e, n_e,eff = sqrt(n_e^2 + ne_floor^2), p_e = sum_s p_s per cell and u+
 * (3 per cell, zero outside fluid cells) from U and W. */
int mhd_gpu_mars_plasma(MhdMesh *mesh, const MhdMarsParams *params, const double *U, const double *W, double *ne, double *ne_eff,
                        double *pe, double *uplus);
/* grad p by Gauss' theorem with the face-averaged p (MarsSolver.cpp:305-325; Ambipolar.cpp:10-31): 3 per cell,
 * zero outside the owned non-solid cells. */
int mhd_gpu_pressure_gradient(MhdMesh *mesh, const double *pe, double *dpe);
/* The explicit sources of fluid_and_sources_ (:400-418): per ion rhs += (w mag_scale J x B - w grad p_e,
 * (the same) . u) with w = n_s / n_e,eff; rhs is added to. */
int mhd_gpu_mars_explicit_sources(MhdMesh *mesh, const MhdMarsParams *params, const double *U, const double *W, const double *Btot,
                                  const double *J, const double *dpe, const double *ne_eff, double *rhs);
/* MarsSolver::ambipolar_emf_ (:529-562): E -= pressure_scale (p_b - p_a) / n_e,eff of the edge, on the owned
 * edges (nodal p_e volume-weighted over the node's fluid cells); needs the mesh's edge_nodes. */
int mhd_gpu_mars_ambipolar_emf(MhdMesh *mesh, const MhdMarsParams *params, const double *pe, const double *ne, double *E);
/* MarsSolver::local_dt_ (:330-376) with its global minimum: each ion alone and the plasma's fast mode. */
int mhd_gpu_mars_time_step(MhdMesh *mesh, const MhdMarsParams *params, double cfl, const double *U, const double *W, const double *Btot,
                           const double *uplus, double *host_dt);
/* MarsSolver::implicit_sources_ (:420-520) on U in place: Crank-Nicolson gyration of the coupled ions,
 * ion-neutral drag and thermal relaxation (backward Euler); neutral: neutral_stride densities per cell [cm^-3]. */
int mhd_gpu_mars_implicit_sources(MhdMesh *mesh, const MhdMarsParams *params, const double *Btot, const double *neutral, double dt,
                                  double *U);
/* The forward-Euler update of MarsSolver::step (:719-726): U += dt rhs on the owned non-solid cells. */
int mhd_gpu_mars_advance(MhdMesh *mesh, int32_t n_species, const double *rhs, double dt, double *U);
/* MarsSolver::floors_ (:686-702). */
int mhd_gpu_mars_floors(MhdMesh *mesh, const MhdMarsParams *params, double *U);

/* The step's Dirichlet wall table (the ten-ion solver's wall_state_, MarsSolver.cpp:147-165, cached per
 * face): host arrays faces[n_wall] (distinct faces of kind wall) and prims[n_species][n_wall][5]; the
 * FP64 and mixed steps use it in the gradients and the face fluxes.  n_wall = 0 removes it.  The
 * differentiated run (mhd_gpu_fn_*) does not take a state with a wall table. */
int mhd_gpu_state_set_wall_ghosts(MhdState *state, int32_t n_wall, const int32_t *faces, const double *prims);

int mhd_gpu_state_set_source_fields(MhdState *state, const double *photo, const double *vst);
/* mercury::gyrate (MercuryUns/physics/Gyration.cpp): exact rotation of the ions' relative velocity
 * about B over dt on the owned fluid cells, UH and UNa (5 per cell) in place; a no-op unless
 * lorentz != 0 and induce_coeff > 0, as in the reference. */
int mhd_gpu_gyrate(MhdMesh *mesh, const MhdStepParams *params, const double *B, double dt, double *UH, double *UNa);

/* Explicit resistive EMF of the FP64 step: with m_edge (host, one value per edge: m_e = eta_e / star1_e)
 * every stage adds m_e (d1^T star2 Phi)_e to the EMF of the owned edges after the ideal UCT EMF and the
 * boundary edge values.  The term is the resistive part of ImplicitInduction::apply_F
 * (Common/induction/ImplicitInduction.cpp:133-137, 182) evaluated explicitly; NULL switches it off. */
int mhd_gpu_state_set_resistivity(MhdState *state, const double *m_edge);

/* ------------------------------------------------------------------ differentiated explicit run
 * Forward / backward (adjoint) / tangent Function of n_steps FP64 SSP-RK2 steps at a fixed dt (the
 * state's parameters, no model sources, one or two species, tetrahedral mesh) with the explicit
 * resistive EMF of the per-cell resistivity eta (m_e = mean of eta over the edge's cells / star1_e),
 * for the functional J = sum over the marked cells of |B_tot|^2 V of the final state.  Parameters:
 * eta (per cell) and the inflow velocity u_inf (every species' free-stream velocity and the inflow
 * edge EMF -u_inf x B_imf); the face kinds and edge modes stay as built.  The run starts from the
 * state's U and Phi at creation.  The reference has no adjoint: this interface is this library's own. */
typedef struct MhdFnParams {
    int32_t n_steps;          /* explicit steps of the run */
    int32_t checkpoint_every; /* the forward run keeps the state every this many steps; the backward
                                 sweep recomputes each segment from its checkpoint */
    double dt;                /* fixed step */
    int32_t uniform_flow;     /* 1: the initial flow moves with the free stream: every species' velocity in
                                 every fluid cell is shifted by u_inf - (u_inf at creation), density and
                                 pressure kept, so J depends on u_inf through the initial state too */
    int32_t pad;
} MhdFnParams;
typedef struct MhdFn MhdFn;

/* eta: per-cell resistivity (host, n_cells); mask: cells of the functional (host int8, n_cells) */
int mhd_gpu_fn_create(MhdState *state, const MhdFnParams *params, const double *eta, const int8_t *mask, MhdFn **out);
int mhd_gpu_fn_destroy(MhdFn *fn);
/* new parameters (either may be NULL: unchanged); sets the state's free-stream velocities and u_inf */
int mhd_gpu_fn_set_params(MhdFn *fn, const double *eta, const double *u_inf);
/* copy the initial state back into the MhdState */
int mhd_gpu_fn_reset(MhdFn *fn);
/* J of the run; keeps the checkpoints and leaves the final state in the MhdState */
int mhd_gpu_fn_forward(MhdFn *fn, double *J);
/* The last J (of a forward or tangent run) as the double-double J_hi_lo[0] + J_hi_lo[1]: J is summed in
 * double-double, so the difference of two runs' J is kept below J's own ulp (finite differences at small
 * steps: (Jp_hi - Jm_hi) + (Jp_lo - Jm_lo)). */
int mhd_gpu_fn_last_J(MhdFn *fn, double *J_hi_lo);
/* dJ/deta (host, n_cells; may be NULL) and dJ/du_inf (3; may be NULL) by the adjoint sweep; needs a
 * forward run with the current parameters */
int mhd_gpu_fn_backward(MhdFn *fn, double *grad_eta, double *grad_u);
/* tangent-linear run: J and its derivative along (d_eta, d_u) (either may be NULL: zero) */
int mhd_gpu_fn_tangent(MhdFn *fn, const double *d_eta, const double *d_u, double *J, double *dJ);
/* One stage as an operator, for dot-product checks.  Host arrays in the state's device layout
 * (U: [(s*5 + m)*n_cells + c], Phi per face, E per edge).  The stage maps (U, Phi; eta, u_inf) to
 * U~ = floors(U + dt rhs) and the edge EMF E.  _tangent: the derivatives of U~ and E along
 * (dU, dPhi, d_eta, d_u).  _adjoint: given adjoints of U~ and E, the adjoints of U, Phi, eta (n_cells)
 * and u_inf (3). */
int mhd_gpu_fn_stage_tangent(MhdFn *fn, const double *U, const double *Phi, const double *dU, const double *dPhi, const double *d_eta,
                             const double *d_u, double *dUt, double *dE);
int mhd_gpu_fn_stage_adjoint(MhdFn *fn, const double *U, const double *Phi, const double *lUt, const double *lE, double *lU, double *lPhi,
                             double *l_eta, double *l_u);
/* Per-class device time of the Function's runs (CUDA events on the mesh stream while enabled; classes:
 * forward_steps, record_steps, adj_floors, adj_edge_emf, adj_face_candidate, adj_cell, adj_face_flux,
 * adj_limited_gradients, adj_prim, adj_misc, tangent_steps), read as in mhd_gpu_state_profile_read. */
int mhd_gpu_fn_profile(MhdFn *fn, int32_t enable);
int mhd_gpu_fn_profile_read(MhdFn *fn, int32_t max_kernels, char *names, double *ms_total, int64_t *count, int32_t *n_out);
/* Switch log of the forward run.  While enabled, every mhd_gpu_fn_forward clears and then fills, per
 * entity, a running 32-bit hash of the discrete choices that the forward kernels make over all steps and
 * stages, so that two runs (J at p + h d and at p - h d) can be compared entity by entity: an entry that
 * differs is an entity where the run crossed a switch, where J is not differentiable along d.  Kinds:
 *   0 limiter [(s*5 + q)*n_cells + c]: which term sets Barth-Jespersen psi (none, upper, lower, relative
 *     bound, clamp at 0) with the neighbour and face slots of the extremes it uses;
 *   1 flux [s*n_faces + f]: the side of the larger Rusanov wave speed, the sign of that side's normal
 *     velocity (not recorded where the two face states are the same state, as on zero-gradient faces,
 *     where the wave speed multiplies zero), and the face states' positivity fallbacks;
 *   2 edge [n_edges]: per face of the edge the cell with the largest |u . m| and its sign, and whether the
 *     2x2 upwind solve ran;
 *   3 floor [s*n_cells + c]: the floor that the update applied (none, density, pressure);
 *   4 face EMF [n_faces]: the face candidate's a_f, the side of the larger |u . n| and its sign.
 * Disabling frees the tables.  _read copies one kind's table (n: its size) to the host. */
int mhd_gpu_fn_switch_log(MhdFn *fn, int32_t enable);
int mhd_gpu_fn_switch_read(MhdFn *fn, int32_t kind, uint32_t *out, int64_t n);

/* Live per-kernel timing of the fused step (CUDA events recorded on the handle's stream around
 * every launch while enabled).  _read synchronises, returns per kernel class its name (32 chars
 * each), summed milliseconds and launch count, and restarts the accumulation. */
int mhd_gpu_state_profile(MhdState *state, int32_t enable);
int mhd_gpu_state_profile_read(MhdState *state, int32_t max_kernels, char *names, double *ms_total, int64_t *count,
                               int32_t *n_out);
/* Number of kernels the fused step has launched since the state was created. */
int mhd_gpu_state_launches(MhdState *state, int64_t *out);

#ifdef __cplusplus
}
#endif
#endif
