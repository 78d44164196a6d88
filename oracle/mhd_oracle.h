/* CPU restatement of the reference's hot path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: the parity tests compare the device library against these
 * functions (and bench.py's CPU-baseline leg may time them); the shipped library never
 * links them.  Each function names the reference function it restates (file:line in the
 * MPCNS_Uns tree).  Pinned against the reference itself: tests/test_oracle.py runs both on
 * the same inputs and checks the golden vectors of tests/golden/ (generated from the
 * compiled reference by tests/golden/make_golden.py).
 *
 * Arrays use the reference layouts (signed CSR; AoS value(i, comp) = a[i*ncomp + comp]). */
#ifndef MHD_ORACLE_H
#define MHD_ORACLE_H
#include <stdint.h>

typedef struct OrMesh {
    int32_t n_nodes, n_edges, n_faces, n_cells, n_owned_cells, n_owned_edges;
    const int64_t *c2f_ptr; const int32_t *c2f_idx; const int8_t *c2f_sgn;
    const int64_t *f2e_ptr; const int32_t *f2e_idx; const int8_t *f2e_sgn;
    const int64_t *e2f_ptr; const int32_t *e2f_idx; const int8_t *e2f_sgn;
    const int64_t *f2c_ptr; const int32_t *f2c_idx; const int8_t *f2c_sgn;
    const int32_t *cell_material;
    const double *edge_vec, *edge_mid, *edge_len, *face_area, *face_center, *face_area_mag, *cell_center, *cell_volume;
    const int64_t *ec_ptr; const int32_t *ec_cell; const double *ec_weight, *ef_weight, *star1, *star2;
    const int8_t *face_kind, *edge_mode;
    const int32_t *edge_nodes; /* start and end node per edge (uns::CellComplex::edge_nodes), for the ambipolar EMF */
} OrMesh;

typedef struct OrPrim { double rho, u, v, w, p; } OrPrim;

void or_to_prim(const double *U, int64_t n, double gamma, double rho_floor, double p_floor, double *W);
/* absorb: wall ghost of this species absorbs (reference: species == 1) */
void or_limited_gradients(const OrMesh *m, const double *W, int32_t absorb, const OrPrim *fs, int32_t limit, double rel_limit,
                          double *grad);
void or_flux_rhs(const OrMesh *m, double gamma, int32_t absorb, const OrPrim *fs, const double *W, const double *grad, double *rhs);
void or_cell_vector(const OrMesh *m, const double *flux, int32_t ncells, double *out);
void or_ideal_emf(const OrMesh *m, const double *u, const double *Bt, const double *Bi, const double *phi_tot, const double *phi_ind,
                  double cuct, double *E);
void or_edge_modes(const OrMesh *m, const double *u_inf, const double *B_imf, double *E);
void or_faraday(const OrMesh *m, const double *E, const double *dt_edge, double dt, double *B);
void or_div_b(const OrMesh *m, const double *B, const double *extra, double *out3);
void or_cell_current(const OrMesh *m, const double *B, double *J);
/* CFL step of mercury::cell_time_steps / local_time_step for n_species ion fluids (W: array of pointers) */
double or_local_time_step(const OrMesh *m, int32_t n_species, const double *const *W, const double *B, double gamma, double cfl,
                          double inver_MA2, double rho_floor_dt);

/* one SSP-RK2 step of the hot path (reference Solver::step without model sources) */
typedef struct OrStepParams {
    int32_t n_species, second_order;
    double gamma, rho_floor, p_floor, cuct, M_ref, ne_floor, rel_limit;
    double u_inf[3], B_imf[3];
    double mass[16];
    OrPrim fs[16];
    int8_t absorb[16];
    /* two-ion model sources: J x B force and the Strang-split exact gyration (needs n_species == 2) */
    int32_t lorentz;
    double induce_coeff, inver_MA2;
    /* explicit resistive EMF: E_e += m_res[e] (d1^T star2 Phi)_e on the owned edges, the resistive part of
     * ImplicitInduction::apply_F (Common/induction/ImplicitInduction.cpp:133-137, 182) with m_e = eta_e / star1_e
     * (NULL: off) */
    const double *m_res;
    /* the rest of add_sources_n and the ambipolar EMF: switches, Scales constants, the chemistry's source fields */
    int32_t ambipolar, chemistry;
    double pressure_coef, a1_Na, a4, a5, a6, state_coeff_H, state_coeff_Na, T_ref, Tn0;
    const double *photo, *vst;
} OrStepParams;
/* mercury::add_sources (MercuryUns/fluid/MercurySources.cpp:13-63), species s: rhs += S; dpe, photo, vst: the
 * SourceFields (NULL: absent) */
void or_add_sources(const OrMesh *m, const OrStepParams *p, int32_t s, const double *WH, const double *WNa, const double *B,
                    const double *J, const double *dpe, const double *photo, const double *vst, double dt, double *rhs);
/* mercury::electron_pressure_gradient (MercuryUns/physics/Ambipolar.cpp:10-31) */
void or_electron_pressure_gradient(const OrMesh *m, const double *WH, const double *WNa, double *dpe);
/* mercury::AmbipolarEMF (Ambipolar.cpp:35-88): node lists and E -= pressure_coef d0 p_e / n_e,eff, E in place */
void or_ambipolar_emf(const OrMesh *m, const OrStepParams *p, const double *WH, const double *WNa, double *E);
/* mercury::gyrate (MercuryUns/physics/Gyration.cpp): exact rotation of the relative ion velocity about B */
void or_gyrate(const OrMesh *m, const OrStepParams *p, const double *B, double dt, double *UH, double *UNa);
/* explicit resistive EMF (see OrStepParams.m_res): E_e += m_e (d1^T star2 phi)_e on the owned edges */
void or_resistive_emf(const OrMesh *m, const double *m_res, const double *phi, double *E);
int or_rk2_step(const OrMesh *m, const OrStepParams *p, double *const *U, double *Phi, const double *PhiAdd, const double *BaddCell,
                double dt);

/* semi-implicit induction (Common/induction/ImplicitInduction.cpp) */
typedef struct OrInduction OrInduction;
typedef struct OrIndParams {
    int32_t hall, max_it, restart;
    double hall_coef, hall_r_min, hall_r_max, rtol;
} OrIndParams;
/* m_edge: per-edge resistive coefficient eta_e / star1_e (NULL or all zero: no resistivity) */
OrInduction *or_ind_create(const OrMesh *m, const OrIndParams *p, const double *m_edge);
void or_ind_free(OrInduction *s);
void or_ind_set_frozen(OrInduction *s, const double *B0, const double *ne);
void or_ind_apply_F(OrInduction *s, const double *phi, double *out);
void or_ind_apply_A(OrInduction *s, const double *x, double dt, double *y);
int32_t or_ind_solve(OrInduction *s, const double *Phi, const double *E_expl, const int8_t *dir, double dt, int32_t warm, double *E,
                     double *rel_res);
/* solve with the per-edge pseudo-time step dte (:299-390 with dte_): A x = x + F(d1 diag(dte) x), Jacobi
 * 1 / (1 + dte m d2), no ILU(0) */
int32_t or_ind_solve_dte(OrInduction *s, const double *Phi, const double *E_expl, const int8_t *dir, const double *dte, int32_t warm,
                         double *E, double *rel_res);
/* the implicit ideal part (Config::implicit_ideal, set_ideal_state :112-116; u NULL: off) and ideal_linear (:118-124) */
void or_ind_set_ideal(OrInduction *s, const double *u_cell, const int8_t *mask, double cuct);
void or_ind_ideal_linear(OrInduction *s, const double *phi, double *out);
/* one semi-implicit step, mercury::Solver::step_first_order (MercuryUns/driver/Solver.cpp:228-277): forward Euler of
 * the fluid (with the opening and closing half-step gyration when lorentz is on), the EMF from ind's solve (frozen
 * total field and n_e,eff of the step, inflow edges Dirichlet, the rhs's EMF as E_expl, warm start) and CT with it;
 * two ions; -1 on bad arguments */
int or_first_order_step(const OrMesh *m, const OrStepParams *p, OrInduction *ind, double *const *U, double *Phi, const double *PhiAdd,
                        const double *BaddCell, double dt, int32_t *iterations, double *rel_res);
/* block-Jacobi ILU(0) (ImplicitInduction.cpp:209-297): enable builds the pattern of the owned rows and makes
 * or_ind_solve factor and apply it in place of the Jacobi scaling.  Ties of the column sort keep the
 * gathering order (the reference's std::sort leaves them in an order of its own), so the diagonal
 * coefficients agree with the reference's to rounding and everything else bit for bit. */
void or_ind_set_ilu(OrInduction *s, int32_t enable, double shift);
/* the pattern (ptr n_owned + 1, col / coef nnz; NULL: skipped); returns nnz, -1 without a pattern */
int64_t or_ind_ilu_pattern(OrInduction *s, int64_t *ptr, int32_t *col, double *coef);
/* factor_precond(dt, dir) then apply_precond(v) -> z (n_edges each; dir may be NULL) */
void or_ind_ilu_precond(OrInduction *s, double dt, const int8_t *dir, const double *v, double *z);
#endif
