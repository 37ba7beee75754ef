/*
 * pdf_oracle.h — C API of the FP64 CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle restates, on the CPU in FP64, the
 * reference's projective-dynamics step loop with dry frictional contact.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, and
 * only as the checker.  The product (climatenet_b200/) never links or calls it.
 *
 * Parity is pinned against the reference's analytic incline known-answer test
 * (replicability/analytic_example_data_processing.py:150-251 on
 * scenes/analytic.json) and against hand-computed cases; the reference itself
 * cannot be built in this environment (Eigen, CGAL and Boost are absent).
 */
#ifndef PDF_ORACLE_H
#define PDF_ORACLE_H
#include "../include/pdf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

int orc_create(const pdf_scene_desc* scene, const pdf_params* params, orc_sim** out);
int orc_step(orc_sim* s, int32_t nsteps, pdf_step_report* report);
int orc_get_state(orc_sim* s, double* q, double* v);
int orc_set_state(orc_sim* s, const double* q, const double* v);
int orc_get_contacts(orc_sim* s, pdf_contact* out, int32_t cap, int32_t* n);
int orc_get_self_contacts(orc_sim* s, pdf_contact* out, int32_t cap, int32_t* n);
int orc_get_self_levels(orc_sim* s, int32_t* level_ptr, int32_t level_cap,
                        int32_t* order, int32_t order_cap, int32_t* n_levels);
int orc_get_residual_history(orc_sim* s, double* out, int32_t cap, int32_t* n);
/* Alart-Curnier trace (SFE:720-752, PRINT_ALART_CURNIER_ERROR): when enabled,
 * every PD iteration of the next steps records (tangential, |normal|) per
 * contact, obstacle contacts first; the trace holds the last step only and is
 * laid out like pdf_get_alart_curnier_trace's. */
int orc_trace_alart_curnier(orc_sim* s, int32_t enable);
/* Per iteration of the last step: mean AC norm evaluated with the force each
 * contact applied in that iteration (zero after a take-off), where the
 * reference's norm uses the stale local force it keeps for such a contact. */
int orc_get_residual_applied_history(orc_sim* s, double* out, int32_t cap, int32_t* n);
int orc_get_alart_curnier_trace(orc_sim* s, double* out, int64_t cap, int32_t* iterations,
                                int32_t* n_contacts, int32_t* n_self);
/* Learned warm start, restated from the product (climatenet_b200/csrc/mlp.cu):
 * weights (5,059 floats), the per-contact sample log, and the MLP forward with
 * the tensor cores' bfloat16 rounding emulated. */
int orc_mlp_set_weights(orc_sim* s, const float* w, int32_t count);
int orc_mlp_log(orc_sim* s, int32_t capacity);
int orc_mlp_samples(orc_sim* s, float* X, float* T, int32_t cap, int32_t* n);
int orc_mlp_forward(const float* w, const float* X, int32_t n, float* Y);
/* rows(A), nnz(A), nnz(LHS) (full symmetric), nnz(L) */
int orc_get_sizes(orc_sim* s, int64_t* sizes4);
/* Projections p (rows x 3) for positions q (3N). */
int orc_projections(orc_sim* s, const double* q, double* p);
/* Base RHS (SimulationSpeed::computeRhs) for q_n, t_n, v^k, q^k given: 3N out. */
int orc_rhs_base(orc_sim* s, const double* qn, const double* tn,
                 const double* vk, double* rhs);
/* The final RHS (with friction) of the last iteration of the last step, 3N. */
int orc_last_rhs(orc_sim* s, double* rhs);
/* Solve LHS x = b for 3 right-hand sides stored vertex-major (3N in/out). */
int orc_solve(orc_sim* s, double* x);
/* LHS in CSR (full symmetric): row_ptr[N+1], col[nnz], val[nnz]; pass NULLs to
 * query nnz through *nnz. */
int orc_lhs_csr(orc_sim* s, int32_t* row_ptr, int32_t* col, double* val, int64_t* nnz);
/* Per-vertex lumped masses (N). */
int orc_masses(orc_sim* s, double* m);
double orc_time(orc_sim* s);
const char* orc_last_error(void);
void orc_destroy(orc_sim* s);

/* Stand-alone detection (one mesh; triangle indices are mesh-local). */
int orc_self_candidates(const double* pos, int32_t n_vertices, const int32_t* tris,
                        int32_t n_triangles, double tolerance, int32_t* pairs,
                        int32_t cap, int32_t* n);
int orc_self_collisions(const double* pos, int32_t n_vertices, const int32_t* tris,
                        int32_t n_triangles, double tolerance, pdf_contact* out,
                        int32_t cap, int32_t* n);
/* Ericson closest point with the reference's early exit; bary[3], cp[3]. */
void orc_closest_point(const double* p, const double* a, const double* b,
                       const double* c, double tol2, double* cp, double* bary);

#ifdef __cplusplus
}
#endif
#endif
