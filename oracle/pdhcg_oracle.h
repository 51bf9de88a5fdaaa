/*
 * pdhcg_oracle.h -- CPU restatement of the reference PDHCG iteration.
 *
 * TEST INFRASTRUCTURE ONLY.  This single-threaded FP64 C code is the checker
 * for the CUDA solver in pdhcg_b200/: only tests/, __graft_entry__.smoke()
 * and the cpu_baseline / reference arms of bench.py may load it.  The
 * product never links or calls it.
 *
 * Parity is pinned two ways (see tests/test_oracle_*.py):
 *   - host logic (rescaling, Q-type detection) is compared bit-for-bit with
 *     the reference's own rescale_problem, compiled from its sources into
 *     oracle/_ref/ by oracle/ref.mk and called on the CPU;
 *   - whole solves reproduce the known answers of the reference's
 *     end-to-end tests (test/test_c_api_working.c, test/test_sparse_q_cones.c,
 *     test/test_diag_q_cones.c, test/test_initial_box_projection.c).
 *
 * Every function names the reference lines it restates.
 */
#pragma once

#include "../include/pdhcg_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Full solve: restates optimize() (reference src/solver.cu:35-210). */
pdhcg_result_t *oracle_solve(const qp_problem_t *prob, const pdhg_parameters_t *params);
void oracle_result_free(pdhcg_result_t *result);

/* Rescaling only: restates rescale_problem (reference src/preconditioner.c:654-713).
 * Outputs have num_constraints / num_variables entries.  Returns 0. */
int oracle_rescale(const qp_problem_t *prob,
                   const pdhg_parameters_t *params,
                   double *con_rescale,
                   double *var_rescale,
                   double *con_bound_rescale,
                   double *obj_vec_rescale);

/* Largest singular value of a CSR matrix by the reference's power method on
 * A A^T (reference src/pdhg_core_op.cu:1673-1788), start vector rand_r(1234). */
double oracle_sigma_max(int m, int n, const int *row_ptr, const int *col_ind, const double *val,
                        int max_iter, double tol);

/* Projection of one cone block of x (scaled space) onto {x : x_i / d_i in K}
 * in the metric sum_i w_i (x_i - r_i)^2 with w_i = 1 + tau*q_i (q may be NULL
 * for w = 1).  type = cone_type_t, block holds cone_length(type, v_dim)
 * slots.  Restates the projection kernels of reference
 * src/kernels/pdhcg_soc_cone_kernels.cu:267-460, 1442-2062 and
 * src/kernels/pdhcg_rsoc_cone_kernels.cu:466-680, 2096-2631. */
void oracle_project_cone_block(int type, int v_dim, double power_alpha, double *x, const double *d,
                               const double *q, double tau);

/* Dual residual of one self-dual block (reference compute_cone_dual_residual
 * kernels, e.g. src/kernels/pdhcg_soc_cone_kernels.cu:470-720):
 * out_i = (rc_i - P_{D^-1 K}(rc)_i) * d_i. */
void oracle_cone_dual_residual_block(int type, int v_dim, double power_alpha, const double *rc,
                                     const double *d, double *out);

/* Blocks with slots fixed by set_cone_fixed (oracle_sections.c): the
 * weighted projection onto the section through the fixed values (x, d,
 * q, fx at the block's first slot; warm: the block's multiplier from the
 * previous call, updated), and the section dual residual (reference
 * src/kernels/pdhcg_*_cone_kernels.cu, fixed-section branches); the latter
 * returns the block's complementarity residual. */
int oracle_block_has_fixed(const char *fx, int len);
void oracle_section_project(int type, int v_dim, double alpha, double *x, const double *d, const double *q,
                            double tau, const char *fx, double *warm);
double oracle_section_dual_residual(int type, int v_dim, double alpha, const double *xp, const double *rc,
                                    const double *d, const char *fx, double *warm, double *out);

/* One PDHG iteration from a given state, for kernel-level parity tests.
 * Inputs are already-scaled data; see oracle_step_t. */
typedef struct {
    int n, m;
    const int *A_row_ptr, *A_col_ind; const double *A_val;     /* m x n */
    const int *At_row_ptr, *At_col_ind; const double *At_val;  /* n x m */
    const double *c, *var_lb, *var_ub, *q_diag;                /* q_diag may be NULL (LP) */
    const double *con_lb, *con_ub, *affine_offset;
    const double *var_rescale;                                 /* for cone projections */
    int num_cones; const int *cone_start, *cone_vdim, *cone_type; const double *cone_alpha;
    double tau, sigma, halpern_weight, reflection;
    /* in/out */
    double *x_init, *x_cur, *y_init, *y_cur;
    /* out */
    double *x_pdhg, *x_refl, *y_pdhg, *y_refl, *Aty, *Ax;
} oracle_step_t;

/* pdhg_update (LP / diagonal-Q, no inner solver) + halpern_update
 * (reference src/pdhg_core_op.cu:705-845). */
void oracle_pdhg_step(oracle_step_t *s);

#ifdef __cplusplus
}
#endif
