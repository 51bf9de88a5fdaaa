/*
 * pdhcg.h -- the PDHCG C interface, served by libpdhcg_b200.so.
 *
 * Every entry point below replaces the function of the same name in the
 * reference solver's public header (reference include/pdhcg.h:31-66) with
 * the same argument meaning, ownership rules and error behaviour:
 *   - builders deep-copy their inputs and return NULL (with a message on
 *     stderr) on invalid input;
 *   - solve_qp_problem returns NULL on invalid input or on a device error,
 *     where the reference would have called exit();
 *   - all returned objects are host memory freed with the *_free calls.
 * The solve runs on the calling thread's current CUDA device.
 */
#pragma once

#include "pdhcg_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Build a problem  min 1/2 x'(Q + R'DR)x + c'x + const  subject to
 * con_lb <= A x <= con_ub, F x + g in K_affine, var_lb <= x <= var_ub,
 * x_J in K_var.  Any matrix descriptor may be NULL (Q = 0, R = 0, D = I).
 * Replaces reference create_qp_problem (include/pdhcg.h:31-46,
 * src/pdhcg.c:365-508). */
qp_problem_t *create_qp_problem(const double *objective_c,
                                const matrix_desc_t *Q_desc,
                                const matrix_desc_t *R_desc,
                                const matrix_desc_t *D_desc,
                                const matrix_desc_t *A_desc,
                                const double *con_lb,
                                const double *con_ub,
                                const double *var_lb,
                                const double *var_ub,
                                const double *objective_constant,
                                int num_var_cones,
                                const cone_spec_t *var_cones,
                                const matrix_desc_t *affine_cone_matrix_desc,
                                const double *affine_cone_offset,
                                int num_affine_cones,
                                const cone_spec_t *affine_cones);

/* Warm start; dual has rows(A) + rows(F) entries.  NULL clears.
 * Replaces reference set_start_values (include/pdhcg.h:49, src/pdhcg.c:569-618). */
void set_start_values(qp_problem_t *prob, const double *primal, const double *dual);

/* Pin one slot of a variable cone (SOC, rotated SOC, exponential or power;
 * not PSD) to a finite value; returns 0 or -1.  The value also becomes that
 * slot's primal start.  solve_qp_problem keeps the slot at the value and
 * projects the block's free slots onto the cone's section through the
 * fixed values; it returns NULL (with a message) when a section is empty.
 * Replaces reference set_cone_fixed (include/pdhcg.h:51, src/pdhcg.c:620-666). */
int set_cone_fixed(qp_problem_t *prob, int cone_idx, int slot, double value);

/* QCQP -> SOCP rewrite: each quadratic constraint (diagonal Q_i, one-sided
 * row) becomes a cone block of type default_type (standard or rotated SOC)
 * with its auxiliary variables and rows; the same layout as the reference's.
 * NULL without quadratic constraints, or with a non-diagonal / mixed-sign
 * Q_i or a two-sided row.  solve_qp_problem applies it by itself.
 * Replaces reference qcqp_to_socp_qp (include/pdhcg.h:53, src/qcqp_transform.c:96). */
qp_problem_t *qcqp_to_socp_qp(const qp_problem_t *orig_qcqp, cone_type_t default_type);

/* Solve on the current CUDA device; params == NULL means defaults.
 * A NaN anywhere in c, the bounds or the matrix values, or an infinite
 * entry of c or of a matrix, gives NULL with a message instead of a run
 * that would iterate on NaN until a limit.
 * Replaces reference solve_qp_problem (include/pdhcg.h:56, src/pdhcg.c:894-922). */
pdhcg_result_t *solve_qp_problem(const qp_problem_t *prob, const pdhg_parameters_t *params);

/* Multi-process solve.  Like the reference's single-GPU build, this library
 * has no distributed path: prints a message and returns NULL.
 * Replaces reference solve_qp_problem_distributed (include/pdhcg.h:59,
 * distributed/distributed_ops_stub.c:78-84). */
pdhcg_result_t *solve_qp_problem_distributed(const pdhg_parameters_t *params, const qp_problem_t *original_problem);

/* Defaults of reference set_default_parameters (include/pdhcg.h:62, src/utils.cu:324-368). */
void set_default_parameters(pdhg_parameters_t *params);

/* Replaces reference pdhcg_result_free (include/pdhcg.h:64, src/pdhcg.c:510-521). */
void pdhcg_result_free(pdhcg_result_t *results);

/* Replaces reference qp_problem_free (include/pdhcg.h:66, src/pdhcg.c:532-567). */
void qp_problem_free(qp_problem_t *prob);

#ifdef __cplusplus
}
#endif
