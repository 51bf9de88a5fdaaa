/*
 * pdhcg_types.h -- value types of the PDHCG C interface.
 *
 * These structs and enums are the binary interface that callers of the
 * reference solver already compile against (reference file
 * include/pdhcg_types.h, lines 28-300).  Field order, field types and enum
 * values are kept identical so that a program built against the reference
 * header links against libpdhcg_b200.so unchanged.  Nothing here depends on
 * CUDA or on any B200 detail; the device side never sees these structs.
 */
#pragma once

#include <stdbool.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Why a solve stopped (reference include/pdhcg_types.h:28-39). */
typedef enum {
    TERMINATION_REASON_UNSPECIFIED,
    TERMINATION_REASON_OPTIMAL,
    TERMINATION_REASON_PRIMAL_INFEASIBLE,
    TERMINATION_REASON_DUAL_INFEASIBLE,
    TERMINATION_REASON_INFEASIBLE_OR_UNBOUNDED,
    TERMINATION_REASON_TIME_LIMIT,
    TERMINATION_REASON_ITERATION_LIMIT,
    TERMINATION_REASON_USER_INTERRUPT,
    TERMINATION_REASON_FEAS_POLISH_SUCCESS
} termination_reason_t;

/* Norm used for residuals and relative errors (reference :41-45). */
typedef enum { NORM_TYPE_L2 = 0, NORM_TYPE_L_INF = 1 } norm_type_t;

/* Host CSR triple owned by qp_problem_t (reference :47-52). */
typedef struct {
    int *row_ptr;
    int *col_ind;
    double *val;
} CsrComponent;

/* Structure of the quadratic objective (reference :54-61). */
typedef enum {
    PDHCG_SPARSE_Q,
    PDHCG_DIAG_Q,
    PDHCG_LOW_RANK_PLUS_SPARSE_Q,
    PDHCG_LOW_RANK_Q,
    PDHCG_NON_Q
} quad_obj_type_t;

/* Cone families (reference :63-71). SOC/RSOC blocks hold v_dim + 2 slots
 * laid out [v(v_dim), w or s, z or t]; EXP and POW hold 3 slots; PSD holds
 * the svec of an order-v_dim symmetric matrix. */
typedef enum {
    CONE_ROTATED_SOC = 0,
    CONE_STANDARD_SOC = 1,
    CONE_EXPONENTIAL = 2,
    CONE_POWER = 3,
    CONE_PSD = 4,
    NUM_CONE_TYPES = 5
} cone_type_t;

/* Owned cone block list inside qp_problem_t (reference :73-82). */
typedef struct {
    int num_cones;
    int *start_idx;
    int *v_dim;
    cone_type_t *type;
    double *power_alpha;
    int fixed_mask_size;
    char *is_fixed;
} cone_blocks_t;

/* One cone as a caller describes it to create_qp_problem (reference :84-91). */
typedef struct {
    cone_type_t type;
    int start_idx;
    int v_dim;
    double power_alpha;
    const char *is_fixed;
} cone_spec_t;

/* Heap-owned problem (reference :93-134). */
typedef struct {
    int num_variables;
    int num_constraints;
    int num_rank_lowrank_obj;
    double *variable_lower_bound;
    double *variable_upper_bound;
    double *objective_vector;
    double objective_constant;

    CsrComponent *constraint_matrix;
    int constraint_matrix_num_nonzeros;

    CsrComponent *objective_sparse_matrix;
    int objective_sparse_matrix_num_nonzeros;

    CsrComponent *objective_lowrank_matrix;
    int objective_lowrank_matrix_num_nonzeros;

    CsrComponent *objective_lowrank_middle_matrix;
    int objective_lowrank_middle_matrix_num_nonzeros;

    double *constraint_lower_bound;
    double *constraint_upper_bound;

    double *affine_cone_offset;
    cone_blocks_t affine_cones;

    int num_quadratic_constraints;
    int *quadratic_constraint_row_indices;
    CsrComponent **quadratic_constraint_matrices;
    int *quadratic_constraint_matrix_num_nonzeros;

    cone_blocks_t cones;
    int num_original_variables;

    double *primal_start;
    double *dual_start;
} qp_problem_t;

/* Restart and PID primal-weight gains (reference :136-145). */
typedef struct {
    double artificial_restart_threshold;
    double sufficient_reduction_for_restart;
    double necessary_reduction_for_restart;
    double k_p;
    double k_i;
    double k_d;
    double i_smooth;
} restart_parameters_t;

/* Stopping rule (reference :147-155). */
typedef struct {
    double eps_optimal_relative;
    double eps_feasible_relative;
    double eps_feas_polish_relative;
    double eps_infeasible;
    double time_sec_limit;
    int iteration_limit;
} termination_criteria_t;

/* Inner projected Barzilai-Borwein solve (reference :157-162). */
typedef struct {
    int iteration_limit;
    double initial_tolerance;
    double min_tolerance;
} inner_solver_parameters_t;

typedef enum { UNIFORM_PARTITION, NNZ_BALANCE_PARTITION } partition_method_t;

typedef enum { NO_PERMUTATION, FULL_RANDOM_PERMUTATION, BLOCK_RANDOM_PERMUTATION } permute_method_t;

typedef struct {
    int row_dims;
    int col_dims;
    bool decided;
} grid_size_t;

/* Solver parameters (reference :183-208). */
typedef struct {
    int curtis_reid_iterations;
    int l_inf_ruiz_iterations;
    bool has_pock_chambolle_alpha;
    double pock_chambolle_alpha;
    bool bound_objective_rescaling;
    bool use_cone_preserving_scaling;
    int verbose;
    int termination_evaluation_frequency;
    int sv_max_iter;
    double sv_tol;
    termination_criteria_t termination_criteria;
    restart_parameters_t restart_params;
    double reflection_coefficient;
    bool feasibility_polishing;
    norm_type_t optimality_norm;
    inner_solver_parameters_t inner_solver_parameters;
    bool presolve;
    bool diag_jacobi_precond;
    cone_type_t default_cone_type;
    partition_method_t partition_method;
    permute_method_t permute_method;
    grid_size_t grid_size;
    int permute_block_size;
} pdhg_parameters_t;

/* Heap-owned result (reference :210-248). */
typedef struct {
    int num_variables;
    int num_constraints;
    int num_nonzeros;

    int num_reduced_variables;
    int num_reduced_constraints;
    int num_reduced_nonzeros;

    double *primal_solution;
    double *dual_solution;
    double *reduced_cost;

    int total_count;
    int total_inner_count;
    double rescaling_time_sec;
    double cumulative_time_sec;

    double absolute_primal_residual;
    double relative_primal_residual;
    double absolute_dual_residual;
    double relative_dual_residual;
    double primal_objective_value;
    double dual_objective_value;
    double objective_gap;
    double relative_objective_gap;
    double max_primal_ray_infeasibility;
    double max_dual_ray_infeasibility;
    double primal_ray_linear_objective;
    double dual_ray_objective;
    termination_reason_t termination_reason;
    double feasibility_polishing_time;
    int feasibility_iteration;

    double presolve_time;
    int presolve_status;
} pdhcg_result_t;

/* Input matrix formats (reference :250-257). */
typedef enum { matrix_dense = 0, matrix_csr = 1, matrix_csc = 2, matrix_coo = 3 } matrix_format_t;

/* Borrowed input matrix (reference :260-300). Entries with
 * |a| <= zero_tolerance are dropped on conversion. */
typedef struct {
    int m;
    int n;
    matrix_format_t fmt;
    double zero_tolerance;
    union MatrixData {
        struct MatrixDense {
            const double *A; /* row-major m*n */
        } dense;
        struct MatrixCSR {
            int nnz;
            const int *row_ptr;
            const int *col_ind;
            const double *vals;
        } csr;
        struct MatrixCSC {
            int nnz;
            const int *col_ptr;
            const int *row_ind;
            const double *vals;
        } csc;
        struct MatrixCOO {
            int nnz;
            const int *row_ind;
            const int *col_ind;
            const double *vals;
        } coo;
    } data;
} matrix_desc_t;

#ifdef __cplusplus
}
#endif
