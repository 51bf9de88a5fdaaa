/*
 * pdhcg_b200.h -- additive entry points of libpdhcg_b200.so beyond the
 * reference interface in pdhcg.h.  None of them changes a struct of
 * pdhcg_types.h; callers that only use pdhcg.h never see them.
 *
 * All functions return 0 on success and a negative code on error, unless
 * stated otherwise; a CUDA error is reported on stderr and returned, never
 * turned into exit().
 */
#pragma once

#include <signal.h>

#include "pdhcg_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Arithmetic of the iteration. */
typedef enum {
    PDHCG_B200_FP64 = 0,       /* every vector and matrix value in double */
    PDHCG_B200_MIXED = 1       /* FP32 matrix values and iterates with FP64 accumulation and FP64
                                  residuals/restarts, then an FP64 polish phase.  Problems that take
                                  the inner BB solve (sparse or low-rank Q, PSD blocks) read FP32
                                  values of Q, R, R^T and of A's long rows in the bulk phase, with
                                  FP64 iterates. */
} pdhcg_b200_precision_t;

typedef struct {
    int precision;                 /* pdhcg_b200_precision_t */
    double polish_threshold;       /* MIXED: relative KKT error at which FP64 takes over (default 1e-5) */
    int has_initial_primal_weight; /* warm start of the primal weight (no counterpart in the reference,
                                      which recomputes it, reference src/pdhg_core_op.cu:962-970) */
    double initial_primal_weight;
    int use_graphs;                /* capture the iterations between two evaluations in a CUDA graph */
    int time_steps;                /* bracket every fused step with CUDA events (fills step_kernel_ms) */
    int solution_on_device;        /* pdhcg_b200_solve_device only: leave x, y, reduced cost in device
                                      memory (result arrays are NULL); see pdhcg_b200_device_solution */
    int has_initial_step_size;     /* skip the power method and use initial_step_size (0.998 / sigma_max
                                      of the scaled A): valid for another problem with the same A and
                                      scaling parameters, e.g. from pdhcg_b200_stats_t.step_size */
    double initial_step_size;
    int reserved[4];
} pdhcg_b200_options_t;

void pdhcg_b200_default_options(pdhcg_b200_options_t *opts);

/* solve_qp_problem with options.  Same ownership and error rules. */
pdhcg_result_t *pdhcg_b200_solve(const qp_problem_t *prob, const pdhg_parameters_t *params,
                                 const pdhcg_b200_options_t *opts);

/* ---- problems resident in device memory -----------------------------------
 * pdhcg_b200_upload copies a problem's raw arrays to the current device
 * once; pdhcg_b200_solve_device then solves from that copy without any
 * host->device traffic for the problem data (each solve rescales a private
 * device copy, so the handle can be solved many times, e.g. with different
 * parameters).  No counterpart in the reference, which uploads inside
 * every solve (reference src/solver_state.cu:688-851). */
typedef struct pdhcg_b200_device_problem_s pdhcg_b200_device_problem_t;

pdhcg_b200_device_problem_t *pdhcg_b200_upload(const qp_problem_t *prob);
pdhcg_result_t *pdhcg_b200_solve_device(pdhcg_b200_device_problem_t *handle, const pdhg_parameters_t *params,
                                        const pdhcg_b200_options_t *opts);
/* Device pointers of the last solution kept with solution_on_device; valid
 * until the next solve on the handle or its release.  Returns 0 or -1. */
int pdhcg_b200_device_solution(const pdhcg_b200_device_problem_t *handle, const double **x, const double **y,
                               const double **reduced_cost);
void pdhcg_b200_device_problem_free(pdhcg_b200_device_problem_t *handle);

/* Device-side statistics of the last solve on the calling thread. */
typedef struct {
    double setup_ms;             /* upload, transpose, rescaling, power method (CUDA events) */
    double loop_ms;              /* main loop on the device, first to last iteration (CUDA events) */
    double step_kernel_ms;       /* summed duration of the fused primal/dual step kernels */
    long long step_kernel_launches;
    long long kernel_launches;   /* all kernels launched by the solve */
    int iterations;
    int fp32_iterations;
    int restarts;
    int evaluations;
    double step_bytes;           /* algorithmic HBM bytes of one primal + dual step */
    double spmv_bytes;           /* algorithmic bytes of the two SpMVs inside one step */
    double host_copy_ms;         /* host-side copy / classification of the problem */
    double upload_ms;            /* allocation and host->device copies */
    double result_ms;            /* result kernel and device->host copies */
    double total_ms;             /* the whole call, wall clock */
    double primal_weight;        /* primal weight at termination (a warm start for a similar solve) */
    double step_size;            /* 0.998 / sigma_max(scaled A), reusable for the same A */
} pdhcg_b200_stats_t;

int pdhcg_b200_last_stats(pdhcg_b200_stats_t *out);

/* The rescaling a solve would apply to prob under params, computed on the
 * device (Curtis-Reid, Ruiz, Pock-Chambolle, bound/objective scaling and
 * the cone-preserving adjustment; reference rescale_problem,
 * src/preconditioner.c:654-713) and copied out: con_rescale[num_constraints]
 * and var_rescale[num_variables] are the cumulative row and column factors
 * (the reference's rescale_info_t con_rescale / var_rescale), bound_obj[0]
 * the bound rescaling and bound_obj[1] the objective rescaling.  Returns 0,
 * or -1 (NULL arguments, a problem the solver refuses, a device error). */
int pdhcg_b200_rescaling(const qp_problem_t *prob, const pdhg_parameters_t *params, double *con_rescale,
                         double *var_rescale, double *bound_obj);

/* Cancellation.  g_pdhcg_cancel_request is the reference's flag (reference
 * src/pdhcg.c:31), exported under the same name so that its Python binding
 * (which declares it extern and sets it from a SIGINT handler, reference
 * python_bindings/_core_bindings.cpp:41-47) links unchanged.  A non-zero
 * value ends the running solve at its next evaluation with
 * TERMINATION_REASON_USER_INTERRUPT. */
extern volatile sig_atomic_t g_pdhcg_cancel_request;
void pdhcg_b200_request_cancel(int on);

/* Length of cone block `block` (3 for EXP/POW, v_dim + 2 for SOC/RSOC,
 * v_dim (v_dim + 1) / 2 for PSD), -1 for an invalid block.  Same name and
 * meaning as the reference's cone_block_length (reference
 * internal/cone_utils.h:27, src/cone_utils.c:40-45), which its Python binding
 * calls. */
int cone_block_length(const cone_blocks_t *blocks, int block);

/* ---- batched solve ----------------------------------------------------------
 * Many small LP / diagonal-QP instances (no cones, at most 65535 rows and
 * columns, each fitting in one SM's shared memory) in persistent launches:
 * each instance runs the same restarted Halpern PDHG as solve_qp_problem
 * inside one thread group with its scaled data held in shared memory, in
 * FP32 with FP64 accumulation, reductions, residuals and step sizes.
 * Instances that do not qualify are solved one by one by solve_qp_problem.
 * No counterpart in the reference (its baseline is one solve_qp_problem call
 * per instance).  results[i] receives a heap result of problem i (free each
 * with pdhcg_result_free); returns 0, or -1 on error. */
typedef struct {
    int shape;         /* launch shape (index into the shapes below), -1: by size */
    int band_shape[7]; /* per size band, 1 + the band's launch shape; 0: not set (shape, or by size).
                          Band b holds the instances that need more than 1/2^(b+1) and at most 1/2^b
                          of a CTA's shared memory (band 6: everything smaller); each band present
                          in a batch is one launch. */
} pdhcg_b200_batch_options_t;

/* Launch shapes {threads per CTA, threads per instance}:
 * 0 {128, 32}, 1 {256, 64}, 2 {256, 128}, 3 {256, 256}, 4 {512, 512}, 5 {1024, 1024},
 * 6 {128, 128}. */
#define PDHCG_B200_BATCH_SHAPES 7

void pdhcg_b200_default_batch_options(pdhcg_b200_batch_options_t *opts);
int pdhcg_b200_solve_batch(int count, const qp_problem_t *const *probs, const pdhg_parameters_t *params,
                           const pdhcg_b200_batch_options_t *opts, pdhcg_result_t **results);
/* Figures of the last pdhcg_b200_solve_batch on the calling thread. */
typedef struct {
    double kernel_ms;   /* device work: the A^T build and the batch kernels, first launch to last (CUDA events) */
    double total_ms;    /* the whole call, wall clock */
    double pack_ms;     /* sizing and packing the instances into page-locked staging memory, wall clock */
    double h2d_bytes;   /* bytes copied host to device (one copy of the packed inputs) */
    double d2h_bytes;   /* bytes copied device to host (one copy of the packed outputs) */
    int launches;       /* kernel launches (the A^T build, then one per size class) */
    int batched;        /* instances solved by the batch kernels */
    int fallback;       /* instances handed to solve_qp_problem */
    int reserved[5];
} pdhcg_b200_batch_stats_t;
int pdhcg_b200_last_batch_stats(pdhcg_b200_batch_stats_t *out);
/* Batch solves keep their page-locked staging buffer and device buffer
 * (sized for the largest batch so far) between calls; this frees both. */
void pdhcg_b200_batch_release(void);

/* Times every launch shape on each size band's instances among the given
 * ones (at most 256 per band, solving them each time), stores each band's
 * fastest in opts->band_shape and the fastest over all bands in
 * opts->shape; shape_ms (may be NULL) receives PDHCG_B200_BATCH_SHAPES wall
 * times in milliseconds, summed over the bands. */
int pdhcg_b200_batch_autotune(int count, const qp_problem_t *const *probs, const pdhg_parameters_t *params,
                              pdhcg_b200_batch_options_t *opts, double *shape_ms);

/* ---- learned warm start --------------------------------------------------------
 * A small MLP from a parametric instance's parameters theta to a starting
 * point and a primal weight (no counterpart in the reference):
 *   h1 = relu(W1 theta + b1), h2 = relu(W2 h1 + b2)      (hidden)
 *   z  = W3 h2 + b3                                       (rank: low-rank head)
 *   o  = U z + bu                                         (out_dim, e.g. n + m)
 *   lw = wp . h2 + bp                                     (log primal weight)
 * BF16 weights in the products with FP32 accumulation, FP32 master weights
 * updated by Adam.  Loss: mean over the batch and the outputs of (o - t)^2,
 * plus the batch mean of (lw - t_lw)^2.  Host arrays are row-major FP32.
 * Parameters are packed in the order W1, b1, W2, b2, W3, b3, U, bu, wp, bp,
 * each weight [out_features x in_features] row-major. */
typedef struct pdhcg_b200_mlp_s pdhcg_b200_mlp_t;

pdhcg_b200_mlp_t *pdhcg_b200_mlp_create(int in_dim, int hidden, int rank, int out_dim, unsigned long long seed);
void pdhcg_b200_mlp_free(pdhcg_b200_mlp_t *net);
long long pdhcg_b200_mlp_num_params(const pdhcg_b200_mlp_t *net);
int pdhcg_b200_mlp_get_params(const pdhcg_b200_mlp_t *net, float *params);
int pdhcg_b200_mlp_set_params(pdhcg_b200_mlp_t *net, const float *params); /* also resets Adam */
/* out: batch x out_dim; logw (may be NULL): batch */
int pdhcg_b200_mlp_predict(pdhcg_b200_mlp_t *net, int batch, const float *theta, float *out, float *logw);
/* loss of one batch and its gradient (packed order; grad may be NULL) */
int pdhcg_b200_mlp_loss_grad(pdhcg_b200_mlp_t *net, int batch, const float *theta, const float *target,
                             const float *target_logw, double *loss, float *grad);
/* `epochs` passes of Adam over `count` samples in minibatches of `batch`
 * (in order, the last partial batch dropped); loss receives the last
 * epoch's mean minibatch loss. */
int pdhcg_b200_mlp_train(pdhcg_b200_mlp_t *net, int count, const float *theta, const float *target,
                         const float *target_logw, int epochs, int batch, float lr, double *loss);

/* ---- problem files -----------------------------------------------------
 * MPS / QPS reader, plain or gzip (name ending in .gz): the reference's
 * read_mps_file (include/mps_parser.h:27, src/mps_parser.c:420-682) with the
 * same conventions (sections ROWS, COLUMNS, RHS, RANGES, BOUNDS, OBJSENSE,
 * QUADOBJ, QMATRIX, QCMATRIX; variables default to [0, inf); OBJSENSE MAX
 * negates the objective).  NULL when the file cannot be read or parsed;
 * release with qp_problem_free. */
qp_problem_t *read_mps_file(const char *filename);

/* ---- kernel-level entry points on device pointers ------------------------
 * For parity tests and embedding.  Pointers are device memory of the current
 * device; stream may be NULL (legacy default stream).  They return after
 * enqueueing (call cudaStreamSynchronize to wait).  pdhcg_b200_csr_spmv
 * allocates nothing; pdhcg_b200_project_cones and pdhcg_b200_pdhg_step take
 * small stream-ordered temporaries (cudaMallocAsync / cudaFreeAsync). */

/* y = M x for a CSR matrix (int32 indices, FP64 values). */
int pdhcg_b200_csr_spmv(int rows, const int *row_ptr, const int *col_ind, const double *val, const double *x,
                        double *y, void *stream);

/* Project each cone block of x (scaled space) onto {x : x_i / d_i in K} in the
 * metric sum_i (1 + tau q_i)(x_i - r_i)^2; q may be NULL.  cone_type holds
 * cone_type_t values: SOC and rotated-SOC blocks of at most 256 slots,
 * exponential blocks, power blocks (exponents in cone_alpha, which may be
 * NULL without power blocks) and PSD blocks of order v_dim <= 22 (svec
 * packing, projected in the plain Frobenius metric as the reference does:
 * d and q do not enter; 2 v_dim^2 doubles of temporary scratch each); -3
 * for a power block without cone_alpha or an unknown type, -2 for a longer
 * block.  Waits for the stream (it reads the block lengths on the host). */
int pdhcg_b200_project_cones(int num_cones, const int *cone_start, const int *cone_vdim, const int *cone_type,
                             const double *cone_alpha, double *x, const double *d, const double *q, double tau,
                             void *stream);

/* Projection of cone blocks with fixed slots onto the sections through the
 * fixed values (set_cone_fixed; reference section projectors,
 * src/kernels/pdhcg_soc_cone_kernels.cu:23-260,
 * src/kernels/pdhcg_rsoc_cone_kernels.cu:23-465,
 * src/kernels/pdhcg_exp_cone_kernels.cu:134-525,
 * src/kernels/pdhcg_power_cone_kernels.cu:135-434).  Arguments as for
 * pdhcg_b200_project_cones, plus fixed: device mask over x (nonzero = the
 * slot keeps its value) and warm: device array of num_cones multipliers
 * carried from call to call (start at 0; may be NULL).  Every block is
 * treated as a section block; PSD blocks are refused with -3 (they cannot
 * be fixed).  Waits for the stream. */
int pdhcg_b200_project_cone_sections(int num_cones, const int *cone_start, const int *cone_vdim,
                                     const int *cone_type, const double *cone_alpha, const unsigned char *fixed,
                                     double *x, const double *d, const double *q, double tau, double *warm,
                                     void *stream);

/* Checks the fixed slots of a problem's variable cones as solve_qp_problem
 * does before solving (reference pdhcg_validate_fixed_cone_sections,
 * src/pdhcg.c:729-892, internal/solver.h:29): the mask has num_variables
 * entries, fixed values are finite, and each block's section through them is
 * nonempty.  0 when valid (or nothing is fixed), -1 with a message on stderr
 * otherwise.  Host only. */
int pdhcg_b200_validate_fixed_sections(const qp_problem_t *prob);

/* pdhcg_b200_project_cones for callers that must not allocate device memory
 * (no cudaMalloc / cudaMallocAsync / cudaFree, no allocating library): e.g.
 * code whose memory is budgeted up front, or that runs while another
 * component owns the allocator.  No counterpart in the reference.
 * Same arguments, results and error codes as pdhcg_b200_project_cones, plus
 * -4 when num_cones > PDHCG_B200_NOALLOC_MAX_CONES (nothing is launched),
 * except that PSD blocks are refused with -3 (their eigen-decomposition
 * scratch grows with the order, so it has no fixed bound).
 * Its scratch is one file-scope device array per device
 * ((PDHCG_B200_NOALLOC_MAX_CONES + 2) ints); every call writes it before
 * reading it, so nothing needs to start at zero.
 * - The first call on each device looks up that array's address
 *   (cudaGetSymbolAddress with the device current) and keeps it for the
 *   life of the process; make that first call before any stream capture.
 *   The kept address belongs to the device's context at that time: after a
 *   cudaDeviceReset of that device, do not call this entry point again in
 *   the same process.
 * - Calls on the same device share the scratch: two calls that overlap in
 *   time (other threads, or other streams before the first has finished)
 *   race.  Serialise them.
 * - Like pdhcg_b200_project_cones it waits for the stream (it reads the
 *   longest block length back to the host). */
#define PDHCG_B200_NOALLOC_MAX_CONES 65536
int pdhcg_b200_project_cones_noalloc(int num_cones, const int *cone_start, const int *cone_vdim,
                                     const int *cone_type, const double *cone_alpha, double *x, const double *d,
                                     const double *q, double tau, void *stream);

/* One restarted-Halpern PDHG step (primal prox with diagonal Q or none, cone
 * projection, dual prox, reflection, Halpern averaging) on device arrays;
 * the layout mirrors oracle_step_t of the oracle.  Sizes: n variables, m rows.
 * -3 with PSD blocks (no scratch is kept for them), -2 for a cone block
 * longer than 256 slots. */
typedef struct {
    int n, m;
    const int *A_row_ptr, *A_col_ind;
    const double *A_val;
    const int *At_row_ptr, *At_col_ind;
    const double *At_val;
    const double *c, *var_lb, *var_ub, *q_diag;
    const double *con_lb, *con_ub, *affine_offset;
    const double *var_rescale;
    int num_cones;
    const int *cone_start, *cone_vdim, *cone_type;
    const double *cone_alpha;
    double tau, sigma, halpern_weight, reflection;
    double *x_init, *x_cur, *y_init, *y_cur;
    double *x_pdhg, *x_refl, *y_pdhg, *y_refl, *Aty, *Ax;
} pdhcg_b200_step_t;

int pdhcg_b200_pdhg_step(const pdhcg_b200_step_t *s, void *stream);

#ifdef __cplusplus
}
#endif
