/*
 * oracle_solver.c -- CPU restatement of the reference restarted Halpern
 * PDHG / PDHCG solve, single-threaded FP64.
 *
 * TEST INFRASTRUCTURE ONLY (see pdhcg_oracle.h).  It is the checker the
 * CUDA solver is compared with; nothing in pdhcg_b200/ links it.
 *
 * The control flow follows the reference line by line where the
 * trajectory depends on it (evaluation cadence, the (k+2) store rule for
 * PDHG iterates, restart tests, PID primal weight, BB tolerance schedule);
 * each function cites the lines it restates.  Vector reductions are plain
 * sequential sums, so results agree with the reference's cuBLAS reductions
 * to rounding, not bit for bit.
 */
#define _POSIX_C_SOURCE 200809L
#include "pdhcg_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------ */
/* small helpers                                                       */
/* ------------------------------------------------------------------ */

typedef struct {
    int rows, cols, nnz;
    int *rp, *ci;
    double *v;
} ocsr;

static void *xmalloc(size_t n) { void *p = malloc(n ? n : 1); if (!p) abort(); return p; }
static void *xcalloc(size_t c, size_t n) { void *p = calloc(c ? c : 1, n ? n : 1); if (!p) abort(); return p; }
static double *dvec(int n) { return (double *)xcalloc((size_t)(n > 0 ? n : 1), sizeof(double)); }
static double *dcopy(const double *s, int n)
{
    double *d = dvec(n);
    if (s && n > 0)
        memcpy(d, s, (size_t)n * sizeof(double));
    return d;
}

static void csr_free(ocsr *M)
{
    free(M->rp); free(M->ci); free(M->v);
    memset(M, 0, sizeof(*M));
}

static void csr_from(ocsr *M, int rows, int cols, int nnz, const CsrComponent *src)
{
    M->rows = rows; M->cols = cols; M->nnz = nnz;
    M->rp = (int *)xcalloc((size_t)rows + 1, sizeof(int));
    M->ci = (int *)xmalloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int));
    M->v = dvec(nnz);
    if (src && src->row_ptr)
        memcpy(M->rp, src->row_ptr, ((size_t)rows + 1) * sizeof(int));
    if (src && nnz > 0) {
        memcpy(M->ci, src->col_ind, (size_t)nnz * sizeof(int));
        memcpy(M->v, src->val, (size_t)nnz * sizeof(double));
    }
}

/* y = M x */
static void spmv(const ocsr *M, const double *x, double *y)
{
    for (int r = 0; r < M->rows; ++r) {
        double s = 0.0;
        for (int k = M->rp[r]; k < M->rp[r + 1]; ++k)
            s += M->v[k] * x[M->ci[k]];
        y[r] = s;
    }
}

/* Explicit transpose; entries of each output row in increasing input-row
 * order (what csr2csc produces, reference src/solver_state.cu:739-770). */
static void csr_transpose(const ocsr *M, ocsr *T)
{
    T->rows = M->cols; T->cols = M->rows; T->nnz = M->nnz;
    T->rp = (int *)xcalloc((size_t)T->rows + 1, sizeof(int));
    T->ci = (int *)xmalloc((size_t)(M->nnz > 0 ? M->nnz : 1) * sizeof(int));
    T->v = dvec(M->nnz);
    for (int k = 0; k < M->nnz; ++k)
        T->rp[M->ci[k] + 1]++;
    for (int i = 0; i < T->rows; ++i)
        T->rp[i + 1] += T->rp[i];
    int *next = (int *)xmalloc((size_t)(T->rows > 0 ? T->rows : 1) * sizeof(int));
    for (int i = 0; i < T->rows; ++i)
        next[i] = T->rp[i];
    for (int r = 0; r < M->rows; ++r)
        for (int k = M->rp[r]; k < M->rp[r + 1]; ++k) {
            int p = next[M->ci[k]]++;
            T->ci[p] = r;
            T->v[p] = M->v[k];
        }
    free(next);
}

static double dot(const double *a, const double *b, int n)
{
    double s = 0.0;
    for (int i = 0; i < n; ++i)
        s += a[i] * b[i];
    return s;
}

static double nrm2(const double *a, int n) { return sqrt(dot(a, a, n)); }

/* |x|_inf as the reference's Idamax + D2H read (src/utils.cu:548-567). */
static double inf_norm(const double *x, int n)
{
    double m = 0.0;
    for (int i = 0; i < n; ++i) {
        if (!isfinite(x[i]))
            return INFINITY;
        double a = fabs(x[i]);
        if (a > m)
            m = a;
    }
    return m;
}

static double vnorm(const double *x, int n, norm_type_t t) { return t == NORM_TYPE_L_INF ? inf_norm(x, n) : nrm2(x, n); }

static double clampd(double lo, double x, double hi) { return fmax(lo, fmin(x, hi)); }

/* reference get_print_frequency, src/utils.cu:535-546 */
static int print_frequency(int iter)
{
    int step = 10;
    long long threshold = 1000;
    while (iter >= threshold) {
        step *= 10;
        threshold *= 10;
    }
    return step;
}

static int cone_len(int type, int v_dim)
{
    if (type == CONE_EXPONENTIAL || type == CONE_POWER)
        return 3;
    if (type == CONE_STANDARD_SOC || type == CONE_ROTATED_SOC)
        return v_dim + 2;
    return v_dim * (v_dim + 1) / 2;
}

static double now_sec(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ------------------------------------------------------------------ */
/* working problem + rescaling (reference src/preconditioner.c)        */
/* ------------------------------------------------------------------ */

typedef struct {
    int n, m, rank;
    ocsr A, Q, R, D;
    int has_D;
    double *c, *l, *u, *lc, *uc, *g;
    double c0;
    int ncones;
    int *cstart, *cvdim, *ctype;
    double *calpha;
    int naff;
    int *astart, *avdim, *atype;
    double *aalpha; /* affine power-cone exponents */
    double *primal_start, *dual_start;
    char *fixed; /* cones.is_fixed over the n variables, or NULL */
} oprob;

static void oprob_free(oprob *P)
{
    csr_free(&P->A); csr_free(&P->Q); csr_free(&P->R); csr_free(&P->D);
    free(P->c); free(P->l); free(P->u); free(P->lc); free(P->uc); free(P->g);
    free(P->cstart); free(P->cvdim); free(P->ctype); free(P->calpha);
    free(P->astart); free(P->avdim); free(P->atype); free(P->aalpha);
    free(P->primal_start); free(P->dual_start);
    free(P->fixed);
}

/* deepcopy_problem + create_problem_with_dummy_constraint
 * (reference src/preconditioner.c:165-252, src/utils.cu:80-135). */
static void oprob_load(oprob *P, const qp_problem_t *prob)
{
    memset(P, 0, sizeof(*P));
    P->n = prob->num_variables;
    P->m = prob->num_constraints;
    P->rank = prob->num_rank_lowrank_obj;
    P->c0 = prob->objective_constant;
    int dummy = (prob->num_constraints == 0 || prob->constraint_matrix == NULL);
    if (dummy) {
        P->m = 1;
        P->A.rows = 1; P->A.cols = P->n; P->A.nnz = 1;
        P->A.rp = (int *)xmalloc(2 * sizeof(int)); P->A.rp[0] = 0; P->A.rp[1] = 1;
        P->A.ci = (int *)xmalloc(sizeof(int)); P->A.ci[0] = 0;
        P->A.v = dvec(1); P->A.v[0] = 1.0;
        P->lc = dvec(1); P->lc[0] = -INFINITY;
        P->uc = dvec(1); P->uc[0] = INFINITY;
        P->g = dvec(1);
    } else {
        csr_from(&P->A, P->m, P->n, prob->constraint_matrix_num_nonzeros, prob->constraint_matrix);
        P->lc = dcopy(prob->constraint_lower_bound, P->m);
        P->uc = dcopy(prob->constraint_upper_bound, P->m);
        P->g = dcopy(prob->affine_cone_offset, P->m);
    }
    if (prob->objective_sparse_matrix && prob->objective_sparse_matrix->row_ptr)
        csr_from(&P->Q, P->n, P->n, prob->objective_sparse_matrix_num_nonzeros, prob->objective_sparse_matrix);
    if (prob->objective_lowrank_matrix && prob->objective_lowrank_matrix->row_ptr && P->rank > 0)
        csr_from(&P->R, P->rank, P->n, prob->objective_lowrank_matrix_num_nonzeros, prob->objective_lowrank_matrix);
    if (prob->objective_lowrank_middle_matrix && prob->objective_lowrank_middle_matrix->row_ptr && P->rank > 0) {
        csr_from(&P->D, P->rank, P->rank, prob->objective_lowrank_middle_matrix_num_nonzeros,
                 prob->objective_lowrank_middle_matrix);
        P->has_D = prob->objective_lowrank_middle_matrix_num_nonzeros > 0;
    }
    P->c = dcopy(prob->objective_vector, P->n);
    P->l = dcopy(prob->variable_lower_bound, P->n);
    P->u = dcopy(prob->variable_upper_bound, P->n);
    P->ncones = prob->cones.num_cones;
    P->cstart = (int *)xcalloc((size_t)P->ncones, sizeof(int));
    P->cvdim = (int *)xcalloc((size_t)P->ncones, sizeof(int));
    P->ctype = (int *)xcalloc((size_t)P->ncones, sizeof(int));
    P->calpha = dvec(P->ncones);
    for (int i = 0; i < P->ncones; ++i) {
        P->cstart[i] = prob->cones.start_idx[i];
        P->cvdim[i] = prob->cones.v_dim[i];
        P->ctype[i] = (int)prob->cones.type[i];
        P->calpha[i] = prob->cones.power_alpha ? prob->cones.power_alpha[i] : 0.0;
    }
    P->naff = dummy ? 0 : prob->affine_cones.num_cones;
    P->astart = (int *)xcalloc((size_t)P->naff, sizeof(int));
    P->avdim = (int *)xcalloc((size_t)P->naff, sizeof(int));
    P->atype = (int *)xcalloc((size_t)P->naff, sizeof(int));
    P->aalpha = (double *)xcalloc((size_t)P->naff, sizeof(double));
    for (int i = 0; i < P->naff; ++i) {
        P->astart[i] = prob->affine_cones.start_idx[i];
        P->avdim[i] = prob->affine_cones.v_dim[i];
        P->atype[i] = (int)prob->affine_cones.type[i];
        P->aalpha[i] = prob->affine_cones.power_alpha ? prob->affine_cones.power_alpha[i] : 0.0;
    }
    if (prob->primal_start)
        P->primal_start = dcopy(prob->primal_start, P->n);
    if (prob->cones.is_fixed) {
        P->fixed = (char *)xmalloc((size_t)(P->n > 0 ? P->n : 1));
        memcpy(P->fixed, prob->cones.is_fixed, (size_t)P->n);
    }
    if (dummy) {
        P->dual_start = dvec(1);
    } else if (prob->dual_start) {
        P->dual_start = dcopy(prob->dual_start, P->m);
    }
}

/* scale_problem, reference src/preconditioner.c:256-309 */
static void scale_problem(oprob *P, const double *cr, const double *vr)
{
    for (int i = 0; i < P->n; ++i) {
        P->c[i] /= vr[i];
        P->u[i] *= vr[i];
        P->l[i] *= vr[i];
    }
    for (int i = 0; i < P->m; ++i) {
        P->lc[i] /= cr[i];
        P->uc[i] /= cr[i];
        P->g[i] /= cr[i];
    }
    for (int r = 0; r < P->m; ++r)
        for (int k = P->A.rp[r]; k < P->A.rp[r + 1]; ++k)
            P->A.v[k] /= (cr[r] * vr[P->A.ci[k]]);
    if (P->Q.rp)
        for (int r = 0; r < P->n; ++r)
            for (int k = P->Q.rp[r]; k < P->Q.rp[r + 1]; ++k)
                P->Q.v[k] /= (vr[r] * vr[P->Q.ci[k]]);
    if (P->R.nnz > 0)
        for (int r = 0; r < P->rank; ++r)
            for (int k = P->R.rp[r]; k < P->R.rp[r + 1]; ++k)
                P->R.v[k] /= vr[P->R.ci[k]];
}

#define SCALING_EPSILON 1e-12
#define LOG_SCALING_MIN_ABS 1e-300
#define LOG_SCALING_LIMIT 69.07755278982137
#define PSD_LOG_FACTOR_LIMIT (0.5 * LOG_SCALING_LIMIT)
#define PHASE_TAPER_CONE_THRESHOLD 8

/* project_psd_log_scaling, reference src/preconditioner.c:46-92 */
static void psd_log_projection(double *ls, int start, int order)
{
    double *f = dvec(order);
    int slot = start;
    for (int col = 0; col < order; ++col)
        for (int row = col; row < order; ++row, ++slot) {
            double v = ls[slot];
            if (isnan(v)) v = 0.0;
            else if (v > LOG_SCALING_LIMIT) v = LOG_SCALING_LIMIT;
            else if (v < -LOG_SCALING_LIMIT) v = -LOG_SCALING_LIMIT;
            if (row == col) f[row] += 2.0 * v;
            else { f[row] += v; f[col] += v; }
        }
    double rhs = 0.0;
    for (int i = 0; i < order; ++i) rhs += f[i];
    double corr = rhs / (2.0 * order + 2.0), diag = order + 2.0;
    for (int i = 0; i < order; ++i) {
        f[i] = (f[i] - corr) / diag;
        f[i] = fmax(-PSD_LOG_FACTOR_LIMIT, fmin(PSD_LOG_FACTOR_LIMIT, f[i]));
    }
    slot = start;
    for (int col = 0; col < order; ++col)
        for (int row = col; row < order; ++row, ++slot)
            ls[slot] = f[row] + f[col];
    free(f);
}

/* apply_cone_scaling_adjustment, reference src/preconditioner.c:108-144 */
static void cone_scaling_adjust(double *s, int nb, const int *start, const int *vdim, const int *type, int ruiz,
                                int preserving)
{
    for (int b = 0; b < nb; ++b) {
        if (!preserving) {
            if (type[b] == CONE_PSD) {
                int len = cone_len(CONE_PSD, vdim[b]);
                for (int i = start[b]; i < start[b] + len; ++i)
                    s[i] = log(fmax(s[i], LOG_SCALING_MIN_ABS));
                psd_log_projection(s, start[b], vdim[b]);
                for (int i = start[b]; i < start[b] + len; ++i)
                    s[i] = exp(s[i]);
            }
            continue;
        }
        int st = start[b], len = cone_len(type[b], vdim[b]);
        double mx = 0.0, sq = 0.0;
        for (int i = st; i < st + len; ++i) {
            mx = fmax(mx, s[i]);
            sq += s[i] * s[i];
        }
        double rms = sqrt(sq / (double)len);
        double bs = ruiz ? (len <= PHASE_TAPER_CONE_THRESHOLD ? mx : rms)
                         : (len <= PHASE_TAPER_CONE_THRESHOLD ? rms : sqrt(mx * rms));
        for (int i = st; i < st + len; ++i)
            s[i] = bs;
    }
}

static double cr_exp_clamped(double v)
{
    if (isnan(v)) return 1.0;
    if (v > LOG_SCALING_LIMIT) v = LOG_SCALING_LIMIT;
    else if (v < -LOG_SCALING_LIMIT) v = -LOG_SCALING_LIMIT;
    return exp(v);
}

/* curtis_reid_rescaling, reference src/preconditioner.c:334-495 */
static void curtis_reid(oprob *P, int iters, int preserving, double *cum_cr, double *cum_vr)
{
    int m = P->m, n = P->n, nnz = P->A.nnz;
    double *cr = dvec(m), *vr = dvec(n);
    for (int i = 0; i < m; ++i) cr[i] = 1.0;
    for (int i = 0; i < n; ++i) vr[i] = 1.0;
    if (iters > 0 && m > 0 && n > 0 && nnz > 0) {
        const ocsr *M = &P->A;
        double *rls = dvec(m), *cls = dvec(n), *rsum = dvec(m), *csum = dvec(n), *cs = dvec(n);
        int *ccount = (int *)xcalloc((size_t)n, sizeof(int));
        for (int r = 0; r < m; ++r)
            for (int k = M->rp[r]; k < M->rp[r + 1]; ++k) {
                double la = log(fmax(fabs(M->v[k]), LOG_SCALING_MIN_ABS));
                rsum[r] += la;
                csum[M->ci[k]] += la;
                ++ccount[M->ci[k]];
            }
        for (int it = 0; it < iters; ++it) {
            for (int r = 0; r < m; ++r) {
                int b = M->rp[r], e = M->rp[r + 1];
                double s = rsum[r];
                for (int k = b; k < e; ++k) s -= cls[M->ci[k]];
                rls[r] = (e > b) ? s / (double)(e - b) : 0.0;
            }
            for (int blk = 0; blk < P->naff; ++blk) {
                if (!preserving) {
                    if (P->atype[blk] == CONE_PSD) psd_log_projection(rls, P->astart[blk], P->avdim[blk]);
                    continue;
                }
                int st = P->astart[blk], len = cone_len(P->atype[blk], P->avdim[blk]);
                double bsum = 0.0; int bcount = 0;
                for (int r = st; r < st + len; ++r) {
                    int b = M->rp[r], e = M->rp[r + 1];
                    bsum += rsum[r];
                    bcount += e - b;
                    for (int k = b; k < e; ++k) bsum -= cls[M->ci[k]];
                }
                double bl = bcount > 0 ? bsum / (double)bcount : 0.0;
                for (int r = st; r < st + len; ++r) rls[r] = bl;
            }
            memcpy(cs, csum, (size_t)n * sizeof(double));
            for (int r = 0; r < m; ++r)
                for (int k = M->rp[r]; k < M->rp[r + 1]; ++k) cs[M->ci[k]] -= rls[r];
            for (int c = 0; c < n; ++c) cls[c] = ccount[c] > 0 ? cs[c] / (double)ccount[c] : 0.0;
            for (int blk = 0; blk < P->ncones; ++blk) {
                if (!preserving) {
                    if (P->ctype[blk] == CONE_PSD) psd_log_projection(cls, P->cstart[blk], P->cvdim[blk]);
                    continue;
                }
                int st = P->cstart[blk], len = cone_len(P->ctype[blk], P->cvdim[blk]);
                double bsum = 0.0; int bcount = 0;
                for (int c = st; c < st + len; ++c) { bsum += cs[c]; bcount += ccount[c]; }
                double bl = bcount > 0 ? bsum / (double)bcount : 0.0;
                for (int c = st; c < st + len; ++c) cls[c] = bl;
            }
        }
        for (int r = 0; r < m; ++r) cr[r] = cr_exp_clamped(rls[r]);
        for (int c = 0; c < n; ++c) vr[c] = cr_exp_clamped(cls[c]);
        free(rls); free(cls); free(rsum); free(csum); free(cs); free(ccount);
    }
    scale_problem(P, cr, vr);
    for (int r = 0; r < m; ++r) cum_cr[r] *= cr[r];
    for (int c = 0; c < n; ++c) cum_vr[c] *= vr[c];
    free(cr); free(vr);
}

/* ruiz_rescaling, reference src/preconditioner.c:497-556 */
static void ruiz(oprob *P, int iters, int preserving, double *cum_cr, double *cum_vr)
{
    int m = P->m, n = P->n;
    double *cr = dvec(m), *vr = dvec(n);
    for (int it = 0; it < iters; ++it) {
        for (int i = 0; i < n; ++i) vr[i] = 0.0;
        for (int i = 0; i < m; ++i) cr[i] = 0.0;
        for (int r = 0; r < m; ++r)
            for (int k = P->A.rp[r]; k < P->A.rp[r + 1]; ++k) {
                int c = P->A.ci[k];
                double a = fabs(P->A.v[k]);
                if (a > vr[c]) vr[c] = a;
                if (a > cr[r]) cr[r] = a;
            }
        for (int i = 0; i < n; ++i) vr[i] = (vr[i] < SCALING_EPSILON) ? 1.0 : sqrt(vr[i]);
        for (int i = 0; i < m; ++i) cr[i] = (cr[i] < SCALING_EPSILON) ? 1.0 : sqrt(cr[i]);
        cone_scaling_adjust(vr, P->ncones, P->cstart, P->cvdim, P->ctype, 1, preserving);
        cone_scaling_adjust(cr, P->naff, P->astart, P->avdim, P->atype, 1, preserving);
        scale_problem(P, cr, vr);
        for (int i = 0; i < n; ++i) cum_vr[i] *= vr[i];
        for (int i = 0; i < m; ++i) cum_cr[i] *= cr[i];
    }
    free(cr); free(vr);
}

/* pock_chambolle_rescaling, reference src/preconditioner.c:558-600 */
static void pock_chambolle(oprob *P, double alpha, int preserving, double *cum_cr, double *cum_vr)
{
    int m = P->m, n = P->n;
    double *cr = dvec(m), *vr = dvec(n);
    for (int r = 0; r < m; ++r)
        for (int k = P->A.rp[r]; k < P->A.rp[r + 1]; ++k) {
            double a = fabs(P->A.v[k]);
            vr[P->A.ci[k]] += pow(a, 2.0 - alpha);
            cr[r] += pow(a, alpha);
        }
    for (int i = 0; i < n; ++i) vr[i] = (vr[i] < SCALING_EPSILON) ? 1.0 : sqrt(vr[i]);
    for (int i = 0; i < m; ++i) cr[i] = (cr[i] < SCALING_EPSILON) ? 1.0 : sqrt(cr[i]);
    cone_scaling_adjust(vr, P->ncones, P->cstart, P->cvdim, P->ctype, 0, preserving);
    cone_scaling_adjust(cr, P->naff, P->astart, P->avdim, P->atype, 0, preserving);
    scale_problem(P, cr, vr);
    for (int i = 0; i < n; ++i) cum_vr[i] *= vr[i];
    for (int i = 0; i < m; ++i) cum_cr[i] *= cr[i];
    free(cr); free(vr);
}

/* bound_obj_rescaling, reference src/preconditioner.c:602-652 */
static void bound_obj(oprob *P, double *sb, double *sc)
{
    double b2 = 0.0;
    for (int i = 0; i < P->m; ++i) {
        if (isfinite(P->lc[i]) && P->lc[i] != P->uc[i]) b2 += P->lc[i] * P->lc[i];
        if (isfinite(P->uc[i])) b2 += P->uc[i] * P->uc[i];
    }
    for (int i = 0; i < P->m; ++i) b2 += P->g[i] * P->g[i];
    double c2 = 0.0;
    for (int i = 0; i < P->n; ++i) c2 += P->c[i] * P->c[i];
    *sb = 1.0 / (sqrt(b2) + 1.0);
    *sc = 1.0 / (sqrt(c2) + 1.0);
    for (int i = 0; i < P->m; ++i) {
        P->lc[i] *= *sb;
        P->uc[i] *= *sb;
        P->g[i] *= *sb;
    }
    for (int i = 0; i < P->n; ++i) {
        P->l[i] *= *sb;
        P->u[i] *= *sb;
        P->c[i] *= *sc;
    }
    for (int k = 0; k < P->Q.nnz; ++k) P->Q.v[k] *= *sc / *sb;
    if (P->R.nnz > 0) {
        double f = sqrt(*sc / *sb);
        for (int k = 0; k < P->R.nnz; ++k) P->R.v[k] *= f;
    }
}

/* rescale_problem, reference src/preconditioner.c:654-713 */
static void rescale(oprob *P, const pdhg_parameters_t *prm, double *cr, double *vr, double *sb, double *sc)
{
    for (int i = 0; i < P->m; ++i) cr[i] = 1.0;
    for (int i = 0; i < P->n; ++i) vr[i] = 1.0;
    int pres = prm->use_cone_preserving_scaling;
    if (prm->curtis_reid_iterations > 0) curtis_reid(P, prm->curtis_reid_iterations, pres, cr, vr);
    if (prm->l_inf_ruiz_iterations > 0) ruiz(P, prm->l_inf_ruiz_iterations, pres, cr, vr);
    if (prm->has_pock_chambolle_alpha) pock_chambolle(P, prm->pock_chambolle_alpha, pres, cr, vr);
    if (prm->bound_objective_rescaling) bound_obj(P, sb, sc);
    else { *sb = 1.0; *sc = 1.0; }
    /* pin_scaled_fixed_cone_bounds, reference src/preconditioner.c:311-327 */
    if (P->fixed)
        for (int j = 0; j < P->n; ++j) {
            if (!P->fixed[j]) continue;
            double v = (P->primal_start ? P->primal_start[j] : 0.0) * vr[j] * *sb;
            P->l[j] = v;
            P->u[j] = v;
        }
}

int oracle_rescale(const qp_problem_t *prob, const pdhg_parameters_t *params, double *con_rescale,
                   double *var_rescale, double *con_bound_rescale, double *obj_vec_rescale)
{
    oprob P;
    oprob_load(&P, prob);
    double *cr = dvec(P.m), *vr = dvec(P.n);
    rescale(&P, params, cr, vr, con_bound_rescale, obj_vec_rescale);
    memcpy(con_rescale, cr, (size_t)prob->num_constraints * sizeof(double));
    memcpy(var_rescale, vr, (size_t)P.n * sizeof(double));
    free(cr); free(vr);
    oprob_free(&P);
    return 0;
}

/* ------------------------------------------------------------------ */
/* power methods (reference src/pdhg_core_op.cu:1498-1788)            */
/* ------------------------------------------------------------------ */

static double sigma_max_csr(const ocsr *A, const ocsr *At, int max_iter, double tol)
{
    int m = A->rows, n = A->cols;
    double *v = dvec(m), *nv = dvec(m), *dp = dvec(n);
    unsigned int seed = 1234;
    for (int i = 0; i < m; ++i)
        v[i] = ((double)rand_r(&seed) / (double)RAND_MAX) * 2.0 - 1.0;
    double nrm = nrm2(v, m);
    for (int i = 0; i < m; ++i) v[i] *= 1.0 / nrm;
    double s2 = 1.0;
    for (int it = 0; it < max_iter; ++it) {
        spmv(At, v, dp);
        spmv(A, dp, nv);
        s2 = dot(nv, v, m);
        for (int i = 0; i < m; ++i) nv[i] += -s2 * v[i];
        if (nrm2(nv, m) < tol) break;
        for (int i = 0; i < m; ++i) nv[i] += s2 * v[i];
        nrm = nrm2(nv, m);
        double inv = 1.0 / nrm;
        for (int i = 0; i < m; ++i) nv[i] *= inv;
        double *t = v; v = nv; nv = t;
    }
    free(v); free(nv); free(dp);
    return sqrt(s2);
}

double oracle_sigma_max(int m, int n, const int *row_ptr, const int *col_ind, const double *val, int max_iter,
                        double tol)
{
    ocsr A = {m, n, row_ptr[m], (int *)row_ptr, (int *)col_ind, (double *)val}, At;
    csr_transpose(&A, &At);
    double s = sigma_max_csr(&A, &At, max_iter, tol);
    csr_free(&At);
    return s;
}

static double max_eig(const ocsr *Q, int max_iter, double tol)
{
    int n = Q->rows;
    double *v = dvec(n), *av = dvec(n);
    unsigned int seed = 1234;
    for (int i = 0; i < n; ++i) v[i] = (double)rand_r(&seed) / RAND_MAX;
    double lam = 0.0;
    for (int it = 0; it < max_iter; ++it) {
        double nrm = nrm2(v, n), inv = 1.0 / nrm;
        for (int i = 0; i < n; ++i) v[i] *= inv;
        spmv(Q, v, av);
        double old = lam;
        lam = dot(v, av, n);
        if (it > 0 && fabs(lam - old) < tol) break;
        memcpy(v, av, (size_t)n * sizeof(double));
    }
    free(v); free(av);
    return lam;
}

static double min_eig(const ocsr *Q, double lmax, int max_iter, double tol)
{
    int n = Q->rows;
    double *v = dvec(n), *av = dvec(n), *sv = dvec(n);
    unsigned int seed = 1234;
    for (int i = 0; i < n; ++i) v[i] = (double)rand_r(&seed) / RAND_MAX;
    double mu = 0.0;
    for (int it = 0; it < max_iter; ++it) {
        double nrm = nrm2(v, n), inv = 1.0 / nrm;
        for (int i = 0; i < n; ++i) v[i] *= inv;
        spmv(Q, v, av);
        double old = mu;
        for (int i = 0; i < n; ++i) sv[i] = -av[i] + lmax * v[i];
        mu = dot(v, sv, n);
        if (it > 0 && fabs(mu - old) < tol) break;
        memcpy(v, sv, (size_t)n * sizeof(double));
    }
    free(v); free(av); free(sv);
    return lmax - mu;
}

/* ------------------------------------------------------------------ */
/* solver state                                                        */
/* ------------------------------------------------------------------ */

typedef struct {
    int n, m;
    oprob P; /* scaled */
    ocsr At;
    double *cr, *vr, sb, sc;
    double *lc_fin, *uc_fin, *l_fin, *u_fin;
    int qtype; /* quad_obj_type_t */
    double *qdiag;
    int dkind; double *Ddiag, *Ddense;
    double q_norm, nonconvexity;
    double *qx, *Rx, *Rxbuf, *eff;
    int is_lp;
    /* iterates */
    double *x0, *x, *xp, *xr, *Aty, *y0, *y, *yp, *yr, *Ax;
    double *dual_slack, *primal_slack, *dual_residual, *primal_residual, *dx, *dy;
    double step, omega;
    int k;
    int is_major;
    double pw_err_sum, pw_last_err, best_omega, best_gap;
    double cnorm, bnorm;
    double abs_p, rel_p, abs_d, rel_d, pobj, dobj, gap, rel_gap;
    double max_p_ray, max_d_ray, p_ray_obj, d_ray_obj;
    termination_reason_t reason;
    double fpe, fpe0, fpe_last;
    int inner_count;
    int inner_total;
    /* BB */
    int use_bb, precond;
    double *grad, *dir, *pbuf, *diag_h, *m_diag, *m_inv, *Ms;
    double cached_inv_tau, tol_scale, bb_tol, bb_min_tol;
    int bb_limit;
    double *snap;
    double cum_time;
    /* per cone block: warm starts of the section projectors (the step's
     * projections and those of the residual, reference
     * projection_warm_start / residual_warm_start), complementarity */
    double *proj_warm, *res_warm, *compl;
} ostate;

static void project_affine(ostate *S, double *v);


static void apply_middle(ostate *S)
{
    int r = S->P.rank;
    if (S->dkind == 0 || r <= 0) return;
    if (S->dkind == 1) {
        for (int i = 0; i < r; ++i) S->Rx[i] *= S->Ddiag[i];
        return;
    }
    /* cublasDsymv, lower fill mode on the row-major array seen as
     * column-major: entry (i,j) comes from the row-major upper triangle. */
    for (int i = 0; i < r; ++i) {
        double s = 0.0;
        for (int j = 0; j < r; ++j) {
            int a = i < j ? i : j, b = i < j ? j : i;
            s += S->Ddense[(size_t)a * r + b] * S->Rx[j];
        }
        S->Rxbuf[i] = s;
    }
    memcpy(S->Rx, S->Rxbuf, (size_t)r * sizeof(double));
}

/* update_obj_product, reference src/pdhg_core_op.cu:305-413 */
static void update_obj_product(ostate *S, const double *x)
{
    int n = S->n;
    switch (S->qtype) {
    case PDHCG_NON_Q: return;
    case PDHCG_DIAG_Q:
        for (int i = 0; i < n; ++i) S->qx[i] = S->qdiag[i] * x[i];
        break;
    case PDHCG_SPARSE_Q:
        spmv(&S->P.Q, x, S->qx);
        break;
    case PDHCG_LOW_RANK_Q: {
        spmv(&S->P.R, x, S->Rx);
        apply_middle(S);
        ocsr Rt; csr_transpose(&S->P.R, &Rt);
        spmv(&Rt, S->Rx, S->qx);
        csr_free(&Rt);
        break;
    }
    case PDHCG_LOW_RANK_PLUS_SPARSE_Q: {
        spmv(&S->P.Q, x, S->qx);
        spmv(&S->P.R, x, S->Rx);
        apply_middle(S);
        ocsr Rt; csr_transpose(&S->P.R, &Rt);
        double *t = dvec(n);
        spmv(&Rt, S->Rx, t);
        for (int i = 0; i < n; ++i) S->qx[i] += t[i];
        free(t);
        csr_free(&Rt);
        break;
    }
    }
    if (S->eff)
        for (int i = 0; i < n; ++i) S->eff[i] = S->P.c[i] + S->qx[i];
}

/* project_cone_runtime (reference src/cone_dispatch.cu:38-58): blocks with
 * fixed slots take the section projectors, with the warm starts in warm */
static void project_cones_w(ostate *S, double *vec, const double *q, double tau, double *warm)
{
    for (int b = 0; b < S->P.ncones; ++b) {
        int st = S->P.cstart[b];
        int len = cone_len(S->P.ctype[b], S->P.cvdim[b]);
        if (S->P.fixed && oracle_block_has_fixed(S->P.fixed + st, len))
            oracle_section_project(S->P.ctype[b], S->P.cvdim[b], S->P.calpha[b], vec + st, S->vr + st,
                                   q ? q + st : NULL, tau, S->P.fixed + st, warm + b);
        else
            oracle_project_cone_block(S->P.ctype[b], S->P.cvdim[b], S->P.calpha[b], vec + st, S->vr + st,
                                      q ? q + st : NULL, tau);
    }
}

static void project_cones(ostate *S, double *vec, const double *q, double tau)
{
    project_cones_w(S, vec, q, tau, S->proj_warm);
}

static void cone_reflection(ostate *S)
{
    for (int b = 0; b < S->P.ncones; ++b) {
        int st = S->P.cstart[b], len = cone_len(S->P.ctype[b], S->P.cvdim[b]);
        for (int i = st; i < st + len; ++i) S->xr[i] = 2.0 * S->xp[i] - S->x[i];
    }
}

/* primal_BB_step_size_update, reference src/pdhg_core_op.cu:495-669 */
static void bb_update(ostate *S, double tau)
{
    int n = S->n;
    double inv_tau = 1.0 / tau;
    int it = 1;
    double alpha0 = 1.0 / inv_tau;
    if (S->precond && S->cached_inv_tau != inv_tau) {
        double sum = 0.0;
        for (int i = 0; i < n; ++i) {
            double mm = S->diag_h[i] + inv_tau;
            if (mm <= 0.0) mm = 1.0;
            S->m_diag[i] = mm;
            S->m_inv[i] = 1.0 / mm;
            sum += fabs(mm);
        }
        S->cached_inv_tau = inv_tau;
        S->tol_scale = n > 0 ? sqrt(sum / (double)n) : 1.0;
    }
    if (S->precond) alpha0 *= S->tol_scale * S->tol_scale;
    update_obj_product(S, S->x);
    for (int i = 0; i < n; ++i) {
        double g = S->qx[i] + S->P.c[i] - S->Aty[i];
        double nx = S->x[i] - alpha0 * (S->precond ? S->m_inv[i] : 1.0) * g;
        nx = clampd(S->P.l[i], nx, S->P.u[i]);
        S->xp[i] = nx;
        S->grad[i] = g;
        S->dir[i] = nx - S->x[i];
    }
    int cones = S->P.ncones > 0;
    if (cones) {
        project_cones(S, S->xp, NULL, 0.0);
        for (int i = 0; i < n; ++i) S->dir[i] = S->xp[i] - S->x[i];
    }
    double stMs = 0.0, nrm = 0.0;
    while (it < S->bb_limit) {
        if (S->precond) {
            for (int i = 0; i < n; ++i) S->Ms[i] = S->m_diag[i] * S->dir[i];
            stMs = dot(S->dir, S->Ms, n);
            nrm = sqrt(stMs);
        } else {
            nrm = sqrt(dot(S->dir, S->dir, n));
        }
        if (nrm <= S->bb_tol) break;
        update_obj_product(S, S->xp);
        for (int i = 0; i < n; ++i) {
            double last = S->grad[i];
            double cur = S->qx[i] + S->P.c[i] - S->Aty[i] + inv_tau * (S->xp[i] - S->x[i]);
            S->pbuf[i] = cur - last;
            S->grad[i] = cur;
        }
        double tmp = dot(S->dir, S->pbuf, n);
        if (cones) memcpy(S->snap, S->xp, (size_t)n * sizeof(double));
        double alpha = S->precond ? stMs / tmp : (nrm * nrm) / tmp;
        for (int i = 0; i < n; ++i) {
            double cur = S->xp[i];
            double nx = cur - alpha * (S->precond ? S->m_inv[i] : 1.0) * S->grad[i];
            nx = clampd(S->P.l[i], nx, S->P.u[i]);
            S->dir[i] = nx - cur;
            S->xp[i] = nx;
        }
        if (cones) {
            project_cones(S, S->xp, NULL, 0.0);
            for (int i = 0; i < n; ++i) S->dir[i] = S->xp[i] - S->snap[i];
        }
        ++it;
    }
    for (int i = 0; i < n; ++i) S->xr[i] = 2.0 * S->xp[i] - S->x[i];
    S->inner_total += it - 1;
}

/* pdhg_update, reference src/pdhg_core_op.cu:705-830 */
static void pdhg_update(ostate *S)
{
    int n = S->n, m = S->m;
    double tau = S->step / S->omega;
    if (S->nonconvexity < 0) {
        tau = fmax(tau, -1.01 * fmin(0.0, S->nonconvexity));
        tau /= 100;
    }
    double sigma = S->step * S->omega;
    spmv(&S->At, S->y, S->Aty);
    int cones = S->P.ncones > 0;
    int store_rule = ((S->k + 2) % print_frequency(S->k + 2)) == 0;
    if (S->use_bb) {
        bb_update(S, tau);
    } else if (S->qtype == PDHCG_NON_Q) {
        int store = S->is_major || cones || store_rule;
        for (int i = 0; i < n; ++i) {
            double xi = S->x[i];
            double t = xi - tau * (S->P.c[i] - S->Aty[i]);
            double p = clampd(S->P.l[i], t, S->P.u[i]);
            S->xr[i] = 2.0 * p - xi;
            if (store) {
                S->xp[i] = p;
                S->dual_slack[i] = (p - t) / tau;
            }
        }
        if (cones) {
            project_cones(S, S->xp, NULL, 0.0);
            cone_reflection(S);
        }
    } else { /* DIAG_Q without PSD */
        int store = S->is_major || store_rule || cones;
        for (int i = 0; i < n; ++i) {
            double xi = S->x[i];
            double t = (xi - tau * (S->P.c[i] - S->Aty[i])) / (1.0 + tau * S->qdiag[i]);
            double p = clampd(S->P.l[i], t, S->P.u[i]);
            S->xr[i] = 2.0 * p - xi;
            if (store) S->xp[i] = p;
        }
        if (cones) {
            project_cones(S, S->xp, S->qdiag, tau);
            cone_reflection(S);
        }
    }
    S->inner_total++;
    spmv(&S->P.A, S->xr, S->Ax);
    int store_dual = S->is_major || store_rule;
    /* with affine cones the clamped point is projected onto the cones of the
     * affine rows before the update (reference pdhg_update,
     * src/pdhg_core_op.cu:810-829, prepare / finish_constraint_dual_update) */
    double *pr = dvec(m);
    for (int i = 0; i < m; ++i)
        pr[i] = clampd(S->P.lc[i], S->Ax[i] + S->P.g[i] - S->y[i] / sigma, S->P.uc[i]);
    if (S->P.naff > 0) project_affine(S, pr);
    for (int i = 0; i < m; ++i) {
        double cur = S->y[i];
        double v = S->Ax[i] + S->P.g[i];
        double nx = cur - sigma * v + sigma * pr[i];
        if (store_dual) S->yp[i] = nx;
        S->yr[i] = 2.0 * nx - cur;
    }
    free(pr);
}

/* Projection of the affine-cone rows of a row vector v onto their cones in
 * the unit metric of the scaled space, K defined on v / d with d = 1 / cr
 * (the reference's affine coordinate rescaling, src/solver_state.cu:625-638;
 * project_cone_runtime on the affine runtime, src/cone_dispatch.cu:38-57). */
static void project_affine(ostate *S, double *v)
{
    for (int b = 0; b < S->P.naff; ++b) {
        int st = S->P.astart[b], len = cone_len(S->P.atype[b], S->P.avdim[b]);
        double *d = dvec(len);
        for (int i = 0; i < len; ++i) d[i] = 1.0 / S->cr[st + i];
        oracle_project_cone_block(S->P.atype[b], S->P.avdim[b], S->P.aalpha[b], v + st, d, NULL, 0.0);
        free(d);
    }
}

/* halpern_update, reference src/pdhg_core_op.cu:832-845 */
static void halpern(ostate *S, double rho)
{
    double w = (double)(S->inner_count + 1) / (S->inner_count + 2);
    for (int i = 0; i < S->n; ++i) {
        double r = rho * S->xr[i] + (1.0 - rho) * S->x[i];
        S->x[i] = w * r + (1.0 - w) * S->x0[i];
    }
    for (int i = 0; i < S->m; ++i) {
        double r = rho * S->yr[i] + (1.0 - rho) * S->y[i];
        S->y[i] = w * r + (1.0 - w) * S->y0[i];
    }
}

/* compute_fixed_point_error, reference src/pdhg_core_op.cu:973-1035 */
static void fixed_point_error(ostate *S)
{
    for (int i = 0; i < S->n; ++i) S->dx[i] = S->xr[i] - S->x[i];
    for (int i = 0; i < S->m; ++i) S->dy[i] = S->yr[i] - S->y[i];
    spmv(&S->At, S->dy, S->Aty);
    double dn = nrm2(S->dy, S->m), pn = nrm2(S->dx, S->n);
    double movement = pn * pn * S->omega + dn * dn / S->omega;
    double cross = dot(S->Aty, S->dx, S->n);
    double interaction = 2 * S->step * cross;
    S->fpe = sqrt(movement + interaction);
    if (!S->is_lp && S->use_bb)
        S->bb_tol = fmin(S->bb_tol, fmax(0.0005 * pn / S->step * S->omega, S->bb_min_tol));
}

/* cone dual residual + projected-gradient augmentation + cone dual slack,
 * reference src/cone_dispatch.cu:88-154 and src/pdhg_core_op.cu:67-90 */
/* compute_cone_dual_residual, reference src/cone_dispatch.cu:86-108 */
static void cone_dual_residual(ostate *S, const double *eff)
{
    for (int b = 0; b < S->P.ncones; ++b) {
        int st = S->P.cstart[b], len = cone_len(S->P.ctype[b], S->P.cvdim[b]);
        double *rc = dvec(len);
        for (int i = 0; i < len; ++i) rc[i] = eff[st + i] - S->Aty[st + i];
        S->compl[b] = 0.0;
        if (S->P.fixed && oracle_block_has_fixed(S->P.fixed + st, len))
            S->compl[b] = oracle_section_dual_residual(S->P.ctype[b], S->P.cvdim[b], S->P.calpha[b], S->xp + st, rc,
                                                       S->vr + st, S->P.fixed + st, S->res_warm + b,
                                                       S->dual_residual + st);
        else
            oracle_cone_dual_residual_block(S->P.ctype[b], S->P.cvdim[b], S->P.calpha[b], rc, S->vr + st,
                                            S->dual_residual + st);
        free(rc);
    }
}

static void augment_projected_gradient(ostate *S, const double *eff)
{
    int n = S->n;
    double s = S->step / S->omega;
    if (!(s > 0.0) || !isfinite(s)) s = 1.0;
    for (int i = 0; i < n; ++i) {
        double g = eff[i] - S->Aty[i];
        S->dx[i] = clampd(S->P.l[i], S->xp[i] - s * g, S->P.u[i]);
    }
    project_cones_w(S, S->dx, NULL, 0.0, S->res_warm);
    for (int i = 0; i < n; ++i) {
        double r = (S->xp[i] - S->dx[i]) / s * S->vr[i];
        if (!isfinite(r)) r = copysign(INFINITY, r);
        if (fabs(r) > fabs(S->dual_residual[i])) S->dual_residual[i] = r;
    }
}

/* compute_residual, reference src/pdhg_core_op.cu:1037-1294 (affine cones:
 * compute_affine_cone_residuals, :109-212, and
 * src/kernels/pdhcg_affine_cone_kernels.cu) */
static void compute_residual(ostate *S, norm_type_t nt)
{
    int n = S->n, m = S->m;
    spmv(&S->P.A, S->xp, S->Ax);
    spmv(&S->At, S->yp, S->Aty);
    update_obj_product(S, S->xp);
    int cones = S->P.ncones > 0;
    double *pp = dvec(m);
    for (int i = 0; i < m; ++i) {
        pp[i] = clampd(S->P.lc[i], S->Ax[i] + S->P.g[i], S->P.uc[i]);
        S->primal_slack[i] = fmax(S->yp[i], 0.0) * S->lc_fin[i] + fmin(S->yp[i], 0.0) * S->uc_fin[i] -
            S->P.g[i] * S->yp[i];
    }
    if (S->P.naff > 0) project_affine(S, pp); /* affine rows: distance to their cone */
    for (int i = 0; i < m; ++i)
        S->primal_residual[i] = (S->Ax[i] + S->P.g[i] - pp[i]) * S->cr[i];
    free(pp);
    /* affine rows: dual membership proj_K(-y) (zero when y is in the dual
     * cone) in the 1 / cr scaling, and per-block complementarity
     * |y . (A x + g)| / sb */
    double mem_norm = 0.0, compl_norm = 0.0;
    if (S->P.naff > 0) {
        double *mv = dvec(m), *cpl = dvec(S->P.naff);
        for (int b = 0; b < S->P.naff; ++b) {
            int st = S->P.astart[b], len = cone_len(S->P.atype[b], S->P.avdim[b]);
            double d = 0.0;
            for (int i = st; i < st + len; ++i) {
                mv[i] = -S->yp[i];
                d += S->yp[i] * (S->Ax[i] + S->P.g[i]);
            }
            cpl[b] = fabs(d) / S->sb;
        }
        project_affine(S, mv);
        for (int b = 0; b < S->P.naff; ++b) {
            int st = S->P.astart[b], len = cone_len(S->P.atype[b], S->P.avdim[b]);
            for (int i = st; i < st + len; ++i) mv[i] /= S->cr[i];
        }
        mem_norm = vnorm(mv, m, nt);
        compl_norm = vnorm(cpl, S->P.naff, nt);
        free(mv);
        free(cpl);
    }
    if (S->is_lp) {
        for (int i = 0; i < n; ++i)
            S->dual_residual[i] = (S->P.c[i] - S->Aty[i] - S->dual_slack[i]) * S->vr[i];
    } else {
        double tau = S->step / S->omega;
        for (int i = 0; i < n; ++i) {
            double g = S->qx[i] + S->P.c[i] - S->Aty[i];
            double t = S->xp[i] - tau * g;
            double p = fmax(S->P.l[i], fmin(S->P.u[i], t));
            double ds = (p - t) / tau;
            S->dual_residual[i] = (g - ds) * S->vr[i];
            S->dual_slack[i] = ds;
        }
    }
    const double *eff = S->eff ? S->eff : S->P.c;
    if (cones) {
        cone_dual_residual(S, eff);
        augment_projected_gradient(S, eff);
    }
    S->abs_p = vnorm(S->primal_residual, m, nt) / S->sb;
    double lin_abs_p = S->abs_p;
    /* power-cone primal violation (reference compute_power_cone_primal_violation,
     * src/pdhg_core_op.cu:214-250, kernel src/kernels/pdhcg_power_cone_kernels.cu:623-669) */
    double pv_abs = 0.0, pv_rel = 0.0;
    for (int b = 0; cones && b < S->P.ncones; ++b) {
        if (S->P.ctype[b] != CONE_POWER) continue;
        int st = S->P.cstart[b];
        double x = S->xp[st] / S->vr[st], y = S->xp[st + 1] / S->vr[st + 1], z = S->xp[st + 2] / S->vr[st + 2];
        double va, vrel;
        if (!isfinite(x) || !isfinite(y) || !isfinite(z)) {
            va = vrel = INFINITY;
        } else {
            double v = fmax(-x, -y), az = fabs(z);
            int inside = 0;
            if (az > 0.0) {
                double bound = 0.0;
                if (x > 0.0 && y > 0.0) {
                    double a = S->P.calpha[b];
                    double lb = a * log(x) + (1.0 - a) * log(y), lz = log(az);
                    double tol = 64.0 * DBL_EPSILON * (1.0 + fabs(lb) + fabs(lz));
                    if (lb + tol >= lz) inside = 1;
                    else bound = exp(lb);
                }
                if (!inside) v = fmax(v, az - bound);
            }
            va = fmax(v, 0.0);
            vrel = va / (S->sb + fmax(fabs(x), fmax(fabs(y), az)));
        }
        if (nt == NORM_TYPE_L_INF) {
            pv_abs = fmax(pv_abs, va);
            pv_rel = fmax(pv_rel, vrel);
        } else {
            pv_abs += va * va;
            pv_rel += vrel * vrel;
        }
    }
    if (nt != NORM_TYPE_L_INF) {
        pv_abs = sqrt(pv_abs);
        pv_rel = sqrt(pv_rel);
    }
    if (cones)
        S->abs_p = nt == NORM_TYPE_L_INF ? fmax(S->abs_p, pv_abs) : hypot(S->abs_p, pv_abs);
    /* cone complementarity (nonzero only on power blocks with fixed slots),
     * reference compute_cone_complementarity_norm, src/pdhg_core_op.cu:92-100 */
    double ccompl = cones ? vnorm(S->compl, S->P.ncones, nt) : 0.0;
    S->abs_d = vnorm(S->dual_residual, n, nt);
    if (nt == NORM_TYPE_L_INF)
        S->abs_d = fmax(fmax(S->abs_d, ccompl), fmax(mem_norm, compl_norm));
    else
        S->abs_d = sqrt(S->abs_d * S->abs_d + ccompl * ccompl + mem_norm * mem_norm + compl_norm * compl_norm);
    S->abs_d /= S->sc;
    double half_xqx = S->qtype == PDHCG_NON_Q ? 0.0 : 0.5 * dot(S->xp, S->qx, n);
    S->pobj = (dot(S->P.c, S->xp, n) + half_xqx) / (S->sb * S->sc) + S->P.c0;
    if (cones)
        for (int b = 0; b < S->P.ncones; ++b) {
            int st = S->P.cstart[b], len = cone_len(S->P.ctype[b], S->P.cvdim[b]);
            for (int i = st; i < st + len; ++i) S->dual_slack[i] = eff[i] - S->Aty[i];
        }
    double base = dot(S->dual_slack, S->xp, n);
    double ssum = 0.0;
    for (int i = 0; i < m; ++i) ssum += S->primal_slack[i];
    S->dobj = (base + ssum - half_xqx) / (S->sb * S->sc) + S->P.c0;
    S->rel_p = lin_abs_p / (1.0 + S->bnorm);
    if (cones)
        S->rel_p = nt == NORM_TYPE_L_INF ? fmax(S->rel_p, pv_rel) : hypot(S->rel_p, pv_rel);
    double den;
    if (S->is_lp) {
        den = 1.0 + S->cnorm;
    } else {
        for (int i = 0; i < n; ++i) {
            S->Aty[i] *= S->vr[i];
            S->qx[i] *= S->vr[i];
        }
        double qn = vnorm(S->qx, n, nt), an = vnorm(S->Aty, n, nt);
        den = 1.0 + fmax(S->cnorm, fmax(qn / S->sc, an / S->sc));
    }
    S->rel_d = S->abs_d / den;
    S->gap = fabs(S->pobj - S->dobj);
    S->rel_gap = S->gap / (1.0 + fabs(S->pobj) + fabs(S->dobj));
}

/* compute_infeasibility_information, reference src/pdhg_core_op.cu:1296-1429 */
static void infeasibility_info(ostate *S)
{
    int n = S->n, m = S->m;
    for (int i = 0; i < n; ++i) {
        if (isfinite(S->P.l[i])) S->dx[i] = fmax(S->dx[i], 0.0);
        if (isfinite(S->P.u[i])) S->dx[i] = fmin(S->dx[i], 0.0);
    }
    for (int i = 0; i < m; ++i) {
        if (!isfinite(S->P.lc[i])) S->dy[i] = fmin(S->dy[i], 0.0);
        if (!isfinite(S->P.uc[i])) S->dy[i] = fmax(S->dy[i], 0.0);
    }
    double pr = inf_norm(S->dx, n);
    if (pr > 0.0) {
        double sc = 1.0 / pr;
        for (int i = 0; i < n; ++i) S->dx[i] *= sc;
    }
    double dr = inf_norm(S->dy, m);
    spmv(&S->P.A, S->dx, S->Ax);
    spmv(&S->At, S->dy, S->Aty);
    S->p_ray_obj = dot(S->P.c, S->dx, n) / (S->sb * S->sc);
    for (int i = 0; i < m; ++i)
        S->primal_slack[i] = fmax(S->dy[i], 0.0) * S->lc_fin[i] + fmin(S->dy[i], 0.0) * S->uc_fin[i] -
            S->P.g[i] * S->dy[i];
    for (int i = 0; i < n; ++i)
        S->dual_slack[i] = fmax(-S->Aty[i], 0.0) * S->l_fin[i] + fmin(-S->Aty[i], 0.0) * S->u_fin[i];
    double sp = 0.0, sd = 0.0;
    for (int i = 0; i < m; ++i) sp += S->primal_slack[i];
    for (int i = 0; i < n; ++i) sd += S->dual_slack[i];
    S->d_ray_obj = (sp + sd) / (S->sb * S->sc);
    for (int i = 0; i < m; ++i) {
        double pp = S->Ax[i];
        S->primal_slack[i] = (fmax(0.0, -pp) * isfinite(S->P.lc[i]) + fmax(0.0, pp) * isfinite(S->P.uc[i])) * S->cr[i];
    }
    for (int i = 0; i < n; ++i) {
        double dp = -S->Aty[i];
        S->dual_slack[i] = (fmax(0.0, dp) * !isfinite(S->P.l[i]) - fmin(0.0, dp) * !isfinite(S->P.u[i])) * S->vr[i];
    }
    S->max_p_ray = inf_norm(S->primal_slack, m);
    if (!S->is_lp && S->qtype != PDHCG_NON_Q) {
        update_obj_product(S, S->dx);
        double qr = inf_norm(S->qx, n);
        S->max_p_ray = fmax(S->max_p_ray, qr / S->sc);
    }
    double dsn = inf_norm(S->dual_slack, n);
    S->max_d_ray = dsn;
    double f = fmax(dr, dsn);
    if (f > 0.0) {
        S->max_d_ray /= f;
        S->d_ray_obj /= f;
    } else {
        S->max_d_ray = 0.0;
        S->d_ray_obj = 0.0;
    }
}

/* check_termination_criteria, reference src/utils.cu:219-289 */
static void check_termination(ostate *S, const termination_criteria_t *c)
{
    if (S->rel_d < c->eps_feasible_relative && S->rel_p < c->eps_feasible_relative &&
        S->rel_gap < c->eps_optimal_relative) {
        S->reason = TERMINATION_REASON_OPTIMAL;
        return;
    }
    if (S->P.ncones == 0) {
        if (S->d_ray_obj > 0.0 && S->max_d_ray / S->d_ray_obj <= c->eps_infeasible) {
            S->reason = TERMINATION_REASON_PRIMAL_INFEASIBLE;
            return;
        }
        if (S->p_ray_obj < 0.0 && S->max_p_ray / (-S->p_ray_obj) <= c->eps_infeasible) {
            S->reason = TERMINATION_REASON_DUAL_INFEASIBLE;
            return;
        }
    }
    if (S->k >= c->iteration_limit) {
        S->reason = TERMINATION_REASON_ITERATION_LIMIT;
        return;
    }
    if (S->cum_time >= c->time_sec_limit) {
        S->reason = TERMINATION_REASON_TIME_LIMIT;
        return;
    }
}

/* should_do_adaptive_restart, reference src/utils.cu:291-322 */
static int should_restart(ostate *S, const restart_parameters_t *rp, int freq)
{
    int r = 0;
    if (S->k == freq) r = 1;
    else if (S->k > freq) {
        if (S->fpe <= rp->sufficient_reduction_for_restart * S->fpe0) r = 1;
        if (S->fpe <= rp->necessary_reduction_for_restart * S->fpe0 && S->fpe > S->fpe_last) r = 1;
        if (S->inner_count >= rp->artificial_restart_threshold * S->k) r = 1;
    }
    S->fpe_last = S->fpe;
    return r;
}

/* perform_restart, reference src/pdhg_core_op.cu:859-931 */
static void perform_restart(ostate *S, const pdhg_parameters_t *prm)
{
    for (int i = 0; i < S->n; ++i) S->dx[i] = S->xp[i] - S->x0[i];
    for (int i = 0; i < S->m; ++i) S->dy[i] = S->yp[i] - S->y0[i];
    double pd = nrm2(S->dx, S->n), dd = nrm2(S->dy, S->m);
    double ratio = S->rel_d / S->rel_p;
    if (pd > 1e-16 && dd > 1e-16 && pd < 1e12 && dd < 1e12 && ratio > 1e-8 && ratio < 1e8) {
        double err = log(dd) - log(pd) - log(S->omega);
        S->pw_err_sum *= prm->restart_params.i_smooth;
        S->pw_err_sum += err;
        double derr = err - S->pw_last_err;
        S->omega *= exp(prm->restart_params.k_p * err + prm->restart_params.k_i * S->pw_err_sum +
                        prm->restart_params.k_d * derr);
        S->pw_last_err = err;
    } else {
        S->omega = S->best_omega;
        S->pw_err_sum = 0.0;
        S->pw_last_err = 0.0;
    }
    double g = fabs(log10(S->rel_d / S->rel_p));
    if (g < S->best_gap) {
        S->best_gap = g;
        S->best_omega = S->omega;
    }
    memcpy(S->x0, S->xp, (size_t)S->n * sizeof(double));
    memcpy(S->x, S->xp, (size_t)S->n * sizeof(double));
    memcpy(S->y0, S->yp, (size_t)S->m * sizeof(double));
    memcpy(S->y, S->yp, (size_t)S->m * sizeof(double));
    S->inner_count = 0;
    S->fpe_last = INFINITY;
}

/* preprocess_qp_problem (Q type, D kind, diag Q),
 * reference src/preconditioner.c:715-830 and detect_q_type src/utils.cu:834-885 */
static void classify_q(ostate *S)
{
    oprob *P = &S->P;
    int n = P->n, r = P->rank;
    S->dkind = 0;
    if (P->has_D && r > 0) {
        int diag_only = 1;
        for (int i = 0; i < r && diag_only; ++i)
            for (int k = P->D.rp[i]; k < P->D.rp[i + 1]; ++k)
                if (P->D.ci[k] != i) { diag_only = 0; break; }
        if (diag_only) {
            S->dkind = 1;
            S->Ddiag = dvec(r);
            for (int i = 0; i < r; ++i)
                for (int k = P->D.rp[i]; k < P->D.rp[i + 1]; ++k) S->Ddiag[i] = P->D.v[k];
        } else {
            S->dkind = 2;
            S->Ddense = dvec(r * r);
            for (int i = 0; i < r; ++i)
                for (int k = P->D.rp[i]; k < P->D.rp[i + 1]; ++k) S->Ddense[(size_t)i * r + P->D.ci[k]] = P->D.v[k];
        }
    }
    int nnzq = P->Q.rp ? P->Q.nnz : 0;
    int nnzr = P->R.rp ? P->R.nnz : 0;
    if (nnzq == 0 && nnzr == 0) S->qtype = PDHCG_NON_Q;
    else if (nnzr > 0) S->qtype = nnzq > 0 ? PDHCG_LOW_RANK_PLUS_SPARSE_Q : PDHCG_LOW_RANK_Q;
    else {
        S->qtype = PDHCG_DIAG_Q;
        for (int i = 0; i < n && S->qtype == PDHCG_DIAG_Q; ++i)
            for (int k = P->Q.rp[i]; k < P->Q.rp[i + 1]; ++k)
                if (P->Q.ci[k] != i) { S->qtype = PDHCG_SPARSE_Q; break; }
    }
    if (S->qtype == PDHCG_DIAG_Q) {
        S->qdiag = dvec(n);
        for (int i = 0; i < n; ++i)
            for (int k = P->Q.rp[i]; k < P->Q.rp[i + 1]; ++k)
                if (P->Q.ci[k] < n) S->qdiag[P->Q.ci[k]] = P->Q.v[k] + 1e-12;
    }
}

static void state_free(ostate *S)
{
    oprob_free(&S->P);
    csr_free(&S->At);
    double *arrs[] = {S->cr, S->vr, S->lc_fin, S->uc_fin, S->l_fin, S->u_fin, S->qdiag, S->Ddiag, S->Ddense,
                      S->qx, S->Rx, S->Rxbuf, S->eff, S->x0, S->x, S->xp, S->xr, S->Aty, S->y0, S->y, S->yp,
                      S->yr, S->Ax, S->dual_slack, S->primal_slack, S->dual_residual, S->primal_residual, S->dx,
                      S->dy, S->grad, S->dir, S->pbuf, S->diag_h, S->m_diag, S->m_inv, S->Ms, S->snap, S->proj_warm, S->res_warm, S->compl};
    for (size_t i = 0; i < sizeof(arrs) / sizeof(arrs[0]); ++i) free(arrs[i]);
}

/* optimize, reference src/solver.cu:35-210, with initialize_solver_state
 * (src/solver_state.cu:688-1058) and initialize_step_size_and_primal_weight
 * (src/pdhg_core_op.cu:933-971). */
pdhcg_result_t *oracle_solve(const qp_problem_t *prob, const pdhg_parameters_t *params_in)
{
    pdhg_parameters_t prm;
    if (params_in) prm = *params_in;
    else return NULL;
    if (!prob) return NULL;
    if (prob->affine_cones.is_fixed || prob->num_quadratic_constraints > 0) {
        fprintf(stderr, "[oracle] fixed affine slots and quadratic constraints are not restated\n");
        return NULL;
    }
    ostate Sv;
    ostate *S = &Sv;
    memset(S, 0, sizeof(*S));
    oprob_load(&S->P, prob);
    int n = S->P.n, m = S->P.m;
    S->n = n;
    S->m = m;

    /* unscaled norms for relative errors (src/solver_state.cu:854-934) */
    {
        double mx = 0.0, ss = 0.0;
        for (int i = 0; i < n; ++i) {
            if (prm.optimality_norm == NORM_TYPE_L_INF) mx = fmax(mx, fabs(S->P.c[i]));
            else ss += S->P.c[i] * S->P.c[i];
        }
        S->cnorm = prm.optimality_norm == NORM_TYPE_L_INF ? mx : sqrt(ss);
        mx = 0.0; ss = 0.0;
        for (int i = 0; i < m; ++i) {
            double lo = S->P.lc[i], up = S->P.uc[i];
            if (prm.optimality_norm == NORM_TYPE_L_INF) {
                if (isfinite(lo) && lo != up) mx = fmax(mx, fabs(lo));
                if (isfinite(up)) mx = fmax(mx, fabs(up));
            } else {
                if (isfinite(lo) && lo != up) ss += lo * lo;
                if (isfinite(up)) ss += up * up;
            }
        }
        for (int i = 0; i < m; ++i) {
            if (prm.optimality_norm == NORM_TYPE_L_INF) mx = fmax(mx, fabs(S->P.g[i]));
            else ss += S->P.g[i] * S->P.g[i];
        }
        S->bnorm = prm.optimality_norm == NORM_TYPE_L_INF ? mx : sqrt(ss);
    }

    S->cr = dvec(m);
    S->vr = dvec(n);
    rescale(&S->P, &prm, S->cr, S->vr, &S->sb, &S->sc);
    classify_q(S);
    S->is_lp = S->qtype == PDHCG_NON_Q;
    csr_transpose(&S->P.A, &S->At);

    S->x0 = dvec(n); S->x = dvec(n); S->xp = dvec(n); S->xr = dvec(n); S->Aty = dvec(n);
    S->dual_slack = dvec(n); S->dual_residual = dvec(n); S->dx = dvec(n);
    S->y0 = dvec(m); S->y = dvec(m); S->yp = dvec(m); S->yr = dvec(m); S->Ax = dvec(m);
    S->primal_slack = dvec(m); S->primal_residual = dvec(m); S->dy = dvec(m);
    S->qx = dvec(n); S->Rx = dvec(S->P.rank); S->Rxbuf = dvec(S->P.rank);
    if (S->P.primal_start)
        for (int i = 0; i < n; ++i) {
            double v = S->P.primal_start[i] * S->vr[i] * S->sb;
            S->x0[i] = v; S->x[i] = v; S->xp[i] = v;
        }
    if (S->P.dual_start)
        for (int i = 0; i < m; ++i) {
            double v = S->P.dual_start[i] * S->cr[i] * S->sc;
            S->y0[i] = v; S->y[i] = v; S->yp[i] = v;
        }
    S->lc_fin = dvec(m); S->uc_fin = dvec(m); S->l_fin = dvec(n); S->u_fin = dvec(n);
    for (int i = 0; i < m; ++i) {
        S->lc_fin[i] = isfinite(S->P.lc[i]) ? S->P.lc[i] : 0.0;
        S->uc_fin[i] = isfinite(S->P.uc[i]) ? S->P.uc[i] : 0.0;
    }
    for (int i = 0; i < n; ++i) {
        S->l_fin[i] = isfinite(S->P.l[i]) ? S->P.l[i] : 0.0;
        S->u_fin[i] = isfinite(S->P.u[i]) ? S->P.u[i] : 0.0;
    }
    /* cone runtime: effective gradient, interior starting points
     * (src/solver_state.cu:578-686) */
    int cones = S->P.ncones > 0;
    if (cones && S->qtype != PDHCG_NON_Q) S->eff = dvec(n);
    S->proj_warm = dvec(S->P.ncones);
    S->res_warm = dvec(S->P.ncones);
    S->compl = dvec(S->P.ncones);
    const double INV_SQRT2 = 0.7071067811865475;
    for (int b = 0; b < S->P.ncones; ++b) {
        int aux0 = S->P.cstart[b] + S->P.cvdim[b];
        const char *fx = S->P.fixed;
        if (S->P.ctype[b] == CONE_STANDARD_SOC) {
            double wv = -INV_SQRT2 * S->sb * S->vr[aux0];
            double zv = INV_SQRT2 * S->sb * S->vr[aux0 + 1];
            double *d4[4] = {S->x0, S->x, S->xp, S->xr};
            for (int w = 0; w < 4; ++w) {
                if (!(fx && fx[aux0])) d4[w][aux0] = wv;
                if (!(fx && fx[aux0 + 1])) d4[w][aux0 + 1] = zv;
            }
        } else if (S->P.ctype[b] == CONE_ROTATED_SOC) {
            double tv = S->sb * S->vr[aux0 + 1];
            double *d4[4] = {S->x0, S->x, S->xp, S->xr};
            for (int w = 0; w < 4; ++w)
                if (!(fx && fx[aux0 + 1])) d4[w][aux0 + 1] = tv;
        }
    }
    if (cones) project_cones(S, S->x0, NULL, 0.0);
    for (int i = 0; i < n; ++i) S->x0[i] = fmax(S->P.l[i], fmin(S->x0[i], S->P.u[i]));
    memcpy(S->x, S->x0, (size_t)n * sizeof(double));
    memcpy(S->xp, S->x0, (size_t)n * sizeof(double));
    memcpy(S->xr, S->x0, (size_t)n * sizeof(double));

    /* quadratic term information (src/solver_state.cu:380-420) */
    if (S->qtype == PDHCG_SPARSE_Q) {
        S->q_norm = max_eig(&S->P.Q, prm.sv_max_iter, prm.sv_tol);
        S->nonconvexity = min_eig(&S->P.Q, S->q_norm, prm.sv_max_iter, prm.sv_tol);
    } else if (S->qtype == PDHCG_DIAG_Q) {
        double mx = 0.0, mn = 0.0;
        for (int i = 0; i < n; ++i) {
            mx = fmax(mx, fabs(S->qdiag[i]));
            mn = fmin(mn, S->qdiag[i]);
        }
        S->q_norm = mx;
        S->nonconvexity = mn;
    }
    /* inner solver (src/solver_state.cu:280-370): diagonal Q with PSD blocks
     * also takes the BB solve (a nonuniform diagonal metric has no one-EVD
     * PSD prox), without the Jacobi preconditioner (:307, :323) */
    int has_psd = 0;
    for (int b = 0; b < S->P.ncones; ++b)
        has_psd |= S->P.ctype[b] == CONE_PSD;
    S->use_bb = !(S->qtype == PDHCG_NON_Q || (S->qtype == PDHCG_DIAG_Q && !has_psd));
    if (S->use_bb) {
        int lim = prm.inner_solver_parameters.iteration_limit;
        double it0 = prm.inner_solver_parameters.initial_tolerance, mt = prm.inner_solver_parameters.min_tolerance;
        if (lim < 1) lim = 1;
        if (it0 <= 0.0) it0 = 1e-3;
        if (mt <= 0.0) mt = 1e-9;
        S->bb_limit = lim;
        S->bb_tol = it0;
        S->bb_min_tol = mt;
        S->grad = dvec(n); S->dir = dvec(n); S->pbuf = dvec(n);
        if (cones) S->snap = dvec(n);
        S->precond = prm.diag_jacobi_precond && !has_psd;
        if (S->precond) {
            S->diag_h = dvec(n); S->m_diag = dvec(n); S->m_inv = dvec(n); S->Ms = dvec(n);
            S->cached_inv_tau = -1.0;
            S->tol_scale = 1.0;
            if (S->qtype == PDHCG_SPARSE_Q || S->qtype == PDHCG_LOW_RANK_PLUS_SPARSE_Q)
                for (int i = 0; i < n; ++i) {
                    double s = 0.0;
                    for (int k = S->P.Q.rp[i]; k < S->P.Q.rp[i + 1]; ++k)
                        if (S->P.Q.ci[k] == i) s += S->P.Q.v[k];
                    S->diag_h[i] = s;
                }
            if (S->qtype == PDHCG_LOW_RANK_Q || S->qtype == PDHCG_LOW_RANK_PLUS_SPARSE_Q) {
                ocsr Rt; csr_transpose(&S->P.R, &Rt);
                int r = S->P.rank;
                for (int i = 0; i < n; ++i) {
                    double s = 0.0;
                    int b0 = Rt.rp[i], e0 = Rt.rp[i + 1];
                    if (S->dkind == 1) {
                        for (int k = b0; k < e0; ++k) s += S->Ddiag[Rt.ci[k]] * Rt.v[k] * Rt.v[k];
                    } else if (S->dkind == 2) {
                        for (int ka = b0; ka < e0; ++ka)
                            for (int kb = b0; kb < e0; ++kb)
                                s += Rt.v[ka] * Rt.v[kb] * S->Ddense[(size_t)Rt.ci[ka] * r + Rt.ci[kb]];
                    } else {
                        for (int k = b0; k < e0; ++k) s += Rt.v[k] * Rt.v[k];
                    }
                    S->diag_h[i] += s;
                }
                csr_free(&Rt);
            }
        }
    }
    if (S->q_norm != S->q_norm) S->q_norm = 0.0;
    int bb_limit_one = S->nonconvexity < 0;
    if (bb_limit_one) S->bb_limit = 1;

    /* step size and primal weight (src/pdhg_core_op.cu:933-971) */
    if (S->P.A.nnz == 0) S->step = 1.0;
    else {
        double sv = sigma_max_csr(&S->P.A, &S->At, prm.sv_max_iter, prm.sv_tol);
        S->step = sv < 1e-12 ? 1.0 : 0.998 / sv;
    }
    S->omega = prm.bound_objective_rescaling ? 1.0 : (S->cnorm + 1.0) / (S->bnorm + 1.0);
    S->best_omega = S->omega;
    S->best_gap = INFINITY;
    S->fpe_last = INFINITY;
    S->reason = TERMINATION_REASON_UNSPECIFIED;

    double t0 = now_sec();
    int do_restart = 0;
    int freq = prm.termination_evaluation_frequency;
    while (S->k < prm.termination_criteria.iteration_limit) {
        if (S->is_major || S->k == 0 || (S->k % print_frequency(S->k)) == 0) {
            compute_residual(S, prm.optimality_norm);
            if (!cones && S->P.naff == 0 && S->is_major && S->k < 3 * freq) infeasibility_info(S);
            S->cum_time = now_sec() - t0;
            check_termination(S, &prm.termination_criteria);
            if (S->reason != TERMINATION_REASON_UNSPECIFIED) break;
        }
        if (S->is_major || S->k == 0) {
            do_restart = should_restart(S, &prm.restart_params, freq);
            if (do_restart) perform_restart(S, &prm);
        }
        S->is_major = ((S->k + 1) % freq) == 0;
        pdhg_update(S);
        if (S->is_major || do_restart) {
            fixed_point_error(S);
            if (do_restart) {
                S->fpe0 = S->fpe;
                do_restart = 0;
            }
        }
        halpern(S, prm.reflection_coefficient);
        S->inner_count++;
        S->k++;
    }
    if (S->reason == TERMINATION_REASON_UNSPECIFIED) {
        S->reason = TERMINATION_REASON_ITERATION_LIMIT;
        compute_residual(S, prm.optimality_norm);
    }

    /* create_result_from_state, reference src/pdhg_core_op.cu:1431-1496 */
    pdhcg_result_t *res = (pdhcg_result_t *)xcalloc(1, sizeof(pdhcg_result_t));
    spmv(&S->At, S->yp, S->Aty);
    update_obj_product(S, S->xp);
    res->primal_solution = dvec(n);
    res->dual_solution = dvec(m);
    res->reduced_cost = dvec(n);
    for (int i = 0; i < n; ++i) {
        double g = S->P.c[i] + (S->qtype != PDHCG_NON_Q ? S->qx[i] : 0.0);
        double rc = (g - S->Aty[i]) * S->vr[i] / S->sc;
        if (!isfinite(S->P.l[i])) rc = fmin(rc, 0.0);
        if (!isfinite(S->P.u[i])) rc = fmax(rc, 0.0);
        res->reduced_cost[i] = rc;
        res->primal_solution[i] = S->xp[i] / S->vr[i] / S->sb;
    }
    for (int i = 0; i < m; ++i) res->dual_solution[i] = S->yp[i] / S->cr[i] / S->sc;
    res->num_variables = prob->num_variables;
    res->num_constraints = prob->num_constraints;
    res->num_nonzeros = prob->constraint_matrix_num_nonzeros;
    res->total_count = S->k;
    res->total_inner_count = S->inner_total;
    res->cumulative_time_sec = S->cum_time;
    res->relative_primal_residual = S->rel_p;
    res->relative_dual_residual = S->rel_d;
    res->absolute_primal_residual = S->abs_p;
    res->absolute_dual_residual = S->abs_d;
    res->primal_objective_value = S->pobj;
    res->dual_objective_value = S->dobj;
    res->objective_gap = S->gap;
    res->relative_objective_gap = S->rel_gap;
    res->max_primal_ray_infeasibility = S->max_p_ray;
    res->max_dual_ray_infeasibility = S->max_d_ray;
    res->primal_ray_linear_objective = S->p_ray_obj;
    res->dual_ray_objective = S->d_ray_obj;
    res->termination_reason = S->reason;
    state_free(S);
    return res;
}

/* ------------------------------------------------------------------ */
/* one step for kernel-level parity                                    */
/* ------------------------------------------------------------------ */

void oracle_pdhg_step(oracle_step_t *s)
{
    int n = s->n, m = s->m;
    for (int j = 0; j < n; ++j) {
        double acc = 0.0;
        for (int k = s->At_row_ptr[j]; k < s->At_row_ptr[j + 1]; ++k) acc += s->At_val[k] * s->y_cur[s->At_col_ind[k]];
        s->Aty[j] = acc;
    }
    for (int j = 0; j < n; ++j) {
        double xi = s->x_cur[j];
        double t = xi - s->tau * (s->c[j] - s->Aty[j]);
        if (s->q_diag) t /= (1.0 + s->tau * s->q_diag[j]);
        double p = clampd(s->var_lb[j], t, s->var_ub[j]);
        s->x_pdhg[j] = p;
        s->x_refl[j] = 2.0 * p - xi;
    }
    for (int b = 0; b < s->num_cones; ++b) {
        int st = s->cone_start[b];
        int len = cone_len(s->cone_type[b], s->cone_vdim[b]);
        oracle_project_cone_block(s->cone_type[b], s->cone_vdim[b], s->cone_alpha ? s->cone_alpha[b] : 0.0,
                                  s->x_pdhg + st, s->var_rescale + st, s->q_diag ? s->q_diag + st : NULL, s->tau);
        for (int i = st; i < st + len; ++i) s->x_refl[i] = 2.0 * s->x_pdhg[i] - s->x_cur[i];
    }
    for (int i = 0; i < m; ++i) {
        double acc = 0.0;
        for (int k = s->A_row_ptr[i]; k < s->A_row_ptr[i + 1]; ++k) acc += s->A_val[k] * s->x_refl[s->A_col_ind[k]];
        s->Ax[i] = acc;
    }
    for (int i = 0; i < m; ++i) {
        double cur = s->y_cur[i];
        double v = s->Ax[i] + (s->affine_offset ? s->affine_offset[i] : 0.0);
        double pr = clampd(s->con_lb[i], v - cur / s->sigma, s->con_ub[i]);
        double nx = cur - s->sigma * v + s->sigma * pr;
        s->y_pdhg[i] = nx;
        s->y_refl[i] = 2.0 * nx - cur;
    }
    double w = s->halpern_weight, rho = s->reflection;
    for (int j = 0; j < n; ++j) {
        double r = rho * s->x_refl[j] + (1.0 - rho) * s->x_cur[j];
        s->x_cur[j] = w * r + (1.0 - w) * s->x_init[j];
    }
    for (int i = 0; i < m; ++i) {
        double r = rho * s->y_refl[i] + (1.0 - rho) * s->y_cur[i];
        s->y_cur[i] = w * r + (1.0 - w) * s->y_init[i];
    }
}

void oracle_result_free(pdhcg_result_t *r)
{
    if (!r)
        return;
    free(r->primal_solution);
    free(r->dual_solution);
    free(r->reduced_cost);
    free(r);
}
