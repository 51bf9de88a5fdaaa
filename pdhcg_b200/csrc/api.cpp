// api.cpp -- host side of the PDHCG C interface: problem building,
// validation, warm starts, fixed cone slots, defaults and deallocation.
//
// Semantics follow the reference so that a qp_problem_t built here is
// field-for-field what the reference builds from the same inputs
// (reference src/pdhcg.c:35-666, src/cone_utils.c:26-211,
// src/utils.cu:324-368, 591-833).  The solve itself lives in solver.cu.

#include <cfloat>
#include <climits>
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.h"

namespace {

void *xmalloc(size_t n)
{
    void *p = std::malloc(n ? n : 1);
    if (!p) {
        std::perror("pdhcg_b200: malloc failed");
        std::abort();
    }
    return p;
}
void *xcalloc(size_t c, size_t n)
{
    void *p = std::calloc(c ? c : 1, n ? n : 1);
    if (!p) {
        std::perror("pdhcg_b200: calloc failed");
        std::abort();
    }
    return p;
}

void csr_release(CsrComponent *c)
{
    if (!c)
        return;
    std::free(c->row_ptr);
    std::free(c->col_ind);
    std::free(c->val);
    std::memset(c, 0, sizeof(*c));
}

// ---- matrix descriptor checks (reference src/pdhcg.c:35-168) -------------
// The two compressed formats are one check over a view: a pointer array
// over the major dimension spanning [0, nnz], and minor indices in range.
// The messages are the reference's (callers match on them).
struct CompressedView {
    const char *fmt;        // "CSR" / "CSC"
    const char *ptrs;       // "row pointers" / "column pointers"
    const char *major;      // "row" / "column"
    const char *minor;      // "column" / "row"
    int nmajor, nminor, nnz;
    const int *ptr, *idx;
    const double *vals;
};

int check_compressed(const CompressedView &v, const char *name)
{
    if (v.nnz < 0 || !v.ptr || (v.nnz > 0 && (!v.idx || !v.vals))) {
        std::fprintf(stderr, "[create_qp_problem] %s %s storage is incomplete.\n", name, v.fmt);
        return -1;
    }
    if (v.ptr[0] != 0 || v.ptr[v.nmajor] != v.nnz) {
        std::fprintf(stderr, "[create_qp_problem] %s %s %s do not span [0, nnz].\n", name, v.fmt, v.ptrs);
        return -1;
    }
    for (int r = 0; r < v.nmajor; ++r)
        if (v.ptr[r] > v.ptr[r + 1] || v.ptr[r] < 0 || v.ptr[r + 1] > v.nnz) {
            std::fprintf(stderr, "[create_qp_problem] %s %s %s are invalid at %s %d.\n", name, v.fmt, v.ptrs,
                         v.major, r);
            return -1;
        }
    for (int k = 0; k < v.nnz; ++k)
        if (v.idx[k] < 0 || v.idx[k] >= v.nminor) {
            std::fprintf(stderr, "[create_qp_problem] %s %s %s index %d is out of range [0, %d).\n", name, v.fmt,
                         v.minor, v.idx[k], v.nminor);
            return -1;
        }
    return 0;
}

int check_descriptor(const matrix_desc_t *d, const char *name)
{
    if (!d)
        return 0;
    if (d->m < 0 || d->n < 0) {
        std::fprintf(stderr, "[create_qp_problem] %s matrix has negative shape (%d, %d).\n", name, d->m, d->n);
        return -1;
    }
    switch (d->fmt) {
    case matrix_csr: {
        const auto &c = d->data.csr;
        return check_compressed({"CSR", "row pointers", "row", "column", d->m, d->n, c.nnz, c.row_ptr, c.col_ind,
                                 c.vals},
                                name);
    }
    case matrix_csc: {
        const auto &c = d->data.csc;
        return check_compressed({"CSC", "column pointers", "column", "row", d->n, d->m, c.nnz, c.col_ptr, c.row_ind,
                                 c.vals},
                                name);
    }
    case matrix_dense:
        if (d->m > 0 && d->n > INT_MAX / d->m) {
            std::fprintf(stderr, "[create_qp_problem] %s dense matrix is too large to index with int.\n", name);
            return -1;
        }
        if (d->m > 0 && d->n > 0 && !d->data.dense.A) {
            std::fprintf(stderr, "[create_qp_problem] %s dense matrix data is NULL.\n", name);
            return -1;
        }
        return 0;
    case matrix_coo: {
        const auto &c = d->data.coo;
        if (c.nnz < 0 || (c.nnz > 0 && (!c.row_ind || !c.col_ind || !c.vals))) {
            std::fprintf(stderr, "[create_qp_problem] %s COO storage is incomplete.\n", name);
            return -1;
        }
        for (int k = 0; k < c.nnz; ++k)
            if (c.row_ind[k] < 0 || c.row_ind[k] >= d->m || c.col_ind[k] < 0 || c.col_ind[k] >= d->n) {
                std::fprintf(stderr,
                             "[create_qp_problem] %s COO index (%d, %d) is out of range for shape (%d, %d).\n", name,
                             c.row_ind[k], c.col_ind[k], d->m, d->n);
                return -1;
            }
        return 0;
    }
    default:
        std::fprintf(stderr, "[create_qp_problem] %s matrix has unsupported format %d.\n", name, (int)d->fmt);
        return -1;
    }
}

// ---- format conversion to CSR (reference src/utils.cu:591-833) -----------
// Dense: entries with |a| > tol kept, tol defaults to 1e-12 when not given.
int dense_to_csr(const matrix_desc_t *d, CsrComponent *out, int *nnz_out)
{
    int m = d->m, n = d->n;
    double tol = d->zero_tolerance > 0 ? d->zero_tolerance : 1e-12;
    const double *A = d->data.dense.A;
    int nnz = 0;
    for (long long i = 0; i < (long long)m * n; ++i)
        if (std::fabs(A[i]) > tol)
            ++nnz;
    out->row_ptr = (int *)xmalloc((size_t)(m + 1) * sizeof(int));
    out->col_ind = (int *)xmalloc((size_t)nnz * sizeof(int));
    out->val = (double *)xmalloc((size_t)nnz * sizeof(double));
    int z = 0;
    for (int i = 0; i < m; ++i) {
        out->row_ptr[i] = z;
        for (int j = 0; j < n; ++j) {
            double v = A[(size_t)i * n + j];
            if (std::fabs(v) > tol) {
                out->col_ind[z] = j;
                out->val[z] = v;
                ++z;
            }
        }
    }
    out->row_ptr[m] = z;
    *nnz_out = z;
    return 0;
}

// CSC / COO: bucket by row, stable in input order; zero tolerance 0 keeps all.
int triplets_to_csr(int m, int n, int count, const int *rows, const int *cols_or_null, const int *colptr_or_null,
                    const double *vals, double tol, CsrComponent *out, int *nnz_out, const char *fmt)
{
    std::vector<int> rowcount(m + 1, 0);
    int kept = 0;
    auto col_of = [&](int k, int col_from_ptr) { return cols_or_null ? cols_or_null[k] : col_from_ptr; };
    // pass 1: count
    if (colptr_or_null) {
        for (int j = 0; j < n; ++j)
            for (int k = colptr_or_null[j]; k < colptr_or_null[j + 1]; ++k) {
                int r = rows[k];
                if (r < 0 || r >= m) {
                    std::fprintf(stderr, "[interface] %s: row index out of range\n", fmt);
                    return -1;
                }
                if (tol > 0 && std::fabs(vals[k]) <= tol)
                    continue;
                ++rowcount[r + 1];
                ++kept;
            }
    } else {
        for (int k = 0; k < count; ++k) {
            if (tol > 0 && std::fabs(vals[k]) <= tol)
                continue;
            int r = rows[k];
            if (r < 0 || r >= m) {
                std::fprintf(stderr, "[interface] %s: row index out of range\n", fmt);
                return -1;
            }
            ++rowcount[r + 1];
            ++kept;
        }
    }
    for (int i = 0; i < m; ++i)
        rowcount[i + 1] += rowcount[i];
    out->row_ptr = (int *)xmalloc((size_t)(m + 1) * sizeof(int));
    std::memcpy(out->row_ptr, rowcount.data(), (size_t)(m + 1) * sizeof(int));
    out->col_ind = (int *)xmalloc((size_t)kept * sizeof(int));
    out->val = (double *)xmalloc((size_t)kept * sizeof(double));
    std::vector<int> next(rowcount.begin(), rowcount.end() - 1);
    auto place = [&](int k, int c) -> int {
        if (c < 0 || c >= n) {
            std::fprintf(stderr, "[interface] %s: col index out of range\n", fmt);
            return -1;
        }
        int p = next[rows[k]]++;
        out->col_ind[p] = c;
        out->val[p] = vals[k];
        return 0;
    };
    if (colptr_or_null) {
        for (int j = 0; j < n; ++j)
            for (int k = colptr_or_null[j]; k < colptr_or_null[j + 1]; ++k) {
                if (tol > 0 && std::fabs(vals[k]) <= tol)
                    continue;
                if (place(k, j))
                    return -1;
            }
    } else {
        for (int k = 0; k < count; ++k) {
            if (tol > 0 && std::fabs(vals[k]) <= tol)
                continue;
            if (place(k, col_of(k, 0)))
                return -1;
        }
    }
    *nnz_out = kept;
    return 0;
}

int desc_to_csr(const matrix_desc_t *d, const char *name, CsrComponent *out, int *nnz)
{
    int rc = 0;
    double tol = d->zero_tolerance > 0 ? d->zero_tolerance : 0.0;
    switch (d->fmt) {
    case matrix_dense:
        rc = dense_to_csr(d, out, nnz);
        break;
    case matrix_csc:
        rc = triplets_to_csr(d->m, d->n, d->data.csc.nnz, d->data.csc.row_ind, nullptr, d->data.csc.col_ptr,
                             d->data.csc.vals, tol, out, nnz, "CSC");
        break;
    case matrix_coo:
        rc = triplets_to_csr(d->m, d->n, d->data.coo.nnz, d->data.coo.row_ind, d->data.coo.col_ind, nullptr,
                             d->data.coo.vals, tol, out, nnz, "COO");
        break;
    case matrix_csr: {
        int k = d->data.csr.nnz;
        out->row_ptr = (int *)xmalloc((size_t)(d->m + 1) * sizeof(int));
        std::memcpy(out->row_ptr, d->data.csr.row_ptr, (size_t)(d->m + 1) * sizeof(int));
        if (k > 0) {
            out->col_ind = (int *)xmalloc((size_t)k * sizeof(int));
            out->val = (double *)xmalloc((size_t)k * sizeof(double));
            std::memcpy(out->col_ind, d->data.csr.col_ind, (size_t)k * sizeof(int));
            std::memcpy(out->val, d->data.csr.vals, (size_t)k * sizeof(double));
        }
        *nnz = k;
        break;
    }
    default:
        rc = -1;
    }
    if (rc != 0) {
        std::fprintf(stderr, "[create_qp_problem] failed to convert %s matrix to CSR.\n", name);
        csr_release(out);
    }
    return rc;
}

int append_rows(const matrix_desc_t *d, const char *name, int cur_rows, CsrComponent *dst, int *nnz)
{
    if (!d)
        return 0;
    CsrComponent conv{};
    const int *rp, *ci;
    const double *v;
    int add;
    if (d->fmt == matrix_csr) {
        rp = d->data.csr.row_ptr;
        ci = d->data.csr.col_ind;
        v = d->data.csr.vals;
        add = d->data.csr.nnz;
    } else {
        if (desc_to_csr(d, name, &conv, &add) != 0)
            return -1;
        rp = conv.row_ptr;
        ci = conv.col_ind;
        v = conv.val;
    }
    if (add > INT_MAX - *nnz) {
        std::fprintf(stderr, "[create_qp_problem] combined A and F matrices have too many nonzeros.\n");
        csr_release(&conv);
        return -1;
    }
    int base = *nnz, total = base + add;
    size_t rows = (size_t)cur_rows + (size_t)d->m;
    dst->row_ptr = (int *)std::realloc(dst->row_ptr, (rows + 1) * sizeof(int));
    for (int r = 1; r <= d->m; ++r)
        dst->row_ptr[cur_rows + r] = base + rp[r];
    if (add > 0) {
        dst->col_ind = (int *)std::realloc(dst->col_ind, (size_t)total * sizeof(int));
        dst->val = (double *)std::realloc(dst->val, (size_t)total * sizeof(double));
        std::memcpy(dst->col_ind + base, ci, (size_t)add * sizeof(int));
        std::memcpy(dst->val + base, v, (size_t)add * sizeof(double));
    }
    *nnz = total;
    csr_release(&conv);
    return 0;
}

double *fill_or_copy(int n, const double *src, double fill)
{
    double *d = (double *)xmalloc((size_t)n * sizeof(double));
    if (src)
        std::memcpy(d, src, (size_t)n * sizeof(double));
    else
        for (int i = 0; i < n; ++i)
            d[i] = fill;
    return d;
}

} // namespace

// ---- cone metadata (reference src/cone_utils.c:26-211) -------------------
int pdhcg_b200_cone_length(cone_type_t type, int v_dim)
{
    if (type == CONE_EXPONENTIAL || type == CONE_POWER)
        return 3;
    if (type == CONE_STANDARD_SOC || type == CONE_ROTATED_SOC)
        return v_dim >= 0 && v_dim <= INT_MAX - 2 ? v_dim + 2 : -1;
    if (type == CONE_PSD && v_dim > 0) {
        long long len = (long long)v_dim * (v_dim + 1LL) / 2LL;
        return len <= INT_MAX ? (int)len : -1;
    }
    return -1;
}

// Length of cone block i (reference cone_block_length, src/cone_utils.c:40-45);
// exported under the reference's name because its Python binding calls it.
extern "C" int cone_block_length(const cone_blocks_t *b, int i)
{
    if (!b || i < 0 || i >= b->num_cones || !b->type || !b->v_dim)
        return -1;
    return pdhcg_b200_cone_length(b->type[i], b->v_dim[i]);
}

static void cones_release(cone_blocks_t *b)
{
    if (!b)
        return;
    std::free(b->start_idx);
    std::free(b->v_dim);
    std::free(b->type);
    std::free(b->power_alpha);
    std::free(b->is_fixed);
    std::memset(b, 0, sizeof(*b));
}

static int cones_from_specs(cone_blocks_t *b, int num, const cone_spec_t *specs, int ambient, bool allow_fixed,
                            const char *label)
{
    if (num < 0 || ambient < 0 || (num > 0 && !specs)) {
        std::fprintf(stderr,
                     "[create_qp_problem] Invalid %s cone metadata (num_cones=%d, ambient_dimension=%d, specs=%p).\n",
                     label, num, ambient, (const void *)specs);
        return -1;
    }
    cones_release(b);
    if (num == 0)
        return 0;
    std::vector<char> owner((size_t)ambient, 0);
    bool any_fixed = false, any_power = false;
    for (int c = 0; c < num; ++c) {
        int len = pdhcg_b200_cone_length(specs[c].type, specs[c].v_dim);
        int st = specs[c].start_idx;
        if (len <= 0 || st < 0 || (long long)st + len > ambient) {
            std::fprintf(stderr,
                         "[create_qp_problem] %s cone %d has invalid type, size, or range (start=%d, length=%d, "
                         "ambient_dimension=%d).\n",
                         label, c, st, len, ambient);
            return -1;
        }
        if (!allow_fixed && specs[c].is_fixed) {
            std::fprintf(stderr, "[create_qp_problem] %s cone %d does not support fixed slots.\n", label, c);
            return -1;
        }
        if (specs[c].type == CONE_PSD && specs[c].is_fixed) {
            for (int s = 0; s < len; ++s)
                if (specs[c].is_fixed[s]) {
                    std::fprintf(stderr, "[create_qp_problem] %s PSD cone %d does not support fixed slots.\n", label,
                                 c);
                    return -1;
                }
        }
        if (specs[c].type == CONE_POWER && !(std::isfinite(specs[c].power_alpha) && specs[c].power_alpha > 0.0 &&
                                             specs[c].power_alpha < 1.0)) {
            std::fprintf(stderr, "[create_qp_problem] %s power cone %d requires alpha in (0,1); got %.6g.\n", label, c,
                         specs[c].power_alpha);
            return -1;
        }
        for (int i = st; i < st + len; ++i) {
            if (owner[i]) {
                std::fprintf(stderr, "[create_qp_problem] %s cone %d overlaps at index %d.\n", label, c, i);
                return -1;
            }
            owner[i] = 1;
        }
        any_fixed |= specs[c].is_fixed != nullptr;
        any_power |= specs[c].type == CONE_POWER;
    }
    b->num_cones = num;
    b->start_idx = (int *)xmalloc((size_t)num * sizeof(int));
    b->v_dim = (int *)xmalloc((size_t)num * sizeof(int));
    b->type = (cone_type_t *)xmalloc((size_t)num * sizeof(cone_type_t));
    b->power_alpha = any_power ? (double *)xcalloc((size_t)num, sizeof(double)) : nullptr;
    if (any_fixed) {
        b->fixed_mask_size = ambient;
        b->is_fixed = (char *)xcalloc((size_t)ambient, sizeof(char));
    }
    for (int c = 0; c < num; ++c) {
        int len = pdhcg_b200_cone_length(specs[c].type, specs[c].v_dim);
        b->start_idx[c] = specs[c].start_idx;
        b->v_dim[c] = (specs[c].type == CONE_EXPONENTIAL || specs[c].type == CONE_POWER) ? 1 : specs[c].v_dim;
        b->type[c] = specs[c].type;
        if (b->power_alpha && specs[c].type == CONE_POWER)
            b->power_alpha[c] = specs[c].power_alpha;
        if (b->is_fixed && specs[c].is_fixed)
            for (int s = 0; s < len; ++s)
                b->is_fixed[specs[c].start_idx + s] = specs[c].is_fixed[s] ? 1 : 0;
    }
    return 0;
}

static void cones_clone(cone_blocks_t *dst, const cone_blocks_t *src)
{
    cones_release(dst);
    dst->num_cones = src->num_cones;
    if (src->num_cones <= 0)
        return;
    size_t k = (size_t)src->num_cones;
    dst->start_idx = (int *)xmalloc(k * sizeof(int));
    dst->v_dim = (int *)xmalloc(k * sizeof(int));
    dst->type = (cone_type_t *)xmalloc(k * sizeof(cone_type_t));
    std::memcpy(dst->start_idx, src->start_idx, k * sizeof(int));
    std::memcpy(dst->v_dim, src->v_dim, k * sizeof(int));
    std::memcpy(dst->type, src->type, k * sizeof(cone_type_t));
    if (src->power_alpha) {
        dst->power_alpha = (double *)xmalloc(k * sizeof(double));
        std::memcpy(dst->power_alpha, src->power_alpha, k * sizeof(double));
    }
    if (src->is_fixed && src->fixed_mask_size > 0) {
        dst->fixed_mask_size = src->fixed_mask_size;
        dst->is_fixed = (char *)xmalloc((size_t)src->fixed_mask_size);
        std::memcpy(dst->is_fixed, src->is_fixed, (size_t)src->fixed_mask_size);
    }
}

static CsrComponent *csr_clone(const CsrComponent *src, size_t rows, size_t nnz)
{
    if (!src)
        return nullptr;
    if (!src->row_ptr && nnz == 0)
        return nullptr;
    CsrComponent *c = (CsrComponent *)xcalloc(1, sizeof(CsrComponent));
    c->row_ptr = (int *)xcalloc(rows + 1, sizeof(int));
    c->col_ind = (int *)xmalloc(nnz * sizeof(int));
    c->val = (double *)xmalloc(nnz * sizeof(double));
    std::memcpy(c->row_ptr, src->row_ptr, (rows + 1) * sizeof(int));
    if (nnz > 0) {
        std::memcpy(c->col_ind, src->col_ind, nnz * sizeof(int));
        std::memcpy(c->val, src->val, nnz * sizeof(double));
    }
    return c;
}

// Deep copy of a qp_problem_t (reference deepcopy_problem, src/preconditioner.c:165-252).
qp_problem_t *pdhcg_b200_problem_clone(const qp_problem_t *p)
{
    qp_problem_t *q = (qp_problem_t *)xcalloc(1, sizeof(qp_problem_t));
    q->num_variables = p->num_variables;
    q->num_constraints = p->num_constraints;
    q->constraint_matrix_num_nonzeros = p->constraint_matrix_num_nonzeros;
    q->objective_sparse_matrix_num_nonzeros = p->objective_sparse_matrix_num_nonzeros;
    q->objective_lowrank_matrix_num_nonzeros = p->objective_lowrank_matrix_num_nonzeros;
    q->objective_constant = p->objective_constant;
    q->num_rank_lowrank_obj = p->num_rank_lowrank_obj;
    size_t vb = (size_t)p->num_variables * sizeof(double), cb = (size_t)p->num_constraints * sizeof(double);
    q->variable_lower_bound = (double *)xmalloc(vb);
    q->variable_upper_bound = (double *)xmalloc(vb);
    q->objective_vector = (double *)xmalloc(vb);
    q->constraint_lower_bound = (double *)xmalloc(cb);
    q->constraint_upper_bound = (double *)xmalloc(cb);
    q->affine_cone_offset = (double *)xmalloc(cb);
    std::memcpy(q->variable_lower_bound, p->variable_lower_bound, vb);
    std::memcpy(q->variable_upper_bound, p->variable_upper_bound, vb);
    std::memcpy(q->objective_vector, p->objective_vector, vb);
    if (cb) {
        std::memcpy(q->constraint_lower_bound, p->constraint_lower_bound, cb);
        std::memcpy(q->constraint_upper_bound, p->constraint_upper_bound, cb);
        std::memcpy(q->affine_cone_offset, p->affine_cone_offset, cb);
    }
    q->constraint_matrix = csr_clone(p->constraint_matrix, p->num_constraints, p->constraint_matrix_num_nonzeros);
    q->objective_sparse_matrix =
        csr_clone(p->objective_sparse_matrix, p->num_variables, p->objective_sparse_matrix_num_nonzeros);
    q->objective_lowrank_matrix =
        csr_clone(p->objective_lowrank_matrix, p->num_rank_lowrank_obj, p->objective_lowrank_matrix_num_nonzeros);
    q->objective_lowrank_middle_matrix = csr_clone(p->objective_lowrank_middle_matrix, p->num_rank_lowrank_obj,
                                                   p->objective_lowrank_middle_matrix_num_nonzeros);
    q->objective_lowrank_middle_matrix_num_nonzeros = p->objective_lowrank_middle_matrix_num_nonzeros;
    if (p->primal_start) {
        q->primal_start = (double *)xmalloc(vb);
        std::memcpy(q->primal_start, p->primal_start, vb);
    }
    if (p->dual_start) {
        q->dual_start = (double *)xmalloc(cb);
        std::memcpy(q->dual_start, p->dual_start, cb);
    }
    q->num_original_variables = p->num_original_variables;
    cones_clone(&q->cones, &p->cones);
    cones_clone(&q->affine_cones, &p->affine_cones);
    return q;
}

extern "C" {

void qp_problem_free(qp_problem_t *p)
{
    if (!p)
        return;
    csr_release(p->objective_sparse_matrix);
    std::free(p->objective_sparse_matrix);
    csr_release(p->objective_lowrank_matrix);
    std::free(p->objective_lowrank_matrix);
    csr_release(p->constraint_matrix);
    std::free(p->constraint_matrix);
    std::free(p->variable_lower_bound);
    std::free(p->variable_upper_bound);
    std::free(p->objective_vector);
    std::free(p->constraint_lower_bound);
    std::free(p->constraint_upper_bound);
    std::free(p->affine_cone_offset);
    std::free(p->primal_start);
    std::free(p->dual_start);
    csr_release(p->objective_lowrank_middle_matrix);
    std::free(p->objective_lowrank_middle_matrix);
    if (p->quadratic_constraint_matrices) {
        for (int i = 0; i < p->num_quadratic_constraints; ++i) {
            csr_release(p->quadratic_constraint_matrices[i]);
            std::free(p->quadratic_constraint_matrices[i]);
        }
        std::free(p->quadratic_constraint_matrices);
    }
    std::free(p->quadratic_constraint_row_indices);
    std::free(p->quadratic_constraint_matrix_num_nonzeros);
    cones_release(&p->cones);
    cones_release(&p->affine_cones);
    std::memset(p, 0, sizeof(*p));
    std::free(p);
}

qp_problem_t *create_qp_problem(const double *objective_c, const matrix_desc_t *Q_desc, const matrix_desc_t *R_desc,
                                const matrix_desc_t *D_desc, const matrix_desc_t *A_desc, const double *con_lb,
                                const double *con_ub, const double *var_lb, const double *var_ub,
                                const double *objective_constant, int num_var_cones, const cone_spec_t *var_cones,
                                const matrix_desc_t *F_desc, const double *affine_offset, int num_affine_cones,
                                const cone_spec_t *affine_cones)
{
    qp_problem_t *prob = (qp_problem_t *)xcalloc(1, sizeof(qp_problem_t));
    int n = 0, m = 0, p = 0;
    if (!F_desc && (affine_offset || num_affine_cones != 0 || affine_cones)) {
        std::fprintf(stderr, "[create_qp_problem] affine cone data requires affine_cone_matrix_desc.\n");
        goto failure;
    }
    // shapes (reference src/pdhcg.c:170-230)
    if (!A_desc && !F_desc && !Q_desc && !R_desc) {
        std::fprintf(stderr, "[create_qp_problem] at least one of A, F, Q, or R must be provided.\n");
        goto failure;
    }
    if (check_descriptor(A_desc, "A") || check_descriptor(F_desc, "F") || check_descriptor(Q_desc, "Q") ||
        check_descriptor(R_desc, "R"))
        goto failure;
    n = A_desc ? A_desc->n : (F_desc ? F_desc->n : (Q_desc ? Q_desc->n : R_desc->n));
    m = A_desc ? A_desc->m : 0;
    p = F_desc ? F_desc->m : 0;
    if (F_desc && F_desc->n != n) {
        std::fprintf(stderr, "[create_qp_problem] F matrix shape (%d, %d) must have %d columns.\n", F_desc->m,
                     F_desc->n, n);
        goto failure;
    }
    if (Q_desc && (Q_desc->m != n || Q_desc->n != n)) {
        std::fprintf(stderr, "[create_qp_problem] Q matrix shape (%d, %d) must be (%d, %d).\n", Q_desc->m, Q_desc->n,
                     n, n);
        goto failure;
    }
    if (R_desc && R_desc->n != n) {
        std::fprintf(stderr, "[create_qp_problem] R matrix shape (%d, %d) must have %d columns.\n", R_desc->m,
                     R_desc->n, n);
        goto failure;
    }
    if (D_desc && R_desc && R_desc->m > 0) {
        int rank = R_desc->m;
        if (check_descriptor(D_desc, "D") != 0 || D_desc->m != rank || D_desc->n != rank) {
            std::fprintf(stderr, "[create_qp_problem] D matrix shape (%d, %d) must be (%d, %d).\n", D_desc->m,
                         D_desc->n, rank, rank);
            goto failure;
        }
    }
    if (p > INT_MAX - m) {
        std::fprintf(stderr, "[create_qp_problem] combined A and F matrices have too many rows.\n");
        goto failure;
    }

    prob->num_variables = n;
    prob->num_constraints = m + p;
    prob->affine_cone_offset =
        prob->num_constraints > 0 ? (double *)xcalloc((size_t)prob->num_constraints, sizeof(double)) : nullptr;
    prob->constraint_matrix = (CsrComponent *)xcalloc(1, sizeof(CsrComponent));
    if (A_desc) {
        if (desc_to_csr(A_desc, "A", prob->constraint_matrix, &prob->constraint_matrix_num_nonzeros) != 0)
            goto failure;
    } else {
        prob->constraint_matrix->row_ptr = (int *)xcalloc((size_t)m + 1, sizeof(int));
        prob->constraint_matrix_num_nonzeros = 0;
    }
    if (append_rows(F_desc, "F", m, prob->constraint_matrix, &prob->constraint_matrix_num_nonzeros) != 0)
        goto failure;

    prob->objective_sparse_matrix = (CsrComponent *)xcalloc(1, sizeof(CsrComponent));
    if (Q_desc) {
        if (desc_to_csr(Q_desc, "Q", prob->objective_sparse_matrix, &prob->objective_sparse_matrix_num_nonzeros) != 0)
            goto failure;
    } else {
        prob->objective_sparse_matrix->row_ptr = (int *)xcalloc((size_t)n + 1, sizeof(int));
        prob->objective_sparse_matrix_num_nonzeros = 0;
    }
    prob->objective_lowrank_matrix = (CsrComponent *)xcalloc(1, sizeof(CsrComponent));
    prob->num_rank_lowrank_obj = 0;
    if (R_desc) {
        prob->num_rank_lowrank_obj = R_desc->m;
        if (desc_to_csr(R_desc, "R", prob->objective_lowrank_matrix, &prob->objective_lowrank_matrix_num_nonzeros) !=
            0)
            goto failure;
    } else {
        prob->objective_lowrank_matrix->row_ptr = (int *)xcalloc(1, sizeof(int));
        prob->objective_lowrank_matrix_num_nonzeros = 0;
    }
    prob->objective_lowrank_middle_matrix = nullptr;
    prob->objective_lowrank_middle_matrix_num_nonzeros = 0;
    if (D_desc) {
        if (prob->num_rank_lowrank_obj <= 0)
            std::fprintf(stderr, "[interface] D matrix ignored: problem has no low-rank component.\n");
        else {
            prob->objective_lowrank_middle_matrix = (CsrComponent *)xcalloc(1, sizeof(CsrComponent));
            if (desc_to_csr(D_desc, "D", prob->objective_lowrank_middle_matrix,
                            &prob->objective_lowrank_middle_matrix_num_nonzeros) != 0)
                goto failure;
        }
    }
    prob->objective_constant = objective_constant ? *objective_constant : 0.0;
    prob->objective_vector = fill_or_copy(n, objective_c, 0.0);
    prob->variable_lower_bound = fill_or_copy(n, var_lb, -INFINITY);
    prob->variable_upper_bound = fill_or_copy(n, var_ub, INFINITY);
    prob->constraint_lower_bound = fill_or_copy(prob->num_constraints, nullptr, -INFINITY);
    prob->constraint_upper_bound = fill_or_copy(prob->num_constraints, nullptr, INFINITY);
    if (m > 0 && con_lb)
        std::memcpy(prob->constraint_lower_bound, con_lb, (size_t)m * sizeof(double));
    if (m > 0 && con_ub)
        std::memcpy(prob->constraint_upper_bound, con_ub, (size_t)m * sizeof(double));

    // affine cones: indices are rows of F, shifted past the scalar rows
    // (reference src/pdhcg.c:331-363)
    if (cones_from_specs(&prob->affine_cones, num_affine_cones, affine_cones, p, false, "affine") != 0)
        goto failure;
    {
        int covered = 0;
        for (int c = 0; c < num_affine_cones; ++c) {
            covered += cone_block_length(&prob->affine_cones, c);
            prob->affine_cones.start_idx[c] += m;
        }
        if (covered != p) {
            std::fprintf(stderr, "[create_qp_problem] affine cone blocks cover %d of %d rows of F.\n", covered, p);
            goto failure;
        }
        if (affine_offset && p > 0)
            std::memcpy(prob->affine_cone_offset + m, affine_offset, (size_t)p * sizeof(double));
    }
    if (cones_from_specs(&prob->cones, num_var_cones, var_cones, n, true, "variable") != 0)
        goto failure;
    {
        // cone slots must be free (reference src/pdhcg.c:468-503)
        int n_orig = n;
        for (int c = 0; c < prob->cones.num_cones; ++c) {
            int st = prob->cones.start_idx[c], len = cone_block_length(&prob->cones, c);
            for (int v = st; v < st + len; ++v) {
                double lo = prob->variable_lower_bound[v], hi = prob->variable_upper_bound[v];
                bool lo_fin = std::isfinite(lo) && lo > -1e30, hi_fin = std::isfinite(hi) && hi < 1e30;
                if (lo_fin || hi_fin) {
                    std::fprintf(stderr,
                                 "[create_qp_problem] cone %d slot %d has a finite box bound (lb=%.6g, ub=%.6g); cone "
                                 "variables must be free. Introduce an auxiliary x_cone with x_cone = x_box and put "
                                 "the box on the non-cone copy.\n",
                                 c, v, lo, hi);
                    goto failure;
                }
            }
            if (st < n_orig)
                n_orig = st;
        }
        if (prob->cones.num_cones > 0)
            prob->num_original_variables = n_orig;
    }
    return prob;

failure:
    qp_problem_free(prob);
    return nullptr;
}

void set_start_values(qp_problem_t *prob, const double *primal, const double *dual)
{
    if (!prob)
        return;
    int n = prob->num_variables, m = prob->num_constraints;
    if (primal && prob->cones.is_fixed && prob->primal_start) {
        for (int i = 0; i < n; ++i)
            if (prob->cones.is_fixed[i] && primal[i] != prob->primal_start[i]) {
                std::fprintf(stderr,
                             "[set_start_values] slot %d is fixed at %.17g but caller provided %.17g; rejecting (use "
                             "set_cone_fixed to change fixed value).\n",
                             i, prob->primal_start[i], primal[i]);
                return;
            }
    }
    double *np_ = nullptr, *nd = nullptr;
    if (primal) {
        np_ = (double *)xmalloc((size_t)n * sizeof(double));
        std::memcpy(np_, primal, (size_t)n * sizeof(double));
    } else if (prob->cones.is_fixed && prob->primal_start) {
        np_ = (double *)xcalloc((size_t)n, sizeof(double));
        for (int i = 0; i < n; ++i)
            if (prob->cones.is_fixed[i])
                np_[i] = prob->primal_start[i];
    }
    if (dual) {
        nd = (double *)xmalloc((size_t)m * sizeof(double));
        std::memcpy(nd, dual, (size_t)m * sizeof(double));
    }
    std::free(prob->primal_start);
    std::free(prob->dual_start);
    prob->primal_start = np_;
    prob->dual_start = nd;
}

int set_cone_fixed(qp_problem_t *prob, int cone_idx, int slot, double value)
{
    if (!prob) {
        std::fprintf(stderr, "[set_cone_fixed] prob is NULL\n");
        return -1;
    }
    if (cone_idx < 0 || cone_idx >= prob->cones.num_cones) {
        std::fprintf(stderr, "[set_cone_fixed] cone_idx %d out of range [0, %d)\n", cone_idx, prob->cones.num_cones);
        return -1;
    }
    if (prob->cones.type[cone_idx] == CONE_PSD) {
        std::fprintf(stderr, "[set_cone_fixed] fixed PSD cone sections are not supported.\n");
        return -1;
    }
    int len = cone_block_length(&prob->cones, cone_idx);
    if (slot < 0 || slot >= len) {
        std::fprintf(stderr, "[set_cone_fixed] slot %d out of range [0, %d) for cone %d\n", slot, len, cone_idx);
        return -1;
    }
    int idx = prob->cones.start_idx[cone_idx] + slot;
    if (idx < 0 || idx >= prob->num_variables) {
        std::fprintf(stderr, "[set_cone_fixed] computed index %d out of range [0, %d)\n", idx, prob->num_variables);
        return -1;
    }
    if (!std::isfinite(value)) {
        std::fprintf(stderr, "[set_cone_fixed] fixed value must be finite; got %.17g\n", value);
        return -1;
    }
    if (!prob->cones.is_fixed) {
        prob->cones.is_fixed = (char *)xcalloc((size_t)prob->num_variables, sizeof(char));
        prob->cones.fixed_mask_size = prob->num_variables;
    }
    prob->cones.is_fixed[idx] = 1;
    if (!prob->primal_start)
        prob->primal_start = (double *)xcalloc((size_t)prob->num_variables, sizeof(double));
    prob->primal_start[idx] = value;
    return 0;
}

// Is the fixed exponential section {(x, y, z) : y e^{x/y} <= z} closure,
// with the fixed coordinates at their values, nonempty?  (reference
// fixed_exp_section_is_nonempty, src/pdhcg.c:682-727)
static bool exp_section_nonempty(bool fx, bool fy, bool fz, double x, double y, double z)
{
    if ((fx && !std::isfinite(x)) || (fy && !std::isfinite(y)) || (fz && !std::isfinite(z)))
        return false;
    if (fy) {
        if (y < 0.0)
            return false;
        if (y == 0.0) // only the closure's face {x <= 0, z >= 0}
            return (!fx || x <= 0.0) && (!fz || z >= 0.0);
        if (fz && !(z > 0.0))
            return false;
        if (fx && fz) {
            const double lb = std::log(y) + x / y, lz = std::log(z);
            return lb <= lz + 64.0 * DBL_EPSILON * (1.0 + std::fabs(lb) + std::fabs(lz));
        }
        return true;
    }
    if (!fz)
        return true;
    if (z < 0.0)
        return false;
    if (z == 0.0)
        return !fx || x <= 0.0;
    if (!fx || x <= 0.0)
        return true;
    // the smallest y e^{x/y} over y > 0 is e x for x > 0
    const double lmin = 1.0 + std::log(x), lz = std::log(z);
    return lmin <= lz + 64.0 * DBL_EPSILON * (1.0 + std::fabs(lmin) + std::fabs(lz));
}

// Checks the fixed slots of the variable cones: a mask of the problem's
// size, finite values, and a nonempty section through them in every block
// (reference pdhcg_validate_fixed_cone_sections, src/pdhcg.c:729-892, with
// its messages).  0 when valid or without fixed slots, -1 otherwise.
int pdhcg_b200_validate_fixed_sections(const qp_problem_t *prob)
{
    if (!prob || !prob->cones.is_fixed)
        return 0;
    if (prob->cones.fixed_mask_size != prob->num_variables) {
        std::fprintf(stderr, "[solve_qp_problem] variable cone fixed mask has size %d; expected %d.\n",
                     prob->cones.fixed_mask_size, prob->num_variables);
        return -1;
    }
    const char *fx = prob->cones.is_fixed;
    auto val = [&](int j) { return prob->primal_start ? prob->primal_start[j] : 0.0; };
    for (int c = 0; c < prob->cones.num_cones; ++c) {
        const int st = prob->cones.start_idx[c], vd = prob->cones.v_dim[c];
        const int len = cone_block_length(&prob->cones, c);
        bool any = false;
        for (int i = 0; i < len; ++i)
            any |= fx[st + i] != 0;
        if (!any)
            continue;
        const cone_type_t t = prob->cones.type[c];
        if (t == CONE_EXPONENTIAL) {
            if (!exp_section_nonempty(fx[st], fx[st + 1], fx[st + 2], val(st), val(st + 1), val(st + 2))) {
                std::fprintf(stderr,
                             "[solve_qp_problem] exponential cone %d has an empty or non-finite fixed section.\n", c);
                return -1;
            }
            continue;
        }
        if (t == CONE_STANDARD_SOC || t == CONE_ROTATED_SOC) {
            const bool std_soc = t == CONE_STANDARD_SOC;
            for (int i = 0; i < vd + 2; ++i)
                if (fx[st + i] && !std::isfinite(val(st + i))) {
                    std::fprintf(stderr, "[solve_qp_problem] %s SOC %d has a non-finite fixed value.\n",
                                 std_soc ? "standard" : "rotated", c);
                    return -1;
                }
            // norm of the fixed vector slots (v and, for the standard cone, w)
            double fnorm = 0.0;
            for (int i = 0; i < (std_soc ? vd + 1 : vd); ++i)
                if (fx[st + i])
                    fnorm = std::hypot(fnorm, val(st + i));
            if (std_soc) {
                const int zi = st + vd + 1;
                const double z = val(zi);
                if (fx[zi] && (!(z >= 0.0) || fnorm > z)) {
                    std::fprintf(stderr,
                                 "[solve_qp_problem] standard SOC %d has an empty fixed section "
                                 "(fixed vector norm=%.17g, fixed z=%.17g).\n",
                                 c, fnorm, z);
                    return -1;
                }
                continue;
            }
            const int si = st + vd, ti = si + 1;
            const bool fs = fx[si] != 0, ft = fx[ti] != 0;
            const double sv = val(si), tv = val(ti);
            bool empty = (fs && sv < 0.0) || (ft && tv < 0.0);
            if (!empty && fs && ft)
                empty = fnorm > 1.41421356237309504880 * std::sqrt(sv) * std::sqrt(tv);
            else if (fs && sv == 0.0)
                empty |= fnorm > 0.0;
            else if (ft && tv == 0.0)
                empty |= fnorm > 0.0;
            if (empty) {
                std::fprintf(stderr,
                             "[solve_qp_problem] rotated SOC %d has an empty fixed section "
                             "(fixed vector norm=%.17g, s=%.17g%s, t=%.17g%s).\n",
                             c, fnorm, sv, fs ? " fixed" : "", tv, ft ? " fixed" : "");
                return -1;
            }
            continue;
        }
        if (t != CONE_POWER)
            continue;
        const bool f0 = fx[st] != 0, f1 = fx[st + 1] != 0, f2 = fx[st + 2] != 0;
        const double x = val(st), y = val(st + 1), z = val(st + 2);
        if ((f0 && (!std::isfinite(x) || x < 0.0)) || (f1 && (!std::isfinite(y) || y < 0.0)) ||
            (f2 && !std::isfinite(z))) {
            std::fprintf(stderr,
                         "[solve_qp_problem] power cone %d has an invalid fixed value "
                         "(x=%.17g%s, y=%.17g%s, z=%.17g%s).\n",
                         c, x, f0 ? " fixed" : "", y, f1 ? " fixed" : "", z, f2 ? " fixed" : "");
            return -1;
        }
        if (f2 && z != 0.0 && ((f0 && x == 0.0) || (f1 && y == 0.0))) {
            std::fprintf(stderr,
                         "[solve_qp_problem] power cone %d has an empty fixed section: "
                         "|z| is positive while a fixed nonnegative axis is zero.\n",
                         c);
            return -1;
        }
        if (f0 && f1 && f2 && z != 0.0) {
            const double a = prob->cones.power_alpha[c];
            const double lb = (x > 0.0 && y > 0.0) ? a * std::log(x) + (1.0 - a) * std::log(y) : -INFINITY;
            const double lz = std::log(std::fabs(z));
            if (lb + 64.0 * DBL_EPSILON * (1.0 + std::fabs(lb) + std::fabs(lz)) < lz) {
                std::fprintf(stderr,
                             "[solve_qp_problem] power cone %d has an infeasible fully fixed point "
                             "(x=%.17g, y=%.17g, z=%.17g, alpha=%.17g).\n",
                             c, x, y, z, a);
                return -1;
            }
        }
    }
    return 0;
}

void set_default_parameters(pdhg_parameters_t *p)
{
    std::memset(p, 0, sizeof(*p));
    p->curtis_reid_iterations = 0;
    p->l_inf_ruiz_iterations = 10;
    p->has_pock_chambolle_alpha = true;
    p->pock_chambolle_alpha = 1.0;
    p->bound_objective_rescaling = true;
    p->use_cone_preserving_scaling = true;
    p->verbose = 1;
    p->termination_evaluation_frequency = 200;
    p->feasibility_polishing = false;
    p->reflection_coefficient = 1.0;
    p->presolve = false;
    p->sv_max_iter = 5000;
    p->sv_tol = 1e-4;
    p->termination_criteria.eps_optimal_relative = 1e-4;
    p->termination_criteria.eps_feasible_relative = 1e-4;
    p->termination_criteria.eps_infeasible = 1e-12;
    p->termination_criteria.time_sec_limit = 3600.0;
    p->termination_criteria.iteration_limit = INT32_MAX;
    p->termination_criteria.eps_feas_polish_relative = 1e-6;
    p->restart_params.artificial_restart_threshold = 0.36;
    p->restart_params.sufficient_reduction_for_restart = 0.2;
    p->restart_params.necessary_reduction_for_restart = 0.8;
    p->restart_params.k_p = 0.99;
    p->restart_params.k_i = 0.01;
    p->restart_params.k_d = 0.0;
    p->restart_params.i_smooth = 0.3;
    p->optimality_norm = NORM_TYPE_L_INF;
    p->inner_solver_parameters.iteration_limit = 1000;
    p->inner_solver_parameters.initial_tolerance = 1e-3;
    p->inner_solver_parameters.min_tolerance = 1e-9;
    p->grid_size.decided = false;
    p->partition_method = NNZ_BALANCE_PARTITION;
    p->permute_method = BLOCK_RANDOM_PERMUTATION;
    p->diag_jacobi_precond = true;
    p->default_cone_type = CONE_ROTATED_SOC;
}

void pdhcg_result_free(pdhcg_result_t *r)
{
    if (!r)
        return;
    std::free(r->primal_solution);
    std::free(r->dual_solution);
    std::free(r->reduced_cost);
    std::free(r);
}

pdhcg_result_t *solve_qp_problem_distributed(const pdhg_parameters_t *params, const qp_problem_t *original_problem)
{
    (void)params;
    (void)original_problem;
    std::fprintf(stderr, "[interface] distributed support is not enabled in this build.\n");
    return nullptr;
}

} // extern "C"
