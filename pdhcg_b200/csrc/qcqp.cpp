// qcqp.cpp -- quadratic constraints rewritten as SOC / rotated-SOC blocks.
//
// Restates the reference transform qcqp_to_socp_qp (src/qcqp_transform.c:
// 96-552) so that the same problem gives the same extended problem, field
// for field, and the result trim restore_qcqp_result_dimensions (:15-58).
//
// Constraint i is a_i . x + x' Q_i x <= b_i (Q_i diagonal, every nonzero
// positive, row one-sided <=), or the same with every nonzero negative and a
// one-sided >= row (negated: "flipped").  With k_i nonzeros it adds k_i
// variables v = sqrt(2 q_jj) x_j (k_i rows -sqrt(2 q_jj) x_j + v_j = 0), two
// auxiliary variables s, t and one cone block [v, s, t]:
//   rotated SOC  (|v|^2 <= 2 s t):  a . x + s = b, and t = 1;
//   standard SOC (|(v, s)| <= t):   sqrt2 (a . x) + s + t = sqrt2 b, and
//                                   -s + t = sqrt2,
// which are x' Q x <= b - a . x in either form.  A constraint without a
// linear part keeps its row with a zero right-hand side, an empty last row,
// and its s, t slots fixed (fixed cone slots) at the values the two forms
// give, with a primal start there.  Variables: n, then per block k_i + 2;
// rows: m, then sum k_i, then one per block.  Q, R and D are copied with Q
// extended by empty rows; c by zeros.
#include "internal.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

template <typename T>
T *copy_array(const T *src, size_t k)
{
    T *p = (T *)std::malloc(std::max<size_t>(k, 1) * sizeof(T));
    if (k)
        std::memcpy(p, src, k * sizeof(T));
    return p;
}

// a copy of a CSR component with `rows` rows (rows past `src_rows` empty)
CsrComponent *copy_csr(const CsrComponent *m, int src_rows, int rows, int nnz)
{
    auto *c = (CsrComponent *)std::calloc(1, sizeof(CsrComponent));
    c->row_ptr = (int *)std::malloc(((size_t)rows + 1) * sizeof(int));
    std::memcpy(c->row_ptr, m->row_ptr, ((size_t)src_rows + 1) * sizeof(int));
    for (int r = src_rows + 1; r <= rows; ++r)
        c->row_ptr[r] = m->row_ptr[src_rows];
    if (nnz > 0) {
        c->col_ind = copy_array(m->col_ind, (size_t)nnz);
        c->val = copy_array(m->val, (size_t)nnz);
    }
    return c;
}

struct Block {
    std::vector<int> cols;
    std::vector<double> root; // sqrt(2 |q_jj|)
    bool flip = false, pinned = false;
    double b = 0.0;
};

} // namespace

extern "C" qp_problem_t *qcqp_to_socp_qp(const qp_problem_t *orig, cone_type_t default_type)
{
    if (!orig)
        return nullptr;
    if (orig->num_quadratic_constraints == 0) {
        std::fprintf(stderr, "[qcqp_to_socp_qp] no quadratic constraints; nothing to do.\n");
        return nullptr;
    }
    if (orig->affine_cones.num_cones > 0) {
        std::fprintf(stderr, "[qcqp_to_socp_qp] native affine cones combined with quadratic constraints "
                             "are not supported by this transform.\n");
        return nullptr;
    }
    const int n = orig->num_variables, m = orig->num_constraints, K = orig->num_quadratic_constraints;
    const bool std_form = default_type == CONE_STANDARD_SOC;
    const double R2 = 1.4142135623730951;
    const CsrComponent *A = orig->constraint_matrix;
    std::vector<Block> blk(K);
    long total_v = 0;
    int num_pin = 0;
    for (int i = 0; i < K; ++i) {
        const CsrComponent *Q = orig->quadratic_constraint_matrices[i];
        int sign = 0;
        bool ok = true;
        for (int r = 0; r < n && ok; ++r)
            for (int k = Q->row_ptr[r]; k < Q->row_ptr[r + 1]; ++k) {
                const double v = Q->val[k];
                if (Q->col_ind[k] != r) {
                    ok = false;
                    break;
                }
                if (v == 0.0)
                    continue;
                const int sg = v > 0.0 ? 1 : -1;
                if (sign != 0 && sg != sign) {
                    ok = false;
                    break;
                }
                sign = sg;
                blk[i].cols.push_back(r);
                blk[i].root.push_back(std::sqrt(2.0 * std::fabs(v)));
            }
        if (!ok) {
            std::fprintf(stderr, "[qcqp_to_socp_qp] Q_%d is non-diagonal or has mixed signs; diagonal PSD (or "
                                 "all-NSD with >= sense) required.\n", i);
            return nullptr;
        }
        const int row = orig->quadratic_constraint_row_indices[i];
        const double lhs = orig->constraint_lower_bound[row], rhs = orig->constraint_upper_bound[row];
        if (sign >= 0) {
            if (std::isfinite(lhs) || !std::isfinite(rhs)) {
                std::fprintf(stderr, "[qcqp_to_socp_qp] QC row %d (Q PSD) requires one-sided <= (lhs=-inf, rhs "
                                     "finite); got lhs=%.3g rhs=%.3g.\n", row, lhs, rhs);
                return nullptr;
            }
            blk[i].b = rhs;
        } else {
            if (!std::isfinite(lhs) || std::isfinite(rhs)) {
                std::fprintf(stderr, "[qcqp_to_socp_qp] QC row %d (Q NSD) requires one-sided >= (lhs finite, rhs="
                                     "+inf); got lhs=%.3g rhs=%.3g.\n", row, lhs, rhs);
                return nullptr;
            }
            blk[i].flip = true;
            blk[i].b = -lhs;
        }
        blk[i].pinned = A->row_ptr[row + 1] == A->row_ptr[row];
        num_pin += blk[i].pinned;
        total_v += (long)blk[i].cols.size();
    }
    const long n_ext = (long)n + total_v + 2L * K, m_ext = (long)m + total_v + K;
    const long per = std_form ? 2 : 1;
    const long nnz_ext = (long)orig->constraint_matrix_num_nonzeros + 2 * per * (K - num_pin) + 2 * total_v;
    if (n_ext > INT32_MAX || m_ext > INT32_MAX || nnz_ext > INT32_MAX) {
        std::fprintf(stderr, "[qcqp_to_socp_qp] extended problem size overflows int32.\n");
        return nullptr;
    }
    auto *out = (qp_problem_t *)std::calloc(1, sizeof(qp_problem_t));
    out->num_variables = (int)n_ext;
    out->num_constraints = (int)m_ext;
    out->num_original_variables = n;
    out->objective_constant = orig->objective_constant;
    out->affine_cone_offset = (double *)std::calloc((size_t)m_ext, sizeof(double));
    std::memcpy(out->affine_cone_offset, orig->affine_cone_offset, (size_t)m * sizeof(double));
    out->objective_vector = (double *)std::calloc((size_t)n_ext, sizeof(double));
    std::memcpy(out->objective_vector, orig->objective_vector, (size_t)n * sizeof(double));
    out->variable_lower_bound = (double *)std::malloc((size_t)n_ext * sizeof(double));
    out->variable_upper_bound = (double *)std::malloc((size_t)n_ext * sizeof(double));
    std::memcpy(out->variable_lower_bound, orig->variable_lower_bound, (size_t)n * sizeof(double));
    std::memcpy(out->variable_upper_bound, orig->variable_upper_bound, (size_t)n * sizeof(double));
    for (long j = n; j < n_ext; ++j) {
        out->variable_lower_bound[j] = -INFINITY;
        out->variable_upper_bound[j] = INFINITY;
    }
    // cone blocks [v, s, t], one per constraint, after the original variables
    out->cones.num_cones = K;
    out->cones.start_idx = (int *)std::malloc((size_t)K * sizeof(int));
    out->cones.v_dim = (int *)std::malloc((size_t)K * sizeof(int));
    out->cones.type = (cone_type_t *)std::malloc((size_t)K * sizeof(cone_type_t));
    {
        long at = n;
        for (int i = 0; i < K; ++i) {
            out->cones.start_idx[i] = (int)at;
            out->cones.v_dim[i] = (int)blk[i].cols.size();
            out->cones.type[i] = default_type;
            at += (long)blk[i].cols.size() + 2;
        }
    }
    // row bounds: constraint rows, then the v rows (= 0), then the last rows
    out->constraint_lower_bound = (double *)std::malloc((size_t)m_ext * sizeof(double));
    out->constraint_upper_bound = (double *)std::malloc((size_t)m_ext * sizeof(double));
    std::memcpy(out->constraint_lower_bound, orig->constraint_lower_bound, (size_t)m * sizeof(double));
    std::memcpy(out->constraint_upper_bound, orig->constraint_upper_bound, (size_t)m * sizeof(double));
    std::vector<int> block_of(m, -1);
    for (int i = 0; i < K; ++i) {
        const int row = orig->quadratic_constraint_row_indices[i];
        block_of[row] = i;
        const double v = blk[i].pinned ? 0.0 : (std_form ? blk[i].b * R2 : blk[i].b);
        out->constraint_lower_bound[row] = out->constraint_upper_bound[row] = v;
    }
    for (long r = m; r < m + total_v; ++r)
        out->constraint_lower_bound[r] = out->constraint_upper_bound[r] = 0.0;
    for (int i = 0; i < K; ++i) {
        const long r = m + total_v + i;
        const double v = blk[i].pinned ? 0.0 : (std_form ? R2 : 1.0);
        out->constraint_lower_bound[r] = out->constraint_upper_bound[r] = v;
    }
    // extended A
    auto *E = (CsrComponent *)std::calloc(1, sizeof(CsrComponent));
    out->constraint_matrix = E;
    out->constraint_matrix_num_nonzeros = (int)nnz_ext;
    E->row_ptr = (int *)std::calloc((size_t)m_ext + 1, sizeof(int));
    E->col_ind = (int *)std::malloc(std::max<long>(nnz_ext, 1) * sizeof(int));
    E->val = (double *)std::malloc(std::max<long>(nnz_ext, 1) * sizeof(double));
    for (int r = 0; r < m; ++r) {
        const int b = block_of[r];
        E->row_ptr[r + 1] = A->row_ptr[r + 1] - A->row_ptr[r] + ((b >= 0 && !blk[b].pinned) ? (int)per : 0);
    }
    {
        long r = m;
        for (int i = 0; i < K; ++i)
            for (size_t j = 0; j < blk[i].cols.size(); ++j)
                E->row_ptr[++r] = 2;
        for (int i = 0; i < K; ++i)
            E->row_ptr[++r] = blk[i].pinned ? 0 : (int)per;
    }
    for (long r = 1; r <= m_ext; ++r)
        E->row_ptr[r] += E->row_ptr[r - 1];
    auto put = [&](long &d, int c, double v) {
        E->col_ind[d] = c;
        E->val[d] = v;
        ++d;
    };
    for (int r = 0; r < m; ++r) {
        long d = E->row_ptr[r];
        const int b = block_of[r];
        const double sgn = (b >= 0 && blk[b].flip) ? -1.0 : 1.0;
        const double scale = (std_form && b >= 0) ? sgn * R2 : sgn;
        for (int k = A->row_ptr[r]; k < A->row_ptr[r + 1]; ++k)
            put(d, A->col_ind[k], scale * A->val[k]);
        if (b >= 0 && !blk[b].pinned) {
            const int aux = out->cones.start_idx[b] + out->cones.v_dim[b];
            put(d, aux, 1.0);
            if (std_form)
                put(d, aux + 1, 1.0);
        }
    }
    {
        long r = m;
        for (int i = 0; i < K; ++i)
            for (size_t j = 0; j < blk[i].cols.size(); ++j, ++r) {
                long d = E->row_ptr[r];
                put(d, blk[i].cols[j], -blk[i].root[j]);
                put(d, out->cones.start_idx[i] + (int)j, 1.0);
            }
        for (int i = 0; i < K; ++i, ++r) {
            if (blk[i].pinned)
                continue;
            long d = E->row_ptr[r];
            const int aux = out->cones.start_idx[i] + out->cones.v_dim[i];
            if (std_form) {
                put(d, aux, -1.0);
                put(d, aux + 1, 1.0);
            } else {
                put(d, aux + 1, 1.0);
            }
        }
    }
    // objective terms
    out->num_rank_lowrank_obj = orig->num_rank_lowrank_obj;
    out->objective_sparse_matrix_num_nonzeros = orig->objective_sparse_matrix_num_nonzeros;
    out->objective_lowrank_matrix_num_nonzeros = orig->objective_lowrank_matrix_num_nonzeros;
    out->objective_lowrank_middle_matrix_num_nonzeros = orig->objective_lowrank_middle_matrix_num_nonzeros;
    if (orig->objective_sparse_matrix)
        out->objective_sparse_matrix =
            copy_csr(orig->objective_sparse_matrix, n, (int)n_ext, orig->objective_sparse_matrix_num_nonzeros);
    const int k = orig->num_rank_lowrank_obj;
    if (orig->objective_lowrank_matrix)
        out->objective_lowrank_matrix =
            copy_csr(orig->objective_lowrank_matrix, k, k, orig->objective_lowrank_matrix_num_nonzeros);
    if (orig->objective_lowrank_middle_matrix)
        out->objective_lowrank_middle_matrix = copy_csr(orig->objective_lowrank_middle_matrix, k, k,
                                                        orig->objective_lowrank_middle_matrix_num_nonzeros);
    // constraints without a linear part: s, t fixed
    if (num_pin > 0) {
        out->cones.fixed_mask_size = (int)n_ext;
        out->cones.is_fixed = (char *)std::calloc((size_t)n_ext, sizeof(char));
        out->primal_start = (double *)std::calloc((size_t)n_ext, sizeof(double));
        for (int i = 0; i < K; ++i) {
            if (!blk[i].pinned)
                continue;
            const int s = out->cones.start_idx[i] + out->cones.v_dim[i], t = s + 1;
            out->cones.is_fixed[s] = out->cones.is_fixed[t] = 1;
            if (std_form) {
                out->primal_start[s] = (blk[i].b - 1.0) * R2 * 0.5;
                out->primal_start[t] = (blk[i].b + 1.0) * R2 * 0.5;
            } else {
                out->primal_start[s] = blk[i].b;
                out->primal_start[t] = 1.0;
            }
        }
    }
    return out;
}

// Trim a result of the extended problem to the original sizes.
void pdhcg_b200_restore_qcqp_result(pdhcg_result_t *r, const qp_problem_t *orig)
{
    if (!r || !orig)
        return;
    const int n = orig->num_variables, m = orig->num_constraints;
    auto trim = [](double *&a, int k) {
        if (!a)
            return;
        double *t = k > 0 ? copy_array(a, (size_t)k) : nullptr;
        std::free(a);
        a = t;
    };
    if (n >= 0 && n < r->num_variables) {
        trim(r->primal_solution, n);
        trim(r->reduced_cost, n);
        r->num_variables = n;
    }
    if (m >= 0 && m < r->num_constraints) {
        trim(r->dual_solution, m);
        r->num_constraints = m;
    }
    r->num_nonzeros = orig->constraint_matrix_num_nonzeros;
}
