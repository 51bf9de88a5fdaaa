// mps.cpp -- MPS / QPS reader (plain or gzip) producing a qp_problem_t.
//
// Restates the reference reader read_mps_file (src/mps_parser.c:420-682,
// declared in include/mps_parser.h:27) so that the same file gives the same
// problem, field for field:
//   - lines starting with '*' and blank lines are skipped; a line is split
//     on blanks into at most six tokens; a line of one token starting with a
//     letter opens a section (ROWS, COLUMNS, RHS, RANGES, BOUNDS, OBJSENSE,
//     QUADOBJ, QMATRIX, ENDATA; any other such token closes the current
//     one), "QCMATRIX <row>" opens the quadratic block of a row;
//   - ROWS: the first N row is the objective (the first row when there is
//     none); other N rows are dropped; L / G / E rows become constraints in
//     file order with bounds (-inf, 0], [0, inf), [0, 0];
//   - COLUMNS: a line with an odd token count starts a column, an even one
//     continues the last; 'MARKER' lines are skipped; entries of unknown
//     rows are dropped; objective entries add up;
//   - RHS: pairs after the set name; the objective's value gives the
//     constant -value; L rows set the upper bound, G the lower, E both;
//   - RANGES: G [rhs, rhs + |R|], L [rhs - |R|, rhs], E [rhs, rhs + R] for
//     R >= 0 and [rhs + R, rhs] otherwise;
//   - BOUNDS: LO, UP, FX, FR, MI, PL, BV (other types are ignored);
//     variables default to [0, inf);
//   - QUADOBJ entries (upper triangle) are mirrored, QMATRIX entries are
//     taken as given; zero values and unknown names are skipped;
//   - QCMATRIX entries go to the row's quadratic constraint (the objective
//     row's to Q), not mirrored;
//   - a data line under OBJSENSE whose first token is MAX or MAXIMIZE
//     negates c, the constant, Q and the quadratic constraints.  A line of
//     that one token alone is taken as a section header first (it starts
//     with a letter), as in the reference, so it leaves the sense at
//     minimize;
//   - CSR rows keep the file order of their entries; duplicates stay.
// The layout of the result is the one qp_problem_free releases.
#include "internal.h"

#include <zlib.h>

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

// Line source over a plain or gzip file.
struct LineReader {
    gzFile gz = nullptr;
    FILE *f = nullptr;
    explicit LineReader(const char *name)
    {
        const size_t n = std::strlen(name);
        if (n > 3 && std::strcmp(name + n - 3, ".gz") == 0)
            gz = gzopen(name, "rb");
        else
            f = std::fopen(name, "r");
    }
    ~LineReader()
    {
        if (gz)
            gzclose(gz);
        if (f)
            std::fclose(f);
    }
    bool ok() const { return gz || f; }
    bool next(char *buf, int size)
    {
        if (gz)
            return gzgets(gz, buf, size) != nullptr;
        return std::fgets(buf, size, f) != nullptr;
    }
};

struct Coo {
    std::vector<int> r, c;
    std::vector<double> v;
    void add(int i, int j, double x)
    {
        r.push_back(i);
        c.push_back(j);
        v.push_back(x);
    }
};

// COO -> CSR with `rows` rows, entries of a row in COO order.
CsrComponent *to_csr(const Coo &m, int rows)
{
    auto *csr = (CsrComponent *)std::calloc(1, sizeof(CsrComponent));
    csr->row_ptr = (int *)std::calloc((size_t)rows + 1, sizeof(int));
    const size_t nnz = m.v.size();
    if (nnz == 0)
        return csr;
    csr->col_ind = (int *)std::malloc(nnz * sizeof(int));
    csr->val = (double *)std::malloc(nnz * sizeof(double));
    for (size_t k = 0; k < nnz; ++k)
        csr->row_ptr[m.r[k] + 1]++;
    for (int i = 0; i < rows; ++i)
        csr->row_ptr[i + 1] += csr->row_ptr[i];
    std::vector<int> pos(csr->row_ptr, csr->row_ptr + rows);
    for (size_t k = 0; k < nnz; ++k) {
        const int d = pos[m.r[k]]++;
        csr->col_ind[d] = m.c[k];
        csr->val[d] = m.v[k];
    }
    return csr;
}

double *copy_out(const std::vector<double> &v)
{
    double *p = (double *)std::malloc(std::max<size_t>(v.size(), 1) * sizeof(double));
    if (!v.empty())
        std::memcpy(p, v.data(), v.size() * sizeof(double));
    return p;
}

enum Section { NONE, ROWS, COLUMNS, RHS, RANGES, BOUNDS, OBJSENSE, QUADOBJ, QMATRIX, QCMATRIX, ENDATA };

struct Parser {
    // rows as listed, resolved when ROWS ends
    std::vector<std::pair<char, std::string>> listed;
    bool rows_done = false;
    std::string obj_row;
    bool has_obj = false;
    std::unordered_map<std::string, int> row_of, col_of;
    std::vector<char> row_type;
    std::vector<double> lc, uc;
    // columns
    std::string cur_col;
    bool has_col = false;
    std::vector<double> c, lb, ub;
    Coo A, Q;
    double obj_const = 0.0;
    bool maximize = false;
    // quadratic constraints: row index and entries, in order of first use
    std::vector<std::pair<int, Coo>> qc;
    int qc_cur = -1;
    bool qc_obj = false;

    int row(const char *name) const
    {
        auto it = row_of.find(name);
        return it == row_of.end() ? -1 : it->second;
    }
    int col(const char *name) const
    {
        auto it = col_of.find(name);
        return it == col_of.end() ? -1 : it->second;
    }
    bool is_obj(const char *name) const { return has_obj && obj_row == name; }

    void finish_rows()
    {
        if (rows_done)
            return;
        rows_done = true;
        int oi = -1;
        for (size_t i = 0; i < listed.size(); ++i)
            if (listed[i].first == 'N') {
                oi = (int)i;
                break;
            }
        if (oi < 0 && !listed.empty())
            oi = 0;
        if (oi >= 0) {
            obj_row = listed[oi].second;
            has_obj = true;
        }
        for (size_t i = 0; i < listed.size(); ++i) {
            const char t = listed[i].first;
            if ((int)i == oi || !(t == 'E' || t == 'L' || t == 'G'))
                continue;
            if (row_of.count(listed[i].second))
                continue; // a repeated name keeps its first row
            row_of.emplace(listed[i].second, (int)row_type.size());
            row_type.push_back(t);
            lc.push_back(t == 'L' ? -INFINITY : 0.0);
            uc.push_back(t == 'G' ? INFINITY : 0.0);
        }
    }

    void columns(char **tk, int nt)
    {
        if (nt < 2 || std::strcmp(tk[1], "'MARKER'") == 0)
            return;
        int first = 0;
        if (nt % 2 != 0) {
            cur_col = tk[0];
            has_col = true;
            first = 1;
        } else if (!has_col) {
            std::fprintf(stderr, "ERROR: Column data found before any column name was defined.\n");
            error = true;
            return;
        }
        int j = col(cur_col.c_str());
        if (j < 0) {
            j = (int)c.size();
            col_of.emplace(cur_col, j);
            c.push_back(0.0);
            lb.push_back(0.0);
            ub.push_back(INFINITY);
        }
        for (int k = first; k + 1 < nt; k += 2) {
            const double v = std::atof(tk[k + 1]);
            if (is_obj(tk[k])) {
                c[j] += v;
            } else {
                const int i = row(tk[k]);
                if (i >= 0)
                    A.add(i, j, v);
            }
        }
    }

    void rhs(char **tk, int nt)
    {
        for (int k = 1; k + 1 < nt; k += 2) {
            const double v = std::atof(tk[k + 1]);
            if (is_obj(tk[k])) {
                obj_const = -v;
                continue;
            }
            const int i = row(tk[k]);
            if (i < 0)
                continue;
            if (row_type[i] == 'L')
                uc[i] = v;
            else if (row_type[i] == 'G')
                lc[i] = v;
            else
                lc[i] = uc[i] = v;
        }
    }

    void ranges(char **tk, int nt)
    {
        for (int k = 1; k + 1 < nt; k += 2) {
            const double r = std::atof(tk[k + 1]);
            const int i = row(tk[k]);
            if (i < 0)
                continue;
            const char t = row_type[i];
            const double base = t == 'L' ? uc[i] : lc[i];
            if (t == 'G')
                uc[i] = base + std::fabs(r);
            else if (t == 'L')
                lc[i] = base - std::fabs(r);
            else if (r >= 0)
                uc[i] = base + r;
            else
                lc[i] = base + r;
        }
    }

    void bounds(char **tk, int nt)
    {
        if (nt < 3)
            return;
        const int j = col(tk[2]);
        if (j < 0)
            return;
        const double v = nt > 3 ? std::atof(tk[3]) : 0.0;
        const std::string t = tk[0];
        if (t == "LO")
            lb[j] = v;
        else if (t == "UP")
            ub[j] = v;
        else if (t == "FX")
            lb[j] = ub[j] = v;
        else if (t == "FR") {
            lb[j] = -INFINITY;
            ub[j] = INFINITY;
        } else if (t == "MI")
            lb[j] = -INFINITY;
        else if (t == "PL")
            ub[j] = INFINITY;
        else if (t == "BV") {
            lb[j] = 0.0;
            ub[j] = 1.0;
        }
    }

    void quad(char **tk, int nt, bool mirror)
    {
        if (nt < 3)
            return;
        const double v = std::atof(tk[2]);
        if (v == 0.0)
            return;
        const int a = col(tk[0]), b = col(tk[1]);
        if (a < 0 || b < 0) {
            std::fprintf(stderr, "Warning: Variable '%s' or '%s' not found in COLUMNS. Skipping Q-entry.\n", tk[0],
                         tk[1]);
            return;
        }
        Q.add(a, b, v);
        if (mirror && a != b)
            Q.add(b, a, v);
    }

    void open_qc(const char *name)
    {
        qc_cur = -1;
        qc_obj = false;
        if (is_obj(name)) {
            qc_obj = true;
            return;
        }
        const int i = row(name);
        if (i < 0) {
            std::fprintf(stderr, "Warning: QCMATRIX references unknown row '%s'. Skipping.\n", name);
            return;
        }
        for (size_t k = 0; k < qc.size(); ++k)
            if (qc[k].first == i) {
                qc_cur = (int)k;
                return;
            }
        qc.emplace_back(i, Coo{});
        qc_cur = (int)qc.size() - 1;
    }

    void qcmatrix(char **tk, int nt)
    {
        if (nt < 3 || (qc_cur < 0 && !qc_obj))
            return;
        const double v = std::atof(tk[2]);
        if (v == 0.0)
            return;
        const int a = col(tk[0]), b = col(tk[1]);
        if (a < 0 || b < 0) {
            std::fprintf(stderr, "Warning: QCMATRIX references unknown variable '%s' or '%s'. Skipping entry.\n",
                         tk[0], tk[1]);
            return;
        }
        (qc_obj ? Q : qc[qc_cur].second).add(a, b, v);
    }

    bool error = false;
};

} // namespace

extern "C" qp_problem_t *read_mps_file(const char *filename)
{
    if (!filename)
        return nullptr;
    LineReader in(filename);
    if (!in.ok()) {
        std::fprintf(stderr, "ERROR: Could not open file %s\n", filename);
        return nullptr;
    }
    Parser P;
    Section sec = NONE;
    static thread_local char line[4096];
    while (!P.error && in.next(line, sizeof(line))) {
        if (line[0] == '*' || line[0] == '\n' || line[0] == '\r')
            continue;
        char *tk[6] = {nullptr};
        int nt = 0;
        char *save = nullptr;
        for (char *t = strtok_r(line, " \t\n\r", &save); t && nt < 6; t = strtok_r(nullptr, " \t\n\r", &save))
            tk[nt++] = t;
        if (nt == 0)
            continue;
        if (nt == 1 && std::isalpha((unsigned char)tk[0][0])) {
            const std::string h = tk[0];
            Section next = h == "ROWS"       ? ROWS
                           : h == "COLUMNS"  ? COLUMNS
                           : h == "RHS"      ? RHS
                           : h == "RANGES"   ? RANGES
                           : h == "BOUNDS"   ? BOUNDS
                           : h == "OBJSENSE" ? OBJSENSE
                           : h == "QUADOBJ"  ? QUADOBJ
                           : h == "QMATRIX"  ? QMATRIX
                           : h == "ENDATA"   ? ENDATA
                                             : NONE;
            if (sec == ROWS && next != ROWS)
                P.finish_rows();
            sec = next;
            if (sec == ENDATA)
                break;
            continue;
        }
        if (nt == 2 && std::strcmp(tk[0], "QCMATRIX") == 0) {
            if (sec == ROWS)
                P.finish_rows();
            sec = QCMATRIX;
            P.open_qc(tk[1]);
            continue;
        }
        switch (sec) {
        case OBJSENSE:
            if (std::strcmp(tk[0], "MAX") == 0 || std::strcmp(tk[0], "MAXIMIZE") == 0)
                P.maximize = true;
            break;
        case ROWS:
            if (nt >= 2)
                P.listed.emplace_back(tk[0][0], tk[1]);
            break;
        case COLUMNS: P.columns(tk, nt); break;
        case RHS: P.rhs(tk, nt); break;
        case RANGES: P.ranges(tk, nt); break;
        case BOUNDS: P.bounds(tk, nt); break;
        case QUADOBJ: P.quad(tk, nt, true); break;
        case QMATRIX: P.quad(tk, nt, false); break;
        case QCMATRIX: P.qcmatrix(tk, nt); break;
        default: break;
        }
    }
    if (P.error) {
        std::fprintf(stderr, "ERROR: Failed to parse MPS file.\n");
        return nullptr;
    }
    const int n = (int)P.c.size(), m = (int)P.row_type.size();
    const double sgn = P.maximize ? -1.0 : 1.0;
    auto *prob = (qp_problem_t *)std::calloc(1, sizeof(qp_problem_t));
    prob->num_variables = n;
    prob->num_constraints = m;
    prob->affine_cone_offset = m > 0 ? (double *)std::calloc((size_t)m, sizeof(double)) : nullptr;
    prob->objective_constant = sgn * P.obj_const;
    for (double &v : P.c)
        v *= sgn;
    for (double &v : P.Q.v)
        v *= sgn;
    prob->objective_vector = copy_out(P.c);
    prob->variable_lower_bound = copy_out(P.lb);
    prob->variable_upper_bound = copy_out(P.ub);
    prob->constraint_lower_bound = m > 0 ? copy_out(P.lc) : nullptr;
    prob->constraint_upper_bound = m > 0 ? copy_out(P.uc) : nullptr;
    prob->constraint_matrix = to_csr(P.A, m);
    prob->constraint_matrix_num_nonzeros = (int)P.A.v.size();
    prob->objective_sparse_matrix = to_csr(P.Q, n);
    prob->objective_sparse_matrix_num_nonzeros = (int)P.Q.v.size();
    prob->objective_lowrank_matrix = to_csr(Coo{}, 0);
    size_t kept = 0;
    for (auto &q : P.qc)
        kept += !q.second.v.empty();
    if (kept > 0) {
        prob->num_quadratic_constraints = (int)kept;
        prob->quadratic_constraint_row_indices = (int *)std::calloc(kept, sizeof(int));
        prob->quadratic_constraint_matrices = (CsrComponent **)std::calloc(kept, sizeof(CsrComponent *));
        prob->quadratic_constraint_matrix_num_nonzeros = (int *)std::calloc(kept, sizeof(int));
        size_t k = 0;
        for (auto &q : P.qc) {
            if (q.second.v.empty())
                continue;
            for (double &v : q.second.v)
                v *= sgn;
            prob->quadratic_constraint_row_indices[k] = q.first;
            prob->quadratic_constraint_matrix_num_nonzeros[k] = (int)q.second.v.size();
            prob->quadratic_constraint_matrices[k] = to_csr(q.second, n);
            ++k;
        }
    }
    return prob;
}
