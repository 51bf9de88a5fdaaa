// setup.cuh -- device preprocessing: transposition, rescaling, starting
// point, power method.  Rescaling restates the reference's host code
// (src/preconditioner.c:256-713) operation for operation so that Ruiz and
// Pock-Chambolle factors are bit-identical: per-row maxima and sums run
// sequentially in CSR order, per-column ones sequentially over the rows of
// A^T (increasing row index, the order of the reference's scatter loop).
#pragma once

#include <cooperative_groups.h>

#include "kernels.cuh"

namespace pdhcg {

namespace cg = cooperative_groups;

// Row-wise set-up kernels run one thread per row.  With skip_long set, rows
// of more than LONG_ROW entries are skipped and left to the companion
// kernel over the long-row table, one block per long row, so that a dense
// row does not hold one thread for its whole length.

__global__ void expand_rows_kernel(const int *rp, int rows, int *row_of, int skip_long)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        if (skip_long && rp[r + 1] - rp[r] > LONG_ROW)
            continue;
        for (int k = rp[r]; k < rp[r + 1]; ++k)
            row_of[k] = r;
    }
}

__global__ void expand_long_rows_kernel(LongRows L, const int *rp, int *row_of)
{
    for (int i = blockIdx.x; i < L.n; i += gridDim.x) {
        const int r = L.rows[i];
        for (int k = rp[r] + threadIdx.x; k < rp[r + 1]; k += blockDim.x)
            row_of[k] = r;
    }
}

// fixed-order block reductions of one value per thread (blockDim.x == TPB)
__device__ __forceinline__ double block_sum_fixed(double v)
{
    __shared__ double sh[TPB];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = TPB / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ double block_max(double v)
{
    __shared__ double sh[TPB];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = TPB / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// bad != 0 unless the CSR holds exactly the columns 0..cols-1 in order in every row
__global__ void dense_rows_check_kernel(int rows, int cols, const int *rp, const int *ci, int *bad)
{
    const long long nnz = (long long)rows * cols;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x) {
        if (ci[k] != (int)(k % cols))
            atomicOr(bad, 1);
        if (k <= rows && rp[k] != (int)(k * cols)) // row pointers (rows + 1 <= nnz + 1 entries)
            atomicOr(bad, 1);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && rp[rows] != (int)nnz)
        atomicOr(bad, 1);
}

// *flag = 1 when an entry of v[0, n) is NaN (strict = 0: bounds, where
// +-inf means "no bound") or not finite (strict = 1: objective, matrices)
__global__ void nonfinite_kernel(const double *v, long long n, int strict, int *flag)
{
    bool bad = false;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double x = v[i];
        bad |= strict ? !isfinite(x) : isnan(x);
    }
    if (__any_sync(FULL, bad) && (threadIdx.x & 31) == 0)
        atomicOr(flag, 1);
}

__global__ void iota_kernel(int *v, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v[i] = i;
}

// rp_t[c] = first position of key >= c in the sorted column keys
__global__ void col_ptr_kernel(const int *keys, int nnz, int ncols, int *rp_t)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= ncols; c += gridDim.x * blockDim.x) {
        int lo = 0, hi = nnz;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (keys[mid] < c)
                lo = mid + 1;
            else
                hi = mid;
        }
        rp_t[c] = lo;
    }
}

__global__ void gather_transpose_kernel(const int *perm, const int *row_of, const double *val, int nnz, int *ci_t,
                                        double *v_t)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x) {
        int p = perm[k];
        ci_t[k] = row_of[p];
        v_t[k] = val[p];
    }
}

__global__ void row_absmax_kernel(const int *rp, const double *v, int rows, double *out, int skip_long)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        if (skip_long && rp[r + 1] - rp[r] > LONG_ROW)
            continue;
        double mx = 0.0;
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            double a = fabs(v[k]);
            if (a > mx)
                mx = a;
        }
        out[r] = mx;
    }
}

// the maximum is exact in any order, so a long row's value is the same
__global__ void long_row_absmax_kernel(LongRows L, const int *rp, const double *v, double *out)
{
    for (int i = blockIdx.x; i < L.n; i += gridDim.x) {
        const int r = L.rows[i];
        double mx = 0.0;
        for (int k = rp[r] + threadIdx.x; k < rp[r + 1]; k += blockDim.x)
            mx = fmax(mx, fabs(v[k]));
        mx = block_max(mx);
        if (threadIdx.x == 0)
            out[r] = mx;
    }
}

// sum_k |a_k|^p per row; p == 1 uses |a| itself (pow(x, 1) == x exactly)
__global__ void row_powsum_kernel(const int *rp, const double *v, int rows, double p, double *out, int skip_long)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        if (skip_long && rp[r + 1] - rp[r] > LONG_ROW)
            continue;
        double s = 0.0;
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            double a = fabs(v[k]);
            s += (p == 1.0) ? a : pow(a, p);
        }
        out[r] = s;
    }
}

// a long row's sum in a fixed order (thread-strided, then a tree): the same
// on every run, but associated differently from a sequential sum
__global__ void long_row_powsum_kernel(LongRows L, const int *rp, const double *v, double p, double *out)
{
    for (int i = blockIdx.x; i < L.n; i += gridDim.x) {
        const int r = L.rows[i];
        double s = 0.0;
        for (int k = rp[r] + threadIdx.x; k < rp[r + 1]; k += blockDim.x) {
            const double a = fabs(v[k]);
            s += (p == 1.0) ? a : pow(a, p);
        }
        s = block_sum_fixed(s);
        if (threadIdx.x == 0)
            out[r] = s;
    }
}

__global__ void sqrt_or_one_kernel(double *v, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v[i] = v[i] < 1e-12 ? 1.0 : sqrt(v[i]);
}

// Cone-preserving aggregation of a scaling vector over each cone block
// (reference apply_cone_scaling_adjustment, src/preconditioner.c:108-144).
__global__ void cone_scaling_adjust_kernel(double *s, int ncones, const int *start, const int *len, int ruiz_phase)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < ncones; b += gridDim.x * blockDim.x) {
        int st = start[b], L = len[b];
        double mx = 0.0, sq = 0.0;
        for (int i = st; i < st + L; ++i) {
            mx = fmax(mx, s[i]);
            sq += s[i] * s[i];
        }
        double rms = sqrt(sq / (double)L);
        double bs = ruiz_phase ? (L <= 8 ? mx : rms) : (L <= 8 ? rms : sqrt(mx * rms));
        for (int i = st; i < st + L; ++i)
            s[i] = bs;
    }
}

// Diagonal-congruence projection of the log scaling of a PSD block, used
// when cone-preserving scaling is off (reference project_psd_log_scaling,
// src/preconditioner.c:46-92); one thread per block, order <= 64.
// log_space: s already holds log scales (Curtis-Reid) and receives log scales
__global__ void psd_scaling_kernel(double *s, int ncones, const int *start, const int *vdim, const int *type,
                                   int log_space)
{
    const double LIM = 69.07755278982137;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < ncones; b += gridDim.x * blockDim.x) {
        if (type[b] != 4)
            continue;
        int st = start[b], order = vdim[b];
        if (order > 64)
            continue;
        double f[64];
        for (int i = 0; i < order; ++i)
            f[i] = 0.0;
        int slot = st;
        for (int col = 0; col < order; ++col)
            for (int row = col; row < order; ++row, ++slot) {
                double v = log_space ? s[slot] : log(fmax(s[slot], 1e-300));
                if (isnan(v))
                    v = 0.0;
                else if (v > LIM)
                    v = LIM;
                else if (v < -LIM)
                    v = -LIM;
                if (row == col)
                    f[row] += 2.0 * v;
                else {
                    f[row] += v;
                    f[col] += v;
                }
            }
        double rhs = 0.0;
        for (int i = 0; i < order; ++i)
            rhs += f[i];
        double corr = rhs / (2.0 * order + 2.0), diag = order + 2.0;
        for (int i = 0; i < order; ++i) {
            f[i] = (f[i] - corr) / diag;
            f[i] = fmax(-0.5 * LIM, fmin(0.5 * LIM, f[i]));
        }
        slot = st;
        for (int col = 0; col < order; ++col)
            for (int row = col; row < order; ++row, ++slot)
                s[slot] = log_space ? f[row] + f[col] : exp(f[row] + f[col]);
    }
}

// v_k /= (rs[r] * cs[col]) : A with (cr, vr), A^T with (vr, cr), Q with (vr, vr)
__global__ void scale_csr_kernel(const int *rp, const int *ci, double *v, int rows, const double *rs,
                                 const double *cs, int cr_first, int skip_long)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        if (skip_long && rp[r + 1] - rp[r] > LONG_ROW)
            continue;
        double a = rs[r];
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            double b = cs[ci[k]];
            v[k] /= cr_first ? (b * a) : (a * b);
        }
    }
}

__global__ void long_scale_csr_kernel(LongRows L, const int *rp, const int *ci, double *v, const double *rs,
                                      const double *cs, int cr_first)
{
    for (int i = blockIdx.x; i < L.n; i += gridDim.x) {
        const int r = L.rows[i];
        const double a = rs[r];
        for (int k = rp[r] + threadIdx.x; k < rp[r + 1]; k += blockDim.x) {
            const double b = cs[ci[k]];
            v[k] /= cr_first ? (b * a) : (a * b);
        }
    }
}

// v_k /= rs[r] for every entry of row r (rows of at most LONG_ROW entries:
// every caller's matrix has none longer)
__global__ void scale_rows_kernel(const int *rp, double *v, int rows, const double *rs)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        double a = rs[r];
        for (int k = rp[r]; k < rp[r + 1]; ++k)
            v[k] /= a;
    }
}

// v_k /= cs[ci[k]], one thread per entry (no row needed)
__global__ void scale_cols_kernel(const int *ci, double *v, long long nnz, const double *cs)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x)
        v[k] /= cs[ci[k]];
}

__global__ void scale_vectors_kernel(int n, int m, double *c, double *l, double *u, const double *vr, double *lc,
                                     double *uc, double *g, const double *cr, double *cum_vr, double *cum_cr)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
        if (i < n) {
            c[i] /= vr[i];
            u[i] *= vr[i];
            l[i] *= vr[i];
            cum_vr[i] *= vr[i];
        } else {
            int r = i - n;
            lc[r] /= cr[r];
            uc[r] /= cr[r];
            g[r] /= cr[r];
            cum_cr[r] *= cr[r];
        }
    }
}

__global__ void mul_scalar_kernel(double *v, int n, double f)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v[i] *= f;
}

// squares for the bound / objective rescaling norms (reference bound_obj_rescaling,
// src/preconditioner.c:602-652) and max/sq for the unscaled relative-error norms
// (src/solver_state.cu:854-934)
enum NormScalar { NS_B2 = 0, NS_C2, NS_BMAX, NS_CMAX, NS_COUNT };

__global__ void __launch_bounds__(TPB) norms_kernel(int n, int m, const double *c, const double *lc, const double *uc,
                                                    const double *g, double *partials)
{
    const int ops[NS_COUNT] = {RSUM, RSUM, RMAX, RMAX};
    double acc[NS_COUNT] = {0.0, 0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
        if (i < n) {
            double v = c[i];
            acc[NS_C2] += v * v;
            acc[NS_CMAX] = fmax(acc[NS_CMAX], fabs(v));
        } else {
            int r = i - n;
            double lo = lc[r], up = uc[r], gg = g[r];
            double b2 = 0.0, bm = fabs(gg);
            if (isfinite(lo) && lo != up) {
                b2 += lo * lo;
                bm = fmax(bm, fabs(lo));
            }
            if (isfinite(up)) {
                b2 += up * up;
                bm = fmax(bm, fabs(up));
            }
            acc[NS_B2] += b2 + gg * gg;
            acc[NS_BMAX] = fmax(acc[NS_BMAX], bm);
        }
    }
    block_reduce_store<NS_COUNT>(acc, ops, partials);
}

__global__ void bound_obj_scale_kernel(int n, int m, double sb, double sc, double *c, double *l, double *u, double *lc,
                                       double *uc, double *g)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
        if (i < n) {
            l[i] *= sb;
            u[i] *= sb;
            c[i] *= sc;
        } else {
            int r = i - n;
            lc[r] *= sb;
            uc[r] *= sb;
            g[r] *= sb;
        }
    }
}

// diagonal of a diagonal-only Q, plus the reference's 1e-12
// (preprocess_qp_problem, src/preconditioner.c:812-825)
__global__ void q_diag_kernel(const int *rp, const int *ci, const double *v, int n, double *qd)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        for (int k = rp[r]; k < rp[r + 1]; ++k)
            if (ci[k] < n)
                qd[ci[k]] = v[k] + 1e-12;
}

// starting point: warm start scaling, cone interior aux points, box clamp
// (reference initialize_solver_state / initialize_cone_runtime,
// src/solver_state.cu:578-686, 809-829, 983-1000)
__global__ void scale_start_kernel(int n, const double *start, const double *vr, double sb, double *x0)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x0[i] = start[i] * vr[i] * sb;
}

// fixed: slots fixed by set_cone_fixed (NULL: none), which keep their value
__global__ void cone_aux_init_kernel(int ncones, const int *start, const int *vdim, const int *type,
                                     const double *vr, double sb, double *x0, const unsigned char *fixed)
{
    const double INV_SQRT2 = 0.7071067811865475;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < ncones; b += gridDim.x * blockDim.x) {
        int aux0 = start[b] + vdim[b];
        if (type[b] == 1) { // standard SOC: w, z
            if (!(fixed && fixed[aux0]))
                x0[aux0] = -INV_SQRT2 * sb * vr[aux0];
            if (!(fixed && fixed[aux0 + 1]))
                x0[aux0 + 1] = INV_SQRT2 * sb * vr[aux0 + 1];
        } else if (type[b] == 0) { // rotated SOC: t
            if (!(fixed && fixed[aux0 + 1]))
                x0[aux0 + 1] = sb * vr[aux0 + 1];
        }
    }
}

// fixed cone slots: the scaled bounds pinned at value * vr * sb (reference
// pin_scaled_fixed_cone_bounds, src/preconditioner.c:311-327)
__global__ void pin_fixed_kernel(int nfix, const int *idx, const double *val, const double *vr, double sb, double *l,
                                 double *u)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nfix; k += gridDim.x * blockDim.x) {
        const int j = idx[k];
        const double v = val[k] * vr[j] * sb;
        l[j] = v;
        u[j] = v;
    }
}

__global__ void box_clamp_copy_kernel(int n, const double *l, const double *u, double *x0, double *x, double *xp,
                                      double *xr)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double v = fmax(l[i], fmin(x0[i], u[i]));
        x0[i] = v;
        x[i] = v;
        xp[i] = v;
        xr[i] = v;
    }
}

__global__ void dual_start_kernel(int m, const double *start, const double *cr, double sc, double *y0, double *y,
                                  double *yp)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        double v = start ? start[i] * cr[i] * sc : 0.0;
        y0[i] = v;
        y[i] = v;
        yp[i] = v;
    }
}

// warp-per-cone projection of a vector (unit metric, d = rescaling);
// fixed: slots fixed by set_cone_fixed (NULL: none), sect: whether this
// block holds any (then the section projector, with warm start warm)
template <int S>
__device__ __forceinline__ void project_cone_block(int st, int L, int tp, double alpha, double *x, const double *d,
                                                   const double *q, double tau, int lane, double *psd,
                                                   const unsigned char *fixed = nullptr, bool sect = false,
                                                   double *warm = nullptr)
{
    WarpSlots<S> sl;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        sl.x[s] = i < L ? x[st + i] : 0.0;
        sl.d[s] = i < L ? d[st + i] : 1.0;
        sl.w[s] = (i < L && q) ? 1.0 + tau * q[st + i] : 1.0;
    }
    if (sect) {
        warp_section_project<S>(tp, sl, L, lane, section_bits<S>(fixed, st, L, lane), warm, alpha);
    } else {
        bool uni = warp_uniform_unit<S>(sl, L, lane);
        warp_project<S>(tp, sl, L, lane, uni, nullptr, alpha, psd);
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        if (i < L)
            x[st + i] = sl.x[s];
    }
}

// psd_work / psd_off: PSD blocks' scratch and each block's offset in it
// (NULL: no PSD blocks)
template <int S>
__global__ void __launch_bounds__(TPB) project_cones_kernel(int ncones, const int *start, const int *len,
                                                            const int *type, const double *alpha, double *x,
                                                            const double *d, const double *q, double tau,
                                                            double *psd_work, const long long *psd_off,
                                                            const unsigned char *fixed = nullptr,
                                                            const unsigned char *cone_fixed = nullptr,
                                                            double *warm = nullptr)
{
    const int lane = threadIdx.x & 31;
    for (int cb = blockIdx.x * WARPS + (threadIdx.x >> 5); cb < ncones; cb += gridDim.x * WARPS) {
        const int st = start[cb], L = len[cb], tp = type[cb];
        const double a = alpha ? alpha[cb] : 0.0;
        double *psd = psd_work ? psd_work + psd_off[cb] : nullptr;
        const bool sect = cone_fixed && cone_fixed[cb];
        double *wb = warm ? warm + cb : nullptr;
        if (S > 1 && (tp == 2 || tp == 3)) // 3-slot blocks: the one-slot instantiation
            project_cone_block<1>(st, L, tp, a, x, d, q, tau, lane, psd, fixed, sect, wb);
        else if (tp == 4 && L > 32 * S) { // a long PSD block: in place, in memory (no metric)
            if (psd)
                warp_project_psd_mem(x + st, x + st, L, lane, psd);
        } else
            project_cone_block<S>(st, L, tp, a, x, d, q, tau, lane, psd, fixed, sect, wb);
    }
}

// every block a section block (pdhcg_b200_project_cone_sections)
template <int S>
__global__ void __launch_bounds__(TPB) project_sections_kernel(int ncones, const int *start, const int *len,
                                                               const int *type, const double *alpha, double *x,
                                                               const double *d, const double *q, double tau,
                                                               const unsigned char *fixed, double *warm)
{
    const int lane = threadIdx.x & 31;
    for (int cb = blockIdx.x * WARPS + (threadIdx.x >> 5); cb < ncones; cb += gridDim.x * WARPS) {
        const int st = start[cb], L = len[cb], tp = type[cb];
        const double a = alpha ? alpha[cb] : 0.0;
        double *wb = warm ? warm + cb : nullptr;
        if (S > 1 && (tp == 2 || tp == 3))
            project_cone_block<1>(st, L, tp, a, x, d, q, tau, lane, nullptr, fixed, true, wb);
        else
            project_cone_block<S>(st, L, tp, a, x, d, q, tau, lane, nullptr, fixed, true, wb);
    }
}

// restart: x_init = x_cur = x_pdhg, y_init = y_cur = y_pdhg
template <typename VT>
__global__ void restart_copy_kernel(int n, int m, const VT *xp, VT *x0, VT *x, const VT *yp, VT *y0, VT *y)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
        if (i < n) {
            VT v = xp[i];
            x0[i] = v;
            x[i] = v;
        } else {
            int r = i - n;
            VT v = yp[r];
            y0[r] = v;
            y[r] = v;
        }
    }
}

// Final answer: reduced cost and unscaling (reference create_result_from_state
// and compute_and_rescale_reduced_cost_qp_kernel, src/pdhg_core_op.cu:1431-1471,
// src/kernels/pdhcg_kernels.cu:866-894, rescale_solution_kernel :308-327).
template <typename VT>
__global__ void result_kernel(int n, int m, const int *At_rp, const int *At_ci, const double *At_v, const double *c,
                              const double *q, const double *qx, int qmode, const double *l, const double *u,
                              const double *vr, const double *cr, double sb, double sc, const VT *xp,
                              const VT *yp, double *x_out, double *y_out, double *rc_out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
        if (i < n) {
            double aty = row_dot<1>(At_rp, At_ci, At_v, yp, i, 0);
            double g = c[i];
            if (qmode == 1)
                g += q[i] * (double)xp[i];
            else if (qmode == 2)
                g += qx[i];
            double rc = (g - aty) * vr[i] / sc;
            if (!isfinite(l[i]))
                rc = fmin(rc, 0.0);
            if (!isfinite(u[i]))
                rc = fmax(rc, 0.0);
            rc_out[i] = rc;
            x_out[i] = (double)xp[i] / vr[i] / sb;
        } else {
            int r = i - n;
            y_out[r] = (double)yp[r] / cr[r] / sc;
        }
    }
}

// ---------------------------------------------------------------------------
// Power method for sigma_max(A) on A A^T, one cooperative launch (reference
// estimate_maximum_singular_value, src/pdhg_core_op.cu:1673-1788): the same
// sequence of operations, with the vector reductions done as fixed-order
// block folds shared by every block after each grid barrier.
// ---------------------------------------------------------------------------
__device__ double coop_fold(const double *part, int nb)
{
    __shared__ double sh[TPB];
    double a = 0.0;
    for (int b = threadIdx.x; b < nb; b += TPB)
        a += part[b];
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int o = TPB / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}

__device__ void coop_block_partial(double v, double *part)
{
    __shared__ double sh[WARPS];
    double w = warp_sum(v);
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = w;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int i = 0; i < WARPS; ++i)
            a += sh[i];
        part[blockIdx.x] = a;
    }
    __syncthreads();
}

template <typename MT>
__global__ void __launch_bounds__(TPB) power_sigma_kernel(int m, int n, const int *A_rp, const int *A_ci,
                                                          const MT *A_v, const int *At_rp, const int *At_ci,
                                                          const MT *At_v, double *v, double *nv, double *dp,
                                                          double *part /* 4 * gridDim */, int max_iter, double tol,
                                                          double *out /* [sigma, iterations] */, LongRows A_long,
                                                          LongRows At_long)
{
    // The iterate is u with |u| = 1 / inv (v = inv * u is the unit vector):
    //   dp = inv * A^T u;  w = A dp = A A^T v
    //   s2 = v . w = inv * (u . w);  |w - s2 v|^2 = |w|^2 - s2^2  (|v| = 1)
    // then u <- w, inv <- 1 / |w|: two grid barriers per iteration, the
    // buffers of u and w alternate.
    cg::grid_group grid = cg::this_grid();
    __shared__ double stage_all[WARPS][STREAM_CHUNK];
    const int nb = gridDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31, gw = blockIdx.x * WARPS + (threadIdx.x >> 5), nw = gridDim.x * WARPS;
    double *stage = stage_all[threadIdx.x >> 5];
    double *p0 = part, *p1 = part + nb, *p2 = part + 2 * nb;
    double a = 0.0;
    for (int i = tid; i < m; i += nth)
        a += v[i] * v[i];
    coop_block_partial(a, p0);
    grid.sync();
    double inv = 1.0 / sqrt(coop_fold(p0, nb));
    double *u = v, *w = nv;
    double s2 = 1.0;
    int it = 0;
    for (; it < max_iter; ++it) {
        if (At_long.n > 0) { // segment pass of the long rows, then the rows
            long_partials(At_long, At_ci, At_v, u, gw, nw, lane);
            grid.sync();
        }
        for (int t = gw; t < (n + 31) / 32; t += nw) {
            const int r0 = 32 * t, nr = min(32, n - r0);
            double r[1];
            warp_stream_rows<1>(At_rp, At_ci, At_v, u, r0, nr, lane, stage, r, At_long);
            if (lane < nr)
                dp[r0 + lane] = r[0] * inv;
        }
        grid.sync();
        if (A_long.n > 0) {
            long_partials(A_long, A_ci, A_v, dp, gw, nw, lane);
            grid.sync();
        }
        double uw = 0.0, ww = 0.0;
        for (int t = gw; t < (m + 31) / 32; t += nw) {
            const int r0 = 32 * t, nr = min(32, m - r0);
            double r[1];
            warp_stream_rows<1>(A_rp, A_ci, A_v, dp, r0, nr, lane, stage, r, A_long);
            if (lane < nr) {
                w[r0 + lane] = r[0];
                uw += r[0] * u[r0 + lane];
                ww += r[0] * r[0];
            }
        }
        coop_block_partial(uw, p1);
        coop_block_partial(ww, p2);
        grid.sync();
        s2 = inv * coop_fold(p1, nb);
        const double w2 = coop_fold(p2, nb);
        if (sqrt(fmax(w2 - s2 * s2, 0.0)) < tol)
            break;
        inv = 1.0 / sqrt(w2);
        double *t = u;
        u = w;
        w = t;
    }
    if (tid == 0) {
        out[0] = sqrt(s2);
        out[1] = (double)it;
    }
}

// ---- Curtis-Reid scaling (reference curtis_reid_rescaling,
// src/preconditioner.c:334-495): log-space alternating row / column averages
// of log|a_ij|, cone blocks averaged together when scaling is
// cone-preserving.  One thread per row with sequential sums in entry order,
// the order of the reference's host loops.
constexpr double CR_LOG_MIN_ABS = 1e-300;
constexpr double CR_LOG_LIMIT = 69.07755278982137; // log(1e30)

// sum of log max(|a|, 1e-300) over each row of M
__global__ void cr_logsum_kernel(const int *rp, const double *v, int rows, double *sum)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = rp[r]; k < rp[r + 1]; ++k)
            s += log(fmax(fabs(v[k]), CR_LOG_MIN_ABS));
        sum[r] = s;
    }
}

// raw[r] = base[r] - sum_{k in row r} other[col k]; out[r] = raw[r] / len(r),
// 0 for empty rows (raw may be NULL)
__global__ void cr_average_kernel(const int *rp, const int *ci, int rows, const double *base, const double *other,
                                  double *out, double *raw)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        int b = rp[r], e = rp[r + 1];
        double s = base[r];
        for (int k = b; k < e; ++k)
            s -= other[ci[k]];
        if (raw)
            raw[r] = s;
        out[r] = e > b ? s / (double)(e - b) : 0.0;
    }
}

// cone-preserving column step: one value per cone block,
// (sum over the block of cs) / (sum over the block of the column counts)
__global__ void cr_cone_average_kernel(int nc, const int *start, const int *len, const int *At_rp, const double *cs,
                                       double *cls)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nc; b += gridDim.x * blockDim.x) {
        const int st = start[b], L = len[b];
        double bsum = 0.0;
        int bcount = 0;
        for (int c = st; c < st + L; ++c) {
            bsum += cs[c];
            bcount += At_rp[c + 1] - At_rp[c];
        }
        const double bl = bcount > 0 ? bsum / (double)bcount : 0.0;
        for (int c = st; c < st + L; ++c)
            cls[c] = bl;
    }
}

__global__ void cr_exp_kernel(double *v, int k)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        double x = v[i];
        if (isnan(x))
            v[i] = 1.0;
        else
            v[i] = exp(fmin(fmax(x, -CR_LOG_LIMIT), CR_LOG_LIMIT));
    }
}

} // namespace pdhcg
