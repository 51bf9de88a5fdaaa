// bb.cuh -- inner projected Barzilai-Borwein solve of the primal prox for a
// non-diagonal quadratic objective (reference primal_BB_step_size_update,
// src/pdhg_core_op.cu:495-669, kernels src/kernels/pdhcg_kernels.cu:392-636).
//
// The reference runs every inner iteration as a handful of launches plus a
// blocking device-to-host copy of the step norm.  Here the whole inner loop
// is ONE cooperative launch: phases are separated by grid barriers, every
// reduction is a fixed-order fold of per-block partials that all blocks
// compute identically, so the convergence test and the BB step length are
// decided on the device, warp-uniformly, without the host.
//
// Q apply (reference update_obj_product, src/pdhg_core_op.cu:305-413):
//   qx = Q v                       (sparse Q, CSR)
//      + R^T D (R v)               (low rank: R as CSR rows for R v, R^T as
//                                   CSR rows for the back-projection)
// R v is a k-vector reduced over all n columns: each block folds its chunk
// of every row with one warp per row, then block r folds row r's partials.
#pragma once

#include <cooperative_groups.h>

#include "kernels.cuh"

namespace pdhcg {

struct BBData {
    int n;
    // problem (scaled)
    const double *c, *l, *u;
    const double *aty; // A^T y of this outer iteration
    // quadratic term
    int sparse;              // Q CSR present
    const int *Q_rp, *Q_ci;
    const double *Q_v;
    int k;                   // low-rank rank (0: none)
    const int *R_rp, *R_ci;  // R, k rows
    const double *R_v;
    const int *Rt_rp, *Rt_ci; // R^T, n rows (not built when r_width > 0)
    const double *Rt_v;
    int r_width;              // > 0: every row of R holds columns 0..r_width-1 in order, so R_v is
                              // row-major k x r_width (R^T not built); 0: R and R^T as CSR
    int dkind;               // 0 none (D = I), 1 diagonal, 2 dense (row-major, upper triangle used)
    const double *Ddiag, *Ddense;
    // FP32 copies of Q's, R's and R^T's values for the mixed-precision bulk
    // phase (NULL: the FP64 values); products accumulate in FP64 either way
    const float *Q_vf, *R_vf, *Rt_vf;
    // Jacobi preconditioner M = diag(Q) + 1/tau (NULL: none)
    const double *m_diag, *m_inv;
    const double *tol_scale; // device scalar sqrt(sum |M| / n)
    // cones (warp per block) and free variables
    const int *free_idx;
    int n_free;
    const int *cone_start, *cone_len, *cone_type;
    const double *cone_alpha; // power-cone exponents (NULL: none)
    int n_cones;
    const double *vr;
    double *cone_warm;
    const unsigned char *fixed, *cone_fixed; // slots fixed by set_cone_fixed, and per block whether any (NULL: none)
    double *psd_work; // PSD blocks' projection scratch (NULL: none)
    const long long *psd_off;
    // iterates
    const double *x0;
    double *x, *xp, *xr, *dx;
    // scratch
    double *grad, *dir, *qx;
    double *part;      // [4][gridDim] scalar partials
    double *rx_part;   // [gridDim][k]
    double *rx;        // [k]
    // controls
    const double *tol; // device scalar, inner tolerance
    int limit;         // inner iteration limit
    int *inner_total;  // device counter, += iterations - 1
};

struct BBParams {
    double tau, w, rho;
    int want_fpe;
};

namespace cgb = cooperative_groups;

__device__ __forceinline__ double bb_fold(const double *part, int nb)
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

__device__ __forceinline__ void bb_block_partial(double v, double *part)
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

// Dense R (every row over columns 0..r_width-1): warp w of block b takes
// rows 4w .. 4w+3, 4(w + WARPS) .., and sums each row's b-th chunk with
// the row's own accumulator, so one load of v serves four rows and four
// loads of R are in flight per lane; each row's lane partials and warp sum
// run in the order of the one-row loop.
template <typename T>
__device__ __forceinline__ void bb_rx_partials_dense(const BBData &D, const T *R, const double *v)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nb = gridDim.x;
    const long long w = D.r_width;
    const int cb = (int)(w * blockIdx.x / nb), ce = (int)(w * (blockIdx.x + 1) / nb);
    for (int r0 = 4 * wid; r0 < D.k; r0 += 4 * WARPS) {
        const int nr = min(4, D.k - r0);
        const T *row[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            row[q] = R + (long long)D.R_rp[r0 + (q < nr ? q : 0)];
        double s[4] = {0.0, 0.0, 0.0, 0.0};
        if (nr == 4) {
#pragma unroll 4
            for (int c = cb + lane; c < ce; c += 32) {
                const double vc = v[c];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    s[q] += (double)row[q][c] * vc;
            }
        } else {
            for (int c = cb + lane; c < ce; c += 32) {
                const double vc = v[c];
                for (int q = 0; q < nr; ++q)
                    s[q] += (double)row[q][c] * vc;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double t = warp_sum(s[q]);
            if (q < nr && lane == 0)
                D.rx_part[(size_t)blockIdx.x * D.k + r0 + q] = t;
        }
    }
}

// Low-rank part, step 1: partials of R v.  Block b owns the b-th chunk of
// every row of R; warp w of the block folds rows w, w + WARPS, ...
__device__ void bb_rx_partials(const BBData &D, const double *v)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nb = gridDim.x;
    if (D.r_width) {
        if (D.R_vf)
            bb_rx_partials_dense(D, D.R_vf, v);
        else
            bb_rx_partials_dense(D, D.R_v, v);
        return;
    }
    for (int r = wid; r < D.k; r += WARPS) {
        int b0 = D.R_rp[r], e0 = D.R_rp[r + 1];
        long long len = e0 - b0;
        int cb = b0 + (int)(len * blockIdx.x / nb), ce = b0 + (int)(len * (blockIdx.x + 1) / nb);
        double s = 0.0;
        if (D.R_vf)
            for (int e = cb + lane; e < ce; e += 32)
                s += (double)D.R_vf[e] * v[D.R_ci[e]];
        else
            for (int e = cb + lane; e < ce; e += 32)
                s += D.R_v[e] * v[D.R_ci[e]];
        s = warp_sum(s);
        if (lane == 0)
            D.rx_part[(size_t)blockIdx.x * D.k + r] = s;
    }
}

// step 2: block r folds row r's partials in block order
__device__ void bb_rx_fold(const BBData &D)
{
    const int nb = gridDim.x;
    for (int r = blockIdx.x; r < D.k; r += nb) {
        __shared__ double sh[TPB];
        double a = 0.0;
        for (int b = threadIdx.x; b < nb; b += TPB)
            a += D.rx_part[(size_t)b * D.k + r];
        sh[threadIdx.x] = a;
        __syncthreads();
        for (int o = TPB / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o)
                sh[threadIdx.x] += sh[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            D.rx[r] = sh[0];
        __syncthreads();
    }
}

// step 3: D (R v) into shared memory (every block, k <= BB_MAX_RANK)
constexpr int BB_MAX_RANK = 512;

__device__ void bb_drx_smem(const BBData &D, double *drx)
{
    for (int r = threadIdx.x; r < D.k; r += TPB) {
        double v;
        if (D.dkind == 1)
            v = D.Ddiag[r] * D.rx[r];
        else if (D.dkind == 2) { // cublasDsymv lower on the row-major array seen column-major
            v = 0.0;
            for (int c = 0; c < D.k; ++c) {
                int a = r < c ? r : c, b = r < c ? c : r;
                v += D.Ddense[(size_t)a * D.k + b] * D.rx[c];
            }
        } else
            v = D.rx[r];
        drx[r] = v;
    }
    __syncthreads();
}

// This lane's share (lanes sub, sub + G, ...) of R^T row j . drx
template <int G>
__device__ __forceinline__ double bb_rt_part(const BBData &D, const double *drx, int j, int sub)
{
    double s = 0.0;
    if (D.r_width) { // column j of the row-major R, rows in increasing order (the order of R^T row j)
        if (j < D.r_width) { // unrolled so that many loads of the column are in flight
            if (D.R_vf) {
                const float *col = D.R_vf + j;
#pragma unroll 16
                for (int r = sub; r < D.k; r += G)
                    s += (double)col[(size_t)r * D.r_width] * drx[r];
            } else {
                const double *col = D.R_v + j;
#pragma unroll 16
                for (int r = sub; r < D.k; r += G)
                    s += col[(size_t)r * D.r_width] * drx[r];
            }
        }
    } else {
        int b = D.Rt_rp[j], e = D.Rt_rp[j + 1];
        if (D.Rt_vf)
            for (int t = b + sub; t < e; t += G)
                s += (double)D.Rt_vf[t] * drx[D.Rt_ci[t]];
        else
            for (int t = b + sub; t < e; t += G)
                s += D.Rt_v[t] * drx[D.Rt_ci[t]];
    }
    return s;
}

// This lane's share (entries sub, sub + G, ...) of Q row j . v
template <int G>
__device__ __forceinline__ double bb_qsp_part(const BBData &D, const double *v, int j, int sub)
{
    const int b = D.Q_rp[j], e = D.Q_rp[j + 1];
    double s = 0.0;
    if (D.Q_vf)
        for (int t = b + sub; t < e; t += G)
            s += (double)D.Q_vf[t] * v[D.Q_ci[t]];
    else
        for (int t = b + sub; t < e; t += G)
            s += D.Q_v[t] * v[D.Q_ci[t]];
    return s;
}

// qx_j for one variable, G lanes: Q row j . v + R^T row j . drx.  Every
// lane of the warp calls it; ok == false gives 0 without reading a row.
template <int G>
__device__ __forceinline__ double bb_q_row(const BBData &D, const double *v, const double *drx, int j, int sub,
                                           bool ok)
{
    double s = 0.0;
    if (ok && D.sparse)
        s = bb_qsp_part<G>(D, v, j, sub);
    if (ok && D.k > 0) {
        s += bb_rt_part<G>(D, drx, j, sub);
    }
    return group_sum<G>(s);
}

// Work items of the variable-wise phases: chunks of 32/G free variables
// (G lanes per variable) and cone blocks (one warp per block, S slots per lane).
template <int G, int S>
struct BBWork {
    int free_tasks, tasks;
    __device__ BBWork(const BBData &D)
    {
        // with cone blocks the free variables are exactly the list (possibly
        // empty, with a NULL list); without, every variable is free
        int nf = D.n_cones > 0 ? D.n_free : D.n;
        free_tasks = (nf + 32 / G - 1) / (32 / G);
        tasks = free_tasks + D.n_cones;
    }
};

// One cone block of bb_var_phase: the warp computes the candidates,
// projects, and takes the step from the values before the update.  SECT:
// the block holds slots fixed by set_cone_fixed (section projectors).
template <int G, int S, bool SECT = false>
__device__ __forceinline__ double bb_cone_block(const BBData &D, const double *drx, bool init, double alpha, int lane,
                                                double *stage, int cb)
{
    const int sub = lane % G;
    double part = 0.0;
    int st = D.cone_start[cb], L = D.cone_len[cb], type = D.cone_type[cb];
    if (init) {
        // Q x for the block's rows, staged through shared memory
        for (int base = 0; base < L; base += 32 / G) {
            int slot = base + lane / G;
            bool ok = slot < L;
            int j = st + (ok ? slot : 0);
            double s = 0.0;
            if (ok && D.sparse)
                s = bb_qsp_part<G>(D, D.x, j, sub);
            if (ok && D.k > 0)
                s += bb_rt_part<G>(D, drx, j, sub);
            s = group_sum<G>(s);
            if (ok && sub == 0)
                stage[slot] = s;
        }
        __syncwarp();
    }
    WarpSlots<S> sl;
    double xo[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        sl.x[s] = 0.0;
        sl.d[s] = 1.0;
        sl.w[s] = 1.0;
        xo[s] = 0.0;
        if (i < L) {
            int j = st + i;
            double mi = D.m_inv ? D.m_inv[j] : 1.0;
            double g;
            if (init) {
                double q = stage[i];
                g = q + D.c[j] - D.aty[j];
                xo[s] = D.x[j];
                D.grad[j] = g;
                D.qx[j] = q;
            } else {
                g = D.grad[j];
                xo[s] = D.xp[j];
            }
            sl.x[s] = clampd(D.l[j], xo[s] - alpha * mi * g, D.u[j]);
            sl.d[s] = D.vr[j];
        }
    }
    __syncwarp();
    if constexpr (SECT) {
        const unsigned fb = section_bits<S>(D.fixed, st, L, lane);
        warp_section_project<S>(type, sl, L, lane, fb, D.cone_warm ? D.cone_warm + cb : nullptr,
                                D.cone_alpha ? D.cone_alpha[cb] : 0.0);
    } else {
        bool uni = warp_uniform_unit<S>(sl, L, lane);
        warp_project<S>(type, sl, L, lane, uni, D.cone_warm ? D.cone_warm + cb : nullptr,
                        D.cone_alpha ? D.cone_alpha[cb] : 0.0, D.psd_work ? D.psd_work + D.psd_off[cb] : nullptr);
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        if (i < L) {
            int j = st + i;
            D.xp[j] = sl.x[s];
            double dd = sl.x[s] - xo[s];
            D.dir[j] = dd;
            part += D.m_diag ? dd * D.m_diag[j] * dd : dd * dd;
        }
    }
    return part;
}

// A PSD block longer than the warp's registers hold: the same step, slot by
// slot, with the candidate staged in the block's scratch and projected in
// memory.
template <int G>
__device__ __noinline__ double bb_psd_long_block(const BBData &D, const double *drx, bool init, double alpha,
                                                 int lane, int cb)
{
    const int st = D.cone_start[cb], L = D.cone_len[cb];
    const int n = psd_order(L);
    double *work = D.psd_work + D.psd_off[cb];
    double *sv = work + 2LL * n * n, *xo_s = sv + L; // candidates, then the values before the step
    for (int i = lane; i < L; i += 32) {
        const int j = st + i;
        const double mi = D.m_inv ? D.m_inv[j] : 1.0;
        double g, xo;
        if (init) {
            double q = 0.0; // (Q x)_j, one lane per slot
            if (D.sparse)
                q = bb_qsp_part<1>(D, D.x, j, 0);
            if (D.k > 0)
                q += bb_rt_part<1>(D, drx, j, 0);
            g = q + D.c[j] - D.aty[j];
            xo = D.x[j];
            D.grad[j] = g;
            D.qx[j] = q;
        } else {
            g = D.grad[j];
            xo = D.xp[j];
        }
        sv[i] = clampd(D.l[j], xo - alpha * mi * g, D.u[j]);
        xo_s[i] = xo;
    }
    __syncwarp();
    warp_project_psd_mem(sv, sv, L, lane, work);
    double part = 0.0;
    for (int i = lane; i < L; i += 32) {
        const int j = st + i;
        D.xp[j] = sv[i];
        const double dd = sv[i] - xo_s[i];
        D.dir[j] = dd;
        part += D.m_diag ? dd * D.m_diag[j] * dd : dd * dd;
    }
    __syncwarp();
    return part;
}

// init: grad = Qx + c - A^T y; x_p = P(x - alpha0 M^-1 grad); dir = x_p - x
// (reference primal_gradient_descent_kernel_bb_init[_precond] and the cone
// projection that follows, src/pdhg_core_op.cu:531-566)
// update: alpha from the previous step; x_p = P(x_p - alpha M^-1 grad);
// dir = x_p(new) - x_p(old) (reference :613-660)
// Both return the partial of dir' M dir (or dir' dir).  SECT: the problem
// has blocks with fixed slots (a kernel of its own, so that the section
// projectors do not weigh on the registers of the others).
template <int G, int S, bool SECT>
__device__ double bb_var_phase(const BBData &D, const double *drx, bool init, double alpha, int lane, int gwarp,
                               int nwarps, double *stage)
{
    BBWork<G, S> W(D);
    double part = 0.0;
    const int sub = lane % G;
    for (int task = gwarp; task < W.tasks; task += nwarps) {
        if (task < W.free_tasks) {
            int r = task * (32 / G) + lane / G;
            int nf = D.n_cones > 0 ? D.n_free : D.n;
            bool ok = r < nf;
            int j = ok ? (D.free_idx ? D.free_idx[r] : r) : 0;
            double q = 0.0;
            if (init) {
                // Q x for the gradient at the prox centre
                if (D.sparse || D.k > 0) {
                    double s = 0.0;
                    if (ok && D.sparse)
                        s = bb_qsp_part<G>(D, D.x, j, sub);
                    if (ok && D.k > 0)
                        s += bb_rt_part<G>(D, drx, j, sub);
                    q = group_sum<G>(s);
                }
            }
            if (ok && sub == 0) {
                double mi = D.m_inv ? D.m_inv[j] : 1.0;
                double xo, xn, g;
                if (init) {
                    g = q + D.c[j] - D.aty[j];
                    xo = D.x[j];
                    D.grad[j] = g;
                    D.qx[j] = q;
                } else {
                    g = D.grad[j];
                    xo = D.xp[j];
                }
                xn = clampd(D.l[j], xo - alpha * mi * g, D.u[j]);
                D.xp[j] = xn;
                double dd = xn - xo;
                D.dir[j] = dd;
                part += D.m_diag ? dd * D.m_diag[j] * dd : dd * dd;
            }
        } else {
            // cone block; 3-slot blocks (exponential, power) take the one-slot
            // instantiation, which alone carries their projection
            const int cb = task - W.free_tasks;
            const bool three = S > 1 && (D.cone_type[cb] == 2 || D.cone_type[cb] == 3);
            if (D.cone_type[cb] == 4 && D.cone_len[cb] > 32 * S)
                part += bb_psd_long_block<G>(D, drx, init, alpha, lane, cb);
            else if (SECT && D.cone_fixed[cb])
                part += three ? bb_cone_block<G, 1, SECT>(D, drx, init, alpha, lane, stage, cb)
                              : bb_cone_block<G, S, SECT>(D, drx, init, alpha, lane, stage, cb);
            else if (three)
                part += bb_cone_block<G, 1>(D, drx, init, alpha, lane, stage, cb);
            else
                part += bb_cone_block<G, S>(D, drx, init, alpha, lane, stage, cb);
        }
    }
    return part;
}

// grad_new = Q x_p + c - A^T y + (x_p - x)/tau; pbuf = grad_new - grad;
// returns the partial of dir . pbuf (reference primal_bb_update_gradient_kernel)
template <int G>
__device__ double bb_grad_phase(const BBData &D, const double *drx, double inv_tau, int lane, int gwarp, int nwarps)
{
    double part = 0.0;
    const int sub = lane % G;
    const int per = 32 / G;
    for (int base = gwarp * per; base < D.n; base += nwarps * per) {
        int j = base + lane / G;
        bool ok = j < D.n;
        double q = bb_q_row<G>(D, D.xp, drx, ok ? j : 0, sub, ok);
        if (ok && sub == 0) {
            double gn = q + D.c[j] - D.aty[j] + inv_tau * (D.xp[j] - D.x[j]);
            double pb = gn - D.grad[j];
            D.grad[j] = gn;
            D.qx[j] = q;
            part += D.dir[j] * pb;
        }
    }
    return part;
}

template <int G, int S, bool SECT>
__global__ void __launch_bounds__(TPB) bb_kernel(BBData D, BBParams P)
{
    cgb::grid_group grid = cgb::this_grid();
    __shared__ double drx[BB_MAX_RANK];
    __shared__ double stage_all[WARPS][32 * S];
    const int lane = threadIdx.x & 31;
    const int gwarp = blockIdx.x * WARPS + (threadIdx.x >> 5), nwarps = gridDim.x * WARPS;
    const int nb = gridDim.x;
    double *stage = stage_all[threadIdx.x >> 5];
    double *p_s = D.part, *p_t = D.part + nb;
    const double inv_tau = 1.0 / P.tau;
    double alpha0 = 1.0 / inv_tau;
    if (D.m_inv) {
        double ts = *D.tol_scale;
        alpha0 *= ts * ts;
    }
    const double tol = *D.tol;

    // Q x at the prox centre
    if (D.k > 0) {
        bb_rx_partials(D, D.x);
        grid.sync();
        bb_rx_fold(D);
        grid.sync();
        bb_drx_smem(D, drx);
    }
    double s = bb_var_phase<G, S, SECT>(D, drx, true, alpha0, lane, gwarp, nwarps, stage);
    bb_block_partial(s, p_s);
    grid.sync();
    int it = 1;
    while (it < D.limit) {
        double stMs = bb_fold(p_s, nb);
        double norm = sqrt(stMs);
        if (norm <= tol)
            break;
        if (D.k > 0) {
            bb_rx_partials(D, D.xp);
            grid.sync();
            bb_rx_fold(D);
            grid.sync();
            bb_drx_smem(D, drx);
        }
        double t = bb_grad_phase<G>(D, drx, inv_tau, lane, gwarp, nwarps);
        bb_block_partial(t, p_t);
        grid.sync();
        double tmp = bb_fold(p_t, nb);
        double alpha = stMs / tmp; // M-metric BB step (precond: sMs/tmp; plain: |s|^2/tmp)
        s = bb_var_phase<G, S, SECT>(D, drx, false, alpha, lane, gwarp, nwarps, stage);
        bb_block_partial(s, p_s);
        grid.sync();
        ++it;
    }
    // x_refl, Halpern average of x (reference primal_bb_final_kernel + halpern)
    for (int j = blockIdx.x * TPB + threadIdx.x; j < D.n; j += nb * TPB) {
        double xi = D.x[j], p = D.xp[j];
        double xr = 2.0 * p - xi;
        D.xr[j] = xr;
        if (P.want_fpe)
            D.dx[j] = xr - xi;
        double refl = P.rho * xr + (1.0 - P.rho) * xi;
        D.x[j] = P.w * refl + (1.0 - P.w) * D.x0[j];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        *D.inner_total += it - 1;
}

// Jacobi preconditioner refresh when tau changes (reference
// refresh_inner_precond_kernel, src/kernels/pdhcg_kernels.cu:482-495, and
// the tol_scale of src/pdhg_core_op.cu:511-523): m = diag_h + 1/tau (1 when
// <= 0), partials of sum |m|.
__global__ void __launch_bounds__(TPB) bb_precond_kernel(int n, const double *diag_h, double inv_tau, double *m_diag,
                                                         double *m_inv, double *partials)
{
    const int ops[1] = {RSUM};
    double acc[1] = {0.0};
    for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) {
        double m = diag_h[i] + inv_tau;
        if (m <= 0.0)
            m = 1.0;
        m_diag[i] = m;
        m_inv[i] = 1.0 / m;
        acc[0] += fabs(m);
    }
    block_reduce_store<1>(acc, ops, partials);
}

__global__ void bb_tol_scale_kernel(const double *sum, int n, double *tol_scale)
{
    *tol_scale = n > 0 ? sqrt(*sum / (double)n) : 1.0;
}

// inner tolerance schedule after a fixed-point error (reference
// compute_fixed_point_error, src/pdhg_core_op.cu:1029-1034)
__global__ void bb_tol_update_kernel(const double *fpe_sums, double step, double omega, double min_tol, double *tol)
{
    double pn = sqrt(fpe_sums[0]);
    *tol = fmin(*tol, fmax(0.0005 * pn / step * omega, min_tol));
}

// diag(Q) + diag(R^T D R) for the preconditioner (reference
// initialize_inner_solver, src/solver_state.cu:321-367)
// R_dense: R row-major k x width over columns 0..width-1 (then R^T is not used)
__global__ void bb_diag_h_kernel(int n, int sparse, const int *Q_rp, const int *Q_ci, const double *Q_v, int k,
                                 const int *Rt_rp, const int *Rt_ci, const double *Rt_v, const double *R_dense,
                                 int width, int dkind, const double *Ddiag, const double *Ddense, double *diag_h)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        if (sparse)
            for (int t = Q_rp[i]; t < Q_rp[i + 1]; ++t)
                if (Q_ci[t] == i)
                    s += Q_v[t];
        double r = 0.0;
        if (k > 0 && R_dense) { // column i (empty past the width), rows in increasing order
            const double *col = R_dense + i;
            const size_t w = width;
            if (i >= width)
                r = 0.0;
            else if (dkind == 1)
                for (int a = 0; a < k; ++a)
                    r += Ddiag[a] * col[a * w] * col[a * w];
            else if (dkind == 2)
                for (int a = 0; a < k; ++a)
                    for (int b = 0; b < k; ++b)
                        r += col[a * w] * col[b * w] * Ddense[(size_t)a * k + b];
            else
                for (int a = 0; a < k; ++a)
                    r += col[a * w] * col[a * w];
        } else if (k > 0) {
            int b = Rt_rp[i], e = Rt_rp[i + 1];
            if (dkind == 1)
                for (int t = b; t < e; ++t)
                    r += Ddiag[Rt_ci[t]] * Rt_v[t] * Rt_v[t];
            else if (dkind == 2)
                for (int ta = b; ta < e; ++ta)
                    for (int tb = b; tb < e; ++tb)
                        r += Rt_v[ta] * Rt_v[tb] * Ddense[(size_t)Rt_ci[ta] * k + Rt_ci[tb]];
            else
                for (int t = b; t < e; ++t)
                    r += Rt_v[t] * Rt_v[t];
        }
        diag_h[i] = s + r;
    }
}

// qx = Q v (+ R^T D R v) for the residual evaluation and the result, one
// cooperative launch (same Q apply as the inner loop).
template <int G>
__global__ void __launch_bounds__(TPB) q_apply_kernel(BBData D, const double *v, double *qx)
{
    cgb::grid_group grid = cgb::this_grid();
    __shared__ double drx[BB_MAX_RANK];
    const int lane = threadIdx.x & 31;
    const int gwarp = blockIdx.x * WARPS + (threadIdx.x >> 5), nwarps = gridDim.x * WARPS;
    if (D.k > 0) {
        bb_rx_partials(D, v);
        grid.sync();
        bb_rx_fold(D);
        grid.sync();
        bb_drx_smem(D, drx);
    }
    const int sub = lane % G, per = 32 / G;
    for (int base = gwarp * per; base < D.n; base += nwarps * per) {
        int j = base + lane / G;
        bool ok = j < D.n;
        double q = bb_q_row<G>(D, v, drx, ok ? j : 0, sub, ok);
        if (ok && sub == 0)
            qx[j] = q;
    }
}

// Power iterations on a sparse Q for its largest eigenvalue and, shifted,
// its smallest (reference estimate_maximum_eigenvalue /
// estimate_minimum_eigenvalue, src/pdhg_core_op.cu:1498-1671), one
// cooperative launch each.  out = {lambda, iterations}.
__global__ void __launch_bounds__(TPB) power_eig_kernel(int n, const int *Q_rp, const int *Q_ci, const double *Q_v,
                                                        double *v, double *av, double *part, int max_iter,
                                                        double tol, int shifted, double lmax, double *out)
{
    cgb::grid_group grid = cgb::this_grid();
    const int nb = gridDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    double *p0 = part, *p1 = part + nb;
    double lam = 0.0;
    int it = 0;
    for (; it < max_iter; ++it) {
        double a = 0.0;
        for (int i = tid; i < n; i += nth)
            a += v[i] * v[i];
        bb_block_partial(a, p0);
        grid.sync();
        double inv = 1.0 / sqrt(bb_fold(p0, nb));
        for (int i = tid; i < n; i += nth)
            v[i] *= inv;
        grid.sync();
        a = 0.0;
        for (int i = tid; i < n; i += nth) {
            double s = 0.0;
            for (int t = Q_rp[i]; t < Q_rp[i + 1]; ++t)
                s += Q_v[t] * v[Q_ci[t]];
            if (shifted)
                s = -s + lmax * v[i];
            av[i] = s;
            a += v[i] * s;
        }
        bb_block_partial(a, p1);
        grid.sync();
        double old = lam;
        lam = bb_fold(p1, nb);
        if (it > 0 && fabs(lam - old) < tol)
            break;
        for (int i = tid; i < n; i += nth)
            v[i] = av[i];
        grid.sync();
    }
    if (tid == 0) {
        out[0] = shifted ? lmax - lam : lam;
        out[1] = (double)it;
    }
}

} // namespace pdhcg
