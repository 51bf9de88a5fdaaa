// batch.cu -- many small LP / diagonal-QP instances in one persistent launch.
//
// Each instance runs the restarted Halpern PDHG of the single-instance
// solver (reference optimize, src/solver.cu:121-170, with the step of
// pdhg_update, the residuals of compute_residual, the restart test and the
// PID primal weight of perform_restart), but entirely inside one thread
// group of a CTA: its scaled matrix (A and A^T, FP32 values, 16-bit column
// indices) and all its vectors live in shared memory for the whole solve,
// so an iteration is two passes over shared memory separated by group
// barriers and never touches HBM.  Groups pull instances from a global
// counter (largest first), so a launch of #SM x k CTAs keeps every SM busy
// until the batch is done.
//
// Precision: FP32 matrix values and iterates, products and every reduction
// accumulated in FP64; the scaling factors, step sizes, primal weight,
// residuals and objectives are FP64.
//
// Launch shapes (threads per group GROUP, groups per CTA) are template
// parameters; pdhcg_b200_batch_autotune times the candidates on a sample of
// the batch and keeps the fastest per size class.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <optional>
#include <thread>
#include <vector>

#include "pdhcg.h"
#include "pdhcg_b200.h"

namespace {

constexpr double SCALE_EPS = 1e-12;
// shared memory one instance may use (the opt-in maximum per CTA, less room
// for the static arrays)
constexpr int SMEM_CAP = 227 * 1024 - 1024;

struct BInst {            // one instance, offsets into the packed arrays
    int n, m;
    long long rp_off;     // A row pointers  (m + 1, local entry offsets)
    long long trp_off;    // A^T row pointers (n + 1)
    long long k_off;      // entries of A (and of A^T, same count)
    long long x_off;      // x-side vectors (n)
    long long y_off;      // y-side vectors (m)
    long long so_off;     // slice tables: A's (m/32 + 2 ints), then A^T's (n/32 + 2 ints)
    int sell_a, sell_at;  // entries of A and A^T in the sliced layout (padding included)
    int smem;             // bytes of shared memory the instance needs
    int qmode;            // 0 LP, 1 diagonal Q
    double obj_const;
};

struct BParams {
    double eps_opt, eps_feas;
    double time_limit_ns;          // per instance, checked at every evaluation
    int iter_limit, freq;
    int l2;
    int ruiz_iters;
    int has_pc;
    double pc_alpha;
    int bound_obj;
    int sv_max_iter;
    double sv_tol;
    double rho;                    // reflection coefficient
    double suff, nec, artificial;  // restart thresholds
    double i_smooth, k_p, k_i, k_d;
};

struct BData {               // packed inputs and outputs of the whole batch
    const int *A_rp, *A_ci, *At_rp, *At_ci;
    const double *A_v, *At_v;
    const double *c, *l, *u, *q;     // x side (q: diagonal, 0 for LP)
    const double *lc, *uc;           // y side
    const double *v0;                // power-method start vector (rand_r(1234) in [-1, 1])
    const int *S_tab;                // slice tables of the sliced layout
    const BInst *inst;
    const int *order;                // instance indices, largest first
    int count;
    int *next;                       // work counter (starts at 0)
    double *x_out, *y_out;           // unscaled solutions
    double *stats;                   // per instance: BS_COUNT doubles
};

enum BStat { BS_STATUS = 0, BS_ITERS, BS_POBJ, BS_DOBJ, BS_ABS_P, BS_ABS_D, BS_REL_P, BS_REL_D, BS_GAP, BS_REL_GAP, BS_COUNT };

__host__ __device__ inline int print_freq(int it)
{
    int step = 10;
    long long th = 1000;
    while (it >= th) {
        step *= 10;
        th *= 10;
    }
    return step;
}

// Matrices in shared memory are sliced (SELL-32): rows in slices of 32,
// slice s holding (max row length in s) x 32 entries, entry k of the slice's
// row r at so[s] + 32 k + (r mod 32), rows shorter than the slice's longest
// padded with (column 0, value 0).  The 32 lanes of a warp own the 32 rows
// of one slice, so a product reads indices and values without bank
// conflicts, every lane of the warp runs the same trip count, and the
// padding adds exact zeros after a row's entries (the sums are those of the
// plain CSR loop).  so[] has one entry per slice plus the end.
__host__ __device__ inline int slices(int rows) { return (rows + 31) >> 5; }

// Shared-memory layout of one instance (byte offsets; every array 16-byte aligned).
struct Layout {
    int arp, atrp, aci, atci, av, atv;                 // matrices: slice tables, indices, values
    int c, l, u, q, x0, x, xp, xr, dx, ds;             // x side, float
    int lc, uc, y0, y, yp, dy;                         // y side, float
    int vr, cr;                                        // scaling, double
    int red;                                           // reduction scratch, double[320]
    int total;
    __host__ __device__ static int al(int b) { return (b + 15) & ~15; }
    __host__ __device__ Layout(int n, int m, int sell_a, int sell_at)
    {
        int o = 0;
        arp = o; o += al(4 * (slices(m) + 1));
        atrp = o; o += al(4 * (slices(n) + 1));
        aci = o; o += al(2 * sell_a);
        atci = o; o += al(2 * sell_at);
        av = o; o += al(4 * sell_a);
        atv = o; o += al(4 * sell_at);
        c = o; o += al(4 * n);
        l = o; o += al(4 * n);
        u = o; o += al(4 * n);
        q = o; o += al(4 * n);
        x0 = o; o += al(4 * n);
        x = o; o += al(4 * n);
        xp = o; o += al(4 * n);
        xr = o; o += al(4 * n);
        dx = o; o += al(4 * n);
        ds = o; o += al(4 * n);
        lc = o; o += al(4 * m);
        uc = o; o += al(4 * m);
        y0 = o; o += al(4 * m);
        y = o; o += al(4 * m);
        yp = o; o += al(4 * m);
        dy = o; o += al(4 * m);
        vr = o; o += al(8 * n);
        cr = o; o += al(8 * m);
        red = o; o += al(8 * 10 * 32); // reduce_n of up to 10 values over up to 32 warps
        total = o;
    }
};

// ---- thread group: GROUP threads of a CTA that own one instance ----------
template <int BT, int GROUP>
struct Grp {
    int id, t;
    __device__ Grp() : id(threadIdx.x / GROUP), t(threadIdx.x % GROUP) {}
    __device__ void sync() const
    {
        if (GROUP == BT)
            __syncthreads();
        else if (GROUP == 32)
            __syncwarp();
        else
            asm volatile("bar.sync %0, %1;" ::"r"(1 + id), "r"(GROUP) : "memory");
    }
    // sum (or max) over the group in a fixed order; every thread gets the result
    __device__ double reduce(double v, bool is_max, double *red) const
    {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double w = __shfl_xor_sync(0xffffffffu, v, o);
            v = is_max ? fmax(v, w) : v + w;
        }
        if (GROUP == 32)
            return v;
        constexpr int NW = GROUP / 32;
        if ((t & 31) == 0)
            red[t >> 5] = v;
        sync();
        double r = red[0];
        for (int i = 1; i < NW; ++i)
            r = is_max ? fmax(r, red[i]) : r + red[i];
        sync();
        return r;
    }
    // K values at once (bit k of is_max: maximum instead of sum), each in the
    // order reduce() uses, with two barriers for all of them; red holds
    // K x GROUP / 32 doubles
    template <int K>
    __device__ void reduce_n(double (&v)[K], unsigned is_max, double *red) const
    {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const bool mx = (is_max >> k) & 1u;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double w = __shfl_xor_sync(0xffffffffu, v[k], o);
                v[k] = mx ? fmax(v[k], w) : v[k] + w;
            }
        }
        if (GROUP == 32)
            return;
        constexpr int NW = GROUP / 32;
        if ((t & 31) == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k)
                red[k * NW + (t >> 5)] = v[k];
        }
        sync();
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const bool mx = (is_max >> k) & 1u;
            double r = red[k * NW];
            for (int i = 1; i < NW; ++i)
                r = mx ? fmax(r, red[k * NW + i]) : r + red[k * NW + i];
            v[k] = r;
        }
        sync();
    }
};

__device__ __forceinline__ double clampd(double lo, double x, double hi) { return fmax(lo, fmin(x, hi)); }
__device__ __forceinline__ double gtimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return (double)t;
}
__device__ __forceinline__ double nterm(double v, int l2) { return l2 ? v * v : (isfinite(v) ? fabs(v) : INFINITY); }

// row r of a sliced matrix times v, FP64 accumulation in entry order
__device__ __forceinline__ double sell_dot(const int *so, const unsigned short *ci, const float *va, const float *v,
                                           int r)
{
    const int sl = r >> 5, ln = r & 31;
    const int o = so[sl], len = (so[sl + 1] - o) >> 5;
    double acc = 0.0;
    for (int k = 0; k < len; ++k) {
        const int e = o + (k << 5) + ln;
        acc += (double)va[e] * (double)v[ci[e]];
    }
    return acc;
}

template <int BT, int GROUP>
__device__ void solve_instance(const BData &D, const BParams &P, int idx, char *sm, const Grp<BT, GROUP> &g)
{
    const BInst I = D.inst[idx];
    const int n = I.n, m = I.m;
    const int *Arp = D.A_rp + I.rp_off, *Atrp = D.At_rp + I.trp_off;
    const int nnz = Arp[m];
    const int *Aci = D.A_ci + I.k_off, *Atci = D.At_ci + I.k_off;
    const double *Av = D.A_v + I.k_off, *Atv = D.At_v + I.k_off;
    const double *gc = D.c + I.x_off, *gl = D.l + I.x_off, *gu = D.u + I.x_off, *gq = D.q + I.x_off;
    const double *glc = D.lc + I.y_off, *guc = D.uc + I.y_off;
    const int nsa = slices(m), nsat = slices(n);
    const int *gsa = D.S_tab + I.so_off, *gsat = gsa + nsa + 1;
    Layout Lo(n, m, I.sell_a, I.sell_at);
    int *arp = (int *)(sm + Lo.arp), *atrp = (int *)(sm + Lo.atrp);
    unsigned short *aci = (unsigned short *)(sm + Lo.aci), *atci = (unsigned short *)(sm + Lo.atci);
    float *av = (float *)(sm + Lo.av), *atv = (float *)(sm + Lo.atv);
    float *c = (float *)(sm + Lo.c), *l = (float *)(sm + Lo.l), *u = (float *)(sm + Lo.u), *q = (float *)(sm + Lo.q);
    float *x0 = (float *)(sm + Lo.x0), *x = (float *)(sm + Lo.x), *xp = (float *)(sm + Lo.xp);
    float *xr = (float *)(sm + Lo.xr), *dx = (float *)(sm + Lo.dx), *ds = (float *)(sm + Lo.ds);
    float *lc = (float *)(sm + Lo.lc), *uc = (float *)(sm + Lo.uc), *y0 = (float *)(sm + Lo.y0);
    float *y = (float *)(sm + Lo.y), *yp = (float *)(sm + Lo.yp), *dy = (float *)(sm + Lo.dy);
    double *vr = (double *)(sm + Lo.vr), *cr = (double *)(sm + Lo.cr), *red = (double *)(sm + Lo.red);
    const int t = g.t;
    const bool hasq = I.qmode == 1;
    const double t_start = g.reduce(t == 0 ? gtimer_ns() : 0.0, true, red); // one clock for the group

    // ---- unscaled norms for the relative errors (reference
    // src/solver_state.cu:854-934) ----------------------------------------
    double c2 = 0.0, cmax = 0.0, b2 = 0.0, bmax = 0.0;
    for (int j = t; j < n; j += GROUP) {
        double v = gc[j];
        c2 += v * v;
        cmax = fmax(cmax, fabs(v));
    }
    for (int i = t; i < m; i += GROUP) {
        double lo = glc[i], up = guc[i], bb = 0.0, bm = 0.0;
        if (isfinite(lo) && lo != up) {
            bb += lo * lo;
            bm = fmax(bm, fabs(lo));
        }
        if (isfinite(up)) {
            bb += up * up;
            bm = fmax(bm, fabs(up));
        }
        b2 += bb;
        bmax = fmax(bmax, bm);
    }
    {
        double rv[4] = {c2, cmax, b2, bmax};
        g.reduce_n(rv, 0xau, red);
        c2 = rv[0];
        cmax = rv[1];
        b2 = rv[2];
        bmax = rv[3];
    }
    const double cnorm = P.l2 ? sqrt(c2) : cmax, bnorm = P.l2 ? sqrt(b2) : bmax;

    // ---- rescaling (reference rescale_problem, src/preconditioner.c:654-713):
    // cumulative factors in FP64, computed from the original FP64 entries ------
    for (int j = t; j < n; j += GROUP)
        vr[j] = 1.0;
    for (int i = t; i < m; i += GROUP)
        cr[i] = 1.0;
    g.sync();
    // Ruiz (max) passes, then one Pock-Chambolle (power-sum) pass; each pass
    // takes both factors from the same scaled matrix, then applies them.  The
    // new factors are parked in the still unused float vector areas.
    double *fr = (double *)(sm + Lo.lc), *fcol = (double *)(sm + Lo.c);
    for (int it = 0; it < P.ruiz_iters + (P.has_pc ? 1 : 0); ++it) {
        const bool ruiz = it < P.ruiz_iters;
        const double a_row = ruiz ? 0.0 : P.pc_alpha, a_col = ruiz ? 0.0 : 2.0 - P.pc_alpha;
        for (int i = t; i < m; i += GROUP) {
            double s = 0.0;
            for (int k = Arp[i]; k < Arp[i + 1]; ++k) {
                double a = fabs(Av[k]) / (cr[i] * vr[Aci[k]]);
                s = ruiz ? fmax(s, a) : s + (a_row == 1.0 ? a : pow(a, a_row));
            }
            fr[i] = s < SCALE_EPS ? 1.0 : sqrt(s);
        }
        for (int j = t; j < n; j += GROUP) {
            double s = 0.0;
            for (int k = Atrp[j]; k < Atrp[j + 1]; ++k) {
                double a = fabs(Atv[k]) / (cr[Atci[k]] * vr[j]);
                s = ruiz ? fmax(s, a) : s + (a_col == 1.0 ? a : pow(a, a_col));
            }
            fcol[j] = s < SCALE_EPS ? 1.0 : sqrt(s);
        }
        g.sync();
        for (int i = t; i < m; i += GROUP)
            cr[i] *= fr[i];
        for (int j = t; j < n; j += GROUP)
            vr[j] *= fcol[j];
        g.sync();
    }
    // bound / objective rescaling (reference bound_obj_rescaling, :602-652)
    double sb = 1.0, sc = 1.0;
    if (P.bound_obj) {
        double bb2 = 0.0, cc2 = 0.0;
        for (int i = t; i < m; i += GROUP) {
            double lo = glc[i] / cr[i], up = guc[i] / cr[i];
            if (isfinite(lo) && lo != up)
                bb2 += lo * lo;
            if (isfinite(up))
                bb2 += up * up;
        }
        for (int j = t; j < n; j += GROUP) {
            double v = gc[j] / vr[j];
            cc2 += v * v;
        }
        double rv[2] = {bb2, cc2};
        g.reduce_n(rv, 0u, red);
        bb2 = rv[0];
        cc2 = rv[1];
        sb = 1.0 / (sqrt(bb2) + 1.0);
        sc = 1.0 / (sqrt(cc2) + 1.0);
    }
    // ---- scaled data in shared memory (sliced matrices) --------------------
    for (int s = t; s <= nsa; s += GROUP)
        arp[s] = gsa[s];
    for (int s = t; s <= nsat; s += GROUP)
        atrp[s] = gsat[s];
    g.sync();
    for (int i = t; i < m; i += GROUP) {
        const int o = arp[i >> 5] + (i & 31), len = (arp[(i >> 5) + 1] - arp[i >> 5]) >> 5;
        const int k0 = Arp[i], rl = Arp[i + 1] - k0;
        for (int k = 0; k < len; ++k) {
            const int col = k < rl ? Aci[k0 + k] : 0;
            aci[o + 32 * k] = (unsigned short)col;
            av[o + 32 * k] = k < rl ? (float)(Av[k0 + k] / (cr[i] * vr[col])) : 0.0f;
        }
    }
    for (int j = t; j < n; j += GROUP) {
        const int o = atrp[j >> 5] + (j & 31), len = (atrp[(j >> 5) + 1] - atrp[j >> 5]) >> 5;
        const int k0 = Atrp[j], cl = Atrp[j + 1] - k0;
        for (int k = 0; k < len; ++k) {
            const int row = k < cl ? Atci[k0 + k] : 0;
            atci[o + 32 * k] = (unsigned short)row;
            atv[o + 32 * k] = k < cl ? (float)(Atv[k0 + k] / (vr[j] * cr[row])) : 0.0f;
        }
    }
    for (int j = t; j < n; j += GROUP) {
        const double vj = vr[j];
        c[j] = (float)(gc[j] / vj * sc);
        l[j] = (float)(gl[j] * vj * sb);
        u[j] = (float)(gu[j] * vj * sb);
        q[j] = hasq ? (float)(gq[j] / (vj * vj) * (sc / sb) + 1e-12) : 0.0f;
        const float x00 = (float)clampd((double)l[j], 0.0, (double)u[j]);
        x0[j] = x[j] = xp[j] = xr[j] = x00;
        dx[j] = ds[j] = 0.0f;
    }
    for (int i = t; i < m; i += GROUP) {
        lc[i] = (float)(glc[i] / cr[i] * sb);
        uc[i] = (float)(guc[i] / cr[i] * sb);
        y0[i] = y[i] = yp[i] = dy[i] = 0.0f;
    }
    g.sync();

    // ---- step size: power method on A A^T (reference
    // estimate_maximum_singular_value, src/pdhg_core_op.cu:1673-1788) ----------
    double step = 1.0;
    if (nnz > 0) {
        float *v = yp, *nv = dy, *dp = xr; // scratch, reset below
        double a = 0.0;
        for (int i = t; i < m; i += GROUP) {
            v[i] = (float)D.v0[i];
            a += D.v0[i] * D.v0[i];
        }
        a = g.reduce(a, false, red);
        double inv = 1.0 / sqrt(a);
        for (int i = t; i < m; i += GROUP)
            v[i] = (float)((double)v[i] * inv);
        g.sync();
        double s2 = 1.0;
        for (int it = 0; it < P.sv_max_iter; ++it) {
            for (int j = t; j < n; j += GROUP)
                dp[j] = (float)sell_dot(atrp, atci, atv, v, j);
            g.sync();
            a = 0.0;
            for (int i = t; i < m; i += GROUP) {
                const double s = sell_dot(arp, aci, av, dp, i);
                nv[i] = (float)s;
                a += s * (double)v[i];
            }
            s2 = g.reduce(a, false, red);
            a = 0.0;
            for (int i = t; i < m; i += GROUP) {
                double r = (double)nv[i] - s2 * (double)v[i];
                a += r * r;
            }
            a = g.reduce(a, false, red);
            if (sqrt(a) < P.sv_tol)
                break;
            a = 0.0;
            for (int i = t; i < m; i += GROUP)
                a += (double)nv[i] * (double)nv[i];
            a = g.reduce(a, false, red);
            inv = 1.0 / sqrt(a);
            for (int i = t; i < m; i += GROUP)
                v[i] = (float)((double)nv[i] * inv);
            g.sync();
        }
        double sv = sqrt(s2);
        step = sv < 1e-12 ? 1.0 : 0.998 / sv;
        for (int i = t; i < m; i += GROUP)
            yp[i] = dy[i] = 0.0f;
        for (int j = t; j < n; j += GROUP)
            xr[j] = x0[j];
        g.sync();
    }
    double omega = P.bound_obj ? 1.0 : (cnorm + 1.0) / (bnorm + 1.0);
    double best_omega = omega, best_gap = INFINITY, pw_sum = 0.0, pw_last = 0.0;
    double fpe = 0.0, fpe0 = 0.0, fpe_last = INFINITY;
    double rel_p = INFINITY, rel_d = INFINITY, rel_gap = INFINITY, abs_p = 0, abs_d = 0, pobj = 0, dobj = 0, gap = 0;
    double dist_x = 0.0, dist_y = 0.0;
    int k = 0, inner = 0, status = TERMINATION_REASON_UNSPECIFIED;
    bool is_major = false, do_restart = false;

    // residual evaluation (compute_residual for LP / diagonal Q without cones)
    auto evaluate = [&](bool want_dist) {
        const double tau = step / omega;
        double pr = 0.0, pslack = 0.0, dy2 = 0.0;
        for (int i = t; i < m; i += GROUP) {
            const double s = sell_dot(arp, aci, av, xp, i);
            double proj = clampd((double)lc[i], s, (double)uc[i]);
            pr = P.l2 ? pr + nterm((s - proj) * cr[i], 1) : fmax(pr, nterm((s - proj) * cr[i], 0));
            double yv = yp[i];
            double lo = lc[i], up = uc[i];
            pslack += fmax(yv, 0.0) * (isfinite(lo) ? lo : 0.0) + fmin(yv, 0.0) * (isfinite(up) ? up : 0.0);
            if (want_dist) {
                double d = yv - (double)y0[i];
                dy2 += d * d;
            }
        }
        double dr = 0.0, cx = 0.0, xqx = 0.0, sx = 0.0, qn = 0.0, an = 0.0, dx2 = 0.0;
        for (int j = t; j < n; j += GROUP) {
            const double s = sell_dot(atrp, atci, atv, yp, j);
            double xv = xp[j], qx = hasq ? (double)q[j] * xv : 0.0;
            double dsl, drr;
            if (!hasq) {
                dsl = ds[j];
                drr = ((double)c[j] - s - dsl) * vr[j];
            } else {
                double gr = qx + (double)c[j] - s;
                double tt = xv - tau * gr;
                double p = fmax((double)l[j], fmin((double)u[j], tt));
                dsl = (p - tt) / tau;
                drr = (gr - dsl) * vr[j];
            }
            dr = P.l2 ? dr + nterm(drr, 1) : fmax(dr, nterm(drr, 0));
            cx += (double)c[j] * xv;
            xqx += xv * qx;
            sx += dsl * xv;
            qn = P.l2 ? qn + nterm(qx * vr[j], 1) : fmax(qn, nterm(qx * vr[j], 0));
            an = P.l2 ? an + nterm(s * vr[j], 1) : fmax(an, nterm(s * vr[j], 0));
            if (want_dist) {
                double d = xv - (double)x0[j];
                dx2 += d * d;
            }
        }
        const bool L2 = P.l2 != 0;
        double rv[10] = {pr, dr, qn, an, pslack, cx, xqx, sx, dx2, dy2};
        g.reduce_n(rv, L2 ? 0u : 0xfu, red);
        pr = rv[0];
        dr = rv[1];
        qn = rv[2];
        an = rv[3];
        pslack = rv[4];
        cx = rv[5];
        xqx = rv[6];
        sx = rv[7];
        dx2 = rv[8];
        dy2 = rv[9];
        auto nrm = [&](double v) { return L2 ? sqrt(v) : v; };
        abs_p = nrm(pr) / sb;
        abs_d = nrm(dr) / sc;
        double hq = hasq ? 0.5 * xqx : 0.0;
        pobj = (cx + hq) / (sb * sc) + I.obj_const;
        dobj = (sx + pslack - hq) / (sb * sc) + I.obj_const;
        rel_p = abs_p / (1.0 + bnorm);
        double den = hasq ? 1.0 + fmax(cnorm, fmax(nrm(qn) / sc, nrm(an) / sc)) : 1.0 + cnorm;
        rel_d = abs_d / den;
        gap = fabs(pobj - dobj);
        rel_gap = gap / (1.0 + fabs(pobj) + fabs(dobj));
        dist_x = sqrt(dx2);
        dist_y = sqrt(dy2);
    };

    // fixed-point error of the last step (compute_fixed_point_error)
    auto fixed_point_error = [&]() {
        double p2 = 0.0, d2 = 0.0, cross = 0.0;
        for (int j = t; j < n; j += GROUP) {
            const double s = sell_dot(atrp, atci, atv, dy, j);
            double d = dx[j];
            p2 += d * d;
            cross += s * d;
        }
        for (int i = t; i < m; i += GROUP) {
            double d = dy[i];
            d2 += d * d;
        }
        double rv[3] = {p2, d2, cross};
        g.reduce_n(rv, 0u, red);
        p2 = rv[0];
        d2 = rv[1];
        cross = rv[2];
        double mv = p2 * omega + d2 / omega;
        return sqrt(mv + 2.0 * step * cross);
    };

    while (k < P.iter_limit) {
        if (is_major || k == 0 || (k % print_freq(k)) == 0) {
            evaluate(is_major || k == 0);
            // elapsed time from thread 0's clock, made uniform by the reduction
            const double el = g.reduce(t == 0 ? gtimer_ns() - t_start : 0.0, true, red);
            if (rel_d < P.eps_feas && rel_p < P.eps_feas && rel_gap < P.eps_opt) {
                status = TERMINATION_REASON_OPTIMAL;
                break;
            }
            if (el >= P.time_limit_ns) {
                status = TERMINATION_REASON_TIME_LIMIT;
                break;
            }
        }
        if (is_major || k == 0) {
            do_restart = false;
            if (k == P.freq)
                do_restart = true;
            else if (k > P.freq) {
                if (fpe <= P.suff * fpe0)
                    do_restart = true;
                if (fpe <= P.nec * fpe0 && fpe > fpe_last)
                    do_restart = true;
                if (inner >= P.artificial * k)
                    do_restart = true;
            }
            fpe_last = fpe;
            if (do_restart) {
                double pd = dist_x, dd = dist_y, ratio = rel_d / rel_p;
                if (pd > 1e-16 && dd > 1e-16 && pd < 1e12 && dd < 1e12 && ratio > 1e-8 && ratio < 1e8) {
                    double err = log(dd) - log(pd) - log(omega);
                    pw_sum = pw_sum * P.i_smooth + err;
                    double derr = err - pw_last;
                    omega *= exp(P.k_p * err + P.k_i * pw_sum + P.k_d * derr);
                    pw_last = err;
                } else {
                    omega = best_omega;
                    pw_sum = 0.0;
                    pw_last = 0.0;
                }
                double gg = fabs(log10(rel_d / rel_p));
                if (gg < best_gap) {
                    best_gap = gg;
                    best_omega = omega;
                }
                for (int j = t; j < n; j += GROUP)
                    x0[j] = x[j] = xp[j];
                for (int i = t; i < m; i += GROUP)
                    y0[i] = y[i] = yp[i];
                g.sync();
                inner = 0;
                fpe_last = INFINITY;
            }
        }
        is_major = ((k + 1) % P.freq) == 0;
        const bool want_fpe = is_major || do_restart;
        const double w = (double)(inner + 1) / (double)(inner + 2);
        const double tau = step / omega, sigma = step * omega;
        const double inv_tau = 1.0 / tau, inv_sigma = 1.0 / sigma;
        // primal step (reference pdhg_update + halpern_update)
        for (int j = t; j < n; j += GROUP) {
            const double s = sell_dot(atrp, atci, atv, y, j);
            double xi = x[j];
            double tt = xi - tau * ((double)c[j] - s);
            if (hasq)
                tt /= (1.0 + tau * (double)q[j]);
            double p = clampd((double)l[j], tt, (double)u[j]);
            double xrr = 2.0 * p - xi;
            xp[j] = (float)p;
            xr[j] = (float)xrr;
            if (!hasq)
                ds[j] = (float)((p - tt) * inv_tau);
            dx[j] = (float)(xrr - xi);
            double refl = P.rho * xrr + (1.0 - P.rho) * xi;
            x[j] = (float)(w * refl + (1.0 - w) * (double)x0[j]);
        }
        g.sync();
        for (int i = t; i < m; i += GROUP) {
            const double s = sell_dot(arp, aci, av, xr, i);
            double yi = y[i];
            double pr = clampd((double)lc[i], s - yi * inv_sigma, (double)uc[i]);
            double yn = yi - sigma * s + sigma * pr;
            double yrr = 2.0 * yn - yi;
            yp[i] = (float)yn;
            dy[i] = (float)(yrr - yi);
            double refl = P.rho * yrr + (1.0 - P.rho) * yi;
            y[i] = (float)(w * refl + (1.0 - w) * (double)y0[i]);
        }
        g.sync();
        if (want_fpe) {
            fpe = fixed_point_error();
            if (do_restart) {
                fpe0 = fpe;
                do_restart = false;
            }
        }
        ++inner;
        ++k;
    }
    if (status == TERMINATION_REASON_UNSPECIFIED) {
        status = TERMINATION_REASON_ITERATION_LIMIT;
        evaluate(false);
    }
    // unscaled solution (reference rescale_solution)
    for (int j = t; j < n; j += GROUP)
        D.x_out[I.x_off + j] = (double)xp[j] / vr[j] / sb;
    for (int i = t; i < m; i += GROUP)
        D.y_out[I.y_off + i] = (double)yp[i] / cr[i] / sc;
    if (t == 0) {
        double *st = D.stats + (size_t)idx * BS_COUNT;
        st[BS_STATUS] = status;
        st[BS_ITERS] = k;
        st[BS_POBJ] = pobj;
        st[BS_DOBJ] = dobj;
        st[BS_ABS_P] = abs_p;
        st[BS_ABS_D] = abs_d;
        st[BS_REL_P] = rel_p;
        st[BS_REL_D] = rel_d;
        st[BS_GAP] = gap;
        st[BS_REL_GAP] = rel_gap;
    }
    g.sync();
}

template <int BT, int GROUP>
__global__ void __launch_bounds__(BT) batch_kernel(BData D, BParams P, int smem_per_group)
{
    extern __shared__ __align__(16) char smem[];
    __shared__ int s_idx[BT / GROUP];
    Grp<BT, GROUP> g;
    char *sm = smem + (size_t)g.id * smem_per_group;
    for (;;) {
        if (g.t == 0)
            s_idx[g.id] = atomicAdd(D.next, 1);
        g.sync();
        const int w = s_idx[g.id];
        g.sync();
        if (w >= D.count)
            break;
        solve_instance<BT, GROUP>(D, P, D.order[w], sm, g);
    }
}

// A^T of every instance, one warp per instance, entries of each column in
// increasing row order (what a counting sort over the rows gives, so the
// batch kernel sums A^T y in the same order as with a host transpose):
// column counts by atomics, a warp scan into the row pointers of A^T, then
// the entries scattered in entry order, 32 at a time; the lanes of a chunk
// that share a column rank themselves with __match_any_sync and the
// column's first lane advances its cursor.  cur: n ints of scratch per
// instance.
__global__ void __launch_bounds__(256) transpose_kernel(const int *A_rp, const int *A_ci, const double *A_v,
                                                        int *At_rp, int *At_ci, double *At_v, int *cur,
                                                        const BInst *inst, int count)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int warps = (int)((gridDim.x * blockDim.x) >> 5);
    for (int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); w < count; w += warps) {
        const BInst b = inst[w];
        const int n = b.n, m = b.m;
        const int *rp = A_rp + b.rp_off;
        const int *ci = A_ci + b.k_off;
        const double *av = A_v + b.k_off;
        int *trp = At_rp + b.trp_off;
        int *cu = cur + b.x_off;
        int *tci = At_ci + b.k_off;
        double *tv = At_v + b.k_off;
        const int nnz = rp[m];
        for (int j = lane; j <= n; j += 32)
            trp[j] = 0;
        __syncwarp();
        for (int k = lane; k < nnz; k += 32)
            atomicAdd(&trp[ci[k] + 1], 1);
        __syncwarp();
        int carry = 0; // inclusive scan of trp[1..n]
        for (int j0 = 1; j0 <= n; j0 += 32) {
            const int j = j0 + lane;
            int v = j <= n ? trp[j] : 0;
            for (int d = 1; d < 32; d <<= 1) {
                const int t = __shfl_up_sync(FULL, v, d);
                if (lane >= d)
                    v += t;
            }
            v += carry;
            if (j <= n)
                trp[j] = v;
            carry = __shfl_sync(FULL, v, 31);
        }
        __syncwarp();
        for (int j = lane; j < n; j += 32)
            cu[j] = trp[j];
        __syncwarp();
        for (int k0 = 0; k0 < nnz; k0 += 32) {
            const int k = k0 + lane;
            const bool ok = k < nnz;
            const int col = ok ? ci[k] : -1 - lane;
            int row = 0;
            if (ok) { // rp[lo] <= k < rp[hi]
                int lo = 0, hi = m;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (rp[mid] <= k)
                        lo = mid;
                    else
                        hi = mid;
                }
                row = lo;
            }
            const unsigned same = __match_any_sync(FULL, col);
            const int rank = __popc(same & ((1u << lane) - 1u));
            const int base = ok ? cu[col] : 0;
            __syncwarp();
            if (ok) {
                tci[base + rank] = row;
                tv[base + rank] = av[k];
                if (rank == 0)
                    cu[col] = base + __popc(same);
            }
            __syncwarp();
        }
    }
}

} // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

thread_local pdhcg_b200_batch_stats_t g_batch_stats;

// f(0) .. f(count - 1) on up to hardware_concurrency host threads
template <typename F>
void parallel_for(int count, F &&f)
{
    int nt = (int)std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 32u);
    nt = std::min(nt, std::max(1, count / 16));
    if (nt <= 1) {
        for (int i = 0; i < count; ++i)
            f(i);
        return;
    }
    std::atomic<int> next{0};
    auto work = [&]() {
        for (int i; (i = next.fetch_add(1)) < count;)
            f(i);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) {
        try {
            pool.emplace_back(work);
        } catch (...) { // fewer threads: the ones there take the rest
            break;
        }
    }
    work(); // the calling thread takes part
    for (auto &th : pool)
        th.join();
}

#define BCK(call)                                                                                                      \
    do {                                                                                                               \
        cudaError_t e_ = (call);                                                                                       \
        if (e_ != cudaSuccess) {                                                                                       \
            std::fprintf(stderr, "[pdhcg_b200_solve_batch] %s: %s\n", #call, cudaGetErrorString(e_));                 \
            return -1;                                                                                                 \
        }                                                                                                              \
    } while (0)

// Page-locked staging memory and device memory that batch solves keep
// between calls (one host buffer, one device buffer per device), grown on
// demand (with 1/8 headroom) and freed by pdhcg_b200_batch_release.  A call
// holds g_arena_mu from packing to the copy of the results, so concurrent
// batch solves in one process take turns.
struct Arena {
    char *p = nullptr;
    size_t cap = 0;
};
std::mutex g_arena_mu;
Arena g_host_arena;
std::map<int, Arena> g_dev_arena;

char *host_arena(size_t need)
{
    Arena &a = g_host_arena;
    if (a.cap < need) {
        if (a.p)
            cudaFreeHost(a.p);
        a = Arena{};
        void *p = nullptr;
        const size_t want = need + need / 8;
        if (cudaHostAlloc(&p, want, cudaHostAllocPortable) != cudaSuccess)
            return nullptr;
        a.p = (char *)p;
        a.cap = want;
    }
    return a.p;
}

char *dev_arena(int dev, size_t need)
{
    Arena &a = g_dev_arena[dev];
    if (a.cap < need) {
        if (a.p)
            cudaFree(a.p);
        a = Arena{};
        void *p = nullptr;
        const size_t want = need + need / 8;
        if (cudaMalloc(&p, want) != cudaSuccess)
            return nullptr;
        a.p = (char *)p;
        a.cap = want;
    }
    return a.p;
}

// Byte offsets of the packed arrays (each 256-byte aligned): the inputs
// first, copied host to device in one piece; then A^T and the scratch
// (device only); then the outputs, copied back in one piece.  The staging
// buffer holds the inputs and, after them (at in_end), the outputs.
struct Pack {
    size_t A_rp, A_ci, A_v, c, l, u, q, lc, uc, v0, S, inst, order, in_end;
    size_t At_rp, At_ci, At_v, cur, next, out, x_out, y_out, stats, end;
    Pack(long long rp, long long trp, long long k, long long x, long long y, long long s, int max_m, int nb,
         int classes)
    {
        size_t o = 0;
        auto put = [&o](long long bytes) {
            const size_t at = o;
            o += ((size_t)std::max(bytes, 1LL) + 255) & ~(size_t)255;
            return at;
        };
        A_rp = put(rp * 4);
        A_ci = put(k * 4);
        A_v = put(k * 8);
        c = put(x * 8);
        l = put(x * 8);
        u = put(x * 8);
        q = put(x * 8);
        lc = put(y * 8);
        uc = put(y * 8);
        v0 = put((long long)max_m * 8);
        S = put(s * 4);
        inst = put((long long)nb * (long long)sizeof(BInst));
        order = put((long long)nb * 4);
        in_end = o;
        At_rp = put(trp * 4);
        At_ci = put(k * 4);
        At_v = put(k * 8);
        cur = put(x * 4);
        next = put((long long)classes * 4);
        out = o;
        x_out = put(x * 8);
        y_out = put(y * 8);
        stats = put((long long)nb * BS_COUNT * 8);
        end = o;
    }
    size_t host_bytes() const { return in_end + (end - out); }
};

// The streams and events of one call's class launches (released on every
// exit path).
struct ClassStreams {
    cudaEvent_t ready = nullptr;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> done;
    ~ClassStreams()
    {
        for (cudaStream_t st : streams)
            cudaStreamDestroy(st);
        for (cudaEvent_t ev : done)
            cudaEventDestroy(ev);
        if (ready)
            cudaEventDestroy(ready);
    }
};

// A launch shape: threads per CTA, threads per instance group.
struct Shape {
    int bt, group;
};
const Shape SHAPES[] = {{128, 32}, {256, 64}, {256, 128}, {256, 256}, {512, 512}, {1024, 1024}, {128, 128}};
constexpr int NSHAPES = sizeof(SHAPES) / sizeof(SHAPES[0]);

template <int BT, int GROUP>
cudaError_t launch_shape(const BData &D, const BParams &P, int smem_group, int sms, cudaStream_t s)
{
    constexpr int G = BT / GROUP;
    size_t smem = (size_t)smem_group * G;
    auto kern = batch_kernel<BT, GROUP>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BT, smem);
    if (e != cudaSuccess)
        return e;
    if (per_sm < 1)
        return cudaErrorInvalidConfiguration;
    int groups = (D.count + G - 1) / G;
    int grid = std::max(1, std::min(groups, sms * per_sm));
    kern<<<grid, BT, smem, s>>>(D, P, smem_group);
    return cudaGetLastError();
}

cudaError_t launch(int shape, const BData &D, const BParams &P, int smem_group, int sms, cudaStream_t s)
{
    switch (shape) {
    case 0: return launch_shape<128, 32>(D, P, smem_group, sms, s);
    case 1: return launch_shape<256, 64>(D, P, smem_group, sms, s);
    case 2: return launch_shape<256, 128>(D, P, smem_group, sms, s);
    case 3: return launch_shape<256, 256>(D, P, smem_group, sms, s);
    case 4: return launch_shape<512, 512>(D, P, smem_group, sms, s);
    case 5: return launch_shape<1024, 1024>(D, P, smem_group, sms, s);
    default: return launch_shape<128, 128>(D, P, smem_group, sms, s);
    }
}

// Q diagonal-only?  (the batch supports LP and diagonal Q; reference
// detect_q_type, src/utils.cu:834-885)
bool diag_q(const qp_problem_t *p, std::vector<double> &q)
{
    q.assign(p->num_variables, 0.0);
    if (p->num_rank_lowrank_obj > 0 && p->objective_lowrank_matrix_num_nonzeros > 0)
        return false;
    if (!p->objective_sparse_matrix || p->objective_sparse_matrix_num_nonzeros == 0)
        return true;
    const CsrComponent *Q = p->objective_sparse_matrix;
    for (int r = 0; r < p->num_variables; ++r)
        for (int k = Q->row_ptr[r]; k < Q->row_ptr[r + 1]; ++k) {
            if (Q->col_ind[k] != r && Q->val[k] != 0.0)
                return false;
            if (Q->col_ind[k] == r)
                q[r] += Q->val[k];
        }
    return true;
}

// Size band of an instance by its shared-memory need: band b holds the
// needs in (CAP / 2^(b+1), CAP / 2^b], band BATCH_BANDS - 1 everything
// smaller.  Instances of one band form one launch (a size class).
constexpr int BATCH_BANDS = 7;
int size_band(int smem)
{
    int b = 0;
    while (b < BATCH_BANDS - 1 && (long long)smem * 2 <= (long long)(SMEM_CAP >> b))
        ++b;
    return b;
}

// The slice tables of p's A and A^T for the sliced layout: T holds, for
// each 32 rows of A, the offset of its slice (32 x its longest row), then
// the end, then the same for A^T.  False when A is not valid CSR.
bool slice_tables(const qp_problem_t *p, std::vector<int> &T)
{
    const int n = p->num_variables, m = p->num_constraints;
    const int *rp = p->constraint_matrix->row_ptr, *ci = p->constraint_matrix->col_ind;
    bool ok = rp[0] == 0;
    for (int r = 0; ok && r < m; ++r)
        ok = rp[r] <= rp[r + 1];
    const int nnz = ok ? rp[m] : 0;
    for (int k = 0; ok && k < nnz; ++k)
        ok = ci[k] >= 0 && ci[k] < n;
    if (!ok)
        return false;
    const int sa = slices(m), sat = slices(n);
    T.resize(sa + 1 + sat + 1);
    int o = 0;
    for (int s = 0; s < sa; ++s) {
        int mx = 0;
        for (int r = 32 * s; r < std::min(32 * s + 32, m); ++r)
            mx = std::max(mx, rp[r + 1] - rp[r]);
        T[s] = o;
        o += 32 * mx;
    }
    T[sa] = o;
    std::vector<int> cnt(n, 0);
    for (int k = 0; k < nnz; ++k)
        cnt[ci[k]]++;
    int *Tt = T.data() + sa + 1;
    o = 0;
    for (int s = 0; s < sat; ++s) {
        int mx = 0;
        for (int j = 32 * s; j < std::min(32 * s + 32, n); ++j)
            mx = std::max(mx, cnt[j]);
        Tt[s] = o;
        o += 32 * mx;
    }
    Tt[sat] = o;
    return true;
}

// The batch kernel's problem class (LP or diagonal Q, no cones, rows and
// columns below 65536, a constraint matrix)
bool batchable(const qp_problem_t *p, std::vector<double> &qd)
{
    const int n = p->num_variables, m = p->num_constraints;
    return n > 0 && m > 0 && n < 65536 && m < 65536 && p->cones.num_cones == 0 && p->affine_cones.num_cones == 0 &&
           p->constraint_matrix && diag_q(p, qd);
}

// smallest-group shape that holds the class's largest instance
int default_shape(int max_smem, int max_dim)
{
    const int cap = SMEM_CAP;
    int want = max_dim <= 256 ? 32 : (max_dim <= 1024 ? 128 : 256);
    for (int sh = 0; sh < NSHAPES; ++sh) {
        if (SHAPES[sh].group < want)
            continue;
        if ((long long)max_smem * (SHAPES[sh].bt / SHAPES[sh].group) <= cap)
            return sh;
    }
    return (long long)max_smem <= cap ? 4 : -1; // {512, 512}: one instance per CTA
}

} // namespace

extern "C" void pdhcg_b200_default_batch_options(pdhcg_b200_batch_options_t *o)
{
    std::memset(o, 0, sizeof(*o));
    o->shape = -1;
}

extern "C" int pdhcg_b200_solve_batch(int count, const qp_problem_t *const *probs, const pdhg_parameters_t *params,
                                      const pdhcg_b200_batch_options_t *opts, pdhcg_result_t **results)
{
    if (count < 0 || (count > 0 && (!probs || !results))) {
        std::fprintf(stderr, "[pdhcg_b200_solve_batch] invalid arguments.\n");
        return -1;
    }
    pdhcg_b200_batch_options_t o;
    if (opts)
        o = *opts;
    else
        pdhcg_b200_default_batch_options(&o);
    pdhg_parameters_t prm;
    if (params)
        prm = *params;
    else
        set_default_parameters(&prm);
    for (int i = 0; i < count; ++i)
        results[i] = nullptr;
    if (count == 0)
        return 0;
    auto t0 = std::chrono::steady_clock::now();
    // ---- pack: a sizing pass, then every instance copied (and A transposed)
    // by a pool of host threads into its slot of the packed arrays ----------
    std::vector<int> batched, fallback;
    std::vector<BInst> inst;
    long long tot_rp = 0, tot_trp = 0, tot_k = 0, tot_x = 0, tot_y = 0, tot_s = 0;
    int max_m = 1;
    std::vector<std::vector<int>> tab(count); // slice tables of the candidates
    {
        // cheap checks here; the matrix checks and the slice tables of the
        // sliced layout (max row length of A and of A^T per 32 rows) on the
        // thread pool
        std::vector<char> cand(count, 0), valid(count, 1);
        std::vector<double> qd;
        for (int i = 0; i < count; ++i) {
            const qp_problem_t *p = probs[i];
            if (!p) {
                std::fprintf(stderr, "[pdhcg_b200_solve_batch] problem %d is NULL.\n", i);
                return -1;
            }
            cand[i] = batchable(p, qd);
        }
        parallel_for(count, [&](int i) {
            if (cand[i] && !slice_tables(probs[i], tab[i]))
                valid[i] = 0;
        });
        for (int i = 0; i < count; ++i)
            if (cand[i] && !valid[i]) {
                std::fprintf(stderr, "[pdhcg_b200_solve_batch] problem %d: the constraint matrix is not valid CSR "
                                     "(row pointers must start at 0 and not decrease, columns must lie in [0, n)).\n",
                             i);
                return -1;
            }
        for (int i = 0; i < count; ++i) {
            const qp_problem_t *p = probs[i];
            const int n = p->num_variables, m = p->num_constraints;
            BInst b{};
            bool ok = cand[i];
            if (ok) {
                b.sell_a = tab[i][slices(m)];
                b.sell_at = tab[i].back();
                const Layout Lo(n, m, b.sell_a, b.sell_at);
                ok = Lo.total <= SMEM_CAP;
                b.smem = Lo.total;
            }
            if (!ok) { // solved on its own by the single-instance path
                fallback.push_back(i);
                continue;
            }
            const int nnz = p->constraint_matrix->row_ptr[m];
            b.n = n;
            b.m = m;
            b.rp_off = tot_rp;
            b.trp_off = tot_trp;
            b.k_off = tot_k;
            b.x_off = tot_x;
            b.y_off = tot_y;
            b.so_off = tot_s;
            b.qmode = (p->objective_sparse_matrix && p->objective_sparse_matrix_num_nonzeros > 0) ? 1 : 0;
            b.obj_const = p->objective_constant;
            tot_rp += m + 1;
            tot_trp += n + 1;
            tot_k += nnz;
            tot_x += n;
            tot_y += m;
            tot_s += (long long)tab[i].size();
            max_m = std::max(max_m, m);
            inst.push_back(b);
            batched.push_back(i);
        }
    }
    const int nb = (int)inst.size();
    // power-method start vector (reference: rand_r with seed 1234 in [-1, 1])
    std::vector<double> v0(max_m);
    unsigned int seed = 1234;
    for (int i = 0; i < max_m; ++i)
        v0[i] = ((double)rand_r(&seed) / (double)RAND_MAX) * 2.0 - 1.0;
    BParams P{};
    P.eps_opt = prm.termination_criteria.eps_optimal_relative;
    P.eps_feas = prm.termination_criteria.eps_feasible_relative;
    P.time_limit_ns = prm.termination_criteria.time_sec_limit * 1e9;
    P.iter_limit = prm.termination_criteria.iteration_limit;
    P.freq = prm.termination_evaluation_frequency > 0 ? prm.termination_evaluation_frequency : 200;
    P.l2 = prm.optimality_norm == NORM_TYPE_L2;
    P.ruiz_iters = prm.l_inf_ruiz_iterations;
    P.has_pc = prm.has_pock_chambolle_alpha;
    P.pc_alpha = prm.pock_chambolle_alpha;
    P.bound_obj = prm.bound_objective_rescaling;
    P.sv_max_iter = prm.sv_max_iter;
    P.sv_tol = prm.sv_tol;
    P.rho = prm.reflection_coefficient;
    P.suff = prm.restart_params.sufficient_reduction_for_restart;
    P.nec = prm.restart_params.necessary_reduction_for_restart;
    P.artificial = prm.restart_params.artificial_restart_threshold;
    P.i_smooth = prm.restart_params.i_smooth;
    P.k_p = prm.restart_params.k_p;
    P.k_i = prm.restart_params.k_i;
    P.k_d = prm.restart_params.k_d;

    double kernel_ms = 0.0, pack_ms = 0.0;
    size_t h2d = 0, d2h = 0;
    int launches = 0;
    std::unique_lock<std::mutex> lock(g_arena_mu, std::defer_lock);
    std::optional<Pack> pk;
    if (nb > 0) {
        // classes by size: instances sorted by shared-memory need, largest
        // first; one launch per class of similar size (a new class starts
        // when the need drops below half)
        std::vector<int> order(nb);
        for (int i = 0; i < nb; ++i)
            order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return inst[a].smem > inst[b].smem; });
        // size classes: the runs of one size band in that order
        std::vector<std::pair<int, int>> classes; // [begin, end) in order
        for (int b = 0; b < nb;) {
            int e = b + 1;
            while (e < nb && size_band(inst[order[e]].smem) == size_band(inst[order[b]].smem))
                ++e;
            classes.push_back({b, e});
            b = e;
        }
        pk.emplace(tot_rp, tot_trp, tot_k, tot_x, tot_y, tot_s, max_m, nb, (int)classes.size());
        const Pack &L = *pk;
        int dev = 0, sms = 0;
        BCK(cudaGetDevice(&dev));
        BCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        lock.lock();
        char *H = host_arena(L.host_bytes());
        char *G = dev_arena(dev, L.end);
        if (!H || !G) {
            std::fprintf(stderr, "[pdhcg_b200_solve_batch] cannot allocate %zu bytes of page-locked or %zu bytes of "
                                 "device memory.\n", L.host_bytes(), L.end);
            return -1;
        }
        int *hA_rp = (int *)(H + L.A_rp), *hA_ci = (int *)(H + L.A_ci);
        double *hA_v = (double *)(H + L.A_v), *hc = (double *)(H + L.c), *hl = (double *)(H + L.l);
        double *hu = (double *)(H + L.u), *hq = (double *)(H + L.q), *hlc = (double *)(H + L.lc);
        double *huc = (double *)(H + L.uc);
        int *hS = (int *)(H + L.S);
        // pack: every instance copied by a pool of host threads into its slot
        // of the staging buffer (A^T is built on the device).  The instances
        // form NG groups of consecutive slots; the thread that packs a
        // group's last instance queues that group's host-to-device copies, so
        // the copies of early groups overlap the packing of later ones.
        const int NG = std::min(nb, 16);
        std::vector<int> gstart(NG + 1);
        for (int g = 0; g <= NG; ++g)
            gstart[g] = (int)((long long)nb * g / NG);
        std::unique_ptr<std::atomic<int>[]> left(new std::atomic<int>[NG]);
        for (int g = 0; g < NG; ++g)
            left[g] = gstart[g + 1] - gstart[g];
        std::atomic<int> copy_err{0};
        auto copy_group = [&](int g) {
            if (cudaSetDevice(dev) != cudaSuccess) { // the pool's threads start on device 0
                copy_err = 1;
                return;
            }
            const BInst &f = inst[gstart[g]];
            const bool last = g + 1 == NG;
            const BInst *e = last ? nullptr : &inst[gstart[g + 1]];
            // {region, element size, first element, end element}
            const struct {
                size_t base, es;
                long long a, b;
            } rg[] = {{L.S, 4, f.so_off, last ? tot_s : e->so_off},
                      {L.A_rp, 4, f.rp_off, last ? tot_rp : e->rp_off},
                      {L.A_ci, 4, f.k_off, last ? tot_k : e->k_off},
                      {L.A_v, 8, f.k_off, last ? tot_k : e->k_off},
                      {L.c, 8, f.x_off, last ? tot_x : e->x_off},
                      {L.l, 8, f.x_off, last ? tot_x : e->x_off},
                      {L.u, 8, f.x_off, last ? tot_x : e->x_off},
                      {L.q, 8, f.x_off, last ? tot_x : e->x_off},
                      {L.lc, 8, f.y_off, last ? tot_y : e->y_off},
                      {L.uc, 8, f.y_off, last ? tot_y : e->y_off}};
            for (const auto &r : rg) {
                const size_t off = r.base + (size_t)r.a * r.es, len = (size_t)(r.b - r.a) * r.es;
                if (len > 0 && cudaMemcpyAsync(G + off, H + off, len, cudaMemcpyHostToDevice, 0) != cudaSuccess)
                    copy_err = 1;
            }
        };
        parallel_for(nb, [&](int bi) {
            const qp_problem_t *p = probs[batched[bi]];
            const BInst &b = inst[bi];
            const int n = b.n, m = b.m;
            const CsrComponent *A = p->constraint_matrix;
            const int nnz = A->row_ptr[m];
            const std::vector<int> &T = tab[batched[bi]];
            std::memcpy(hS + b.so_off, T.data(), T.size() * sizeof(int));
            std::memcpy(hA_rp + b.rp_off, A->row_ptr, (m + 1) * sizeof(int));
            std::memcpy(hA_ci + b.k_off, A->col_ind, nnz * sizeof(int));
            std::memcpy(hA_v + b.k_off, A->val, nnz * sizeof(double));
            std::vector<double> qd;
            diag_q(p, qd);
            for (int j = 0; j < n; ++j)
                hc[b.x_off + j] = p->objective_vector ? p->objective_vector[j] : 0.0;
            std::memcpy(hl + b.x_off, p->variable_lower_bound, n * sizeof(double));
            std::memcpy(hu + b.x_off, p->variable_upper_bound, n * sizeof(double));
            std::memcpy(hq + b.x_off, qd.data(), n * sizeof(double));
            std::memcpy(hlc + b.y_off, p->constraint_lower_bound, m * sizeof(double));
            std::memcpy(huc + b.y_off, p->constraint_upper_bound, m * sizeof(double));
            const int g = (int)(std::upper_bound(gstart.begin(), gstart.end(), bi) - gstart.begin()) - 1;
            if (left[g].fetch_sub(1) == 1)
                copy_group(g);
        });
        BCK(cudaSetDevice(dev));
        if (copy_err) {
            std::fprintf(stderr, "[pdhcg_b200_solve_batch] host-to-device copy failed.\n");
            return -1;
        }
        std::memcpy(H + L.v0, v0.data(), v0.size() * sizeof(double));
        std::memcpy(H + L.inst, inst.data(), inst.size() * sizeof(BInst));
        std::memcpy(H + L.order, order.data(), order.size() * sizeof(int));
        pack_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

        BData D{};
        D.A_rp = (const int *)(G + L.A_rp);
        D.A_ci = (const int *)(G + L.A_ci);
        D.A_v = (const double *)(G + L.A_v);
        D.At_rp = (const int *)(G + L.At_rp);
        D.At_ci = (const int *)(G + L.At_ci);
        D.At_v = (const double *)(G + L.At_v);
        D.c = (const double *)(G + L.c);
        D.l = (const double *)(G + L.l);
        D.u = (const double *)(G + L.u);
        D.q = (const double *)(G + L.q);
        D.lc = (const double *)(G + L.lc);
        D.uc = (const double *)(G + L.uc);
        D.v0 = (const double *)(G + L.v0);
        D.S_tab = (const int *)(G + L.S);
        D.inst = (const BInst *)(G + L.inst);
        D.x_out = (double *)(G + L.x_out);
        D.y_out = (double *)(G + L.y_out);
        D.stats = (double *)(G + L.stats);
        const int *d_order = (const int *)(G + L.order);
        int *d_next = (int *)(G + L.next);
        h2d = L.in_end;
        d2h = L.end - L.out;
        // the parts no group copied: the power-method start vector, then the
        // instance table and the order
        BCK(cudaMemcpyAsync(G + L.v0, H + L.v0, L.S - L.v0, cudaMemcpyHostToDevice, 0));
        BCK(cudaMemcpyAsync(G + L.inst, H + L.inst, L.in_end - L.inst, cudaMemcpyHostToDevice, 0));
        BCK(cudaMemsetAsync(G + L.next, 0, L.out - L.next, 0));
        BCK(cudaMemsetAsync(G + L.out, 0, d2h, 0));
        cudaEvent_t e0, e1;
        BCK(cudaEventCreate(&e0));
        BCK(cudaEventCreate(&e1));
        BCK(cudaEventRecord(e0, 0));
        {
            const int warps_per_cta = 8;
            const int grid = std::max(1, std::min((nb + warps_per_cta - 1) / warps_per_cta, sms * 8));
            transpose_kernel<<<grid, 32 * warps_per_cta, 0, 0>>>(D.A_rp, D.A_ci, D.A_v, (int *)(G + L.At_rp),
                                                                 (int *)(G + L.At_ci), (double *)(G + L.At_v),
                                                                 (int *)(G + L.cur), D.inst, nb);
            ++launches;
            BCK(cudaGetLastError());
        }
        // every class on a stream of its own, all queued at once: a class's
        // CTAs take the SMs that the previous class's CTAs leave when its
        // instances run out, so the classes' tails overlap instead of adding
        // up (each class still runs its instances largest first)
        ClassStreams cs;
        BCK(cudaEventCreateWithFlags(&cs.ready, cudaEventDisableTiming));
        BCK(cudaEventRecord(cs.ready, 0));
        for (size_t ci = 0; ci < classes.size(); ++ci) {
            cudaStream_t st = nullptr;
            cudaEvent_t done = nullptr;
            BCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            cs.streams.push_back(st);
            BCK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
            cs.done.push_back(done);
            BCK(cudaStreamWaitEvent(st, cs.ready, 0));
        }
        for (size_t ci = 0; ci < classes.size(); ++ci) {
            const int b = classes[ci].first, e = classes[ci].second;
            int max_smem = 0, max_dim = 0;
            for (int i = b; i < e; ++i) {
                max_smem = std::max(max_smem, inst[order[i]].smem);
                max_dim = std::max(max_dim, std::max(inst[order[i]].n, inst[order[i]].m));
            }
            const int bs = o.band_shape[size_band(inst[order[b]].smem)] - 1;
            int sh = bs >= 0 && bs < NSHAPES ? bs
                     : o.shape >= 0 && o.shape < NSHAPES ? o.shape
                                                         : default_shape(max_smem, max_dim);
            if (sh < 0 || (long long)max_smem * (SHAPES[sh].bt / SHAPES[sh].group) > SMEM_CAP)
                sh = default_shape(max_smem, max_dim);
            BData Dc = D;
            Dc.order = d_order + b;
            Dc.count = e - b;
            Dc.next = d_next + ci;
            cudaError_t err = launch(sh, Dc, P, max_smem, sms, cs.streams[ci]);
            ++launches;
            if (err != cudaSuccess) {
                std::fprintf(stderr, "[pdhcg_b200_solve_batch] launch: %s\n", cudaGetErrorString(err));
                return -1;
            }
            BCK(cudaEventRecord(cs.done[ci], cs.streams[ci]));
            BCK(cudaStreamWaitEvent(0, cs.done[ci], 0));
        }
        BCK(cudaEventRecord(e1, 0));
        BCK(cudaMemcpyAsync(H + L.in_end, G + L.out, d2h, cudaMemcpyDeviceToHost, 0));
        BCK(cudaStreamSynchronize(0));
        float ms = 0.0f;
        BCK(cudaEventElapsedTime(&ms, e0, e1));
        kernel_ms = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    // ---- results (from the staging buffer, still held) -------------------
    std::atomic<int> alloc_failed{0};
    parallel_for(nb, [&](int bi) {
        const Pack &L = *pk;
        const char *H = g_host_arena.p;
        const int i = batched[bi];
        const qp_problem_t *p = probs[i];
        const BInst &b = inst[bi];
        const double *xo = (const double *)(H + L.in_end + (L.x_out - L.out));
        const double *yo = (const double *)(H + L.in_end + (L.y_out - L.out));
        const double *s = (const double *)(H + L.in_end + (L.stats - L.out)) + (size_t)bi * BS_COUNT;
        const int *arp = (const int *)(H + L.A_rp) + b.rp_off;
        const int *aci = (const int *)(H + L.A_ci) + b.k_off;
        const double *av = (const double *)(H + L.A_v) + b.k_off;
        const double *q = (const double *)(H + L.q) + b.x_off;
        pdhcg_result_t *r = (pdhcg_result_t *)std::calloc(1, sizeof(pdhcg_result_t));
        if (!r) {
            alloc_failed = 1;
            return;
        }
        r->num_variables = b.n;
        r->num_constraints = b.m;
        r->primal_solution = (double *)std::malloc(b.n * sizeof(double));
        r->dual_solution = (double *)std::malloc(b.m * sizeof(double));
        r->reduced_cost = (double *)std::malloc(b.n * sizeof(double));
        results[i] = r;
        if (!r->primal_solution || !r->dual_solution || !r->reduced_cost) {
            alloc_failed = 1;
            return;
        }
        std::memcpy(r->primal_solution, xo + b.x_off, b.n * sizeof(double));
        std::memcpy(r->dual_solution, yo + b.y_off, b.m * sizeof(double));
        // reduced cost c + Qx - A^T y, clamped on infinite bounds (reference
        // compute_and_rescale_reduced_cost_qp_kernel)
        for (int j = 0; j < b.n; ++j)
            r->reduced_cost[j] = (p->objective_vector ? p->objective_vector[j] : 0.0) + q[j] * r->primal_solution[j];
        for (int row = 0; row < b.m; ++row)
            for (int k = arp[row]; k < arp[row + 1]; ++k)
                r->reduced_cost[aci[k]] -= av[k] * r->dual_solution[row];
        for (int j = 0; j < b.n; ++j) {
            if (!std::isfinite(p->variable_lower_bound[j]))
                r->reduced_cost[j] = std::fmin(r->reduced_cost[j], 0.0);
            if (!std::isfinite(p->variable_upper_bound[j]))
                r->reduced_cost[j] = std::fmax(r->reduced_cost[j], 0.0);
        }
        r->termination_reason = (termination_reason_t)(int)s[BS_STATUS];
        r->total_count = (int)s[BS_ITERS];
        r->primal_objective_value = s[BS_POBJ];
        r->dual_objective_value = s[BS_DOBJ];
        r->absolute_primal_residual = s[BS_ABS_P];
        r->absolute_dual_residual = s[BS_ABS_D];
        r->relative_primal_residual = s[BS_REL_P];
        r->relative_dual_residual = s[BS_REL_D];
        r->objective_gap = s[BS_GAP];
        r->relative_objective_gap = s[BS_REL_GAP];
        r->cumulative_time_sec = kernel_ms * 1e-3;
    });
    if (lock.owns_lock())
        lock.unlock();
    if (alloc_failed) {
        for (int i = 0; i < count; ++i)
            if (results[i]) {
                pdhcg_result_free(results[i]);
                results[i] = nullptr;
            }
        return -1;
    }
    for (int i : fallback) {
        results[i] = solve_qp_problem(probs[i], &prm);
        if (!results[i])
            return -1;
    }
    std::memset(&g_batch_stats, 0, sizeof(g_batch_stats));
    g_batch_stats.kernel_ms = kernel_ms;
    g_batch_stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    g_batch_stats.pack_ms = pack_ms;
    g_batch_stats.h2d_bytes = (double)h2d;
    g_batch_stats.d2h_bytes = (double)d2h;
    g_batch_stats.launches = launches;
    g_batch_stats.batched = nb;
    g_batch_stats.fallback = (int)fallback.size();
    return 0;
}

extern "C" int pdhcg_b200_last_batch_stats(pdhcg_b200_batch_stats_t *out)
{
    if (!out)
        return -1;
    *out = g_batch_stats;
    return 0;
}

extern "C" void pdhcg_b200_batch_release(void)
{
    std::lock_guard<std::mutex> lock(g_arena_mu);
    if (g_host_arena.p)
        cudaFreeHost(g_host_arena.p);
    g_host_arena = Arena{};
    int cur = 0;
    const bool have = cudaGetDevice(&cur) == cudaSuccess;
    for (auto &kv : g_dev_arena) {
        if (!kv.second.p)
            continue;
        cudaSetDevice(kv.first);
        cudaFree(kv.second.p);
    }
    g_dev_arena.clear();
    if (have)
        cudaSetDevice(cur);
}

extern "C" int pdhcg_b200_batch_autotune(int count, const qp_problem_t *const *probs, const pdhg_parameters_t *params,
                                         pdhcg_b200_batch_options_t *opts, double *shape_ms)
{
    if (count <= 0 || !probs || !opts) {
        std::fprintf(stderr, "[pdhcg_b200_batch_autotune] invalid arguments.\n");
        return -1;
    }
    // the batched instances by size band (at most 256 of each band)
    std::vector<std::vector<const qp_problem_t *>> band(BATCH_BANDS);
    {
        std::vector<double> qd;
        std::vector<int> T;
        for (int i = 0; i < count; ++i) {
            const qp_problem_t *p = probs[i];
            if (!p || !batchable(p, qd) || !slice_tables(p, T))
                continue;
            const int n = p->num_variables, m = p->num_constraints;
            const Layout Lo(n, m, T[slices(m)], T.back());
            if (Lo.total > SMEM_CAP)
                continue;
            auto &v = band[size_band(Lo.total)];
            if (v.size() < 256)
                v.push_back(p);
        }
    }
    // every shape on every band's sample; a band keeps its fastest shape,
    // opts->shape the fastest over all bands together
    double tot[NSHAPES] = {};
    for (int b = 0; b < BATCH_BANDS; ++b) {
        if (band[b].empty())
            continue;
        std::vector<pdhcg_result_t *> res(band[b].size());
        double best = INFINITY;
        int best_shape = -1;
        for (int sh = 0; sh < NSHAPES; ++sh) {
            pdhcg_b200_batch_options_t o = *opts;
            o.shape = sh;
            for (int k = 0; k < BATCH_BANDS; ++k)
                o.band_shape[k] = 0;
            // an untimed pass first (the kernel's first launch, the buffers'
            // growth), then the timed one
            double ms = 0.0;
            for (int pass = 0; pass < 2; ++pass) {
                cudaDeviceSynchronize();
                auto t0 = std::chrono::steady_clock::now();
                int rc = pdhcg_b200_solve_batch((int)band[b].size(), band[b].data(), params, &o, res.data());
                ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
                for (auto *r : res)
                    if (r)
                        pdhcg_result_free(r);
                if (rc != 0)
                    return rc;
            }
            tot[sh] += ms;
            if (ms < best) {
                best = ms;
                best_shape = sh;
            }
        }
        opts->band_shape[b] = best_shape + 1;
    }
    int best_shape = 0;
    for (int sh = 0; sh < NSHAPES; ++sh) {
        if (shape_ms)
            shape_ms[sh] = tot[sh];
        if (tot[sh] < tot[best_shape])
            best_shape = sh;
    }
    opts->shape = best_shape;
    return 0;
}
