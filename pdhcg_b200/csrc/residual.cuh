// residual.cuh -- KKT residual, objectives and restart distances in one
// launch (reference compute_residual, src/pdhg_core_op.cu:1037-1294, with
// compute_qp_residual_kernel / compute_lp_residual_kernel,
// src/kernels/pdhcg_kernels.cu:628-738, the cone dual residual and the
// projected-gradient augmentation, src/cone_dispatch.cu:88-116 and
// src/pdhg_core_op.cu:67-90, and the distances of perform_restart,
// src/pdhg_core_op.cu:859-880).  Three block ranges: constraint rows, free
// variables, cone blocks (a warp each).  Every block leaves NS partial
// scalars; fold_partials_kernel folds them in a fixed order, so the result
// is deterministic.
#pragma once

#include "kernels.cuh"

namespace pdhcg {

enum ResidualScalar {
    RS_PRIMAL_RES = 0, // max |r_p| or sum r_p^2 (scaled by D_con)
    RS_PRIMAL_SLACK,   // sum of bound * y terms of the dual objective
    RS_DUAL_RES,       // max |r_d| or sum r_d^2
    RS_CX,             // c . x
    RS_XQX,            // x . Qx
    RS_SLACKX,         // dual_slack . x
    RS_QX_NORM,        // |Qx * D_var|
    RS_ATY_NORM,       // |A^T y * D_var|
    RS_DIST_X,         // |x_pdhg - x_init|^2
    RS_DIST_Y,         // |y_pdhg - y_init|^2
    RS_POW_ABS,        // power-cone primal violation (max, or sum of squares)
    RS_POW_REL,        // the same relative to the point's size
    RS_AFF_MEM,        // affine rows: dual membership proj_K(-y) / cr (max, or sum of squares)
    RS_AFF_COMPL,      // affine blocks: |y . (A x + g)| / sb (max, or sum of squares)
    RS_CONE_COMPL,     // variable cone blocks with fixed slots: complementarity (max, or sum of squares)
    RS_COUNT
};

struct ResidualParams {
    int l2;           // 1: Euclidean norms, 0: infinity norms
    int is_lp;        // NON_Q problem type (dual slack comes from the primal step)
    int qmode;        // 0 none, 1 diagonal q, 2 precomputed qx vector
    int has_cones;
    int want_dist;    // restart distances
    double tau;       // step / primal weight (QP dual slack)
    double s_aug;     // step of the projected-gradient augmentation
    double sb;        // constraint-bound rescaling (power-cone relative violation)
};

// VT: storage type of the iterates (FP32 during the mixed bulk phase); the
// matrices and problem data are read in FP64 so residuals are exact FP64
// evaluations of the stored iterates.
template <typename VT>
struct ResidualData {
    int n, m;
    const int *A_rp, *A_ci;
    const double *A_v;
    const int *At_rp, *At_ci;
    const double *At_v;
    const double *c, *l, *u, *q, *qx;
    const double *lc, *uc, *g, *cr, *vr;
    const VT *xp, *yp, *x0, *y0;
    const VT *dual_slack;
    const int *free_idx; int n_free;
    const int2 *free_tiles; int n_free_tiles; // tiles of consecutive free rows (NULL: all n rows)
    const int *cone_start, *cone_len, *cone_type; int n_cones;
    const double *cone_alpha;     // power-cone exponents (NULL: none)
    double *warm_dual, *warm_aug; // per-cone warm starts of the two projections
    const unsigned char *fixed, *cone_fixed; // slots fixed by set_cone_fixed, per block whether any (NULL: none)
    double *partials;
    int rows_blocks, free_blocks, cone_blocks;
    LongRows A_long, At_long; // passes over x_pdhg and y_pdhg
    double *psd_work;         // PSD blocks' projection scratch (NULL: none)
    const long long *psd_off;
    // affine cone blocks of rows and the rows outside them (tiles; NULL: all)
    const int2 *row_tiles;
    int n_row_tiles;
    const int *aff_start, *aff_len, *aff_type;
    const double *aff_alpha;
    const long long *aff_psd_off;
    int n_aff, aff_blocks;
};

__device__ __forceinline__ double norm_term(double v, int l2) { return l2 ? v * v : abs_or_inf(v); }

// One cone block of the residual: A^T y over the block, the dual-cone
// residual and the augmented projected gradient, folded into acc.  SECT:
// the block holds slots fixed by set_cone_fixed (section projectors).
template <int S, typename VT, bool SECT = false>
__device__ __forceinline__ void residual_cone_block(const ResidualData<VT> &D, const ResidualParams &P, int cb,
                                                    int lane, double *stage, double (&acc)[RS_COUNT],
                                                    const int (&ops)[RS_COUNT])
{
    auto fold = [&](int s, double v) { acc[s] = ops[s] == RMAX ? fmax(acc[s], v) : acc[s] + v; };
    const int st = D.cone_start[cb], L = D.cone_len[cb], type = D.cone_type[cb];
    double atys[S];
    warp_stream_rows<S>(D.At_rp, D.At_ci, D.At_v, D.yp, st, L, lane, stage, atys, D.At_long);
    WarpSlots<S> dual, aug;
    double xv[S], rc[S], qxv[S], atyv[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        dual.x[s] = aug.x[s] = 0.0;
        dual.d[s] = aug.d[s] = 1.0;
        dual.w[s] = aug.w[s] = 1.0;
        xv[s] = rc[s] = qxv[s] = atyv[s] = 0.0;
        if (i < L) {
            int j = st + i;
            double aty = atys[s];
            double x = D.xp[j];
            double qx = P.qmode == 1 ? D.q[j] * x : (P.qmode == 2 ? D.qx[j] : 0.0);
            double eff = P.qmode ? D.c[j] + qx : D.c[j];
            xv[s] = x;
            atyv[s] = aty;
            qxv[s] = qx;
            rc[s] = eff - aty;
            // dual cone of {x : x/d in K} is {s : s*d in K}: metric 1/d
            dual.x[s] = rc[s];
            dual.d[s] = 1.0 / D.vr[j];
            aug.x[s] = clampd(D.l[j], x - P.s_aug * rc[s], D.u[j]);
            aug.d[s] = D.vr[j];
        }
    }
    const double alpha = D.cone_alpha ? D.cone_alpha[cb] : 0.0;
    double dres[S]; // the block's dual residual, scaled (before the augmentation)
    if constexpr (SECT) {
        // fixed slots: x - P_section(x - rc) in the d metric, and the
        // projected gradient on the section; both projections share the
        // block's residual warm start, as in the reference
        const unsigned fb = section_bits<S>(D.fixed, st, L, lane);
        double vrs[S];
#pragma unroll
        for (int s = 0; s < S; ++s)
            vrs[s] = aug.d[s];
        double *wa = D.warm_aug ? D.warm_aug + cb : nullptr;
        const double cplx = warp_section_dual<S>(type, L, lane, fb, xv, rc, vrs, alpha, wa, dres);
        warp_section_project<S>(type, aug, L, lane, fb, wa, alpha);
        if (lane == 0)
            fold(RS_CONE_COMPL, norm_term(cplx, P.l2));
    } else {
    bool uni = warp_uniform_unit<S>(aug, L, lane); // d uniform <=> 1/d uniform
    double *psd = D.psd_work ? D.psd_work + D.psd_off[cb] : nullptr;
    if (type == 0 || type == 1 || type == 4) {
        // self-dual: projection onto the dual cone in the 1/d metric
        // (PSD: without a metric, as the reference projects it)
        warp_project<S>(type, dual, L, lane, uni, D.warm_dual ? D.warm_dual + cb : nullptr, 0.0, psd);
    } else {
        // Moreau: rc - proj_{K*}(rc) = -proj_K(-rc), in the inverse scaling
        // (exponential) or on rc d in the unit metric (power) (reference
        // compute_cone_dual_residual_exp_kernel / _power_kernel)
        WarpSlots<S> neg;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const double vr = dual.d[s] > 0.0 ? 1.0 / dual.d[s] : 1.0;
            neg.x[s] = type == 2 ? -dual.x[s] : -dual.x[s] * vr;
            neg.d[s] = type == 2 ? dual.d[s] : 1.0;
            neg.w[s] = 1.0;
        }
        warp_project<S>(type, neg, L, lane, false, nullptr, alpha);
        // keep dual.x = proj_{K*} so that (rc - dual.x) vr is the residual below
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const double vr = dual.d[s] > 0.0 ? 1.0 / dual.d[s] : 1.0;
            dual.x[s] = type == 2 ? rc[s] + neg.x[s] : rc[s] + neg.x[s] / vr;
        }
    }
    warp_project<S>(type, aug, L, lane, uni, D.warm_aug ? D.warm_aug + cb : nullptr, alpha, psd);
#pragma unroll
    for (int s = 0; s < S; ++s)
        dres[s] = (rc[s] - dual.x[s]) * aug.d[s];
    }
    if (type == 3 && lane == 0) {
        // power-cone primal violation (reference compute_power_cone_primal_violation_kernel,
        // src/kernels/pdhcg_power_cone_kernels.cu:623-669): lane 0 holds slot 0 and
        // reads slots 1, 2 from the block's storage
        const double x = xv[0] / D.vr[st], y = (double)D.xp[st + 1] / D.vr[st + 1],
                     z = (double)D.xp[st + 2] / D.vr[st + 2];
        double va, vrel;
        if (!isfinite(x) || !isfinite(y) || !isfinite(z)) {
            va = vrel = INFINITY;
        } else {
            double v = fmax(-x, -y);
            const double az = fabs(z);
            if (az > 0.0) {
                double bound = 0.0;
                bool in = false;
                if (x > 0.0 && y > 0.0) {
                    const double lb = alpha * log(x) + (1.0 - alpha) * log(y), lz = log(az);
                    in = lb + 64.0 * DBL_EPSILON * (1.0 + fabs(lb) + fabs(lz)) >= lz;
                    bound = in ? 0.0 : exp(lb);
                }
                if (!in)
                    v = fmax(v, az - bound);
            }
            va = fmax(v, 0.0);
            vrel = va / (P.sb + fmax(fabs(x), fmax(fabs(y), az)));
        }
        fold(RS_POW_ABS, norm_term(va, P.l2));
        fold(RS_POW_REL, norm_term(vrel, P.l2));
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        if (i < L) {
            int j = st + i;
            double vr = D.vr[j];
            double dr = dres[s];
            double rr = (xv[s] - aug.x[s]) / P.s_aug * vr;
            if (!isfinite(rr))
                rr = copysign(INFINITY, rr);
            if (fabs(rr) > fabs(dr))
                dr = rr;
            fold(RS_DUAL_RES, norm_term(dr, P.l2));
            fold(RS_CX, D.c[j] * xv[s]);
            fold(RS_XQX, xv[s] * qxv[s]);
            fold(RS_SLACKX, rc[s] * xv[s]);
            fold(RS_QX_NORM, norm_term(qxv[s] * vr, P.l2));
            fold(RS_ATY_NORM, norm_term(atyv[s] * vr, P.l2));
            if (P.want_dist) {
                double d = xv[s] - D.x0[j];
                fold(RS_DIST_X, d * d);
            }
        }
    }
}

// A PSD block longer than the warp's registers hold: the terms of
// residual_cone_block slot by slot, with rc, the augmented point and A^T y
// staged in the block's scratch and the two projections (no metric, as for
// every PSD block) taken in memory.
template <int S, typename VT>
__device__ __forceinline__ void residual_psd_long_block(const ResidualData<VT> &D, const ResidualParams &P, int cb,
                                                     int lane, double *stage, double (&acc)[RS_COUNT],
                                                     const int (&ops)[RS_COUNT])
{
    auto fold = [&](int s, double v) { acc[s] = ops[s] == RMAX ? fmax(acc[s], v) : acc[s] + v; };
    const int st = D.cone_start[cb], L = D.cone_len[cb];
    const int n = psd_order(L);
    double *work = D.psd_work + D.psd_off[cb];
    double *rcv = work + 2LL * n * n, *augv = rcv + L, *atyv = augv + L;
    auto qx_of = [&](int j, double x) {
        return P.qmode == 1 ? D.q[j] * x : (P.qmode == 2 ? D.qx[j] : 0.0);
    };
    for (int c0 = 0; c0 < L; c0 += 32 * S) {
        const int nr = min(32 * S, L - c0);
        double atys[S];
        warp_stream_rows<S>(D.At_rp, D.At_ci, D.At_v, D.yp, st + c0, nr, lane, stage, atys, D.At_long);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int i = lane + 32 * s;
            if (i < nr) {
                const int j = st + c0 + i;
                const double x = D.xp[j];
                const double eff = P.qmode ? D.c[j] + qx_of(j, x) : D.c[j];
                const double rc = eff - atys[s];
                rcv[c0 + i] = rc;
                augv[c0 + i] = clampd(D.l[j], x - P.s_aug * rc, D.u[j]);
                atyv[c0 + i] = atys[s];
            }
        }
    }
    __syncwarp();
    double *psd = D.psd_work + D.psd_off[cb];
    warp_project_psd_mem(rcv, rcv, L, lane, psd);   // the dual cone (self-dual) of rc
    warp_project_psd_mem(augv, augv, L, lane, psd); // the augmented point
    for (int i = lane; i < L; i += 32) {
        const int j = st + i;
        const double x = D.xp[j], qx = qx_of(j, x), aty = atyv[i];
        const double eff = P.qmode ? D.c[j] + qx : D.c[j];
        const double rc = eff - aty, vr = D.vr[j];
        double dr = (rc - rcv[i]) * vr;
        double rr = (x - augv[i]) / P.s_aug * vr;
        if (!isfinite(rr))
            rr = copysign(INFINITY, rr);
        if (fabs(rr) > fabs(dr))
            dr = rr;
        fold(RS_DUAL_RES, norm_term(dr, P.l2));
        fold(RS_CX, D.c[j] * x);
        fold(RS_XQX, x * qx);
        fold(RS_SLACKX, rc * x);
        fold(RS_QX_NORM, norm_term(qx * vr, P.l2));
        fold(RS_ATY_NORM, norm_term(aty * vr, P.l2));
        if (P.want_dist) {
            const double d = x - (double)D.x0[j];
            fold(RS_DIST_X, d * d);
        }
    }
    __syncwarp();
}

// One affine cone block of rows (reference compute_residual with affine
// cones, src/pdhg_core_op.cu:1037-1294, and compute_affine_cone_residuals,
// :109-212): v = A x + g; the primal residual is v - proj_K(v) scaled by
// cr; the dual membership proj_K(-y) / cr (zero when y is in the dual
// cone); the complementarity |y . v| / sb; the bound terms of the dual
// objective as for other rows.  Projections as in the dual step (d = 1 / cr).
template <int S, typename VT>
__device__ __forceinline__ void residual_affine_block(const ResidualData<VT> &D, const ResidualParams &P, int ab,
                                                      int lane, double *stage, double (&acc)[RS_COUNT],
                                                      const int (&ops)[RS_COUNT])
{
    auto fold = [&](int s, double v) { acc[s] = ops[s] == RMAX ? fmax(acc[s], v) : acc[s] + v; };
    const int st = D.aff_start[ab], L = D.aff_len[ab], type = D.aff_type[ab];
    const double alpha = D.aff_alpha ? D.aff_alpha[ab] : 0.0;
    double *psd = D.psd_work ? D.psd_work + D.aff_psd_off[ab] : nullptr;
    double axr[S];
    warp_stream_rows<S>(D.A_rp, D.A_ci, D.A_v, D.xp, st, L, lane, stage, axr, D.A_long);
    WarpSlots<S> pv, mv;
    double vv[S], yv[S];
    double ydv = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        pv.x[s] = mv.x[s] = 0.0;
        pv.d[s] = mv.d[s] = 1.0;
        pv.w[s] = mv.w[s] = 1.0;
        vv[s] = yv[s] = 0.0;
        if (i < L) {
            const int j = st + i;
            vv[s] = axr[s] + D.g[j];
            yv[s] = D.yp[j];
            pv.x[s] = clampd(D.lc[j], vv[s], D.uc[j]);
            mv.x[s] = -yv[s];
            pv.d[s] = mv.d[s] = 1.0 / D.cr[j];
            ydv += yv[s] * vv[s];
            const double lcf = isfinite(D.lc[j]) ? D.lc[j] : 0.0, ucf = isfinite(D.uc[j]) ? D.uc[j] : 0.0;
            fold(RS_PRIMAL_SLACK, fmax(yv[s], 0.0) * lcf + fmin(yv[s], 0.0) * ucf - D.g[j] * yv[s]);
            if (P.want_dist) {
                const double d = yv[s] - D.y0[j];
                fold(RS_DIST_Y, d * d);
            }
        }
    }
    const bool uni = warp_uniform_unit<S>(pv, L, lane);
    warp_project<S>(type, pv, L, lane, uni, nullptr, alpha, psd);
    warp_project<S>(type, mv, L, lane, uni, nullptr, alpha, psd);
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        if (i < L) {
            const int j = st + i;
            fold(RS_PRIMAL_RES, norm_term((vv[s] - pv.x[s]) * D.cr[j], P.l2));
            fold(RS_AFF_MEM, norm_term(mv.x[s] / D.cr[j], P.l2));
        }
    }
    ydv = warp_sum(ydv);
    if (lane == 0)
        fold(RS_AFF_COMPL, norm_term(fabs(ydv) / P.sb, P.l2));
}

// SECT: the problem has blocks with fixed slots (an instantiation of its
// own, so that the section projectors do not weigh on the registers of the
// others)
template <int S, typename VT, bool SECT>
__global__ void __launch_bounds__(TPB) residual_kernel(ResidualData<VT> D, ResidualParams P)
{
    __shared__ double stage_all[WARPS][STREAM_CHUNK];
    const int NOP = P.l2 ? RSUM : RMAX;
    const int ops[RS_COUNT] = {NOP, RSUM, NOP, RSUM, RSUM, RSUM, NOP, NOP, RSUM, RSUM, NOP, NOP, NOP, NOP, NOP};
    double acc[RS_COUNT];
#pragma unroll
    for (int s = 0; s < RS_COUNT; ++s)
        acc[s] = 0.0;
    auto fold = [&](int s, double v) { acc[s] = ops[s] == RMAX ? fmax(acc[s], v) : acc[s] + v; };
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *stage = stage_all[wib];

    int b = blockIdx.x;
    if (b < D.rows_blocks) {
        // constraint rows, one warp per tile of 32
        const int ntiles = D.row_tiles ? D.n_row_tiles : (D.m + 31) / 32;
        for (int tile = b * WARPS + wib; tile < ntiles; tile += D.rows_blocks * WARPS) {
            int r0, nr;
            if (D.row_tiles) {
                const int2 rt = D.row_tiles[tile];
                r0 = rt.x;
                nr = rt.y;
            } else {
                r0 = 32 * tile;
                nr = min(32, D.m - r0);
            }
            double axr[1];
            warp_stream_rows<1>(D.A_rp, D.A_ci, D.A_v, D.xp, r0, nr, lane, stage, axr, D.A_long);
            if (lane < nr) {
                const int i = r0 + lane;
                double v = axr[0] + D.g[i];
                double proj = clampd(D.lc[i], v, D.uc[i]);
                fold(RS_PRIMAL_RES, norm_term((v - proj) * D.cr[i], P.l2));
                double y = D.yp[i];
                double lcf = isfinite(D.lc[i]) ? D.lc[i] : 0.0, ucf = isfinite(D.uc[i]) ? D.uc[i] : 0.0;
                fold(RS_PRIMAL_SLACK, fmax(y, 0.0) * lcf + fmin(y, 0.0) * ucf - D.g[i] * y);
                if (P.want_dist) {
                    double d = y - D.y0[i];
                    fold(RS_DIST_Y, d * d);
                }
            }
        }
    } else if (b < D.rows_blocks + D.free_blocks) {
        // variables outside cones, one warp per tile of consecutive rows
        b -= D.rows_blocks;
        const int ntiles = D.free_tiles ? D.n_free_tiles : (D.n + 31) / 32;
        for (int tile = b * WARPS + wib; tile < ntiles; tile += D.free_blocks * WARPS) {
            int r0, nr;
            if (D.free_tiles) {
                const int2 ft = D.free_tiles[tile];
                r0 = ft.x;
                nr = ft.y;
            } else {
                r0 = 32 * tile;
                nr = min(32, D.n - r0);
            }
            double atyr[1];
            warp_stream_rows<1>(D.At_rp, D.At_ci, D.At_v, D.yp, r0, nr, lane, stage, atyr, D.At_long);
            if (lane < nr) {
                const int j = r0 + lane;
                const double aty = atyr[0];
                double x = D.xp[j];
                double qx = P.qmode == 1 ? D.q[j] * x : (P.qmode == 2 ? D.qx[j] : 0.0);
                double dr, ds;
                if (P.is_lp) {
                    ds = D.dual_slack[j];
                    dr = (D.c[j] - aty - ds) * D.vr[j];
                } else {
                    double gr = qx + D.c[j] - aty;
                    double t = x - P.tau * gr;
                    double p = fmax(D.l[j], fmin(D.u[j], t));
                    ds = (p - t) / P.tau;
                    dr = (gr - ds) * D.vr[j];
                }
                if (P.has_cones) {
                    double eff = P.qmode ? D.c[j] + qx : D.c[j];
                    double pt = clampd(D.l[j], x - P.s_aug * (eff - aty), D.u[j]);
                    double rr = (x - pt) / P.s_aug * D.vr[j];
                    if (!isfinite(rr))
                        rr = copysign(INFINITY, rr);
                    if (fabs(rr) > fabs(dr))
                        dr = rr;
                }
                fold(RS_DUAL_RES, norm_term(dr, P.l2));
                fold(RS_CX, D.c[j] * x);
                fold(RS_XQX, x * qx);
                fold(RS_SLACKX, ds * x);
                fold(RS_QX_NORM, norm_term(qx * D.vr[j], P.l2));
                fold(RS_ATY_NORM, norm_term(aty * D.vr[j], P.l2));
                if (P.want_dist) {
                    double d = x - D.x0[j];
                    fold(RS_DIST_X, d * d);
                }
            }
        }
    } else if (b < D.rows_blocks + D.free_blocks + D.cone_blocks) {
        b -= D.rows_blocks + D.free_blocks;
        const int nwarps = D.cone_blocks * WARPS;
        for (int cb = b * WARPS + wib; cb < D.n_cones; cb += nwarps) {
            // 3-slot blocks (exponential, power) take the one-slot
            // instantiation, which alone carries their projection
            const int ct = D.cone_type[cb];
            if (SECT && D.cone_fixed[cb]) {
                if (S > 1 && (ct == 2 || ct == 3))
                    residual_cone_block<1, VT, true>(D, P, cb, lane, stage, acc, ops);
                else
                    residual_cone_block<S, VT, true>(D, P, cb, lane, stage, acc, ops);
            } else if (S > 1 && (ct == 2 || ct == 3)) {
                residual_cone_block<1, VT>(D, P, cb, lane, stage, acc, ops);
            } else if (ct == 4 && D.cone_len[cb] > 32 * S) {
                residual_psd_long_block<S, VT>(D, P, cb, lane, stage, acc, ops);
            } else {
                residual_cone_block<S, VT>(D, P, cb, lane, stage, acc, ops);
            }
        }
    } else {
        b -= D.rows_blocks + D.free_blocks + D.cone_blocks;
        const int nwarps = D.aff_blocks * WARPS;
        for (int ab = b * WARPS + wib; ab < D.n_aff; ab += nwarps) {
            const int at = D.aff_type[ab];
            if (S > 1 && (at == 2 || at == 3))
                residual_affine_block<1, VT>(D, P, ab, lane, stage, acc, ops);
            else
                residual_affine_block<S, VT>(D, P, ab, lane, stage, acc, ops);
        }
    }
    block_reduce_store<RS_COUNT>(acc, ops, D.partials);
}

// Fixed-point error pieces (reference compute_fixed_point_error,
// src/pdhg_core_op.cu:973-1035): |dx|^2, |dy|^2 and (A^T dy) . dx, with
// dx = x_refl - x_cur and dy = y_refl - y_cur written by the step kernels.
enum FpeScalar { FP_DX2 = 0, FP_DY2, FP_CROSS, FP_COUNT };

template <typename VT>
__global__ void __launch_bounds__(TPB) fpe_kernel(int n, int m, const int *At_rp, const int *At_ci, const double *At_v,
                                                  const VT *dx, const VT *dy, double *partials,
                                                  int col_blocks, LongRows At_long)
{
    __shared__ double stage_all[WARPS][STREAM_CHUNK];
    const int ops[FP_COUNT] = {RSUM, RSUM, RSUM};
    double acc[FP_COUNT] = {0.0, 0.0, 0.0};
    int b = blockIdx.x;
    if (b < col_blocks) {
        // (A^T dy)_j dx_j, one warp per tile of 32 rows of A^T
        const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
        const int ntiles = (n + 31) / 32;
        for (int tile = b * WARPS + wib; tile < ntiles; tile += col_blocks * WARPS) {
            const int r0 = 32 * tile, nr = min(32, n - r0);
            double a[1];
            warp_stream_rows<1>(At_rp, At_ci, At_v, dy, r0, nr, lane, stage_all[wib], a, At_long);
            if (lane < nr) {
                double d = dx[r0 + lane];
                acc[FP_DX2] += d * d;
                acc[FP_CROSS] += a[0] * d;
            }
        }
    } else {
        b -= col_blocks;
        int nb = gridDim.x - col_blocks;
        for (int i = b * TPB + threadIdx.x; i < m; i += nb * TPB) {
            double d = dy[i];
            acc[FP_DY2] += d * d;
        }
    }
    block_reduce_store<FP_COUNT>(acc, ops, partials);
}

// ---------------------------------------------------------------------------
// Infeasibility certificates (reference compute_infeasibility_information,
// src/pdhg_core_op.cu:1296-1429, kernels src/kernels/pdhcg_kernels.cu:
// 760-859), from the last step's differences dx = x_refl - x_cur and
// dy = y_refl - y_cur, in three launches plus fixed-order folds:
//   ray_project_kernel : dx, dy onto the recession cones of the bounds (in
//                        place), max |dx|, max |dy|
//   ray_scale_kernel   : dx /= max |dx|
//   ray_kernel         : A dx and A^T dy by stream-mode products and the
//                        certificate pieces below
// ---------------------------------------------------------------------------
enum RayNorm { RN_DX = 0, RN_DY, RN_COUNT };
enum RayScalar {
    RY_PSLACK = 0, // sum over rows of the dual-ray objective terms
    RY_DSLACK,     // sum over columns of the reduced-cost objective terms
    RY_CDX,        // c . dx
    RY_PINF,       // max primal-ray infeasibility (scaled by D_con)
    RY_DINF,       // max dual-ray infeasibility (scaled by D_var)
    RY_QDX,        // max |Q dx|
    RY_COUNT
};

template <typename VT>
__global__ void __launch_bounds__(TPB) ray_project_kernel(int n, int m, VT *dx, VT *dy, const double *l,
                                                          const double *u, const double *lc, const double *uc,
                                                          double *partials)
{
    const int ops[RN_COUNT] = {RMAX, RMAX};
    double acc[RN_COUNT] = {0.0, 0.0};
    for (int i = blockIdx.x * TPB + threadIdx.x; i < n + m; i += gridDim.x * TPB) {
        if (i < n) {
            double d = dx[i];
            if (isfinite(l[i]))
                d = fmax(d, 0.0);
            if (isfinite(u[i]))
                d = fmin(d, 0.0);
            dx[i] = (VT)d;
            acc[RN_DX] = fmax(acc[RN_DX], abs_or_inf((double)(VT)d));
        } else {
            const int r = i - n;
            double d = dy[r];
            if (!isfinite(lc[r]))
                d = fmin(d, 0.0);
            if (!isfinite(uc[r]))
                d = fmax(d, 0.0);
            dy[r] = (VT)d;
            acc[RN_DY] = fmax(acc[RN_DY], abs_or_inf((double)(VT)d));
        }
    }
    block_reduce_store<RN_COUNT>(acc, ops, partials);
}

template <typename VT>
__global__ void ray_scale_kernel(int n, VT *dx, const double *norms)
{
    const double nx = norms[RN_DX];
    if (!(nx > 0.0))
        return;
    const double inv = 1.0 / nx;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dx[i] = (VT)((double)dx[i] * inv);
}

struct RayData {
    int n, m;
    const int *A_rp, *A_ci;
    const double *A_v;
    const int *At_rp, *At_ci;
    const double *At_v;
    const double *c, *l, *u, *q, *qx; // q: diagonal Q (qmode 1); qx: Q dx precomputed (qmode 2)
    const double *lc, *uc, *g, *cr, *vr;
    int qmode;
    int rows_blocks; // blocks [0, rows_blocks) take rows of A, the rest columns
    double *partials;
    LongRows A_long, At_long; // passes over the primal and dual rays
};

template <typename VT>
__global__ void __launch_bounds__(TPB) ray_kernel(RayData D, const VT *dx, const VT *dy)
{
    __shared__ double stage_all[WARPS][STREAM_CHUNK];
    const int ops[RY_COUNT] = {RSUM, RSUM, RSUM, RMAX, RMAX, RMAX};
    double acc[RY_COUNT] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *stage = stage_all[wib];
    auto fin = [](double v) { return isfinite(v) ? v : 0.0; };
    if ((int)blockIdx.x < D.rows_blocks) {
        const int ntiles = (D.m + 31) / 32;
        for (int tile = blockIdx.x * WARPS + wib; tile < ntiles; tile += D.rows_blocks * WARPS) {
            const int r0 = 32 * tile, nr = min(32, D.m - r0);
            double pp[1];
            warp_stream_rows<1>(D.A_rp, D.A_ci, D.A_v, dx, r0, nr, lane, stage, pp, D.A_long);
            if (lane < nr) {
                const int i = r0 + lane;
                const double y = dy[i];
                acc[RY_PSLACK] += fmax(y, 0.0) * fin(D.lc[i]) + fmin(y, 0.0) * fin(D.uc[i]) - D.g[i] * y;
                const double pinf = (fmax(0.0, -pp[0]) * (double)isfinite(D.lc[i]) +
                                     fmax(0.0, pp[0]) * (double)isfinite(D.uc[i])) * D.cr[i];
                acc[RY_PINF] = fmax(acc[RY_PINF], abs_or_inf(pinf));
            }
        }
    } else {
        const int b = blockIdx.x - D.rows_blocks, nb = gridDim.x - D.rows_blocks;
        const int ntiles = (D.n + 31) / 32;
        for (int tile = b * WARPS + wib; tile < ntiles; tile += nb * WARPS) {
            const int r0 = 32 * tile, nr = min(32, D.n - r0);
            double dpr[1];
            warp_stream_rows<1>(D.At_rp, D.At_ci, D.At_v, dy, r0, nr, lane, stage, dpr, D.At_long);
            if (lane < nr) {
                const int j = r0 + lane;
                const double dp = -dpr[0];
                const double x = dx[j];
                acc[RY_DSLACK] += fmax(dp, 0.0) * fin(D.l[j]) + fmin(dp, 0.0) * fin(D.u[j]);
                const double dinf =
                    (fmax(0.0, dp) * (double)!isfinite(D.l[j]) - fmin(0.0, dp) * (double)!isfinite(D.u[j])) * D.vr[j];
                acc[RY_DINF] = fmax(acc[RY_DINF], abs_or_inf(dinf));
                acc[RY_CDX] += D.c[j] * x;
                if (D.qmode) {
                    const double qx = D.qmode == 1 ? D.q[j] * x : D.qx[j];
                    acc[RY_QDX] = fmax(acc[RY_QDX], abs_or_inf(qx));
                }
            }
        }
    }
    block_reduce_store<RY_COUNT>(acc, ops, D.partials);
}

} // namespace pdhcg
