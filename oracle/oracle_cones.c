/*
 * oracle_cones.c -- CPU cone projections for the oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see pdhcg_oracle.h).
 *
 * All projections work on one block of the scaled iterate x.  The cone is
 * defined on the unscaled ("actual") coordinates u_i = x_i / d_i, and the
 * projection minimises sum_i w_i (x_i - r_i)^2 with w_i = 1 + tau q_i, i.e.
 * sum_i omega_i (u_i - a_i)^2 with omega_i = w_i d_i^2 and a_i = r_i / d_i
 * (reference internal/cone_projection_utils.h:22-27).  When d is uniform on
 * the block and w == 1 the reference uses closed forms in x-space
 * (src/kernels/pdhcg_soc_cone_kernels.cu:296-324,
 * src/kernels/pdhcg_rsoc_cone_kernels.cu:505-530); they are restated exactly
 * here.  Otherwise the multiplier lambda of the KKT system
 *   u_i = omega_i a_i / (omega_i + lambda)            (vector slots)
 *   u_z = omega_z a_z / (omega_z - lambda)             (SOC apex slot)
 *   [omega_s, -lambda; -lambda, omega_t][s;t] = [omega_s a_s; omega_t a_t]  (RSOC)
 * is found by bracketed Newton as in the reference's block kernels
 * (src/kernels/pdhcg_soc_cone_kernels.cu:1725-2062,
 *  src/kernels/pdhcg_rsoc_cone_kernels.cu:2096-2631).
 */
#include "pdhcg_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_MAX_ROOT_ITERS 200

static int block_length(int type, int v_dim)
{
    if (type == CONE_EXPONENTIAL || type == CONE_POWER)
        return 3;
    if (type == CONE_PSD)
        return v_dim * (v_dim + 1) / 2;
    return v_dim + 2;
}

/* ---------------- standard SOC, weighted, u-space -------------------- */

/* a[0..len-1]: vector part (v then w); az: apex input; om, omz: weights.
 * Writes the projection into u[0..len-1], *uz. */
static void wsoc_u(int len, const double *a, double az, const double *om, double omz, double *u, double *uz)
{
    double norm2 = 0.0, polar2 = 0.0;
    for (int i = 0; i < len; ++i) {
        norm2 += a[i] * a[i];
        polar2 += (om[i] * a[i]) * (om[i] * a[i]);
    }
    if (az >= 0.0 && norm2 <= az * az) { /* inside */
        memcpy(u, a, (size_t)len * sizeof(double));
        *uz = az;
        return;
    }
    if (-omz * az >= sqrt(polar2)) { /* -omega.a in K: projection is the apex */
        for (int i = 0; i < len; ++i)
            u[i] = 0.0;
        *uz = 0.0;
        return;
    }
    if (az == 0.0) {
        double lam = omz, s = 0.0;
        for (int i = 0; i < len; ++i) {
            u[i] = om[i] * a[i] / (om[i] + lam);
            s += u[i] * u[i];
        }
        *uz = sqrt(s);
        return;
    }
    int lower = az > 0.0;
    double lo, hi;
    if (lower) {
        lo = 0.0;
        hi = omz * (1.0 - 1e-14);
    } else {
        lo = omz * (1.0 + 1e-14);
        hi = 2.0 * omz;
        for (int e = 0; e < 200; ++e) {
            double s = 0.0;
            for (int i = 0; i < len; ++i) {
                double t = om[i] * a[i] / (om[i] + hi);
                s += t * t;
            }
            double z = omz * az / (omz - hi);
            if (s - z * z >= 0.0)
                break;
            lo = hi;
            hi *= 2.0;
        }
    }
    double lam = 0.5 * (lo + hi);
    for (int it = 0; it < ORACLE_MAX_ROOT_ITERS; ++it) {
        double s = 0.0, ds = 0.0;
        for (int i = 0; i < len; ++i) {
            double t = om[i] * a[i] / (om[i] + lam);
            s += t * t;
            ds -= 2.0 * t * t / (om[i] + lam);
        }
        double z = omz * az / (omz - lam);
        double f = s - z * z;
        double df = ds - 2.0 * z * z / (omz - lam);
        if ((lower && f > 0.0) || (!lower && f < 0.0))
            lo = lam;
        else
            hi = lam;
        if (fabs(f) <= 1e-13 * (1.0 + s + z * z) || hi - lo <= 1e-13 * (1.0 + hi + lo))
            break;
        double next = lam - f / df;
        if (!isfinite(next) || !(next > lo && next < hi))
            next = 0.5 * (lo + hi);
        lam = next;
    }
    for (int i = 0; i < len; ++i)
        u[i] = om[i] * a[i] / (om[i] + lam);
    *uz = omz * az / (omz - lam);
}

/* ---------------- rotated SOC, weighted, u-space -------------------- */

static void wrsoc_u(int k, const double *a, double as, double at, const double *om, double oms, double omt,
                    double *u, double *us, double *ut)
{
    double norm2 = 0.0, polar2 = 0.0, freeobj = 0.0;
    for (int i = 0; i < k; ++i) {
        norm2 += a[i] * a[i];
        polar2 += (om[i] * a[i]) * (om[i] * a[i]);
        freeobj += om[i] * a[i] * a[i];
    }
    if (as >= 0.0 && at >= 0.0 && norm2 <= 2.0 * as * at) {
        memcpy(u, a, (size_t)k * sizeof(double));
        *us = as;
        *ut = at;
        return;
    }
    double bs = oms * as, bt = omt * at;
    if (bs <= 0.0 && bt <= 0.0 && polar2 <= 2.0 * bs * bt) {
        for (int i = 0; i < k; ++i)
            u[i] = 0.0;
        *us = 0.0;
        *ut = 0.0;
        return;
    }
    double sqs = sqrt(oms), sqt = sqrt(omt);
    double rm = sqs * sqt;
    double balance = sqs * as + sqt * at;
    double bscale = 1.0 + fabs(sqs * as) + fabs(sqt * at);
    double lam, ps, pt;
    if (fabs(balance) <= 64.0 * DBL_EPSILON * bscale) {
        lam = rm;
        double n2 = 0.0;
        for (int i = 0; i < k; ++i) {
            double t = om[i] * a[i] / (om[i] + lam);
            n2 += t * t;
        }
        double product = 0.5 * rm * n2;
        double delta = sqs * as;
        double st = 0.5 * (-delta + sqrt(fmax(0.0, delta * delta + 4.0 * product)));
        double ss = st + delta;
        ps = ss / sqs;
        pt = st / sqt;
    } else {
        int lower = balance > 0.0;
        double lo, hi;
        if (lower) {
            lo = 0.0;
            hi = rm * (1.0 - 1e-14);
        } else {
            lo = rm * (1.0 + 1e-14);
            hi = 2.0 * rm;
            for (int e = 0; e < 200; ++e) {
                double n2 = 0.0;
                for (int i = 0; i < k; ++i) {
                    double t = om[i] * a[i] / (om[i] + hi);
                    n2 += t * t;
                }
                double det = oms * omt - hi * hi;
                double s = omt * (oms * as + hi * at) / det;
                double t = oms * (omt * at + hi * as) / det;
                double f = (s >= 0.0 && t >= 0.0) ? n2 - 2.0 * s * t : INFINITY;
                if (f >= 0.0)
                    break;
                lo = hi;
                hi *= 2.0;
            }
        }
        lam = 0.5 * (lo + hi);
        for (int it = 0; it < ORACLE_MAX_ROOT_ITERS; ++it) {
            double n2 = 0.0, dn2 = 0.0;
            for (int i = 0; i < k; ++i) {
                double t = om[i] * a[i] / (om[i] + lam);
                n2 += t * t;
                dn2 -= 2.0 * t * t / (om[i] + lam);
            }
            double det = oms * omt - lam * lam;
            double s = omt * (oms * as + lam * at) / det;
            double t = oms * (omt * at + lam * as) / det;
            double f = INFINITY, df = dn2;
            if (s >= 0.0 && t >= 0.0) {
                f = n2 - 2.0 * s * t;
                double dsl = (omt * t + lam * s) / det;
                double dtl = (lam * t + oms * s) / det;
                df -= 2.0 * (dsl * t + s * dtl);
            }
            if ((lower && f > 0.0) || (!lower && f < 0.0))
                lo = lam;
            else
                hi = lam;
            if (isfinite(f) && (fabs(f) <= 1e-13 * (1.0 + n2 + 2.0 * s * t) || hi - lo <= 1e-13 * (1.0 + hi + lo)))
                break;
            double next = lam - f / df;
            if (!isfinite(next) || !(next > lo && next < hi))
                next = 0.5 * (lo + hi);
            lam = next;
        }
        double det = oms * omt - lam * lam;
        ps = omt * (oms * as + lam * at) / det;
        pt = oms * (omt * at + lam * as) / det;
    }
    /* The boundary {v = 0, s >= 0, t = 0} and its mirror are not smooth: compare
     * with the axis candidates (reference rsoc block kernel, :2541-2568). */
    double smooth = 0.0;
    for (int i = 0; i < k; ++i) {
        double v = om[i] * a[i] / (om[i] + lam);
        smooth += om[i] * (v - a[i]) * (v - a[i]);
    }
    smooth += oms * (ps - as) * (ps - as) + omt * (pt - at) * (pt - at);
    double s_axis = fmax(as, 0.0), t_axis = fmax(at, 0.0);
    double s_obj = freeobj + oms * (s_axis - as) * (s_axis - as) + omt * at * at;
    double t_obj = freeobj + oms * as * as + omt * (t_axis - at) * (t_axis - at);
    if (s_obj < smooth && s_obj <= t_obj) {
        for (int i = 0; i < k; ++i)
            u[i] = 0.0;
        *us = s_axis;
        *ut = 0.0;
        return;
    }
    if (t_obj < smooth) {
        for (int i = 0; i < k; ++i)
            u[i] = 0.0;
        *us = 0.0;
        *ut = t_axis;
        return;
    }
    for (int i = 0; i < k; ++i)
        u[i] = om[i] * a[i] / (om[i] + lam);
    *us = ps;
    *ut = pt;
}

/* ---------------- closed forms (uniform d, unit metric) ---------------- */

static void soc_closed(int len, double *xv, double *xz)
{
    double s = 0.0;
    for (int i = 0; i < len; ++i)
        s += xv[i] * xv[i];
    double r = sqrt(s);
    double z = *xz;
    if (r <= z)
        return;
    if (r <= -z) {
        for (int i = 0; i < len; ++i)
            xv[i] = 0.0;
        *xz = 0.0;
        return;
    }
    double scale = (z + r) / (2.0 * r);
    for (int i = 0; i < len; ++i)
        xv[i] *= scale;
    *xz = scale * r;
}

static void rsoc_closed(int k, double *x)
{
    const double INV_SQRT2 = 0.7071067811865475;
    double *v = x, *sp = x + k, *tp = x + k + 1;
    double s = *sp, t = *tp;
    double w = (s - t) * INV_SQRT2;
    double z = (s + t) * INV_SQRT2;
    double sumsq = w * w;
    for (int m = 0; m < k; ++m)
        sumsq += v[m] * v[m];
    double r = sqrt(sumsq);
    if (r <= z)
        return;
    if (r <= -z) {
        for (int m = 0; m < k; ++m)
            v[m] = 0.0;
        *sp = 0.0;
        *tp = 0.0;
        return;
    }
    double scale = (z + r) / (2.0 * r);
    for (int m = 0; m < k; ++m)
        v[m] *= scale;
    double w_new = scale * w;
    double z_new = scale * r;
    *sp = (z_new + w_new) * INV_SQRT2;
    *tp = (z_new - w_new) * INV_SQRT2;
}

/* ---------------- public block projection ---------------- */

static int is_uniform(const double *d, int len)
{
    for (int i = 1; i < len; ++i)
        if (d[i] != d[0])
            return 0;
    return 1;
}

static int has_weight(const double *q, int len)
{
    if (!q)
        return 0;
    for (int i = 0; i < len; ++i)
        if (q[i] != 0.0)
            return 1;
    return 0;
}

void oracle_exp_project(double *x, const double *d, const double *q, double tau);
void oracle_pow_project(double *x, const double *d, const double *q, double tau, double alpha);
void oracle_psd_project(int order, double *x);

void oracle_project_cone_block(int type, int v_dim, double power_alpha, double *x, const double *d,
                               const double *q, double tau)
{
    int len = block_length(type, v_dim);
    if (type == CONE_EXPONENTIAL) {
        oracle_exp_project(x, d, q, tau);
        return;
    }
    if (type == CONE_POWER) {
        oracle_pow_project(x, d, q, tau, power_alpha);
        return;
    }
    if (type == CONE_PSD) {
        oracle_psd_project(v_dim, x);
        return;
    }
    if (is_uniform(d, len) && !has_weight(q, len)) {
        if (type == CONE_STANDARD_SOC)
            soc_closed(v_dim + 1, x, x + v_dim + 1);
        else
            rsoc_closed(v_dim, x);
        return;
    }
    double *a = (double *)malloc((size_t)len * sizeof(double));
    double *om = (double *)malloc((size_t)len * sizeof(double));
    double *u = (double *)malloc((size_t)len * sizeof(double));
    for (int i = 0; i < len; ++i) {
        double w = q ? 1.0 + tau * q[i] : 1.0;
        a[i] = x[i] / d[i];
        om[i] = fmax(w * d[i] * d[i], DBL_MIN);
    }
    if (type == CONE_STANDARD_SOC) {
        double uz;
        wsoc_u(v_dim + 1, a, a[v_dim + 1], om, om[v_dim + 1], u, &uz);
        u[v_dim + 1] = uz;
    } else {
        double us, ut;
        wrsoc_u(v_dim, a, a[v_dim], a[v_dim + 1], om, om[v_dim], om[v_dim + 1], u, &us, &ut);
        u[v_dim] = us;
        u[v_dim + 1] = ut;
    }
    for (int i = 0; i < len; ++i)
        x[i] = u[i] * d[i];
    free(a);
    free(om);
    free(u);
}

void oracle_exp_dual_residual(const double *rc, const double *d, double *out);
void oracle_pow_dual_residual(const double *rc, const double *d, double alpha, double *out);
void oracle_psd_dual_residual(int order, const double *rc, const double *d, double *out);

void oracle_cone_dual_residual_block(int type, int v_dim, double power_alpha, const double *rc,
                                     const double *d, double *out)
{
    int len = block_length(type, v_dim);
    if (type == CONE_EXPONENTIAL) {
        oracle_exp_dual_residual(rc, d, out);
        return;
    }
    if (type == CONE_POWER) {
        oracle_pow_dual_residual(rc, d, power_alpha, out);
        return;
    }
    if (type == CONE_PSD) {
        oracle_psd_dual_residual(v_dim, rc, d, out);
        return;
    }
    double *p = (double *)malloc((size_t)len * sizeof(double));
    memcpy(p, rc, (size_t)len * sizeof(double));
    if (is_uniform(d, len)) {
        if (type == CONE_STANDARD_SOC)
            soc_closed(v_dim + 1, p, p + v_dim + 1);
        else
            rsoc_closed(v_dim, p);
    } else {
        /* dual cone of {x : x/d in K} is {s : s*d in K} for self-dual K */
        double *dinv = (double *)malloc((size_t)len * sizeof(double));
        for (int i = 0; i < len; ++i)
            dinv[i] = 1.0 / d[i];
        oracle_project_cone_block(type, v_dim, power_alpha, p, dinv, NULL, 0.0);
        free(dinv);
    }
    for (int i = 0; i < len; ++i)
        out[i] = (rc[i] - p[i]) * d[i];
    free(p);
}
