/*
 * oracle_cones_extra.c -- exponential, power and PSD cone projections for
 * the oracle.  TEST INFRASTRUCTURE ONLY (see pdhcg_oracle.h).
 */
#include "pdhcg_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

/* ---- exponential cone K = cl{(x, y, z) : y > 0, y exp(x / y) <= z} ------
 * Projection of r onto {v : v / d in K} in the unit metric of r's space,
 * restating the reference's point projection (src/kernels/
 * pdhcg_exp_cone_kernels.cu:26-131): the in-cone and polar-cone tests, the
 * (x <= 0, y <= 0) case, then Newton on rho = x / y of the projection
 * (at most 100 steps, step capped at 10, stop below 1e-13 (1 + |rho|),
 * |rho| >= 299 counts as diverged), and the same fallbacks. */
static void exp_point(double r1, double r2, double r3, double d1, double d2, double d3, double *o)
{
    const double e_const = 2.718281828459045;
    const double a1 = r1 / d1, a2 = r2 / d2, a3 = r3 / d3;
    if (a2 > 0.0) {
        double t = a1 / a2;
        if (t < 700.0 && a2 * exp(t) <= a3) {
            o[0] = r1; o[1] = r2; o[2] = r3;
            return;
        }
    } else if (a2 == 0.0 && a1 <= 0.0 && a3 >= 0.0) {
        o[0] = r1; o[1] = r2; o[2] = r3;
        return;
    }
    if (r1 > 0.0) {
        double t = (d2 * r2) / (d1 * r1);
        if (t < 700.0 && d1 * r1 * exp(t) + e_const * d3 * r3 <= 0.0) {
            o[0] = o[1] = o[2] = 0.0;
            return;
        }
    } else if (r1 == 0.0 && r2 <= 0.0 && r3 <= 0.0) {
        o[0] = o[1] = o[2] = 0.0;
        return;
    }
    if (a1 <= 0.0 && a2 <= 0.0) {
        o[0] = r1;
        o[1] = 0.0;
        o[2] = a3 < 0.0 ? 0.0 : r3;
        return;
    }
    const double al = (d3 / d1) * (d3 / d1), be = (d3 / d2) * (d3 / d2);
    double rho = 0.0;
    int diverged = 0;
    for (int it = 0; it < 100; ++it) {
        if (rho >= 299.0 || rho <= -299.0) {
            diverged = 1;
            break;
        }
        double er = exp(rho), e2 = er * er, omr = 1.0 - rho;
        double A = al - be * rho * omr;
        double B = be * a1 * omr - al * a2;
        double f = a1 - a2 * rho + a3 * er * A + e2 * B;
        double dA = -be * (1.0 - 2.0 * rho), dB = -be * a1;
        double df = -a2 + a3 * er * (A + dA) + e2 * (2.0 * B + dB);
        if (fabs(df) < 1e-300)
            break;
        double step = f / df;
        if (step > 10.0) step = 10.0;
        if (step < -10.0) step = -10.0;
        rho -= step;
        if (fabs(step) < 1e-13 * (1.0 + fabs(rho)))
            break;
    }
    double er = exp(rho);
    double u2 = (a1 + al * a3 * er) / (rho + al * er * er);
    if (diverged || !isfinite(u2) || u2 <= 0.0) {
        o[0] = r1 < 0.0 ? r1 : 0.0;
        o[1] = 0.0;
        o[2] = r3 > 0.0 ? r3 : 0.0;
        return;
    }
    o[0] = d1 * rho * u2;
    o[1] = d2 * u2;
    o[2] = d3 * u2 * er;
}

/* weights w = 1 + tau q (diagonal Q; 1 without): the projection in the metric
 * sum w_i (v_i - x_i)^2 is the unit-metric one of sqrt(w) x onto
 * {v : v / (sqrt(w) d) in K}, scaled back (reference
 * project_exp_cone_diag_q_kernel, src/kernels/pdhcg_exp_cone_kernels.cu:624-691) */
void oracle_exp_project(double *x, const double *d, const double *q, double tau)
{
    double sw[3], o[3];
    for (int i = 0; i < 3; ++i) {
        double w = q ? 1.0 + tau * q[i] : 1.0;
        if (!(w > 0.0)) w = 1.0;
        sw[i] = sqrt(w);
    }
    if (!q) {
        exp_point(x[0], x[1], x[2], d[0], d[1], d[2], o);
        x[0] = o[0]; x[1] = o[1]; x[2] = o[2];
        return;
    }
    exp_point(sw[0] * x[0], sw[1] * x[1], sw[2] * x[2], sw[0] * d[0], sw[1] * d[1], sw[2] * d[2], o);
    for (int i = 0; i < 3; ++i)
        x[i] = o[i] / sw[i];
}

/* ---- power cone K_a = {(x, y, z) : x, y >= 0, x^a y^(1-a) >= |z|} ----------
 * Weighted projection min sum w_i (v_i - r_i)^2 over K_a, restating the
 * reference (src/kernels/pdhcg_power_cone_kernels.cu:25-133): in-cone and
 * opposite-cone tests, then 80 bisection steps on log |v_z| with
 * x(rho), y(rho) the positive roots of the KKT quadratics, after scaling the
 * point by its largest magnitude. */
static double pos_root(double r, double q)
{
    if (!(q > 0.0))
        return fmax(r, 0.0);
    double disc = hypot(r, 2.0 * sqrt(q));
    return r >= 0.0 ? 0.5 * (r + disc) : (2.0 * q) / (disc - r);
}

static void pow_point_unit(double rx, double ry, double rz, double wx, double wy, double wz, double a, double *o)
{
    const double az = fabs(rz), sz = rz >= 0.0 ? 1.0 : -1.0, om = 1.0 - a;
    if (az == 0.0) {
        o[0] = fmax(rx, 0.0); o[1] = fmax(ry, 0.0); o[2] = 0.0;
        return;
    }
    if (rx > 0.0 && ry > 0.0 && a * log(rx) + om * log(ry) >= log(az)) {
        o[0] = rx; o[1] = ry; o[2] = rz;
        return;
    }
    if (rx <= 0.0 && ry <= 0.0) {
        double u = rx < 0.0 ? (-wx * rx) / a : 0.0;
        double v = ry < 0.0 ? (-wy * ry) / om : 0.0;
        if (u > 0.0 && v > 0.0 && a * log(u) + om * log(v) >= log(wz) + log(az)) {
            o[0] = o[1] = o[2] = 0.0;
            return;
        }
    }
    const double cx = 4.0 * a * (wz / wx), cy = 4.0 * om * (wz / wy);
    double lo = log(DBL_MIN), hi = log(az);
    if (!(hi > lo)) {
        o[0] = fmax(rx, 0.0); o[1] = fmax(ry, 0.0); o[2] = 0.0;
        return;
    }
    for (int it = 0; it < 80; ++it) {
        double lr = lo + 0.5 * (hi - lo), rho = exp(lr);
        double x = pos_root(rx, 0.25 * cx * rho * (az - rho));
        double y = pos_root(ry, 0.25 * cy * rho * (az - rho));
        if (x > 0.0 && y > 0.0 && a * log(x) + om * log(y) > lr)
            lo = lr;
        else
            hi = lr;
    }
    double rho = exp(lo + 0.5 * (hi - lo));
    o[0] = pos_root(rx, 0.25 * cx * rho * (az - rho));
    o[1] = pos_root(ry, 0.25 * cy * rho * (az - rho));
    o[2] = sz * fmin(rho, exp(a * log(o[0]) + om * log(o[1])));
}

static void pow_point(double rx, double ry, double rz, double wx, double wy, double wz, double a, double *o)
{
    double s = fmax(fabs(rx), fmax(fabs(ry), fabs(rz)));
    if (!(s > 0.0) || !isfinite(s)) {
        pow_point_unit(rx, ry, rz, wx, wy, wz, a, o);
        return;
    }
    pow_point_unit(rx / s, ry / s, rz / s, wx, wy, wz, a, o);
    o[0] *= s; o[1] *= s; o[2] *= s;
}

/* scaled space: v = x / d with weights w d^2 (w = 1 + tau q, 1 without Q)
 * (reference project_power_cone_kernel / project_power_cone_diag_q_kernel) */
void oracle_pow_project(double *x, const double *d, const double *q, double tau, double alpha)
{
    double w[3], o[3];
    for (int i = 0; i < 3; ++i)
        w[i] = (q ? 1.0 + tau * q[i] : 1.0) * d[i] * d[i];
    pow_point(x[0] / d[0], x[1] / d[1], x[2] / d[2], w[0], w[1], w[2], alpha, o);
    for (int i = 0; i < 3; ++i)
        x[i] = o[i] * d[i];
}

/* ---- PSD cone: x holds svec(X) of a symmetric order-n matrix -------------
 * Slots run down the columns of the lower triangle (col 0: rows 0..n-1,
 * col 1: rows 1..n-1, ...), off-diagonal entries scaled by sqrt 2, so that
 * the slot inner product is the trace inner product (reference
 * src/kernels/pdhcg_psd_cone_kernels.cu:65-91, gather / scatter of the
 * packed matrices).  The projection is the Frobenius one, taken in the
 * scaled space as the reference does (:415-475): eigen-decompose X, clip
 * negative eigenvalues, repack.  Order 1 is max(x, 0).
 *
 * The eigen-decomposition is the cyclic Jacobi method with Rutishauser's
 * rotation (theta = (a_qq - a_pp) / (2 a_pq), t = sign(theta) / (|theta| +
 * sqrt(theta^2 + 1)), c = 1 / sqrt(t^2 + 1), s = t c), sweeping pairs
 * p < q in row order until the off-diagonal mass falls below 1e-28 of the
 * matrix's (at most 100 sweeps; the reference's batched Jacobi uses
 * tolerance 1e-12 and 100 sweeps).  The device restates the same steps. */
#define PSD_MAX_SWEEPS 100
#define PSD_OFF_REL 1e-28

static void psd_jacobi(int n, double *A, double *V)
{
    for (int i = 0; i < n * n; ++i) V[i] = 0.0;
    for (int i = 0; i < n; ++i) V[i * n + i] = 1.0;
    for (int sweep = 0; sweep < PSD_MAX_SWEEPS; ++sweep) {
        double off = 0.0, all = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                double a2 = A[i * n + j] * A[i * n + j];
                all += a2;
                if (i != j) off += a2;
            }
        if (!(off > PSD_OFF_REL * all)) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = A[p * n + q];
                if (apq == 0.0) continue;
                double theta = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
                double t = fabs(theta) > 1e150 ? 0.5 / theta
                                               : (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < n; ++k) { /* columns p, q of A and V */
                    double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - sn * akq;
                    A[k * n + q] = sn * akp + c * akq;
                    double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - sn * vkq;
                    V[k * n + q] = sn * vkp + c * vkq;
                }
                for (int k = 0; k < n; ++k) { /* rows p, q of A */
                    double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - sn * aqk;
                    A[q * n + k] = sn * apk + c * aqk;
                }
                A[p * n + q] = A[q * n + p] = 0.0;
            }
    }
}

void oracle_psd_project(int order, double *x)
{
    const int n = order;
    const double r2 = 1.41421356237309504880, ir2 = 0.70710678118654752440;
    if (n == 1) {
        x[0] = fmax(x[0], 0.0);
        return;
    }
    int len = n * (n + 1) / 2, finite = 1;
    for (int i = 0; i < len; ++i) finite &= isfinite(x[i]) != 0;
    if (!finite) { /* the reference's failed decomposition: NaN */
        for (int i = 0; i < len; ++i) x[i] = NAN;
        return;
    }
    double *A = (double *)malloc(sizeof(double) * (size_t)n * n);
    double *V = (double *)malloc(sizeof(double) * (size_t)n * n);
    int slot = 0;
    for (int col = 0; col < n; ++col)
        for (int row = col; row < n; ++row, ++slot) {
            double v = row == col ? x[slot] : x[slot] * ir2;
            A[row * n + col] = A[col * n + row] = v;
        }
    psd_jacobi(n, A, V);
    slot = 0;
    for (int col = 0; col < n; ++col)
        for (int row = col; row < n; ++row, ++slot) {
            double v = 0.0;
            for (int e = 0; e < n; ++e)
                v += fmax(A[e * n + e], 0.0) * V[row * n + e] * V[col * n + e];
            x[slot] = row == col ? v : v * r2;
        }
    free(A);
    free(V);
}

/* Moreau: the dual residual of rc = c_eff - A^T y is -proj_K(-rc) in the
 * inverse scaling (reference compute_cone_dual_residual_exp_kernel,
 * src/kernels/pdhcg_exp_cone_kernels.cu:562-622) */
void oracle_exp_dual_residual(const double *rc, const double *d, double *out)
{
    double o[3];
    exp_point(-rc[0], -rc[1], -rc[2], 1.0 / d[0], 1.0 / d[1], 1.0 / d[2], o);
    for (int i = 0; i < 3; ++i)
        out[i] = -o[i] * d[i];
}

/* -proj_K(-rc d) in the unit metric (reference
 * compute_cone_dual_residual_power_kernel, non-fixed branch) */
void oracle_pow_dual_residual(const double *rc, const double *d, double alpha, double *out)
{
    double o[3];
    pow_point(-rc[0] * d[0], -rc[1] * d[1], -rc[2] * d[2], 1.0, 1.0, 1.0, alpha, o);
    for (int i = 0; i < 3; ++i)
        out[i] = -o[i];
}

/* (rc - proj_PSD(rc)) d: the PSD cone is self-dual and the reference
 * projects rc without a metric (compute_psd_cone_dual_residual,
 * src/kernels/pdhcg_psd_cone_kernels.cu:477-506) */
void oracle_psd_dual_residual(int order, const double *rc, const double *d, double *out)
{
    int len = order * (order + 1) / 2;
    double *p = (double *)malloc(sizeof(double) * (size_t)len);
    for (int i = 0; i < len; ++i) p[i] = rc[i];
    oracle_psd_project(order, p);
    for (int i = 0; i < len; ++i) out[i] = (rc[i] - p[i]) * d[i];
    free(p);
}
