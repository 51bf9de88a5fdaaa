/*
 * oracle_sections.c -- projections onto fixed cross-sections of cones.
 *
 * TEST INFRASTRUCTURE ONLY (see pdhcg_oracle.h).
 *
 * A cone block may have slots fixed by set_cone_fixed (reference
 * src/pdhcg.c:620-666).  Those slots keep the value they hold (the solver
 * pins their scaled bounds, so the box step has already put the value
 * there) and the free slots are projected onto the slice of the cone
 * through the fixed values, in the weighted metric
 *   sum_i omega_i (u_i - a_i)^2,  u = x / d,  a = input / d,
 *   omega_i = max((1 + tau q_i) d_i^2, DBL_MIN)
 * (reference internal/cone_projection_utils.h:22-28).  Each restatement
 * below follows the reference's serial section projector for its cone:
 *   standard SOC  src/kernels/pdhcg_soc_cone_kernels.cu:23-260
 *   rotated SOC   src/kernels/pdhcg_rsoc_cone_kernels.cu:23-465
 *   exponential   src/kernels/pdhcg_exp_cone_kernels.cu:134-525
 *   power         src/kernels/pdhcg_power_cone_kernels.cu:135-434
 * with the same root finders (bisection on the KKT multiplier, golden
 * section on the one-dimensional slices of the exponential cone), the
 * same brackets and the same stopping rules, so that the two agree to
 * the rounding of the arithmetic.
 */
#include "pdhcg_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SECTION_TOL 1e-13
#define SECTION_BISECT 80

static double weight_at(const double *d, const double *q, double tau, int i)
{
    double metric = q ? 1.0 + tau * q[i] : 1.0;
    return fmax(metric * d[i] * d[i], DBL_MIN);
}

/* sum over the free slots i in [0, cnt) of (a_i omega_i / (omega_i + lam))^2 */
static double shrunk_norm2(int cnt, const double *a, const double *om, const char *fx, double lam)
{
    double s = 0.0;
    for (int i = 0; i < cnt; ++i) {
        if (fx[i]) continue;
        double v = a[i] * om[i] / (om[i] + lam);
        s += v * v;
    }
    return s;
}

static int bisect_done(double lo, double hi) { return (hi - lo) <= SECTION_TOL * (1.0 + hi + lo); }

/* Multiplier that pulls the free vector slots inside a ball of radius^2 r2
 * (both SOC endpoints fixed): the vector slots shrink by omega/(omega+lam). */
static double ball_multiplier(int cnt, const double *a, const double *om, const char *fx, double polar2, double r2,
                              double *warm)
{
    double lo = 0.0;
    double hi = sqrt(polar2) / sqrt(r2) * (1.0 + 64.0 * DBL_EPSILON);
    if (!(hi > 0.0) || !isfinite(hi)) {
        hi = warm && *warm > 0.0 && isfinite(*warm) ? *warm : 1.0;
        for (int e = 0; e < 100; ++e) {
            if (shrunk_norm2(cnt, a, om, fx, hi) <= r2) break;
            hi *= 2.0;
        }
    }
    for (int it = 0; it < SECTION_BISECT; ++it) {
        double mid = 0.5 * (lo + hi);
        if (shrunk_norm2(cnt, a, om, fx, mid) > r2) lo = mid;
        else hi = mid;
        if (bisect_done(lo, hi)) break;
    }
    return 0.5 * (lo + hi);
}

/* Upper end of the bracket on the negative branch of a weighted SOC
 * (reference cone_section_negative_soc_upper,
 * internal/cone_projection_utils.h:44-62). */
static double soc_negative_upper(double sing, double endpoint_polar, double fixed2, double polar2, double max_om)
{
    double up;
    if (fixed2 > 0.0) {
        up = sing + endpoint_polar / sqrt(fixed2);
    } else {
        double pn = sqrt(polar2), gap = pn - endpoint_polar;
        if (!(gap > 0.0)) return NAN;
        up = (pn / gap) * sing + (endpoint_polar / gap) * max_om;
    }
    return up * (1.0 + 64.0 * DBL_EPSILON);
}

/* ---------------- standard SOC {(u, z) : |u| <= z}, u = slots 0..k ---------------- */

static void soc_section(int k, double *x, const double *d, const double *q, double tau, const char *fx,
                        double *warm)
{
    const int nu = k + 1, zi = k + 1;
    double *a = (double *)malloc((size_t)(k + 2) * sizeof(double));
    double *om = (double *)malloc((size_t)(k + 2) * sizeof(double));
    double fixed2 = 0.0, free2 = 0.0, polar2 = 0.0, max_om = 0.0;
    int nfree = 0;
    for (int i = 0; i < k + 2; ++i) {
        a[i] = x[i] / d[i];
        om[i] = weight_at(d, q, tau, i);
    }
    for (int i = 0; i < nu; ++i) {
        if (fx[i]) {
            fixed2 += a[i] * a[i];
        } else {
            free2 += a[i] * a[i];
            polar2 += (om[i] * a[i]) * (om[i] * a[i]);
            max_om = fmax(max_om, om[i]);
            ++nfree;
        }
    }
    const double az = a[zi];
    double lam;
    if (fx[zi]) {
        double r2 = fmax(0.0, az * az - fixed2);
        if (nfree == 0 || free2 <= r2) goto done;
        if (!(r2 > 0.0)) {
            for (int i = 0; i < nu; ++i)
                if (!fx[i]) x[i] = 0.0;
            goto done;
        }
        lam = ball_multiplier(nu, a, om, fx, polar2, r2, warm);
        if (warm) *warm = lam;
        for (int i = 0; i < nu; ++i)
            if (!fx[i]) x[i] *= om[i] / (om[i] + lam);
        goto done;
    }
    if (az >= 0.0 && fixed2 + free2 <= az * az) goto done;
    if (nfree == 0) {
        x[zi] = fmax(az, sqrt(fixed2)) * d[zi];
        goto done;
    }
    {
        const double omz = om[zi];
        if (fixed2 == 0.0 && -omz * az >= sqrt(polar2)) {
            for (int i = 0; i < nu; ++i)
                if (!fx[i]) x[i] = 0.0;
            x[zi] = 0.0;
            goto done;
        }
        if (az == 0.0) {
            lam = omz;
            x[zi] = sqrt(fixed2 + shrunk_norm2(nu, a, om, fx, lam)) * d[zi];
        } else {
            /* |u(lam)|^2 = z(lam)^2 with z = omz az / (omz - lam): lam < omz when
             * az > 0, lam > omz when az < 0 */
            const int lower = az > 0.0;
            double lo, hi;
            if (lower) {
                lo = 0.0;
                hi = omz * (1.0 - 1e-14);
            } else {
                lo = omz * (1.0 + 1e-14);
                hi = soc_negative_upper(omz, -omz * az, fixed2, polar2, max_om);
                if (!(hi > lo) || !isfinite(hi)) {
                    hi = 2.0 * omz;
                    for (int e = 0; e < 100; ++e) {
                        double z = omz * az / (omz - hi);
                        if (fixed2 + shrunk_norm2(nu, a, om, fx, hi) >= z * z) break;
                        hi *= 2.0;
                    }
                }
            }
            if (warm && *warm > lo && *warm < hi && isfinite(*warm)) {
                double z = omz * az / (omz - *warm);
                double f = fixed2 + shrunk_norm2(nu, a, om, fx, *warm) - z * z;
                if ((lower && f > 0.0) || (!lower && f < 0.0)) lo = *warm;
                else hi = *warm;
            }
            for (int it = 0; it < SECTION_BISECT; ++it) {
                double mid = 0.5 * (lo + hi);
                double z = omz * az / (omz - mid);
                double f = fixed2 + shrunk_norm2(nu, a, om, fx, mid) - z * z;
                if ((lower && f > 0.0) || (!lower && f < 0.0)) lo = mid;
                else hi = mid;
                if (bisect_done(lo, hi)) break;
            }
            lam = 0.5 * (lo + hi);
            x[zi] *= omz / (omz - lam);
        }
        if (warm) *warm = lam;
        for (int i = 0; i < nu; ++i)
            if (!fx[i]) x[i] *= om[i] / (om[i] + lam);
    }
done:
    free(a);
    free(om);
}

/* ---------------- rotated SOC {(u, s, t) : |u|^2 <= 2 s t, s, t >= 0} ---------------- */

/* Negative-branch bracket of the rotated cone: the rotated cone in
 * sum/difference endpoint coordinates is a standard one (reference
 * cone_section_negative_rsoc_upper, src/kernels/pdhcg_rsoc_cone_kernels.cu:23-45). */
static double rsoc_negative_upper(double oms, double omt, double s, double t, double fixed2, double polar2,
                                  double max_om)
{
    const double r2 = 0.70710678118654752440;
    double ss = sqrt(oms), st = sqrt(omt), root = ss * st;
    double ws = ss * s, wt = st * t;
    double tw = (ws - wt) * r2;
    double endpoint_polar = -(ws + wt) * r2;
    double up = soc_negative_upper(1.0, endpoint_polar, root * fixed2, polar2 / root + tw * tw,
                                   fmax(1.0, max_om / root));
    return root * up;
}

/* weighted distance^2 of (u(lam), s, t) from the input (free slots only) */
static double rsoc_objective(int k, const double *a, const double *om, const char *fx, double lam, double s,
                             double t)
{
    double obj = 0.0;
    for (int i = 0; i < k; ++i) {
        if (fx[i]) continue;
        double v = a[i] * om[i] / (om[i] + lam), dv = v - a[i];
        obj += om[i] * dv * dv;
    }
    double ds = s - a[k], dt = t - a[k + 1];
    return obj + om[k] * ds * ds + om[k + 1] * dt * dt;
}

static void rsoc_section(int k, double *x, const double *d, const double *q, double tau, const char *fx,
                         double *warm)
{
    const int si = k, ti = k + 1;
    double *a = (double *)malloc((size_t)(k + 2) * sizeof(double));
    double *om = (double *)malloc((size_t)(k + 2) * sizeof(double));
    double fixed2 = 0.0, free2 = 0.0, polar2 = 0.0, max_om = 0.0;
    int nfree = 0;
    for (int i = 0; i < k + 2; ++i) {
        a[i] = x[i] / d[i];
        om[i] = weight_at(d, q, tau, i);
    }
    for (int i = 0; i < k; ++i) {
        if (fx[i]) {
            fixed2 += a[i] * a[i];
        } else {
            free2 += a[i] * a[i];
            polar2 += (om[i] * a[i]) * (om[i] * a[i]);
            max_om = fmax(max_om, om[i]);
            ++nfree;
        }
    }
    const double as = a[si], at = a[ti];
    if (fx[si] && fx[ti]) {
        double r2 = fmax(0.0, 2.0 * as * at - fixed2);
        if (nfree == 0 || free2 <= r2) goto done;
        if (!(r2 > 0.0)) {
            for (int i = 0; i < k; ++i)
                if (!fx[i]) x[i] = 0.0;
            goto done;
        }
        double lam = ball_multiplier(k, a, om, fx, polar2, r2, warm);
        if (warm) *warm = lam;
        for (int i = 0; i < k; ++i)
            if (!fx[i]) x[i] *= om[i] / (om[i] + lam);
        goto done;
    }
    if (fx[si] || fx[ti]) {
        /* one endpoint e fixed: |u|^2 <= 2 e f with the other endpoint f free */
        const int fi = fx[si] ? ti : si;
        const double e = fx[si] ? as : at, af = fx[si] ? at : as, omf = om[fi];
        if (!(e > 0.0)) {
            for (int i = 0; i < k; ++i)
                if (!fx[i]) x[i] = 0.0;
            x[fi] = fmax(af, 0.0) * d[fi];
            goto done;
        }
        if (af >= 0.0 && fixed2 + free2 <= 2.0 * e * af) goto done;
        if (nfree == 0) {
            x[fi] = fmax(af, fixed2 / (2.0 * e)) * d[fi];
            goto done;
        }
        double lo = 0.0;
        double viol = fixed2 + free2 - 2.0 * e * af;
        double hi = omf * viol / (2.0 * e * e) * (1.0 + 64.0 * DBL_EPSILON);
        if (!(hi > 0.0) || !isfinite(hi)) {
            hi = warm && *warm > 0.0 && isfinite(*warm) ? *warm : omf;
            for (int it = 0; it < 100; ++it) {
                double f = af + hi * e / omf;
                if (fixed2 + shrunk_norm2(k, a, om, fx, hi) <= 2.0 * e * f) break;
                hi *= 2.0;
            }
        }
        for (int it = 0; it < SECTION_BISECT; ++it) {
            double mid = 0.5 * (lo + hi);
            double f = af + mid * e / omf;
            if (fixed2 + shrunk_norm2(k, a, om, fx, mid) > 2.0 * e * f) lo = mid;
            else hi = mid;
            if (bisect_done(lo, hi)) break;
        }
        double lam = 0.5 * (lo + hi);
        if (warm) *warm = lam;
        for (int i = 0; i < k; ++i)
            if (!fx[i]) x[i] *= om[i] / (om[i] + lam);
        x[fi] = (af + lam * e / omf) * d[fi];
        goto done;
    }
    if (as >= 0.0 && at >= 0.0 && fixed2 + free2 <= 2.0 * as * at) goto done;
    {
        const double oms = om[si], omt = om[ti];
        if (fixed2 == 0.0) {
            double bs = oms * as, bt = omt * at;
            if (bs <= 0.0 && bt <= 0.0 && polar2 <= 2.0 * bs * bt) {
                for (int i = 0; i < k; ++i)
                    if (!fx[i]) x[i] = 0.0;
                x[si] = 0.0;
                x[ti] = 0.0;
                goto done;
            }
        }
        const double root = sqrt(oms) * sqrt(omt);
        const double balance = sqrt(oms) * as + sqrt(omt) * at;
        const double bscale = 1.0 + fabs(sqrt(oms) * as) + fabs(sqrt(omt) * at);
        double lam = root, ps = 0.0, pt = 0.0;
        int smooth = 1;
        if (fabs(balance) <= 64.0 * DBL_EPSILON * bscale) {
            /* lam = sqrt(oms omt): the endpoint system is singular; solve the
             * product condition directly in the metric-scaled endpoints */
            double n2 = fixed2 + shrunk_norm2(k, a, om, fx, lam);
            double prod = 0.5 * root * n2;
            double delta = sqrt(oms) * as;
            double st = 0.5 * (-delta + sqrt(fmax(0.0, delta * delta + 4.0 * prod)));
            double ss = st + delta;
            ps = ss / sqrt(oms);
            pt = st / sqrt(omt);
            smooth = ps >= 0.0 && pt >= 0.0;
        } else {
            const int lower = balance > 0.0;
            double lo = lower ? 0.0 : root * (1.0 + 1e-14);
            double hi = lower ? root * (1.0 - 1e-14) : 2.0 * root;
            if (!lower) {
                hi = rsoc_negative_upper(oms, omt, as, at, fixed2, polar2, max_om);
                if (!(hi > lo) || !isfinite(hi)) {
                    hi = 2.0 * root;
                    for (int e = 0; e < 100; ++e) {
                        double det = oms * omt - hi * hi;
                        double s = omt * (oms * as + hi * at) / det;
                        double t = oms * (omt * at + hi * as) / det;
                        double f = INFINITY;
                        if (s >= 0.0 && t >= 0.0) f = fixed2 + shrunk_norm2(k, a, om, fx, hi) - 2.0 * s * t;
                        if (f >= 0.0) break;
                        hi *= 2.0;
                    }
                }
            }
            for (int it = 0; it < 90; ++it) {
                double mid = 0.5 * (lo + hi);
                double det = oms * omt - mid * mid;
                double s = omt * (oms * as + mid * at) / det;
                double t = oms * (omt * at + mid * as) / det;
                double f = INFINITY;
                if (s >= 0.0 && t >= 0.0) f = fixed2 + shrunk_norm2(k, a, om, fx, mid) - 2.0 * s * t;
                if ((lower && f > 0.0) || (!lower && f < 0.0)) lo = mid;
                else hi = mid;
                if (bisect_done(lo, hi)) break;
            }
            lam = 0.5 * (lo + hi);
            double det = oms * omt - lam * lam;
            ps = omt * (oms * as + lam * at) / det;
            pt = oms * (omt * at + lam * as) / det;
            smooth = isfinite(ps) && isfinite(pt) && ps >= 0.0 && pt >= 0.0;
        }
        /* with no fixed vector slots the two axes {u = 0, t = 0} and
         * {u = 0, s = 0} are candidates too: keep the nearest */
        double best = smooth ? rsoc_objective(k, a, om, fx, lam, ps, pt) : INFINITY;
        int on_axis = !smooth;
        if (fixed2 == 0.0) {
            double vec = 0.0;
            for (int i = 0; i < k; ++i)
                if (!fx[i]) vec += om[i] * a[i] * a[i];
            double sa = fmax(as, 0.0);
            double sobj = vec + oms * (sa - as) * (sa - as) + omt * at * at;
            if (sobj < best) {
                best = sobj;
                ps = sa;
                pt = 0.0;
                on_axis = 1;
            }
            double ta = fmax(at, 0.0);
            double tobj = vec + oms * as * as + omt * (ta - at) * (ta - at);
            if (tobj < best) {
                ps = 0.0;
                pt = ta;
                on_axis = 1;
            }
        }
        if (!on_axis) {
            for (int i = 0; i < k; ++i)
                if (!fx[i]) x[i] *= om[i] / (om[i] + lam);
            if (warm) *warm = lam;
        } else {
            for (int i = 0; i < k; ++i)
                if (!fx[i]) x[i] = 0.0;
            if (warm) *warm = 0.0;
        }
        x[si] = ps * d[si];
        x[ti] = pt * d[ti];
    }
done:
    free(a);
    free(om);
}

/* ---------------- exponential cone {(x, y, z) : y e^{x/y} <= z, y > 0} closure ---------------- */

/* Weighted projection of (x, z) with y > 0 fixed onto the slice
 * {(x, z) : y e^{x/y} <= z}, by safeguarded Newton in u = z / (d_t y)
 * (reference project_2d_exp_persp, src/kernels/pdhcg_exp_cone_kernels.cu:134-231);
 * inputs and outputs carry the square roots of the weights. */
static void exp_slice_fixed_y(double rz0, double ry, double rt0, double d_r, double d_y, double d_t, double *warm,
                              double *rzo, double *rto)
{
    if (d_r <= 0.0 || d_y <= 0.0 || d_t <= 0.0) {
        *rzo = rz0;
        *rto = rt0;
        return;
    }
    double ye = ry / d_y;
    if (ye <= 0.0) {
        *rzo = rz0 < 0.0 ? rz0 : 0.0;
        *rto = rt0 > 0.0 ? rt0 : 0.0;
        return;
    }
    double arg = (rz0 / d_r) / ye;
    if (arg < 700.0 && ye * d_t * exp(arg) <= rt0) {
        *rzo = rz0;
        *rto = rt0;
        return;
    }
    /* stationarity in u: A u^2 - B u + C log u - E = 0 */
    const double A = d_t * d_t * ye, B = d_t * rt0, Cc = d_r * d_r * ye, E = d_r * rz0;
    double u = *warm, ulo = 1e-30, uhi = 1.0;
    for (int g = 0; g < 200; ++g) {
        double f = A * uhi * uhi - B * uhi + Cc * log(uhi) - E;
        if (isfinite(f) && f > 0.0) break;
        uhi *= 4.0;
        if (uhi > 1e150) break;
    }
    for (int g = 0; g < 200; ++g) {
        double f = A * ulo * ulo - B * ulo + Cc * log(ulo) - E;
        if (isfinite(f) && f < 0.0) break;
        ulo *= 0.25;
        if (ulo < 1e-300) break;
    }
    if (ulo >= uhi) {
        *rzo = rz0;
        *rto = rt0;
        return;
    }
    if (!(u > ulo && u < uhi) || !isfinite(u)) u = exp(0.5 * (log(ulo) + log(uhi)));
    for (int it = 0; it < 80; ++it) {
        double f = A * u * u - B * u + Cc * log(u) - E;
        double df = 2.0 * A * u - B + Cc / u;
        if (f > 0.0) uhi = u;
        else ulo = u;
        double un;
        if (df > 1e-300 && isfinite(df) && isfinite(f)) {
            un = u - f / df;
            if (!isfinite(un) || un <= ulo || un >= uhi) un = exp(0.5 * (log(ulo) + log(uhi)));
        } else {
            un = exp(0.5 * (log(ulo) + log(uhi)));
        }
        if (fabs(un - u) < 1e-14 * (1.0 + fabs(un))) {
            u = un;
            break;
        }
        u = un;
    }
    *warm = u;
    *rzo = d_r * ye * log(u);
    *rto = d_t * ye * u;
}

/* z on the boundary for (x, y): y e^{x/y}, in logs */
static double exp_boundary(double x, double y)
{
    if (!(y > 0.0)) return x <= 0.0 ? 0.0 : INFINITY;
    double lv = log(y) + x / y;
    if (lv >= log(DBL_MAX)) return INFINITY;
    if (lv <= log(DBL_MIN)) return 0.0;
    return exp(lv);
}

static int exp_contains(double x, double y, double z)
{
    if (y > 0.0 && z > 0.0) {
        double lhs = log(y) + x / y, rhs = log(z);
        return lhs <= rhs + 64.0 * DBL_EPSILON * (1.0 + fabs(lhs) + fabs(rhs));
    }
    return y == 0.0 && x <= 0.0 && z >= 0.0;
}

/* distance^2 in (y, z) of the boundary point over (x fixed, y) */
static double exp_obj_fixed_x(double y, double x, double iy, double iz, double wy, double wz)
{
    double z = exp_boundary(x, y);
    if (!isfinite(z)) return INFINITY;
    return wy * (y - iy) * (y - iy) + wz * (z - iz) * (z - iz);
}

/* distance^2 in (x, y) of the boundary point over (z fixed, y) */
static double exp_obj_fixed_z(double y, double z, double ix, double iy, double wx, double wy)
{
    double x = y > 0.0 ? y * (log(z) - log(y)) : 0.0;
    return wx * (x - ix) * (x - ix) + wy * (y - iy) * (y - iy);
}

/* log y + x / y - log z, with the closure's signs at y <= 0 or z <= 0 */
static double exp_log_violation(double y, double x, double z)
{
    if (!(y > 0.0) || !(z > 0.0)) return x <= 0.0 ? -INFINITY : INFINITY;
    return log(y) + x / y - log(z);
}

typedef double (*exp_obj_fn)(double, double, double, double, double, double);

/* golden-section minimum of obj(y, p0..p4) over y in [lo, hi] after
 * doubling hi while the objective still falls (reference
 * src/kernels/pdhcg_exp_cone_kernels.cu:422-456, 474-509) */
static double exp_golden(exp_obj_fn obj, double lo, double hi, double p0, double p1, double p2, double p3,
                         double p4)
{
    double prev = obj(0.5 * hi, p0, p1, p2, p3, p4);
    double cur = obj(hi, p0, p1, p2, p3, p4);
    for (int e = 0; e < 80 && cur < prev && hi < DBL_MAX / 4.0; ++e) {
        prev = cur;
        hi *= 2.0;
        cur = obj(hi, p0, p1, p2, p3, p4);
    }
    const double r = 0.6180339887498948482;
    double a = lo, b = hi, c = b - r * (b - a), dd = a + r * (b - a);
    double fc = obj(c, p0, p1, p2, p3, p4), fd = obj(dd, p0, p1, p2, p3, p4);
    for (int it = 0; it < 100; ++it) {
        if (fc <= fd) {
            b = dd;
            dd = c;
            fd = fc;
            c = b - r * (b - a);
            fc = obj(c, p0, p1, p2, p3, p4);
        } else {
            a = c;
            c = dd;
            fc = fd;
            dd = a + r * (b - a);
            fd = obj(dd, p0, p1, p2, p3, p4);
        }
    }
    return 0.5 * (a + b);
}

static void exp_section(double *x, const double *d, const double *q, double tau, const char *fx, double *warm)
{
    const int fxx = fx[0] != 0, fxy = fx[1] != 0, fxz = fx[2] != 0;
    const double ix = x[0] / d[0], iy = x[1] / d[1], iz = x[2] / d[2];
    if (exp_contains(ix, iy, iz) || (fxx && fxy && fxz)) return;
    const double wx = weight_at(d, q, tau, 0), wy = weight_at(d, q, tau, 1), wz = weight_at(d, q, tau, 2);
    double ox = ix, oy = iy, oz = iz;
    if (fxx && fxy) {
        oz = fmax(iz, exp_boundary(ix, iy));
    } else if (fxy && fxz) {
        ox = iy == 0.0 ? fmin(ix, 0.0) : fmin(ix, iy * (log(iz) - log(iy)));
    } else if (fxx && fxz) {
        /* y ranges over the interval where log y + x/y <= log z */
        if (iz == 0.0) {
            oy = 0.0;
        } else if (ix > 0.0) {
            double center = ix;
            double left = fmax(DBL_MIN, ix / 1024.0);
            while (exp_log_violation(left, ix, iz) <= 0.0 && left > DBL_MIN) left *= 0.5;
            double lo = left, hi = center;
            for (int it = 0; it < 100; ++it) {
                double mid = 0.5 * (lo + hi);
                if (exp_log_violation(mid, ix, iz) > 0.0) lo = mid;
                else hi = mid;
            }
            double lower = 0.5 * (lo + hi);
            lo = center;
            hi = fmax(2.0 * center, iz);
            while (exp_log_violation(hi, ix, iz) < 0.0 && hi < DBL_MAX / 4.0) hi *= 2.0;
            for (int it = 0; it < 100; ++it) {
                double mid = 0.5 * (lo + hi);
                if (exp_log_violation(mid, ix, iz) <= 0.0) lo = mid;
                else hi = mid;
            }
            double upper = 0.5 * (lo + hi);
            oy = fmin(fmax(iy, lower), upper);
        } else {
            double lo = 0.0, hi = fmax(1.0, fmax(iz, fabs(ix)));
            while (exp_log_violation(hi, ix, iz) < 0.0 && hi < DBL_MAX / 4.0) hi *= 2.0;
            for (int it = 0; it < 100; ++it) {
                double mid = 0.5 * (lo + hi);
                if (exp_log_violation(mid, ix, iz) <= 0.0) lo = mid;
                else hi = mid;
            }
            oy = fmin(fmax(iy, 0.0), 0.5 * (lo + hi));
        }
    } else if (fxy) {
        if (!(iy > 0.0)) {
            ox = fmin(ix, 0.0);
            oz = fmax(iz, 0.0);
        } else {
            double ex = sqrt(wx), ey = sqrt(wy), ez = sqrt(wz), sx, sz;
            exp_slice_fixed_y(ex * ix, ey * iy, ez * iz, ex, ey, ez, warm, &sx, &sz);
            ox = sx / ex;
            oz = sz / ez;
        }
    } else if (fxx) {
        double scale = 1.0 + fabs(ix) + fabs(iy) + fabs(iz);
        double lo = ix > 0.0 ? fmax(DBL_MIN, ix / 700.0) : 0.0;
        oy = exp_golden(exp_obj_fixed_x, lo, scale, ix, iy, iz, wy, wz);
        oz = exp_boundary(ix, oy);
        if (ix <= 0.0) {
            double cz = fmax(iz, 0.0);
            double closure = wy * iy * iy + wz * (cz - iz) * (cz - iz);
            if (closure <= exp_obj_fixed_x(oy, ix, iy, iz, wy, wz)) {
                oy = 0.0;
                oz = cz;
            }
        }
    } else if (fxz) {
        if (iz == 0.0) {
            ox = fmin(ix, 0.0);
            oy = 0.0;
        } else {
            double scale = 1.0 + fabs(ix) + fabs(iy) + iz;
            oy = exp_golden(exp_obj_fixed_z, 0.0, scale, iz, ix, iy, wx, wy);
            ox = oy > 0.0 ? oy * (log(iz) - log(oy)) : 0.0;
            double cx = fmin(ix, 0.0);
            double closure = wx * (cx - ix) * (cx - ix) + wy * iy * iy;
            if (closure <= exp_obj_fixed_z(oy, iz, ix, iy, wx, wy)) {
                ox = cx;
                oy = 0.0;
            }
        }
    }
    if (!fxx) x[0] = ox * d[0];
    if (!fxy) x[1] = oy * d[1];
    if (!fxz) x[2] = oz * d[2];
}

/* ---------------- power cone {(x, y, z) : x^a y^(1-a) >= |z|, x, y >= 0} ---------------- */

static double pos_root2(double r, double qv)
{
    /* positive root of t^2 - r t - qv = 0 (qv > 0) without cancellation;
     * max(r, 0) when qv <= 0 */
    if (!(qv > 0.0)) return fmax(r, 0.0);
    double disc = hypot(r, 2.0 * sqrt(qv));
    return r >= 0.0 ? 0.5 * (r + disc) : (2.0 * qv) / (disc - r);
}

/* log of x^a y^(1-a) at the KKT point of multiplier lam (z fixed) */
static double pow_xy_log_boundary(double lam, double rx, double ry, double wx, double wy, double a)
{
    double x = pos_root2(rx, (lam / wx) * a);
    double y = pos_root2(ry, (lam / wy) * (1.0 - a));
    if (!(x > 0.0) || !(y > 0.0)) return -INFINITY;
    return a * log(x) + (1.0 - a) * log(y);
}

/* (x, y) with z fixed: onto x^a y^(1-a) >= |z| (reference
 * project_power_xy_fixed_z_normalized, src/kernels/pdhcg_power_cone_kernels.cu:146-215) */
static void pow_xy_fixed_z_unit(double rx, double ry, double fz, double wx, double wy, double a, double *xo,
                                double *yo)
{
    double c = fabs(fz), om = 1.0 - a;
    if (c == 0.0) {
        *xo = fmax(rx, 0.0);
        *yo = fmax(ry, 0.0);
        return;
    }
    if (rx > 0.0 && ry > 0.0 && a * log(rx) + om * log(ry) >= log(c)) {
        *xo = rx;
        *yo = ry;
        return;
    }
    double target = log(c);
    double hi = fmin(wx, wy);
    if (!(hi > 0.0) || !isfinite(hi)) hi = 1.0;
    for (int it = 0; it < 2048; ++it) {
        double lb = pow_xy_log_boundary(hi, rx, ry, wx, wy, a);
        if (lb >= target || isnan(lb)) break;
        if (hi >= 0.5 * DBL_MAX) {
            hi = DBL_MAX;
            break;
        }
        hi *= 2.0;
    }
    double lam;
    if (pow_xy_log_boundary(DBL_MIN, rx, ry, wx, wy, a) >= target) {
        double lo = 0.0, fh = DBL_MIN;
        for (int it = 0; it < 80; ++it) {
            double cnd = lo + 0.5 * (fh - lo);
            if (pow_xy_log_boundary(cnd, rx, ry, wx, wy, a) < target) lo = cnd;
            else fh = cnd;
        }
        lam = lo + 0.5 * (fh - lo);
    } else {
        double llo = log(DBL_MIN), lhi = log(hi);
        for (int it = 0; it < 96; ++it) {
            double ll = llo + 0.5 * (lhi - llo);
            if (pow_xy_log_boundary(exp(ll), rx, ry, wx, wy, a) < target) llo = ll;
            else lhi = ll;
        }
        lam = exp(llo + 0.5 * (lhi - llo));
    }
    *xo = pos_root2(rx, (lam / wx) * a);
    *yo = pos_root2(ry, (lam / wy) * om);
}

static void pow_xy_fixed_z(double rx, double ry, double fz, double wx, double wy, double a, double *xo, double *yo)
{
    double scale = fmax(fabs(rx), fmax(fabs(ry), fabs(fz)));
    if (!(scale > 0.0) || !isfinite(scale)) {
        pow_xy_fixed_z_unit(rx, ry, fz, wx, wy, a, xo, yo);
        return;
    }
    double xn, yn;
    pow_xy_fixed_z_unit(rx / scale, ry / scale, fz / scale, wx, wy, a, &xn, &yn);
    *xo = xn * scale;
    *yo = yn * scale;
}

static double pow_exp_of_log(double lv)
{
    if (lv >= log(DBL_MAX)) return INFINITY;
    if (lv <= log(DBL_MIN)) return 0.0;
    return exp(lv);
}

/* derivative in the free axis of the distance to the slice boundary */
static double pow_section_derivative(double o, double ro, double arz, double wo, double wz, double lcoef, double oexp)
{
    if (!(o > 0.0)) return -INFINITY;
    double lo = log(o);
    double bound = pow_exp_of_log(lcoef + oexp * lo);
    double slope = pow_exp_of_log(lcoef + log(oexp) + (oexp - 1.0) * lo);
    double lin = wo * (o - ro);
    double gap = bound - arz;
    if (gap == 0.0 || slope == 0.0) return lin;
    if (!isfinite(slope)) return copysign(INFINITY, gap);
    return lin + wz * gap * slope;
}

/* one axis fixed at f: (other, z) onto |z| <= f^fexp other^oexp, by
 * bisection in the other axis (reference
 * project_power_section_fixed_axis_normalized, src/kernels/pdhcg_power_cone_kernels.cu:263-333) */
static void pow_fixed_axis_unit(double f, double ro, double rz, double wo, double wz, double fexp, double oexp,
                                double *oo, double *zo)
{
    double arz = fabs(rz);
    if (!(f > 0.0) || arz == 0.0) {
        *oo = fmax(ro, 0.0);
        *zo = 0.0;
        return;
    }
    double lcoef = fexp * log(f);
    if (ro > 0.0 && lcoef + oexp * log(ro) >= log(arz)) {
        *oo = ro;
        *zo = rz;
        return;
    }
    double feas = pow_exp_of_log((log(arz) - lcoef) / oexp);
    if (feas == 0.0) {
        *oo = 0.0;
        *zo = 0.0;
        return;
    }
    double lo = 0.0, hi = fmax(1.0, fmax(ro, 0.0));
    if (isfinite(feas)) hi = fmin(hi, feas);
    for (int it = 0; it < 1024; ++it) {
        if (!(pow_section_derivative(hi, ro, arz, wo, wz, lcoef, oexp) < 0.0)) break;
        if (isfinite(feas) && hi >= feas) break;
        double nh = hi * 2.0;
        if (!isfinite(nh)) {
            hi = isfinite(feas) ? feas : DBL_MAX;
            break;
        }
        hi = isfinite(feas) ? fmin(nh, feas) : nh;
    }
    for (int it = 0; it < 80; ++it) {
        double o = lo + 0.5 * (hi - lo);
        if (o == 0.0) break;
        if (pow_section_derivative(o, ro, arz, wo, wz, lcoef, oexp) < 0.0) lo = o;
        else hi = o;
    }
    double o = lo + 0.5 * (hi - lo);
    double az = o > 0.0 ? pow_exp_of_log(lcoef + oexp * log(o)) : 0.0;
    *oo = o;
    *zo = copysign(fmin(az, arz), rz);
}

static void pow_fixed_axis(double f, double ro, double rz, double wo, double wz, double fexp, double oexp, double *oo,
                           double *zo)
{
    double scale = fmax(f, fmax(fabs(ro), fabs(rz)));
    if (!(scale > 0.0) || !isfinite(scale)) {
        pow_fixed_axis_unit(f, ro, rz, wo, wz, fexp, oexp, oo, zo);
        return;
    }
    double on, zn;
    pow_fixed_axis_unit(f / scale, ro / scale, rz / scale, wo, wz, fexp, oexp, &on, &zn);
    *oo = on * scale;
    *zo = zn * scale;
}

/* the section of the power cone through the fixed axes, in actual
 * coordinates with weights w (reference project_power_cone_point_with_fixed,
 * src/kernels/pdhcg_power_cone_kernels.cu:367-433; the all-free case is not
 * reached here) */
static void pow_section_point(double rx, double ry, double rz, double wx, double wy, double wz, double a, int fxx,
                              int fxy, int fxz, double *xo, double *yo, double *zo)
{
    double om = 1.0 - a;
    *xo = rx;
    *yo = ry;
    *zo = rz;
    if (fxz) {
        if (fxx && fxy) return;
        if (fxx) {
            double lower = fabs(rz) == 0.0 ? 0.0 : exp((log(fabs(rz)) - a * log(rx)) / om);
            *yo = fmax(ry, lower);
            return;
        }
        if (fxy) {
            double lower = fabs(rz) == 0.0 ? 0.0 : exp((log(fabs(rz)) - om * log(ry)) / a);
            *xo = fmax(rx, lower);
            return;
        }
        pow_xy_fixed_z(rx, ry, rz, wx, wy, a, xo, yo);
        return;
    }
    if (fxx && fxy) {
        double bound = 0.0;
        if (rx > 0.0 && ry > 0.0) {
            double lb = a * log(rx) + om * log(ry);
            bound = lb < log(DBL_MAX) ? exp(lb) : INFINITY;
        }
        *zo = fmax(-bound, fmin(rz, bound));
        return;
    }
    if (fxx) {
        pow_fixed_axis(rx, ry, rz, wy, wz, a, om, yo, zo);
        return;
    }
    pow_fixed_axis(ry, rx, rz, wx, wz, om, a, xo, zo);
}

static void pow_section(double *x, const double *d, const double *q, double tau, const char *fx, double alpha)
{
    double xo, yo, zo;
    pow_section_point(x[0] / d[0], x[1] / d[1], x[2] / d[2], weight_at(d, q, tau, 0), weight_at(d, q, tau, 1),
                      weight_at(d, q, tau, 2), alpha, fx[0] != 0, fx[1] != 0, fx[2] != 0, &xo, &yo, &zo);
    x[0] = xo * d[0];
    x[1] = yo * d[1];
    x[2] = zo * d[2];
}

/* ---------------- entry points ---------------- */

int oracle_block_has_fixed(const char *fx, int len)
{
    if (!fx) return 0;
    for (int i = 0; i < len; ++i)
        if (fx[i]) return 1;
    return 0;
}

void oracle_section_project(int type, int v_dim, double alpha, double *x, const double *d, const double *q,
                            double tau, const char *fx, double *warm)
{
    if (type == CONE_STANDARD_SOC) soc_section(v_dim, x, d, q, tau, fx, warm);
    else if (type == CONE_ROTATED_SOC) rsoc_section(v_dim, x, d, q, tau, fx, warm);
    else if (type == CONE_EXPONENTIAL) exp_section(x, d, q, tau, fx, warm);
    else if (type == CONE_POWER) pow_section(x, d, q, tau, fx, alpha);
}

/* Dual residual of a block with fixed slots (reference
 * compute_cone_dual_residual_*_kernel, their fixed-section branches:
 * src/kernels/pdhcg_soc_cone_kernels.cu:471-500,
 * src/kernels/pdhcg_rsoc_cone_kernels.cu:680-717,
 * src/kernels/pdhcg_exp_cone_kernels.cu:562-598,
 * src/kernels/pdhcg_power_cone_kernels.cu:485-604).  xp: the block's scaled
 * primal, rc: its reduced cost c + Qx - A^T y.  SOC / RSOC blocks with
 * v_dim >= 32 take the reference's block projector, whose dual residual is
 * zero (the projected-gradient term alone then measures the block).
 * Returns the block's complementarity residual (nonzero for power cones
 * only). */
double oracle_section_dual_residual(int type, int v_dim, double alpha, const double *xp, const double *rc,
                                    const double *d, const char *fx, double *warm, double *out)
{
    if (type == CONE_POWER) {
        const int f0 = fx[0] != 0, f1 = fx[1] != 0, f2 = fx[2] != 0;
        const double x = xp[0] / d[0], y = xp[1] / d[1], z = xp[2] / d[2];
        const double q[3] = {rc[0] * d[0], rc[1] * d[1], rc[2] * d[2]};
        const int fxa[3] = {f0, f1, f2};
        for (int i = 0; i < 3; ++i) out[i] = fxa[i] ? 0.0 : q[i];
        if (f0 && f1 && f2) return 0.0;
        double az = fabs(z), bound = 0.0;
        int regular = x > 0.0 && y > 0.0 && isfinite(x) && isfinite(y) && isfinite(z);
        if (regular) {
            bound = exp(alpha * log(x) + (1.0 - alpha) * log(y));
            regular = isfinite(bound) && bound > 0.0;
        }
        if (regular && az > 0.0) {
            /* remove the component of q along the boundary's outward normal
             * (free slots only), when q points into the cone */
            double nrm[3] = {-alpha * bound / x, -(1.0 - alpha) * bound / y, copysign(1.0, z)};
            double ns = 0.0;
            for (int i = 0; i < 3; ++i)
                if (!fxa[i]) ns = fmax(ns, fabs(nrm[i]));
            if (!(ns > 0.0) || !isfinite(ns)) regular = 0;
            if (regular) {
                double dot = 0.0, n2 = 0.0;
                for (int i = 0; i < 3; ++i) {
                    if (fxa[i]) continue;
                    double sn = nrm[i] / ns;
                    dot += q[i] * sn;
                    n2 += sn * sn;
                }
                double slam = (dot < 0.0 && n2 > 0.0) ? -dot / n2 : 0.0;
                double lam = slam / ns;
                for (int i = 0; i < 3; ++i)
                    if (!fxa[i]) out[i] = q[i] + slam * (nrm[i] / ns);
                double sscale = fmax(1.0, fmax(bound, az));
                return lam * (fmax(bound - az, 0.0) / sscale);
            }
        }
        if (regular) return 0.0;
        /* nonsmooth points: the projected mapping in the d^2 metric */
        double rx = x - (f0 ? 0.0 : rc[0] / d[0]);
        double ry = y - (f1 ? 0.0 : rc[1] / d[1]);
        double rz = z - (f2 ? 0.0 : rc[2] / d[2]);
        double xo, yo, zo;
        pow_section_point(rx, ry, rz, d[0] * d[0], d[1] * d[1], d[2] * d[2], alpha, f0, f1, f2, &xo, &yo, &zo);
        if (!f0) out[0] = (x - xo) * d[0] * d[0];
        if (!f1) out[1] = (y - yo) * d[1] * d[1];
        if (!f2) out[2] = (z - zo) * d[2] * d[2];
        return 0.0;
    }
    int len = (type == CONE_EXPONENTIAL) ? 3 : v_dim + 2;
    if ((type == CONE_STANDARD_SOC || type == CONE_ROTATED_SOC) && v_dim >= 32) {
        for (int i = 0; i < len; ++i) out[i] = 0.0;
        return 0.0;
    }
    double *p = (double *)malloc((size_t)len * sizeof(double));
    for (int i = 0; i < len; ++i) p[i] = fx[i] ? xp[i] : xp[i] - rc[i];
    oracle_section_project(type, v_dim, alpha, p, d, NULL, 0.0, fx, warm);
    for (int i = 0; i < len; ++i) out[i] = fx[i] ? 0.0 : (xp[i] - p[i]) * d[i];
    free(p);
    return 0.0;
}
