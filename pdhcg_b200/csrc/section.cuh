// section.cuh -- projections onto fixed cross-sections of cone blocks.
//
// set_cone_fixed (reference src/pdhcg.c:620-666) fixes single slots of a
// cone block.  The solve pins their scaled bounds, so the box step leaves
// the fixed value in place, and the block's free slots are then projected
// onto the slice of the cone through the fixed values, in the weighted
// metric sum_i omega_i (u_i - a_i)^2 with u = x / d, a = input / d and
// omega_i = max(w_i d_i^2, DBL_MIN), w = 1 + tau q (reference
// internal/cone_projection_utils.h:22-28).  The root finders, brackets and
// stopping rules are the reference's serial section projectors
// (src/kernels/pdhcg_soc_cone_kernels.cu:23-260,
// src/kernels/pdhcg_rsoc_cone_kernels.cu:23-465,
// src/kernels/pdhcg_exp_cone_kernels.cu:134-525,
// src/kernels/pdhcg_power_cone_kernels.cu:135-434).  Here the SOC and
// rotated SOC sections run on the whole warp: every multiplier trial is a
// warp-wide sum over the free slots, so a block of 256 slots costs eight
// fused multiply-adds per lane and five shuffles per trial.  The 3-slot
// exponential and power sections run on lane 0.
#pragma once

#include "device.cuh"

namespace pdhcg {

constexpr int SECTION_BISECT = 80;
constexpr double SECTION_TOL = 1e-13;

// fixed flags of this lane's slots: bit s <=> slot lane + 32 s
template <int S>
__device__ __forceinline__ unsigned section_bits(const unsigned char *fx, int st, int L, int lane)
{
    unsigned b = 0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        if (i < L && fx[st + i])
            b |= 1u << s;
    }
    return b;
}

__device__ __forceinline__ bool section_done(double lo, double hi) { return (hi - lo) <= SECTION_TOL * (1.0 + hi + lo); }

// warp sum over the free vector slots i < nv of (a omega / (omega + lam))^2
template <int S>
__device__ __forceinline__ double section_shrunk(const double (&a)[S], const double (&om)[S], unsigned fb, int nv,
                                                 int lane, double lam)
{
    double s2 = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        if (i < nv && !((fb >> s) & 1u)) {
            const double v = a[s] * om[s] / (om[s] + lam);
            s2 += v * v;
        }
    }
    return warp_sum(s2);
}

// Vector-slot statistics of a section: |fixed|^2, |free|^2, |omega a|^2 over
// the free slots, the largest free omega and the number of free slots.
template <int S>
__device__ __forceinline__ void section_stats(const double (&a)[S], const double (&om)[S], unsigned fb, int nv,
                                              int lane, double &fixed2, double &free2, double &polar2, double &max_om,
                                              int &nfree)
{
    double f2 = 0.0, g2 = 0.0, p2 = 0.0, mo = 0.0;
    int nf = 0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        if (i < nv) {
            if ((fb >> s) & 1u) {
                f2 += a[s] * a[s];
            } else {
                g2 += a[s] * a[s];
                p2 += (om[s] * a[s]) * (om[s] * a[s]);
                mo = fmax(mo, om[s]);
                ++nf;
            }
        }
    }
    fixed2 = warp_sum(f2);
    free2 = warp_sum(g2);
    polar2 = warp_sum(p2);
    max_om = warp_max(mo);
    nfree = (int)warp_sum((double)nf);
}

// multiplier of the ball |u_free|^2 <= r2 (reference
// src/kernels/pdhcg_soc_cone_kernels.cu:57-118)
template <int S>
__device__ double section_ball(const double (&a)[S], const double (&om)[S], unsigned fb, int nv, int lane,
                               double polar2, double r2, double warm0)
{
    double lo = 0.0, hi = sqrt(polar2) / sqrt(r2) * (1.0 + 64.0 * DBL_EPSILON);
    if (!(hi > 0.0) || !isfinite(hi)) {
        hi = warm0 > 0.0 && isfinite(warm0) ? warm0 : 1.0;
        for (int e = 0; e < 100; ++e) {
            if (section_shrunk<S>(a, om, fb, nv, lane, hi) <= r2)
                break;
            hi *= 2.0;
        }
    }
    for (int it = 0; it < SECTION_BISECT; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (section_shrunk<S>(a, om, fb, nv, lane, mid) > r2)
            lo = mid;
        else
            hi = mid;
        if (section_done(lo, hi))
            break;
    }
    return 0.5 * (lo + hi);
}

__device__ __forceinline__ double section_soc_negative_upper(double sing, double endpoint_polar, double fixed2,
                                                             double polar2, double max_om)
{
    double up;
    if (fixed2 > 0.0) {
        up = sing + endpoint_polar / sqrt(fixed2);
    } else {
        const double pn = sqrt(polar2), gap = pn - endpoint_polar;
        if (!(gap > 0.0))
            return NAN;
        up = (pn / gap) * sing + (endpoint_polar / gap) * max_om;
    }
    return up * (1.0 + 64.0 * DBL_EPSILON);
}

// value of slot `slot` of the block, broadcast from its lane
template <int S>
__device__ __forceinline__ double slot_value(const double (&v)[S], int slot)
{
    double r = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (s == (slot >> 5))
            r = v[s];
    return __shfl_sync(FULL, r, slot & 31);
}

template <int S>
__device__ __forceinline__ bool slot_fixed(unsigned fb, int slot)
{
    const unsigned b = __shfl_sync(FULL, fb, slot & 31);
    return (b >> (slot >> 5)) & 1u;
}

template <int S>
__device__ __forceinline__ void section_scale_free(WarpSlots<S> &sl, const double (&om)[S], unsigned fb, int nv,
                                                   int lane, double lam, bool zero)
{
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        if (i < nv && !((fb >> s) & 1u))
            sl.x[s] = zero ? 0.0 : sl.x[s] * (om[s] / (om[s] + lam));
    }
}

template <int S>
__device__ __forceinline__ void section_set_slot(WarpSlots<S> &sl, int slot, int lane, double v)
{
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (lane + 32 * s == slot)
            sl.x[s] = v;
}

// Standard SOC [v(k), w, z], L = k + 2: u = slots 0..L-2, z = slot L-1.
template <int S>
__device__ void warp_section_soc(WarpSlots<S> &sl, int L, int lane, unsigned fb, double *warm)
{
    const int nv = L - 1, zi = L - 1;
    const double warm0 = warm ? *warm : 0.0;
    double a[S], om[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        a[s] = sl.x[s] / sl.d[s];
        om[s] = fmax(sl.w[s] * sl.d[s] * sl.d[s], DBL_MIN);
    }
    double fixed2, free2, polar2, max_om;
    int nfree;
    section_stats<S>(a, om, fb, nv, lane, fixed2, free2, polar2, max_om, nfree);
    const double az = slot_value<S>(a, zi), omz = slot_value<S>(om, zi), dz = slot_value<S>(sl.d, zi);
    double lam;
    if (slot_fixed<S>(fb, zi)) {
        const double r2 = fmax(0.0, az * az - fixed2);
        if (nfree == 0 || free2 <= r2)
            return;
        if (!(r2 > 0.0)) {
            section_scale_free<S>(sl, om, fb, nv, lane, 0.0, true);
            return;
        }
        lam = section_ball<S>(a, om, fb, nv, lane, polar2, r2, warm0);
        if (warm && lane == 0)
            *warm = lam;
        section_scale_free<S>(sl, om, fb, nv, lane, lam, false);
        return;
    }
    if (az >= 0.0 && fixed2 + free2 <= az * az)
        return;
    if (nfree == 0) {
        section_set_slot<S>(sl, zi, lane, fmax(az, sqrt(fixed2)) * dz);
        return;
    }
    if (fixed2 == 0.0 && -omz * az >= sqrt(polar2)) {
        section_scale_free<S>(sl, om, fb, nv, lane, 0.0, true);
        section_set_slot<S>(sl, zi, lane, 0.0);
        return;
    }
    double zval;
    if (az == 0.0) {
        lam = omz;
        zval = sqrt(fixed2 + section_shrunk<S>(a, om, fb, nv, lane, lam)) * dz;
    } else {
        const bool lower = az > 0.0;
        double lo, hi;
        if (lower) {
            lo = 0.0;
            hi = omz * (1.0 - 1e-14);
        } else {
            lo = omz * (1.0 + 1e-14);
            hi = section_soc_negative_upper(omz, -omz * az, fixed2, polar2, max_om);
            if (!(hi > lo) || !isfinite(hi)) {
                hi = 2.0 * omz;
                for (int e = 0; e < 100; ++e) {
                    const double z = omz * az / (omz - hi);
                    if (fixed2 + section_shrunk<S>(a, om, fb, nv, lane, hi) >= z * z)
                        break;
                    hi *= 2.0;
                }
            }
        }
        if (warm && warm0 > lo && warm0 < hi && isfinite(warm0)) {
            const double z = omz * az / (omz - warm0);
            const double f = fixed2 + section_shrunk<S>(a, om, fb, nv, lane, warm0) - z * z;
            if ((lower && f > 0.0) || (!lower && f < 0.0))
                lo = warm0;
            else
                hi = warm0;
        }
        for (int it = 0; it < SECTION_BISECT; ++it) {
            const double mid = 0.5 * (lo + hi);
            const double z = omz * az / (omz - mid);
            const double f = fixed2 + section_shrunk<S>(a, om, fb, nv, lane, mid) - z * z;
            if ((lower && f > 0.0) || (!lower && f < 0.0))
                lo = mid;
            else
                hi = mid;
            if (section_done(lo, hi))
                break;
        }
        lam = 0.5 * (lo + hi);
        zval = slot_value<S>(sl.x, zi) * (omz / (omz - lam));
    }
    if (warm && lane == 0)
        *warm = lam;
    section_scale_free<S>(sl, om, fb, nv, lane, lam, false);
    section_set_slot<S>(sl, zi, lane, zval);
}

// Rotated SOC [v(k), s, t], L = k + 2: |v|^2 <= 2 s t, s, t >= 0.
template <int S>
__device__ void warp_section_rsoc(WarpSlots<S> &sl, int L, int lane, unsigned fb, double *warm)
{
    const int nv = L - 2, si = L - 2, ti = L - 1;
    const double warm0 = warm ? *warm : 0.0;
    double a[S], om[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        a[s] = sl.x[s] / sl.d[s];
        om[s] = fmax(sl.w[s] * sl.d[s] * sl.d[s], DBL_MIN);
    }
    double fixed2, free2, polar2, max_om;
    int nfree;
    section_stats<S>(a, om, fb, nv, lane, fixed2, free2, polar2, max_om, nfree);
    const double as = slot_value<S>(a, si), at = slot_value<S>(a, ti);
    const double oms = slot_value<S>(om, si), omt = slot_value<S>(om, ti);
    const double ds = slot_value<S>(sl.d, si), dt = slot_value<S>(sl.d, ti);
    const bool fs = slot_fixed<S>(fb, si), ft = slot_fixed<S>(fb, ti);
    if (fs && ft) {
        const double r2 = fmax(0.0, 2.0 * as * at - fixed2);
        if (nfree == 0 || free2 <= r2)
            return;
        if (!(r2 > 0.0)) {
            section_scale_free<S>(sl, om, fb, nv, lane, 0.0, true);
            return;
        }
        const double lam = section_ball<S>(a, om, fb, nv, lane, polar2, r2, warm0);
        if (warm && lane == 0)
            *warm = lam;
        section_scale_free<S>(sl, om, fb, nv, lane, lam, false);
        return;
    }
    if (fs || ft) {
        // one endpoint e fixed; the other endpoint f is free
        const int fi = fs ? ti : si;
        const double e = fs ? as : at, af = fs ? at : as, omf = fs ? omt : oms, df = fs ? dt : ds;
        if (!(e > 0.0)) {
            section_scale_free<S>(sl, om, fb, nv, lane, 0.0, true);
            section_set_slot<S>(sl, fi, lane, fmax(af, 0.0) * df);
            return;
        }
        if (af >= 0.0 && fixed2 + free2 <= 2.0 * e * af)
            return;
        if (nfree == 0) {
            section_set_slot<S>(sl, fi, lane, fmax(af, fixed2 / (2.0 * e)) * df);
            return;
        }
        double lo = 0.0;
        const double viol = fixed2 + free2 - 2.0 * e * af;
        double hi = omf * viol / (2.0 * e * e) * (1.0 + 64.0 * DBL_EPSILON);
        if (!(hi > 0.0) || !isfinite(hi)) {
            hi = warm0 > 0.0 && isfinite(warm0) ? warm0 : omf;
            for (int it = 0; it < 100; ++it) {
                const double f = af + hi * e / omf;
                if (fixed2 + section_shrunk<S>(a, om, fb, nv, lane, hi) <= 2.0 * e * f)
                    break;
                hi *= 2.0;
            }
        }
        for (int it = 0; it < SECTION_BISECT; ++it) {
            const double mid = 0.5 * (lo + hi);
            const double f = af + mid * e / omf;
            if (fixed2 + section_shrunk<S>(a, om, fb, nv, lane, mid) > 2.0 * e * f)
                lo = mid;
            else
                hi = mid;
            if (section_done(lo, hi))
                break;
        }
        const double lam = 0.5 * (lo + hi);
        if (warm && lane == 0)
            *warm = lam;
        section_scale_free<S>(sl, om, fb, nv, lane, lam, false);
        section_set_slot<S>(sl, fi, lane, (af + lam * e / omf) * df);
        return;
    }
    if (as >= 0.0 && at >= 0.0 && fixed2 + free2 <= 2.0 * as * at)
        return;
    if (fixed2 == 0.0) {
        const double bs = oms * as, bt = omt * at;
        if (bs <= 0.0 && bt <= 0.0 && polar2 <= 2.0 * bs * bt) {
            section_scale_free<S>(sl, om, fb, nv, lane, 0.0, true);
            section_set_slot<S>(sl, si, lane, 0.0);
            section_set_slot<S>(sl, ti, lane, 0.0);
            return;
        }
    }
    const double root = sqrt(oms) * sqrt(omt);
    const double balance = sqrt(oms) * as + sqrt(omt) * at;
    const double bscale = 1.0 + fabs(sqrt(oms) * as) + fabs(sqrt(omt) * at);
    double lam = root, ps = 0.0, pt = 0.0;
    bool smooth = true;
    if (fabs(balance) <= 64.0 * DBL_EPSILON * bscale) {
        const double n2 = fixed2 + section_shrunk<S>(a, om, fb, nv, lane, lam);
        const double prod = 0.5 * root * n2;
        const double delta = sqrt(oms) * as;
        const double stt = 0.5 * (-delta + sqrt(fmax(0.0, delta * delta + 4.0 * prod)));
        const double sss = stt + delta;
        ps = sss / sqrt(oms);
        pt = stt / sqrt(omt);
        smooth = ps >= 0.0 && pt >= 0.0;
    } else {
        const bool lower = balance > 0.0;
        double lo = lower ? 0.0 : root * (1.0 + 1e-14);
        double hi = lower ? root * (1.0 - 1e-14) : 2.0 * root;
        if (!lower) {
            // the rotated cone in sum / difference endpoint coordinates is a
            // standard one (reference src/kernels/pdhcg_rsoc_cone_kernels.cu:23-45)
            const double r2 = 0.70710678118654752440;
            const double ws = sqrt(oms) * as, wt = sqrt(omt) * at;
            const double tw = (ws - wt) * r2;
            hi = root * section_soc_negative_upper(1.0, -(ws + wt) * r2, root * fixed2, polar2 / root + tw * tw,
                                                   fmax(1.0, max_om / root));
            if (!(hi > lo) || !isfinite(hi)) {
                hi = 2.0 * root;
                for (int e = 0; e < 100; ++e) {
                    const double det = oms * omt - hi * hi;
                    const double s = omt * (oms * as + hi * at) / det;
                    const double t = oms * (omt * at + hi * as) / det;
                    double f = INFINITY;
                    if (s >= 0.0 && t >= 0.0)
                        f = fixed2 + section_shrunk<S>(a, om, fb, nv, lane, hi) - 2.0 * s * t;
                    if (f >= 0.0)
                        break;
                    hi *= 2.0;
                }
            }
        }
        for (int it = 0; it < 90; ++it) {
            const double mid = 0.5 * (lo + hi);
            const double det = oms * omt - mid * mid;
            const double s = omt * (oms * as + mid * at) / det;
            const double t = oms * (omt * at + mid * as) / det;
            // the shrunk sum is a warp-wide reduction: every lane takes it
            const double n2 = section_shrunk<S>(a, om, fb, nv, lane, mid);
            double f = INFINITY;
            if (s >= 0.0 && t >= 0.0)
                f = fixed2 + n2 - 2.0 * s * t;
            if ((lower && f > 0.0) || (!lower && f < 0.0))
                lo = mid;
            else
                hi = mid;
            if (section_done(lo, hi))
                break;
        }
        lam = 0.5 * (lo + hi);
        const double det = oms * omt - lam * lam;
        ps = omt * (oms * as + lam * at) / det;
        pt = oms * (omt * at + lam * as) / det;
        smooth = isfinite(ps) && isfinite(pt) && ps >= 0.0 && pt >= 0.0;
    }
    // with no fixed vector slots the axes {u = 0, t = 0} and {u = 0, s = 0}
    // are candidates too: keep the nearest (reference
    // src/kernels/pdhcg_rsoc_cone_kernels.cu:410-445)
    double best = INFINITY;
    {
        double obj = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int i = lane + 32 * s;
            if (i < nv && !((fb >> s) & 1u)) {
                const double v = a[s] * om[s] / (om[s] + lam), dv = v - a[s];
                obj += om[s] * dv * dv;
            }
        }
        obj = warp_sum(obj);
        if (smooth)
            best = obj + oms * (ps - as) * (ps - as) + omt * (pt - at) * (pt - at);
    }
    bool on_axis = !smooth;
    if (fixed2 == 0.0) {
        double vec = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int i = lane + 32 * s;
            if (i < nv && !((fb >> s) & 1u))
                vec += om[s] * a[s] * a[s];
        }
        vec = warp_sum(vec);
        const double sa = fmax(as, 0.0);
        const double sobj = vec + oms * (sa - as) * (sa - as) + omt * at * at;
        if (sobj < best) {
            best = sobj;
            ps = sa;
            pt = 0.0;
            on_axis = true;
        }
        const double ta = fmax(at, 0.0);
        const double tobj = vec + oms * as * as + omt * (ta - at) * (ta - at);
        if (tobj < best) {
            ps = 0.0;
            pt = ta;
            on_axis = true;
        }
    }
    if (warm && lane == 0)
        *warm = on_axis ? 0.0 : lam;
    section_scale_free<S>(sl, om, fb, nv, lane, lam, on_axis);
    section_set_slot<S>(sl, si, lane, ps * ds);
    section_set_slot<S>(sl, ti, lane, pt * dt);
}

// ---------------- exponential and power sections (one thread) ----------------

__device__ __forceinline__ double sec_exp_boundary(double x, double y)
{
    if (!(y > 0.0))
        return x <= 0.0 ? 0.0 : INFINITY;
    const double lv = log(y) + x / y;
    if (lv >= log(DBL_MAX))
        return INFINITY;
    if (lv <= log(DBL_MIN))
        return 0.0;
    return exp(lv);
}

__device__ __forceinline__ bool sec_exp_contains(double x, double y, double z)
{
    if (y > 0.0 && z > 0.0) {
        const double lhs = log(y) + x / y, rhs = log(z);
        return lhs <= rhs + 64.0 * DBL_EPSILON * (1.0 + fabs(lhs) + fabs(rhs));
    }
    return y == 0.0 && x <= 0.0 && z >= 0.0;
}

__device__ __forceinline__ double sec_exp_log_violation(double y, double x, double z)
{
    if (!(y > 0.0) || !(z > 0.0))
        return x <= 0.0 ? -INFINITY : INFINITY;
    return log(y) + x / y - log(z);
}

// distance^2 of the boundary point over y, with x fixed (kind 0: (y, z)
// free) or z fixed (kind 1: (x, y) free)
__device__ __forceinline__ double sec_exp_obj(int kind, double y, double p0, double ia, double ib, double wa,
                                              double wb)
{
    if (kind == 0) { // p0 = x; ia = y input, ib = z input; wa = wy, wb = wz
        const double z = sec_exp_boundary(p0, y);
        if (!isfinite(z))
            return INFINITY;
        return wa * (y - ia) * (y - ia) + wb * (z - ib) * (z - ib);
    }
    // p0 = z; ia = x input, ib = y input; wa = wx, wb = wy
    const double x = y > 0.0 ? y * (log(p0) - log(y)) : 0.0;
    return wa * (x - ia) * (x - ia) + wb * (y - ib) * (y - ib);
}

// golden-section minimum over y in [lo, hi] after doubling hi while the
// objective falls (reference src/kernels/pdhcg_exp_cone_kernels.cu:422-456)
__device__ double sec_exp_golden(int kind, double lo, double hi, double p0, double ia, double ib, double wa, double wb)
{
    double prev = sec_exp_obj(kind, 0.5 * hi, p0, ia, ib, wa, wb);
    double cur = sec_exp_obj(kind, hi, p0, ia, ib, wa, wb);
    for (int e = 0; e < 80 && cur < prev && hi < DBL_MAX / 4.0; ++e) {
        prev = cur;
        hi *= 2.0;
        cur = sec_exp_obj(kind, hi, p0, ia, ib, wa, wb);
    }
    const double r = 0.6180339887498948482;
    double a = lo, b = hi, c = b - r * (b - a), d = a + r * (b - a);
    double fc = sec_exp_obj(kind, c, p0, ia, ib, wa, wb), fd = sec_exp_obj(kind, d, p0, ia, ib, wa, wb);
    for (int it = 0; it < 100; ++it) {
        if (fc <= fd) {
            b = d;
            d = c;
            fd = fc;
            c = b - r * (b - a);
            fc = sec_exp_obj(kind, c, p0, ia, ib, wa, wb);
        } else {
            a = c;
            c = d;
            fc = fd;
            d = a + r * (b - a);
            fd = sec_exp_obj(kind, d, p0, ia, ib, wa, wb);
        }
    }
    return 0.5 * (a + b);
}

// (x, z) with y > 0 fixed: safeguarded Newton in u (reference
// project_2d_exp_persp, src/kernels/pdhcg_exp_cone_kernels.cu:134-231)
__device__ void sec_exp_fixed_y(double rz0, double ry, double rt0, double d_r, double d_y, double d_t, double *warm,
                                double &rzo, double &rto)
{
    rzo = rz0;
    rto = rt0;
    if (d_r <= 0.0 || d_y <= 0.0 || d_t <= 0.0)
        return;
    const double ye = ry / d_y;
    if (ye <= 0.0) {
        rzo = rz0 < 0.0 ? rz0 : 0.0;
        rto = rt0 > 0.0 ? rt0 : 0.0;
        return;
    }
    const double arg = (rz0 / d_r) / ye;
    if (arg < 700.0 && ye * d_t * exp(arg) <= rt0)
        return;
    const double A = d_t * d_t * ye, B = d_t * rt0, Cc = d_r * d_r * ye, E = d_r * rz0;
    double u = warm ? *warm : 0.0, ulo = 1e-30, uhi = 1.0;
    for (int g = 0; g < 200; ++g) {
        const double f = A * uhi * uhi - B * uhi + Cc * log(uhi) - E;
        if (isfinite(f) && f > 0.0)
            break;
        uhi *= 4.0;
        if (uhi > 1e150)
            break;
    }
    for (int g = 0; g < 200; ++g) {
        const double f = A * ulo * ulo - B * ulo + Cc * log(ulo) - E;
        if (isfinite(f) && f < 0.0)
            break;
        ulo *= 0.25;
        if (ulo < 1e-300)
            break;
    }
    if (ulo >= uhi)
        return;
    if (!(u > ulo && u < uhi) || !isfinite(u))
        u = exp(0.5 * (log(ulo) + log(uhi)));
    for (int it = 0; it < 80; ++it) {
        const double f = A * u * u - B * u + Cc * log(u) - E;
        const double df = 2.0 * A * u - B + Cc / u;
        if (f > 0.0)
            uhi = u;
        else
            ulo = u;
        double un;
        if (df > 1e-300 && isfinite(df) && isfinite(f)) {
            un = u - f / df;
            if (!isfinite(un) || un <= ulo || un >= uhi)
                un = exp(0.5 * (log(ulo) + log(uhi)));
        } else {
            un = exp(0.5 * (log(ulo) + log(uhi)));
        }
        if (fabs(un - u) < 1e-14 * (1.0 + fabs(un))) {
            u = un;
            break;
        }
        u = un;
    }
    if (warm)
        *warm = u;
    rzo = d_r * ye * log(u);
    rto = d_t * ye * u;
}

// exponential section in actual coordinates i (weights w); fixed slots keep
// their inputs (reference project_exp_cone_section,
// src/kernels/pdhcg_exp_cone_kernels.cu:285-524)
__device__ __noinline__ void sec_exp_point(const double *i3, const double *w3, const bool *f3, double *warm,
                                           double *o3)
{
    const double ix = i3[0], iy = i3[1], iz = i3[2];
    const double wx = w3[0], wy = w3[1], wz = w3[2];
    const bool fxx = f3[0], fxy = f3[1], fxz = f3[2];
    double ox = ix, oy = iy, oz = iz;
    if (!(sec_exp_contains(ix, iy, iz) || (fxx && fxy && fxz))) {
        if (fxx && fxy) {
            oz = fmax(iz, sec_exp_boundary(ix, iy));
        } else if (fxy && fxz) {
            ox = iy == 0.0 ? fmin(ix, 0.0) : fmin(ix, iy * (log(iz) - log(iy)));
        } else if (fxx && fxz) {
            if (iz == 0.0) {
                oy = 0.0;
            } else if (ix > 0.0) {
                const double center = ix;
                double left = fmax(DBL_MIN, ix / 1024.0);
                while (sec_exp_log_violation(left, ix, iz) <= 0.0 && left > DBL_MIN)
                    left *= 0.5;
                double lo = left, hi = center;
                for (int it = 0; it < 100; ++it) {
                    const double mid = 0.5 * (lo + hi);
                    if (sec_exp_log_violation(mid, ix, iz) > 0.0)
                        lo = mid;
                    else
                        hi = mid;
                }
                const double lower = 0.5 * (lo + hi);
                lo = center;
                hi = fmax(2.0 * center, iz);
                while (sec_exp_log_violation(hi, ix, iz) < 0.0 && hi < DBL_MAX / 4.0)
                    hi *= 2.0;
                for (int it = 0; it < 100; ++it) {
                    const double mid = 0.5 * (lo + hi);
                    if (sec_exp_log_violation(mid, ix, iz) <= 0.0)
                        lo = mid;
                    else
                        hi = mid;
                }
                oy = fmin(fmax(iy, lower), 0.5 * (lo + hi));
            } else {
                double lo = 0.0, hi = fmax(1.0, fmax(iz, fabs(ix)));
                while (sec_exp_log_violation(hi, ix, iz) < 0.0 && hi < DBL_MAX / 4.0)
                    hi *= 2.0;
                for (int it = 0; it < 100; ++it) {
                    const double mid = 0.5 * (lo + hi);
                    if (sec_exp_log_violation(mid, ix, iz) <= 0.0)
                        lo = mid;
                    else
                        hi = mid;
                }
                oy = fmin(fmax(iy, 0.0), 0.5 * (lo + hi));
            }
        } else if (fxy) {
            if (!(iy > 0.0)) {
                ox = fmin(ix, 0.0);
                oz = fmax(iz, 0.0);
            } else {
                const double ex = sqrt(wx), ey = sqrt(wy), ez = sqrt(wz);
                double sx, sz;
                sec_exp_fixed_y(ex * ix, ey * iy, ez * iz, ex, ey, ez, warm, sx, sz);
                ox = sx / ex;
                oz = sz / ez;
            }
        } else if (fxx) {
            const double scale = 1.0 + fabs(ix) + fabs(iy) + fabs(iz);
            const double lo = ix > 0.0 ? fmax(DBL_MIN, ix / 700.0) : 0.0;
            oy = sec_exp_golden(0, lo, scale, ix, iy, iz, wy, wz);
            oz = sec_exp_boundary(ix, oy);
            if (ix <= 0.0) {
                const double cz = fmax(iz, 0.0);
                const double closure = wy * iy * iy + wz * (cz - iz) * (cz - iz);
                if (closure <= sec_exp_obj(0, oy, ix, iy, iz, wy, wz)) {
                    oy = 0.0;
                    oz = cz;
                }
            }
        } else if (fxz) {
            if (iz == 0.0) {
                ox = fmin(ix, 0.0);
                oy = 0.0;
            } else {
                const double scale = 1.0 + fabs(ix) + fabs(iy) + iz;
                oy = sec_exp_golden(1, 0.0, scale, iz, ix, iy, wx, wy);
                ox = oy > 0.0 ? oy * (log(iz) - log(oy)) : 0.0;
                const double cx = fmin(ix, 0.0);
                const double closure = wx * (cx - ix) * (cx - ix) + wy * iy * iy;
                if (closure <= sec_exp_obj(1, oy, iz, ix, iy, wx, wy)) {
                    ox = cx;
                    oy = 0.0;
                }
            }
        }
    }
    o3[0] = fxx ? ix : ox;
    o3[1] = fxy ? iy : oy;
    o3[2] = fxz ? iz : oz;
}

__device__ __forceinline__ double sec_pos_root(double r, double qv)
{
    if (!(qv > 0.0))
        return fmax(r, 0.0);
    const double disc = hypot(r, 2.0 * sqrt(qv));
    return r >= 0.0 ? 0.5 * (r + disc) : (2.0 * qv) / (disc - r);
}

__device__ __forceinline__ double sec_pow_xy_log_boundary(double lam, double rx, double ry, double wx, double wy,
                                                          double a)
{
    const double x = sec_pos_root(rx, (lam / wx) * a);
    const double y = sec_pos_root(ry, (lam / wy) * (1.0 - a));
    if (!(x > 0.0) || !(y > 0.0))
        return -INFINITY;
    return a * log(x) + (1.0 - a) * log(y);
}

// (x, y) with z fixed (reference project_power_xy_fixed_z[_normalized],
// src/kernels/pdhcg_power_cone_kernels.cu:146-234)
__device__ void sec_pow_xy_fixed_z(double rx, double ry, double fz, double wx, double wy, double a, double &xo,
                                   double &yo)
{
    double scale = fmax(fabs(rx), fmax(fabs(ry), fabs(fz)));
    if (!(scale > 0.0) || !isfinite(scale))
        scale = 1.0;
    rx /= scale;
    ry /= scale;
    fz /= scale;
    const double c = fabs(fz), om = 1.0 - a;
    if (c == 0.0) {
        xo = fmax(rx, 0.0) * scale;
        yo = fmax(ry, 0.0) * scale;
        return;
    }
    if (rx > 0.0 && ry > 0.0 && a * log(rx) + om * log(ry) >= log(c)) {
        xo = rx * scale;
        yo = ry * scale;
        return;
    }
    const double target = log(c);
    double hi = fmin(wx, wy);
    if (!(hi > 0.0) || !isfinite(hi))
        hi = 1.0;
    for (int it = 0; it < 2048; ++it) {
        const double lb = sec_pow_xy_log_boundary(hi, rx, ry, wx, wy, a);
        if (lb >= target || isnan(lb))
            break;
        if (hi >= 0.5 * DBL_MAX) {
            hi = DBL_MAX;
            break;
        }
        hi *= 2.0;
    }
    double lam;
    if (sec_pow_xy_log_boundary(DBL_MIN, rx, ry, wx, wy, a) >= target) {
        double lo = 0.0, fh = DBL_MIN;
        for (int it = 0; it < 80; ++it) {
            const double cnd = lo + 0.5 * (fh - lo);
            if (sec_pow_xy_log_boundary(cnd, rx, ry, wx, wy, a) < target)
                lo = cnd;
            else
                fh = cnd;
        }
        lam = lo + 0.5 * (fh - lo);
    } else {
        double llo = log(DBL_MIN), lhi = log(hi);
        for (int it = 0; it < 96; ++it) {
            const double ll = llo + 0.5 * (lhi - llo);
            if (sec_pow_xy_log_boundary(exp(ll), rx, ry, wx, wy, a) < target)
                llo = ll;
            else
                lhi = ll;
        }
        lam = exp(llo + 0.5 * (lhi - llo));
    }
    xo = sec_pos_root(rx, (lam / wx) * a) * scale;
    yo = sec_pos_root(ry, (lam / wy) * om) * scale;
}

__device__ __forceinline__ double sec_pow_exp_of_log(double lv)
{
    if (lv >= log(DBL_MAX))
        return INFINITY;
    if (lv <= log(DBL_MIN))
        return 0.0;
    return exp(lv);
}

__device__ __forceinline__ double sec_pow_derivative(double o, double ro, double arz, double wo, double wz,
                                                     double lcoef, double oexp)
{
    if (!(o > 0.0))
        return -INFINITY;
    const double lo = log(o);
    const double bound = sec_pow_exp_of_log(lcoef + oexp * lo);
    const double slope = sec_pow_exp_of_log(lcoef + log(oexp) + (oexp - 1.0) * lo);
    const double lin = wo * (o - ro);
    const double gap = bound - arz;
    if (gap == 0.0 || slope == 0.0)
        return lin;
    if (!isfinite(slope))
        return copysign(INFINITY, gap);
    return lin + wz * gap * slope;
}

// one axis fixed at f: (other, z) onto |z| <= f^fexp other^oexp
// (reference project_power_section_fixed_axis[_normalized],
// src/kernels/pdhcg_power_cone_kernels.cu:263-365)
__device__ void sec_pow_fixed_axis(double f, double ro, double rz, double wo, double wz, double fexp, double oexp,
                                   double &oo, double &zo)
{
    double scale = fmax(f, fmax(fabs(ro), fabs(rz)));
    if (!(scale > 0.0) || !isfinite(scale))
        scale = 1.0;
    f /= scale;
    ro /= scale;
    rz /= scale;
    const double arz = fabs(rz);
    if (!(f > 0.0) || arz == 0.0) {
        oo = fmax(ro, 0.0) * scale;
        zo = 0.0;
        return;
    }
    const double lcoef = fexp * log(f);
    if (ro > 0.0 && lcoef + oexp * log(ro) >= log(arz)) {
        oo = ro * scale;
        zo = rz * scale;
        return;
    }
    const double feas = sec_pow_exp_of_log((log(arz) - lcoef) / oexp);
    if (feas == 0.0) {
        oo = 0.0;
        zo = 0.0;
        return;
    }
    double lo = 0.0, hi = fmax(1.0, fmax(ro, 0.0));
    if (isfinite(feas))
        hi = fmin(hi, feas);
    for (int it = 0; it < 1024; ++it) {
        if (!(sec_pow_derivative(hi, ro, arz, wo, wz, lcoef, oexp) < 0.0))
            break;
        if (isfinite(feas) && hi >= feas)
            break;
        const double nh = hi * 2.0;
        if (!isfinite(nh)) {
            hi = isfinite(feas) ? feas : DBL_MAX;
            break;
        }
        hi = isfinite(feas) ? fmin(nh, feas) : nh;
    }
    for (int it = 0; it < 80; ++it) {
        const double o = lo + 0.5 * (hi - lo);
        if (o == 0.0)
            break;
        if (sec_pow_derivative(o, ro, arz, wo, wz, lcoef, oexp) < 0.0)
            lo = o;
        else
            hi = o;
    }
    const double o = lo + 0.5 * (hi - lo);
    const double az = o > 0.0 ? sec_pow_exp_of_log(lcoef + oexp * log(o)) : 0.0;
    oo = o * scale;
    zo = copysign(fmin(az, arz), rz) * scale;
}

// power section in actual coordinates (reference
// project_power_cone_point_with_fixed, src/kernels/pdhcg_power_cone_kernels.cu:367-433;
// at least one slot is fixed here)
__device__ __noinline__ void sec_pow_point(const double *i3, const double *w3, const bool *f3, double a, double *o3)
{
    const double rx = i3[0], ry = i3[1], rz = i3[2], om = 1.0 - a;
    double xo = rx, yo = ry, zo = rz;
    if (f3[2]) {
        if (f3[0] && f3[1]) {
        } else if (f3[0]) {
            const double lower = fabs(rz) == 0.0 ? 0.0 : exp((log(fabs(rz)) - a * log(rx)) / om);
            yo = fmax(ry, lower);
        } else if (f3[1]) {
            const double lower = fabs(rz) == 0.0 ? 0.0 : exp((log(fabs(rz)) - om * log(ry)) / a);
            xo = fmax(rx, lower);
        } else {
            sec_pow_xy_fixed_z(rx, ry, rz, w3[0], w3[1], a, xo, yo);
        }
    } else if (f3[0] && f3[1]) {
        double bound = 0.0;
        if (rx > 0.0 && ry > 0.0) {
            const double lb = a * log(rx) + om * log(ry);
            bound = lb < log(DBL_MAX) ? exp(lb) : INFINITY;
        }
        zo = fmax(-bound, fmin(rz, bound));
    } else if (f3[0]) {
        sec_pow_fixed_axis(rx, ry, rz, w3[1], w3[2], a, om, yo, zo);
    } else {
        sec_pow_fixed_axis(ry, rx, rz, w3[0], w3[2], om, a, xo, zo);
    }
    o3[0] = xo;
    o3[1] = yo;
    o3[2] = zo;
}

// 3-slot section on lane 0 (slot i sits on lane i, s = 0)
template <int S>
__device__ void warp_section3(int type, WarpSlots<S> &sl, int lane, unsigned fb, double alpha, double *warm)
{
    double i3[3], w3[3], d3[3];
    bool f3[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double x = __shfl_sync(FULL, sl.x[0], k), d = __shfl_sync(FULL, sl.d[0], k),
                     w = __shfl_sync(FULL, sl.w[0], k);
        f3[k] = (__shfl_sync(FULL, fb, k) & 1u) != 0;
        i3[k] = x / d;
        d3[k] = d;
        w3[k] = fmax(w * d * d, DBL_MIN);
    }
    double o3[3] = {i3[0], i3[1], i3[2]};
    if (lane == 0) {
        if (type == 2)
            sec_exp_point(i3, w3, f3, warm, o3);
        else
            sec_pow_point(i3, w3, f3, alpha, o3);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double v = __shfl_sync(FULL, o3[k], 0) * d3[k];
        if (lane == k && !f3[k])
            sl.x[0] = v;
    }
}

// Projection of a block with fixed slots (fb: this lane's fixed bits).
template <int S>
__device__ __forceinline__ void warp_section_project(int type, WarpSlots<S> &sl, int L, int lane, unsigned fb,
                                                     double *warm, double alpha)
{
    if (type == 1) // CONE_STANDARD_SOC
        warp_section_soc<S>(sl, L, lane, fb, warm);
    else if (type == 0) // CONE_ROTATED_SOC
        warp_section_rsoc<S>(sl, L, lane, fb, warm);
    else if (type == 2 || type == 3) // CONE_EXPONENTIAL, CONE_POWER
        warp_section3<S>(type, sl, lane, fb, alpha, warm);
}

// Dual residual of a block with fixed slots (reference
// compute_cone_dual_residual_*_kernel, fixed-section branches,
// src/kernels/pdhcg_soc_cone_kernels.cu:471-500,
// src/kernels/pdhcg_rsoc_cone_kernels.cu:680-717,
// src/kernels/pdhcg_exp_cone_kernels.cu:562-598,
// src/kernels/pdhcg_power_cone_kernels.cu:485-604).  xv: the block's
// scaled primal, rc its reduced cost, vr its rescaling.  Writes the
// residual of each slot to out and returns the complementarity residual
// (nonzero on power blocks only), warp-uniform.  SOC / rotated SOC blocks
// of 32 or more vector slots take the reference's block projector, whose
// dual residual is zero.
template <int S>
__device__ double warp_section_dual(int type, int L, int lane, unsigned fb, const double (&xv)[S],
                                    const double (&rc)[S], const double (&vr)[S], double alpha, double *warm,
                                    double (&out)[S])
{
#pragma unroll
    for (int s = 0; s < S; ++s)
        out[s] = 0.0;
    if (type == 3) {
        double x3[3], q3[3], d3[3], rc3[3];
        bool f3[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            d3[k] = __shfl_sync(FULL, vr[0], k);
            x3[k] = __shfl_sync(FULL, xv[0], k) / d3[k];
            rc3[k] = __shfl_sync(FULL, rc[0], k);
            q3[k] = rc3[k] * d3[k];
            f3[k] = (__shfl_sync(FULL, fb, k) & 1u) != 0;
        }
        double o3[3], cplx = 0.0;
        for (int k = 0; k < 3; ++k)
            o3[k] = f3[k] ? 0.0 : q3[k];
        if (lane == 0 && !(f3[0] && f3[1] && f3[2])) {
            const double x = x3[0], y = x3[1], z = x3[2], az = fabs(z);
            double bound = 0.0;
            bool regular = x > 0.0 && y > 0.0 && isfinite(x) && isfinite(y) && isfinite(z);
            if (regular) {
                bound = exp(alpha * log(x) + (1.0 - alpha) * log(y));
                regular = isfinite(bound) && bound > 0.0;
            }
            bool done = false;
            if (regular && az > 0.0) {
                const double nrm[3] = {-alpha * bound / x, -(1.0 - alpha) * bound / y, copysign(1.0, z)};
                double ns = 0.0;
                for (int k = 0; k < 3; ++k)
                    if (!f3[k])
                        ns = fmax(ns, fabs(nrm[k]));
                if (!(ns > 0.0) || !isfinite(ns))
                    regular = false;
                if (regular) {
                    double dot = 0.0, n2 = 0.0;
                    for (int k = 0; k < 3; ++k) {
                        if (f3[k])
                            continue;
                        const double sn = nrm[k] / ns;
                        dot += q3[k] * sn;
                        n2 += sn * sn;
                    }
                    const double slam = (dot < 0.0 && n2 > 0.0) ? -dot / n2 : 0.0;
                    for (int k = 0; k < 3; ++k)
                        if (!f3[k])
                            o3[k] = q3[k] + slam * (nrm[k] / ns);
                    cplx = (slam / ns) * (fmax(bound - az, 0.0) / fmax(1.0, fmax(bound, az)));
                    done = true;
                }
            }
            if (!done && !regular) {
                // nonsmooth points: the projected mapping in the d^2 metric
                double r3[3], w3[3], p3[3];
                for (int k = 0; k < 3; ++k) {
                    r3[k] = x3[k] - (f3[k] ? 0.0 : rc3[k] / d3[k]);
                    w3[k] = d3[k] * d3[k];
                }
                sec_pow_point(r3, w3, f3, alpha, p3);
                for (int k = 0; k < 3; ++k)
                    if (!f3[k])
                        o3[k] = (x3[k] - p3[k]) * d3[k] * d3[k];
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double v = __shfl_sync(FULL, o3[k], 0);
            if (lane == k)
                out[0] = v;
        }
        return __shfl_sync(FULL, cplx, 0);
    }
    if ((type == 0 || type == 1) && L - 2 >= 32)
        return 0.0;
    WarpSlots<S> p;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const bool f = (fb >> s) & 1u;
        p.x[s] = f ? xv[s] : xv[s] - rc[s];
        p.d[s] = vr[s];
        p.w[s] = 1.0;
    }
    warp_section_project<S>(type, p, L, lane, fb, warm, alpha);
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        const bool f = (fb >> s) & 1u;
        out[s] = (i < L && !f) ? (xv[s] - p.x[s]) * vr[s] : 0.0;
    }
    return 0.0;
}

} // namespace pdhcg
