// device.cuh -- device building blocks of the PDHCG-B200 kernels:
// warp/block reductions, CSR row dot products with a configurable number
// of lanes per row, and warp-cooperative weighted cone projections.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace pdhcg {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(FULL, v, o);
    return v; // identical in every lane: each butterfly step adds the same two operands
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

// |v| for an infinity-norm reduction: a non-finite entry makes the norm +inf
// (reference get_vector_inf_norm, src/utils.cu:548-567).
__device__ __forceinline__ double abs_or_inf(double v) { return isfinite(v) ? fabs(v) : INFINITY; }

// Sum of G consecutive lanes (G a power of two dividing 32).
template <int G>
__device__ __forceinline__ double group_sum(double v)
{
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1)
        v += __shfl_xor_sync(FULL, v, o, G);
    return v;
}

// Row-group loops.  A warp holds 32/G row groups of G lanes, and group_sum
// shuffles over the full warp, so every lane of a warp must run the same
// number of passes: the loop runs over the warp's first row `base`
// (uniform across the warp), each group takes row base + lane / G, and a
// group past the end computes an empty row (ok == false).
//   for (int base = warp_row0<G>(); base < rows; base += warp_row_stride<G>()) {
//       int r = base + (threadIdx.x & 31) / G; bool ok = r < rows;
//       double a = row_dot<G>(rp, ci, val, x, r, sub, ok); ... }
template <int G>
__device__ __forceinline__ int warp_row0(int block = -1)
{
    const int b = block < 0 ? (int)blockIdx.x : block;
    return b * (int)(blockDim.x / G) + (int)(threadIdx.x >> 5) * (32 / G);
}

template <int G>
__device__ __forceinline__ int warp_row_stride(int blocks = -1)
{
    return (blocks < 0 ? (int)gridDim.x : blocks) * (int)(blockDim.x / G);
}

// sum_k val[k] * x[col[k]] over row r, G lanes cooperating (lane = lane in
// group); every lane of the warp must call it, ok == false gives 0 without
// reading the row.
template <int G, typename V>
__device__ __forceinline__ double row_dot(const int *__restrict__ rp, const int *__restrict__ ci,
                                          const V *__restrict__ val, const double *__restrict__ x, int r, int lane,
                                          bool ok = true)
{
    int b = ok ? __ldg(rp + r) : 0, e = ok ? __ldg(rp + r + 1) : 0;
    double s = 0.0;
    for (int k = b + lane; k < e; k += G)
        s += (double)__ldg(val + k) * __ldg(x + __ldg(ci + k));
    return group_sum<G>(s);
}

// Same with the vector held in FP32.
template <int G, typename V>
__device__ __forceinline__ double row_dot(const int *__restrict__ rp, const int *__restrict__ ci,
                                          const V *__restrict__ val, const float *__restrict__ x, int r, int lane,
                                          bool ok = true)
{
    int b = ok ? __ldg(rp + r) : 0, e = ok ? __ldg(rp + r + 1) : 0;
    double s = 0.0;
    for (int k = b + lane; k < e; k += G)
        s += (double)__ldg(val + k) * (double)__ldg(x + __ldg(ci + k));
    return group_sum<G>(s);
}

// Entries [b, e) of one row, G lanes cooperating; every lane of the warp
// must call it (the group reduction shuffles over the full warp).
template <int G, typename V, typename X>
__device__ __forceinline__ double range_dot(const int *__restrict__ ci, const V *__restrict__ val,
                                            const X *__restrict__ x, int b, int e, int lane)
{
    double s = 0.0;
    for (int k = b + lane; k < e; k += G)
        s += (double)__ldg(val + k) * (double)__ldg(x + __ldg(ci + k));
    return group_sum<G>(s);
}

__device__ __forceinline__ double clampd(double lo, double x, double hi) { return fmax(lo, fmin(x, hi)); }

// ---------------------------------------------------------------------------
// Warp-cooperative cone projections.
//
// A warp owns one cone block of L slots; lane l holds slots l, l+32, ...
// in registers (S = slots per lane, compile time).  Inputs are the scaled
// candidate x (after the prox), the variable rescaling d and the metric
// weight w = 1 + tau q (w = 1 without a diagonal Q).  The cone is defined on
// u = x / d, so the projection minimises sum_i w_i d_i^2 (u_i - a_i)^2 with
// a_i = x_i / d_i (reference internal/cone_projection_utils.h:22-27).
// With d uniform and w == 1 the closed forms of the reference's thread
// kernels are used on x directly (src/kernels/pdhcg_soc_cone_kernels.cu:
// 296-324, src/kernels/pdhcg_rsoc_cone_kernels.cu:505-530); otherwise the
// multiplier of the KKT system is found by bracketed Newton, as in the
// reference's block kernels (pdhcg_soc_cone_kernels.cu:1725-2062,
// pdhcg_rsoc_cone_kernels.cu:2096-2631).  All lanes run the same scalar
// iteration on warp-reduced (bitwise identical) sums, so control flow is
// warp-uniform.
// ---------------------------------------------------------------------------

constexpr int ROOT_ITERS = 100;

template <int S>
struct WarpSlots {
    double x[S]; // in: candidate (scaled); out: projection (scaled)
    double d[S];
    double w[S];
};

// Standard SOC [v(k), w, z]: L = k + 2, apex slot index L-1.
// warm: this cone's multiplier from the previous call (NULL: none); on a
// root-finding exit the new multiplier is stored there (the reference keeps
// the same per-cone warm start, internal/internal_types.h:250).
template <int S>
__device__ void warp_project_soc(WarpSlots<S> &sl, int L, int lane, bool uniform_unit, double *warm)
{
    const int apex = L - 1;
    const int apex_lane = apex & 31, apex_s = apex >> 5;
    double xz = 0.0, dz = 1.0, wz = 1.0;
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (s == apex_s) {
            xz = sl.x[s];
            dz = sl.d[s];
            wz = sl.w[s];
        }
    xz = __shfl_sync(FULL, xz, apex_lane);
    dz = __shfl_sync(FULL, dz, apex_lane);
    wz = __shfl_sync(FULL, wz, apex_lane);

    if (uniform_unit) {
        double ss = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            int i = lane + 32 * s;
            if (i < apex)
                ss += sl.x[s] * sl.x[s];
        }
        double r = sqrt(warp_sum(ss));
        if (r <= xz)
            return;
        if (r <= -xz) {
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (lane + 32 * s < L)
                    sl.x[s] = 0.0;
            return;
        }
        double scale = (xz + r) / (2.0 * r);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            int i = lane + 32 * s;
            if (i < apex)
                sl.x[s] *= scale;
            else if (i == apex)
                sl.x[s] = scale * r;
        }
        return;
    }

    // u-space data: a = x / d, omega = w d^2; b = omega * a
    double b[S], om[S];
    double n2 = 0.0, p2 = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        b[s] = 0.0;
        om[s] = 1.0;
        if (i < apex) {
            double a = sl.x[s] / sl.d[s];
            om[s] = fmax(sl.w[s] * sl.d[s] * sl.d[s], DBL_MIN);
            b[s] = om[s] * a;
            n2 += a * a;
            p2 += b[s] * b[s];
        }
    }
    n2 = warp_sum(n2);
    p2 = warp_sum(p2);
    const double az = xz / dz;
    const double omz = fmax(wz * dz * dz, DBL_MIN);
    if (az >= 0.0 && n2 <= az * az)
        return; // inside
    if (-omz * az >= sqrt(p2)) { // -omega.a in the cone: apex
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (lane + 32 * s < L)
                sl.x[s] = 0.0;
        return;
    }
    double lam, uz;
    if (az == 0.0) {
        lam = omz;
        double t2 = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (lane + 32 * s < apex) {
                double t = b[s] / (om[s] + lam);
                t2 += t * t;
            }
        uz = sqrt(warp_sum(t2));
    } else {
        // f(lam) = |U|^2 - Z^2 with U_i = b_i/(om_i+lam), Z = omz az/(omz-lam);
        // root in (0, omz) when az > 0, in (omz, inf) when az < 0.
        const bool lower = az > 0.0;
        const double bz = omz * az;
        double lo = lower ? 0.0 : omz * (1.0 + 1e-14);
        double hi = lower ? omz * (1.0 - 1e-14) : INFINITY;
        double w0 = warm ? *warm : -1.0;
        lam = (w0 > lo && w0 < hi && isfinite(w0)) ? w0 : (lower ? 0.5 * (lo + hi) : 2.0 * omz);
        for (int it = 0; it < ROOT_ITERS; ++it) {
            double t2 = 0.0, dt2 = 0.0;
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (lane + 32 * s < apex) {
                    double inv = 1.0 / (om[s] + lam);
                    double t = b[s] * inv;
                    t2 += t * t;
                    dt2 += t * t * inv;
                }
            t2 = warp_sum(t2);
            dt2 = warp_sum(dt2);
            double izl = 1.0 / (omz - lam);
            double z = bz * izl;
            double f = t2 - z * z;
            double df = -2.0 * dt2 - 2.0 * z * z * izl;
            if ((lower && f > 0.0) || (!lower && f < 0.0))
                lo = lam;
            else
                hi = lam;
            if (fabs(f) <= 1e-13 * (1.0 + t2 + z * z) || (isfinite(hi) && hi - lo <= 1e-13 * (1.0 + hi + lo)))
                break;
            double nx = lam - f / df;
            if (!isfinite(nx) || !(nx > lo && nx < hi))
                nx = isfinite(hi) ? 0.5 * (lo + hi) : 2.0 * lam;
            lam = nx;
        }
        uz = bz / (omz - lam);
        if (warm && lane == 0)
            *warm = lam;
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        if (i < apex)
            sl.x[s] = (b[s] / (om[s] + lam)) * sl.d[s];
        else if (i == apex)
            sl.x[s] = uz * dz;
    }
}

// Rotated SOC [v(k), s, t]: 2 s t >= |v|^2, s, t >= 0.  L = k + 2.
template <int S>
__device__ void warp_project_rsoc(WarpSlots<S> &sl, int L, int lane, bool uniform_unit, double *warm)
{
    const int is = L - 2, it_ = L - 1;
    double xs = 0.0, xt = 0.0, ds = 1.0, dt = 1.0, ws = 1.0, wt = 1.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        if (i == is) {
            xs = sl.x[s];
            ds = sl.d[s];
            ws = sl.w[s];
        }
        if (i == it_) {
            xt = sl.x[s];
            dt = sl.d[s];
            wt = sl.w[s];
        }
    }
    xs = __shfl_sync(FULL, xs, is & 31);
    ds = __shfl_sync(FULL, ds, is & 31);
    ws = __shfl_sync(FULL, ws, is & 31);
    xt = __shfl_sync(FULL, xt, it_ & 31);
    dt = __shfl_sync(FULL, dt, it_ & 31);
    wt = __shfl_sync(FULL, wt, it_ & 31);

    if (uniform_unit) {
        const double INV_SQRT2 = 0.7071067811865475;
        double wv = (xs - xt) * INV_SQRT2, zv = (xs + xt) * INV_SQRT2;
        double ss = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (lane + 32 * s < is)
                ss += sl.x[s] * sl.x[s];
        double r = sqrt(wv * wv + warp_sum(ss));
        if (r <= zv)
            return;
        if (r <= -zv) {
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (lane + 32 * s < L)
                    sl.x[s] = 0.0;
            return;
        }
        double scale = (zv + r) / (2.0 * r);
        double w_new = scale * wv, z_new = scale * r;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            int i = lane + 32 * s;
            if (i < is)
                sl.x[s] *= scale;
            else if (i == is)
                sl.x[s] = (z_new + w_new) * INV_SQRT2;
            else if (i == it_)
                sl.x[s] = (z_new - w_new) * INV_SQRT2;
        }
        return;
    }

    double a[S], om[S];
    double n2 = 0.0, p2 = 0.0, fobj = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        a[s] = 0.0;
        om[s] = 1.0;
        if (i < is) {
            a[s] = sl.x[s] / sl.d[s];
            om[s] = fmax(sl.w[s] * sl.d[s] * sl.d[s], DBL_MIN);
            n2 += a[s] * a[s];
            p2 += (om[s] * a[s]) * (om[s] * a[s]);
            fobj += om[s] * a[s] * a[s];
        }
    }
    n2 = warp_sum(n2);
    p2 = warp_sum(p2);
    fobj = warp_sum(fobj);
    const double as = xs / ds, at = xt / dt;
    const double oms = fmax(ws * ds * ds, DBL_MIN), omt = fmax(wt * dt * dt, DBL_MIN);
    if (as >= 0.0 && at >= 0.0 && n2 <= 2.0 * as * at)
        return;
    const double bs = oms * as, bt = omt * at;
    if (bs <= 0.0 && bt <= 0.0 && p2 <= 2.0 * bs * bt) {
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (lane + 32 * s < L)
                sl.x[s] = 0.0;
        return;
    }
    const double sqs = sqrt(oms), sqt = sqrt(omt), rm = sqs * sqt;
    const double balance = sqs * as + sqt * at;
    const double bscale = 1.0 + fabs(sqs * as) + fabs(sqt * at);
    double lam, ps, pt;
    if (fabs(balance) <= 64.0 * DBL_EPSILON * bscale) {
        lam = rm;
        double t2 = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (lane + 32 * s < is) {
                double t = om[s] * a[s] / (om[s] + lam);
                t2 += t * t;
            }
        t2 = warp_sum(t2);
        double product = 0.5 * rm * t2, delta = sqs * as;
        double st = 0.5 * (-delta + sqrt(fmax(0.0, delta * delta + 4.0 * product)));
        ps = (st + delta) / sqs;
        pt = st / sqt;
    } else {
        // f(lam) = |U|^2 - 2 s t; root in (0, rm) when balance > 0, else (rm, inf)
        const bool lower = balance > 0.0;
        double lo = lower ? 0.0 : rm * (1.0 + 1e-14);
        double hi = lower ? rm * (1.0 - 1e-14) : INFINITY;
        double w0 = warm ? *warm : -1.0;
        lam = (w0 > lo && w0 < hi && isfinite(w0)) ? w0 : (lower ? 0.5 * (lo + hi) : 2.0 * rm);
        for (int itn = 0; itn < ROOT_ITERS; ++itn) {
            double t2 = 0.0, dt2 = 0.0;
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (lane + 32 * s < is) {
                    double inv = 1.0 / (om[s] + lam);
                    double t = om[s] * a[s] * inv;
                    t2 += t * t;
                    dt2 += t * t * inv;
                }
            t2 = warp_sum(t2);
            dt2 = warp_sum(dt2);
            double idet = 1.0 / (oms * omt - lam * lam);
            double sv = omt * (oms * as + lam * at) * idet, tv = oms * (omt * at + lam * as) * idet;
            double f = INFINITY, df = -2.0 * dt2;
            if (sv >= 0.0 && tv >= 0.0) {
                f = t2 - 2.0 * sv * tv;
                double dsl = (omt * tv + lam * sv) * idet, dtl = (lam * tv + oms * sv) * idet;
                df -= 2.0 * (dsl * tv + sv * dtl);
            }
            if ((lower && f > 0.0) || (!lower && f < 0.0))
                lo = lam;
            else
                hi = lam;
            if (isfinite(f) && (fabs(f) <= 1e-13 * (1.0 + t2 + 2.0 * sv * tv) ||
                                (isfinite(hi) && hi - lo <= 1e-13 * (1.0 + hi + lo))))
                break;
            double nx = lam - f / df;
            if (!isfinite(nx) || !(nx > lo && nx < hi))
                nx = isfinite(hi) ? 0.5 * (lo + hi) : 2.0 * lam;
            lam = nx;
        }
        double det = oms * omt - lam * lam;
        ps = omt * (oms * as + lam * at) / det;
        pt = oms * (omt * at + lam * as) / det;
    }
    // axis candidates where the boundary is not smooth
    double sm = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (lane + 32 * s < is) {
            double v = om[s] * a[s] / (om[s] + lam);
            sm += om[s] * (v - a[s]) * (v - a[s]);
        }
    sm = warp_sum(sm) + oms * (ps - as) * (ps - as) + omt * (pt - at) * (pt - at);
    double s_axis = fmax(as, 0.0), t_axis = fmax(at, 0.0);
    double s_obj = fobj + oms * (s_axis - as) * (s_axis - as) + omt * at * at;
    double t_obj = fobj + oms * as * as + omt * (t_axis - at) * (t_axis - at);
    bool axis = false;
    if (s_obj < sm && s_obj <= t_obj) {
        axis = true;
        ps = s_axis;
        pt = 0.0;
    } else if (t_obj < sm) {
        axis = true;
        ps = 0.0;
        pt = t_axis;
    }
    if (warm && lane == 0 && !axis)
        *warm = lam;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        if (i < is)
            sl.x[s] = axis ? 0.0 : (om[s] * a[s] / (om[s] + lam)) * sl.d[s];
        else if (i == is)
            sl.x[s] = ps * ds;
        else if (i == it_)
            sl.x[s] = pt * dt;
    }
}

template <int S>
__device__ __forceinline__ void warp_project(int type, WarpSlots<S> &sl, int L, int lane, bool uniform_unit,
                                             double *warm)
{
    if (type == 1) // CONE_STANDARD_SOC
        warp_project_soc<S>(sl, L, lane, uniform_unit, warm);
    else if (type == 0) // CONE_ROTATED_SOC
        warp_project_rsoc<S>(sl, L, lane, uniform_unit, warm);
}

// Is d uniform over the block and w == 1 everywhere?  (warp vote)
template <int S>
__device__ __forceinline__ bool warp_uniform_unit(const WarpSlots<S> &sl, int L, int lane)
{
    double d0 = __shfl_sync(FULL, sl.d[0], 0);
    bool ok = true;
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (lane + 32 * s < L)
            ok = ok && (sl.d[s] == d0) && (sl.w[s] == 1.0);
    return __all_sync(FULL, ok);
}

} // namespace pdhcg
