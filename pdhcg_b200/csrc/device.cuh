// device.cuh -- device building blocks of the PDHCG-B200 kernels:
// warp/block reductions, CSR row products (stream mode for the hot kernels,
// row groups for set-up), and warp-cooperative weighted cone projections.
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

// ---------------------------------------------------------------------------
// Stream-mode CSR products for the hot step kernels.
//
// A warp owns up to 32 * S consecutive rows [r0, r0 + nr); lane l owns rows
// r0 + l + 32 s.  Their entries are one contiguous range [rp[r0], rp[r0+nr])
// of the CSR arrays, so the warp streams that range in chunks of
// STREAM_CHUNK entries: every lane issues STREAM_U independent coalesced
// loads of (col, val), then STREAM_U gathers of x, and stores the products in
// a per-warp shared buffer; each lane then adds the products of its own rows
// in entry order (the same order as a sequential row loop).
//
// A row longer than STREAM_ROW_MAX would leave one lane adding alone while
// the warp waits, so a warp whose rows include such a row reduces its rows
// one at a time across all 32 lanes instead (warp_sum; a different but
// fixed summation order).
// ---------------------------------------------------------------------------
#ifndef PDHCG_STREAM_U
#define PDHCG_STREAM_U 8
#endif
constexpr int STREAM_U = PDHCG_STREAM_U;
constexpr int STREAM_CHUNK = 32 * STREAM_U;
constexpr int STREAM_ROW_MAX = 64;

__device__ __forceinline__ int warp_max_int(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = max(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

// ---------------------------------------------------------------------------
// Long rows.  A row of more than LONG_ROW entries (a dense constraint row, a
// variable in many rows) is too long for the stream mode below, and one warp
// per row would leave the product to the few warps whose tiles hold such
// rows.  So these rows are cut into segments of at most LONG_SEG entries:
// long_partials_kernel writes one partial product per segment (one warp
// each, fixed order), and the product that reads the row adds its
// segments' partials in segment order, each lane for its own row.  The
// partials belong to the last vector passed to that kernel: every product
// of a matrix with long rows is preceded by its pass.
// ---------------------------------------------------------------------------
constexpr int LONG_ROW = STREAM_ROW_MAX; // every row beyond stream mode
constexpr int LONG_SEG = 4096;

struct LongRows {
    const int *rows;      // [n] long row ids, ascending
    const int *seg_first; // [n + 1] first segment of each long row
    const int2 *seg;      // [nseg] entry range {begin, end} of each segment
    double *part;         // [nseg] partial products of the last pass
    int n, nseg;
};

// index of the first long row >= row (L.n when none)
__device__ __forceinline__ int long_lower_bound(const LongRows &L, int row)
{
    int lo = 0, hi = L.n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(L.rows + mid) < row)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// the same sum computed by the whole warp for one row (every lane calls it)
__device__ __forceinline__ double long_row_sum_warp(const LongRows &L, int row, int lane)
{
    const int i = long_lower_bound(L, row);
    const int f = __ldg(L.seg_first + i), e = __ldg(L.seg_first + i + 1);
    double a = 0.0;
    for (int k = f + lane; k < e; k += 32)
        a += L.part[k];
    return warp_sum(a);
}

// sum of long row i's segment partials, in segment order (one lane)
__device__ __forceinline__ double long_row_fold(const LongRows &L, int i)
{
    const int f = __ldg(L.seg_first + i), e = __ldg(L.seg_first + i + 1);
    double a = 0.0;
    for (int k = f; k < e; ++k)
        a += L.part[k];
    return a;
}

// one warp's dot product over entries [b, e), lane-strided, 4 partial sums
template <typename V, typename X>
__device__ __forceinline__ double warp_range_dot(const int *__restrict__ ci, const V *__restrict__ val,
                                                 const X *__restrict__ x, int b, int e, int lane)
{
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int k = b + lane;
    // two strides of 128 at a time: the eight index and value loads, then the
    // eight gathers, are in flight together; each partial sum still adds its
    // entries in stride order
    for (; k + 224 < e; k += 256) {
        int c[8];
        double v[8], w[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            c[u] = __ldg(ci + k + 32 * u);
            v[u] = (double)__ldg(val + k + 32 * u);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            w[u] = (double)__ldg(x + c[u]);
        a0 += v[0] * w[0];
        a1 += v[1] * w[1];
        a2 += v[2] * w[2];
        a3 += v[3] * w[3];
        a0 += v[4] * w[4];
        a1 += v[5] * w[5];
        a2 += v[6] * w[6];
        a3 += v[7] * w[7];
    }
    for (; k + 96 < e; k += 128) {
        a0 += (double)__ldg(val + k) * (double)__ldg(x + __ldg(ci + k));
        a1 += (double)__ldg(val + k + 32) * (double)__ldg(x + __ldg(ci + k + 32));
        a2 += (double)__ldg(val + k + 64) * (double)__ldg(x + __ldg(ci + k + 64));
        a3 += (double)__ldg(val + k + 96) * (double)__ldg(x + __ldg(ci + k + 96));
    }
    // at most three strides remain (k + 96 >= e): their loads are issued
    // together, then added to a0 in stride order
    const bool p0 = k < e, p1 = k + 32 < e, p2 = k + 64 < e;
    const int c0 = p0 ? __ldg(ci + k) : 0, c1 = p1 ? __ldg(ci + k + 32) : 0, c2 = p2 ? __ldg(ci + k + 64) : 0;
    const double v0 = p0 ? (double)__ldg(val + k) : 0.0, v1 = p1 ? (double)__ldg(val + k + 32) : 0.0,
                 v2 = p2 ? (double)__ldg(val + k + 64) : 0.0;
    const double x0 = p0 ? (double)__ldg(x + c0) : 0.0, x1 = p1 ? (double)__ldg(x + c1) : 0.0,
                 x2 = p2 ? (double)__ldg(x + c2) : 0.0;
    if (p0)
        a0 += v0 * x0;
    if (p1)
        a0 += v1 * x1;
    if (p2)
        a0 += v2 * x2;
    return warp_sum((a0 + a1) + (a2 + a3));
}

// the segment pass over warps gw, gw + nw, ... (a kernel body, or a phase
// of a cooperative kernel followed by a grid barrier)
template <typename V, typename X>
__device__ __forceinline__ void long_partials(const LongRows &L, const int *__restrict__ ci,
                                              const V *__restrict__ val, const X *__restrict__ x, int gw, int nw,
                                              int lane)
{
    // the next segment's bounds are loaded before this segment's sum, so a
    // warp that walks many short segments does not wait for them each time
    int2 r = gw < L.nseg ? L.seg[gw] : make_int2(0, 0);
    for (int sg = gw; sg < L.nseg; sg += nw) {
        const int2 rn = sg + nw < L.nseg ? L.seg[sg + nw] : make_int2(0, 0);
        const double a = warp_range_dot(ci, val, x, r.x, r.y, lane);
        if (lane == 0)
            L.part[sg] = a;
        r = rn;
    }
}

template <typename V, typename X>
__global__ void __launch_bounds__(256) long_partials_kernel(LongRows L, const int *ci, const V *val, const X *x)
{
    long_partials(L, ci, val, x, (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5),
                  (int)((gridDim.x * blockDim.x) >> 5), (int)(threadIdx.x & 31));
}

// number of rows longer than LONG_ROW entries
__global__ void long_count_kernel(int rows, const int *rp, int *count)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
        if (rp[r + 1] - rp[r] > LONG_ROW)
            atomicAdd(count, 1);
}

// out[s] = sum_k val[k] * x[ci[k]] over row r0 + lane + 32 s (0 when that
// row is past nr).  Every lane of the warp must call it with the same r0,
// nr (1 <= nr <= 32 S) and stage (STREAM_CHUNK doubles of this warp's
// shared memory).  Rows longer than LONG_ROW entries take their value from
// the segment partials of lr, which must hold this product's pass.  A tile
// holding such a row is otherwise reduced one row at a time by the whole
// warp (no table, lr.n = 0; or S > 2, where the lane-wise form would cost
// the wide cone kernels their registers).
template <int S, typename V, typename X>
__device__ __forceinline__ void warp_stream_rows(const int *__restrict__ rp, const int *__restrict__ ci,
                                                 const V *__restrict__ val, const X *__restrict__ x, int r0, int nr,
                                                 int lane, double *stage, double (&out)[S], const LongRows &lr)
{
    int rb[S], re[S];
    int longest = 0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        rb[s] = re[s] = 0;
        if (i < nr) {
            rb[s] = __ldg(rp + r0 + i);
            re[s] = __ldg(rp + r0 + i + 1);
        }
        longest = max(longest, re[s] - rb[s]);
        out[s] = 0.0;
    }
    longest = warp_max_int(longest);
    const int b = __shfl_sync(FULL, rb[0], 0);
    int e = 0;
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (s == ((nr - 1) >> 5))
            e = re[s];
    e = __shfl_sync(FULL, e, (nr - 1) & 31);

    if (longest <= STREAM_ROW_MAX) {
        for (int cb = b; cb < e; cb += STREAM_CHUNK) {
            int col[STREAM_U];
            double v[STREAM_U];
#pragma unroll
            for (int u = 0; u < STREAM_U; ++u) {
                const int k = cb + 32 * u + lane;
                col[u] = k < e ? __ldg(ci + k) : -1;
                v[u] = k < e ? (double)__ldg(val + k) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < STREAM_U; ++u)
                stage[32 * u + lane] = col[u] >= 0 ? v[u] * (double)__ldg(x + col[u]) : 0.0;
            __syncwarp();
            const int ce = min(e, cb + STREAM_CHUNK);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int lo = max(rb[s], cb), hi = min(re[s], ce);
                double a = out[s];
                for (int k = lo; k < hi; ++k)
                    a += stage[k - cb];
                out[s] = a;
            }
            __syncwarp();
        }
    } else if (S <= 2 && lr.n > 0) {
        // every row longer than LONG_ROW is in lr: each lane folds its own
        // long row's partials (its table index from one search per tile and
        // a ballot) or adds its own short row in entry order
        const int base = long_lower_bound(lr, r0);
        int before = 0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const bool valid = lane + 32 * s < nr;
            const bool lg = valid && re[s] - rb[s] > LONG_ROW;
            const unsigned mask = __ballot_sync(FULL, lg);
            if (lg) {
                out[s] = long_row_fold(lr, base + before + __popc(mask & ((1u << lane) - 1u)));
            } else if (valid) {
                double a = 0.0;
                for (int k = rb[s]; k < re[s]; ++k)
                    a += (double)__ldg(val + k) * (double)__ldg(x + __ldg(ci + k));
                out[s] = a;
            }
            before += __popc(mask);
        }
    } else {
        for (int i = 0; i < nr; ++i) {
            int bi = 0, ei = 0;
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (s == (i >> 5)) {
                    bi = rb[s];
                    ei = re[s];
                }
            bi = __shfl_sync(FULL, bi, i & 31);
            ei = __shfl_sync(FULL, ei, i & 31);
            // (wide tiles with a long-row table: the warp folds each long row)
            const double a = (lr.n > 0 && ei - bi > LONG_ROW) ? long_row_sum_warp(lr, r0 + i, lane)
                                                                : warp_range_dot(ci, val, x, bi, ei, lane);
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (s == (i >> 5) && lane == (i & 31))
                    out[s] = a;
        }
    }
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

    // u-space data: a = x / d, omega = w d^2; b = omega * a = w d x.  The
    // projection is u_i = b_i / (omega_i + lam), i.e. x_i = x_i omega_i / (omega_i + lam),
    // so the only per-slot reciprocals are 1/d (for the cone tests) and
    // 1/(omega_i + lam) (reused for the output).
    double b[S], om[S], inv[S];
    double n2 = 0.0, p2 = 0.0;
    // d uniform over the block (what cone-preserving scaling gives): one
    // reciprocal serves every slot (the same value each slot would compute)
    bool dsame = true;
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (lane + 32 * s < apex)
            dsame = dsame && sl.d[s] == dz;
    const double rdz = __all_sync(FULL, dsame) ? __drcp_rn(dz) : 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        b[s] = 0.0;
        om[s] = 1.0;
        inv[s] = 1.0;
        if (i < apex) {
            double rd = rdz != 0.0 ? rdz : __drcp_rn(sl.d[s]);
            double a = sl.x[s] * rd;
            om[s] = fmax(sl.w[s] * sl.d[s] * sl.d[s], DBL_MIN);
            b[s] = sl.w[s] * sl.d[s] * sl.x[s];
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
                inv[s] = __drcp_rn(om[s] + lam);
                double t = b[s] * inv[s];
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
        double izl = 0.0;
        bool done = false;
        for (int it = 0; it < ROOT_ITERS; ++it) {
            double t2 = 0.0;
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (lane + 32 * s < apex) {
                    inv[s] = __drcp_rn(om[s] + lam);
                    double t = b[s] * inv[s];
                    t2 += t * t;
                }
            t2 = warp_sum(t2);
            izl = __drcp_rn(omz - lam);
            double z = bz * izl;
            double f = t2 - z * z;
            if ((lower && f > 0.0) || (!lower && f < 0.0))
                lo = lam;
            else
                hi = lam;
            if (fabs(f) <= 1e-13 * (1.0 + t2 + z * z) || (isfinite(hi) && hi - lo <= 1e-13 * (1.0 + hi + lo))) {
                done = true;
                break;
            }
            // f' only when a Newton step follows (a warm-started search
            // usually stops at its first evaluation)
            double dt2 = 0.0;
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (lane + 32 * s < apex) {
                    double t = b[s] * inv[s];
                    dt2 += t * t * inv[s];
                }
            dt2 = warp_sum(dt2);
            double df = -2.0 * dt2 - 2.0 * z * z * izl;
            double nx = lam - f / df;
            // a Newton step below the resolution of lam cannot improve it:
            // stop there (without this, rounding that keeps |f| above its
            // tolerance sent the search into ~40 bisections of the bracket,
            // and the warp holding that block set the length of the launch)
            if (isfinite(nx) && fabs(nx - lam) <= 2.0 * DBL_EPSILON * fabs(lam)) {
                done = true;
                break;
            }
            if (!isfinite(nx) || !(nx > lo && nx < hi))
                nx = isfinite(hi) ? 0.5 * (lo + hi) : 2.0 * lam;
            lam = nx;
        }
        if (!done) { // iteration cap: inv and izl of the final lam
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (lane + 32 * s < apex)
                    inv[s] = __drcp_rn(om[s] + lam);
            izl = __drcp_rn(omz - lam);
        }
        uz = bz * izl;
        if (warm && lane == 0)
            *warm = lam;
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int i = lane + 32 * s;
        if (i < apex)
            sl.x[s] = sl.x[s] * om[s] * inv[s];
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
            if (isfinite(f) && isfinite(nx) && fabs(nx - lam) <= 2.0 * DBL_EPSILON * fabs(lam))
                break; // step below the resolution of lam (as for the SOC)
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

// ---------------------------------------------------------------------------
// Three-dimensional cones, projected by one thread.
//
// Exponential cone K = cl{(x, y, z) : y > 0, y exp(x / y) <= z}: the
// projection of r onto {v : v / d in K} in the unit metric of r's space,
// with the reference's sequence of tests and its Newton iteration on
// rho = x / y (src/kernels/pdhcg_exp_cone_kernels.cu:26-131): in-cone test,
// polar-cone test, the x <= 0, y <= 0 case, then at most 100 capped Newton
// steps with the same fallbacks.
// ---------------------------------------------------------------------------
__device__ inline void exp_cone_point(double r1, double r2, double r3, double d1, double d2, double d3, double &o1,
                                      double &o2, double &o3)
{
    const double a1 = r1 / d1, a2 = r2 / d2, a3 = r3 / d3;
    const bool inside = a2 > 0.0 ? (a1 / a2 < 700.0 && a2 * exp(a1 / a2) <= a3)
                                 : (a2 == 0.0 && a1 <= 0.0 && a3 >= 0.0);
    if (inside) {
        o1 = r1;
        o2 = r2;
        o3 = r3;
        return;
    }
    const bool polar = r1 > 0.0 ? ((d2 * r2) / (d1 * r1) < 700.0 &&
                                   d1 * r1 * exp((d2 * r2) / (d1 * r1)) + 2.718281828459045 * d3 * r3 <= 0.0)
                                : (r1 == 0.0 && r2 <= 0.0 && r3 <= 0.0);
    if (polar) {
        o1 = o2 = o3 = 0.0;
        return;
    }
    if (a1 <= 0.0 && a2 <= 0.0) {
        o1 = r1;
        o2 = 0.0;
        o3 = a3 < 0.0 ? 0.0 : r3;
        return;
    }
    const double al = (d3 / d1) * (d3 / d1), be = (d3 / d2) * (d3 / d2);
    double rho = 0.0;
    bool diverged = false;
    for (int it = 0; it < 100; ++it) {
        if (fabs(rho) >= 299.0) {
            diverged = true;
            break;
        }
        const double er = exp(rho), e2 = er * er, omr = 1.0 - rho;
        const double A = al - be * rho * omr, B = be * a1 * omr - al * a2;
        const double f = a1 - a2 * rho + a3 * er * A + e2 * B;
        const double df = -a2 + a3 * er * (A - be * (1.0 - 2.0 * rho)) + e2 * (2.0 * B - be * a1);
        if (fabs(df) < 1e-300)
            break;
        const double step = fmin(fmax(f / df, -10.0), 10.0);
        rho -= step;
        if (fabs(step) < 1e-13 * (1.0 + fabs(rho)))
            break;
    }
    const double er = exp(rho);
    const double u2 = (a1 + al * a3 * er) / (rho + al * er * er);
    if (diverged || !isfinite(u2) || u2 <= 0.0) {
        o1 = r1 < 0.0 ? r1 : 0.0;
        o2 = 0.0;
        o3 = r3 > 0.0 ? r3 : 0.0;
        return;
    }
    o1 = d1 * rho * u2;
    o2 = d2 * u2;
    o3 = d3 * u2 * er;
}

// Power cone K_a = {(x, y, z) : x, y >= 0, x^a y^(1-a) >= |z|}: weighted
// projection min sum w_i (v_i - r_i)^2 over K_a, by the reference's steps
// (src/kernels/pdhcg_power_cone_kernels.cu:25-133): in-cone and
// opposite-cone tests, then 80 bisection steps on log |v_z| with x, y the
// positive roots of the KKT quadratics, on the point scaled by its largest
// magnitude.
__device__ inline double pow_pos_root(double r, double q)
{
    if (!(q > 0.0))
        return fmax(r, 0.0);
    const double disc = hypot(r, 2.0 * sqrt(q));
    return r >= 0.0 ? 0.5 * (r + disc) : (2.0 * q) / (disc - r);
}

__device__ inline void pow_cone_point(double rx, double ry, double rz, double wx, double wy, double wz, double a,
                                      double &ox, double &oy, double &oz)
{
    double s = fmax(fabs(rx), fmax(fabs(ry), fabs(rz)));
    if (!(s > 0.0) || !isfinite(s))
        s = 1.0;
    rx /= s;
    ry /= s;
    rz /= s;
    const double az = fabs(rz), om = 1.0 - a;
    if (az == 0.0) {
        ox = fmax(rx, 0.0) * s;
        oy = fmax(ry, 0.0) * s;
        oz = 0.0;
        return;
    }
    if (rx > 0.0 && ry > 0.0 && a * log(rx) + om * log(ry) >= log(az)) {
        ox = rx * s;
        oy = ry * s;
        oz = rz * s;
        return;
    }
    if (rx <= 0.0 && ry <= 0.0) {
        const double u = rx < 0.0 ? (-wx * rx) / a : 0.0, v = ry < 0.0 ? (-wy * ry) / om : 0.0;
        if (u > 0.0 && v > 0.0 && a * log(u) + om * log(v) >= log(wz) + log(az)) {
            ox = oy = oz = 0.0;
            return;
        }
    }
    const double cx = 4.0 * a * (wz / wx), cy = 4.0 * om * (wz / wy);
    double lo = log(DBL_MIN), hi = log(az);
    if (!(hi > lo)) {
        ox = fmax(rx, 0.0) * s;
        oy = fmax(ry, 0.0) * s;
        oz = 0.0;
        return;
    }
    for (int it = 0; it < 80; ++it) {
        const double lr = lo + 0.5 * (hi - lo), rho = exp(lr);
        const double x = pow_pos_root(rx, 0.25 * cx * rho * (az - rho));
        const double y = pow_pos_root(ry, 0.25 * cy * rho * (az - rho));
        if (x > 0.0 && y > 0.0 && a * log(x) + om * log(y) > lr)
            lo = lr;
        else
            hi = lr;
    }
    const double rho = exp(lo + 0.5 * (hi - lo));
    const double x = pow_pos_root(rx, 0.25 * cx * rho * (az - rho));
    const double y = pow_pos_root(ry, 0.25 * cy * rho * (az - rho));
    ox = x * s;
    oy = y * s;
    oz = (rz >= 0.0 ? 1.0 : -1.0) * fmin(rho, exp(a * log(x) + om * log(y))) * s;
}

// Projection of one 3-slot EXP (type 2) or POW (type 3) block: metric w,
// scaling d.  Only the one-slot (S = 1) instantiations of the cone-block
// bodies reach it, so its Newton / bisection loops stay out of the wide SOC
// bodies' register allocation.
__device__ __forceinline__ double3 cone3_point(int type, double3 x, double3 d, double3 w, double alpha)
{
    double3 o;
    if (type == 2) { // exponential: the sqrt(w) change of variables
        const double s0 = sqrt(w.x > 0.0 ? w.x : 1.0), s1 = sqrt(w.y > 0.0 ? w.y : 1.0),
                     s2 = sqrt(w.z > 0.0 ? w.z : 1.0);
        exp_cone_point(s0 * x.x, s1 * x.y, s2 * x.z, s0 * d.x, s1 * d.y, s2 * d.z, o.x, o.y, o.z);
        o.x /= s0;
        o.y /= s1;
        o.z /= s2;
    } else { // power: scaled space, weights w d^2
        pow_cone_point(x.x / d.x, x.y / d.y, x.z / d.z, w.x * d.x * d.x, w.y * d.y * d.y, w.z * d.z * d.z, alpha,
                       o.x, o.y, o.z);
        o.x *= d.x;
        o.y *= d.y;
        o.z *= d.z;
    }
    return o;
}

// A 3-slot block held in lanes 0..2 (S = 1 slot each): lane 0 gathers it,
// projects it and hands the result back.
template <int S>
__device__ __forceinline__ void warp_project3(int type, WarpSlots<S> &sl, int lane, double alpha)
{
    double3 x, d, w;
    x.x = __shfl_sync(FULL, sl.x[0], 0);
    x.y = __shfl_sync(FULL, sl.x[0], 1);
    x.z = __shfl_sync(FULL, sl.x[0], 2);
    d.x = __shfl_sync(FULL, sl.d[0], 0);
    d.y = __shfl_sync(FULL, sl.d[0], 1);
    d.z = __shfl_sync(FULL, sl.d[0], 2);
    w.x = __shfl_sync(FULL, sl.w[0], 0);
    w.y = __shfl_sync(FULL, sl.w[0], 1);
    w.z = __shfl_sync(FULL, sl.w[0], 2);
    double3 o = make_double3(0.0, 0.0, 0.0);
    if (lane == 0)
        o = cone3_point(type, x, d, w, alpha);
    const double r0 = __shfl_sync(FULL, o.x, 0), r1 = __shfl_sync(FULL, o.y, 0), r2 = __shfl_sync(FULL, o.z, 0);
    if (lane < 3)
        sl.x[0] = lane == 0 ? r0 : (lane == 1 ? r1 : r2);
}

// Cone kinds an instantiation carries: SOC / RSOC (any S), and the 3-slot
// exponential / power cones (S = 1 only; callers route those blocks there).
// ---------------------------------------------------------------------------
// PSD blocks.  The block's L = n (n + 1) / 2 slots hold svec(X): the lower
// triangle down the columns, off-diagonal entries scaled by sqrt 2 (the
// reference's packing, src/kernels/pdhcg_psd_cone_kernels.cu:65-91).  The
// projection is the Frobenius one in the scaled space, as the reference
// takes it (:415-475; no metric): the warp unpacks X into work[0, n^2)
// (this block's device scratch, row-major), runs cyclic Jacobi with
// Rutishauser's rotation on it while accumulating the eigenvectors in
// work[n^2, 2 n^2), clips the negative eigenvalues and repacks.  Every
// lane takes the same rotation from the same entries; lane k updates row /
// column entry k of the two rotated rows and columns, so the arithmetic of
// each entry is that of the sequential method.  Stops when the
// off-diagonal mass is below 1e-28 of the whole (at most 100 sweeps).
// n <= PSD_MAX_ORDER (L <= 256 slots, S <= 8).
// ---------------------------------------------------------------------------
constexpr int PSD_MAX_ORDER = 22;
constexpr int PSD_MAX_SWEEPS = 100;
constexpr double PSD_OFF_REL = 1e-28;

// (row, col) of svec slot i of an order-n block
__device__ __forceinline__ void psd_slot_rc(int i, int n, int &row, int &col)
{
    int c = 0, first = 0;
    while (i >= first + (n - c)) {
        first += n - c;
        ++c;
    }
    col = c;
    row = c + (i - first);
}

template <int S>
__device__ void warp_project_psd(WarpSlots<S> &sl, int L, int lane, double *work)
{
    int n = 0;
    while (n * (n + 1) / 2 < L)
        ++n;
    if (n == 1) {
        if (lane == 0)
            sl.x[0] = fmax(sl.x[0], 0.0);
        return;
    }
    bool finite = true;
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (lane + 32 * s < L)
            finite &= isfinite(sl.x[s]) != 0;
    if (!__all_sync(FULL, finite)) { // the reference's failed decomposition gives NaN
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (lane + 32 * s < L)
                sl.x[s] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const double R2 = 1.41421356237309504880, IR2 = 0.70710678118654752440;
    double *A = work, *V = work + n * n;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        if (i < L) {
            int row, col;
            psd_slot_rc(i, n, row, col);
            const double v = row == col ? sl.x[s] : sl.x[s] * IR2;
            A[row * n + col] = v;
            A[col * n + row] = v;
        }
    }
    for (int e = lane; e < n * n; e += 32)
        V[e] = (e / n == e % n) ? 1.0 : 0.0;
    __syncwarp();
    for (int sweep = 0; sweep < PSD_MAX_SWEEPS; ++sweep) {
        double off = 0.0, all = 0.0;
        for (int e = lane; e < n * n; e += 32) {
            const double a2 = A[e] * A[e];
            all += a2;
            if (e / n != e % n)
                off += a2;
        }
        off = warp_sum(off);
        all = warp_sum(all);
        if (!(off > PSD_OFF_REL * all))
            break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[p * n + q];
                if (apq == 0.0)
                    continue;
                const double theta = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
                const double t = fabs(theta) > 1e150
                                     ? 0.5 / theta
                                     : (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
                __syncwarp(); // every lane has read a_pp, a_qq, a_pq
                if (lane < n) { // columns p, q of A and V
                    const int k = lane;
                    const double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - sn * akq;
                    A[k * n + q] = sn * akp + c * akq;
                    const double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - sn * vkq;
                    V[k * n + q] = sn * vkp + c * vkq;
                }
                __syncwarp();
                if (lane < n) { // rows p, q of A
                    const int k = lane;
                    const double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - sn * aqk;
                    A[q * n + k] = sn * apk + c * aqk;
                }
                __syncwarp();
                if (lane == 0) {
                    A[p * n + q] = 0.0;
                    A[q * n + p] = 0.0;
                }
                __syncwarp();
            }
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        if (i < L) {
            int row, col;
            psd_slot_rc(i, n, row, col);
            double v = 0.0;
            for (int e = 0; e < n; ++e)
                v += fmax(A[e * n + e], 0.0) * V[row * n + e] * V[col * n + e];
            sl.x[s] = row == col ? v : v * R2;
        }
    }
    __syncwarp(); // the scratch may be reused by this warp's next projection
}

// PSD blocks of any order ("long" blocks: more slots than a warp's
// registers hold, L > 32 S).  The svec lies in memory (in, L doubles; out
// may alias it); the warp unpacks it into work[0, n^2), runs the same
// cyclic Jacobi as warp_project_psd with every row / column loop strided
// over the lanes, clips and repacks into out.  Callers stage the block's
// candidate in its scratch (after the 2 n^2 doubles of the decomposition)
// and call this instead of the register form.
__device__ __forceinline__ int psd_order(int L)
{
    int n = (int)floor(sqrt(2.0 * L));
    while (n * (n + 1) / 2 < L)
        ++n;
    while (n > 1 && (n - 1) * n / 2 >= L)
        --n;
    return n;
}

// L doubles of candidate staging per long block, after its 2 n^2 doubles
// (the residual stages three vectors, so 3 L are kept)
__host__ __device__ inline long long psd_scratch_doubles(int order, bool is_long)
{
    const long long L = (long long)order * (order + 1) / 2;
    return 2LL * order * order + (is_long ? 3 * L : 0);
}

__device__ void warp_project_psd_mem(const double *in, double *out, int L, int lane, double *work)
{
    const int n = psd_order(L);
    if (n == 1) {
        if (lane == 0)
            out[0] = fmax(in[0], 0.0);
        __syncwarp();
        return;
    }
    bool finite = true;
    for (int i = lane; i < L; i += 32)
        finite &= isfinite(in[i]) != 0;
    if (!__all_sync(FULL, finite)) { // the reference's failed decomposition gives NaN
        for (int i = lane; i < L; i += 32)
            out[i] = __longlong_as_double(0x7ff8000000000000LL);
        __syncwarp();
        return;
    }
    const double R2 = 1.41421356237309504880, IR2 = 0.70710678118654752440;
    double *A = work, *V = work + (size_t)n * n;
    for (int col = 0, first = 0; col < n; first += n - col, ++col)
        for (int row = col + lane; row < n; row += 32) {
            const double x = in[first + row - col];
            const double v = row == col ? x : x * IR2;
            A[(size_t)row * n + col] = v;
            A[(size_t)col * n + row] = v;
        }
    for (long long e = lane; e < (long long)n * n; e += 32)
        V[e] = (e / n == e % n) ? 1.0 : 0.0;
    __syncwarp();
    for (int sweep = 0; sweep < PSD_MAX_SWEEPS; ++sweep) {
        double off = 0.0, all = 0.0;
        for (long long e = lane; e < (long long)n * n; e += 32) {
            const double a2 = A[e] * A[e];
            all += a2;
            if (e / n != e % n)
                off += a2;
        }
        off = warp_sum(off);
        all = warp_sum(all);
        if (!(off > PSD_OFF_REL * all))
            break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[(size_t)p * n + q];
                if (apq == 0.0)
                    continue;
                const double theta = (A[(size_t)q * n + q] - A[(size_t)p * n + p]) / (2.0 * apq);
                const double t = fabs(theta) > 1e150
                                     ? 0.5 / theta
                                     : (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
                __syncwarp(); // every lane has read a_pp, a_qq, a_pq
                for (int k = lane; k < n; k += 32) { // columns p, q of A and V
                    const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * akp - sn * akq;
                    A[(size_t)k * n + q] = sn * akp + c * akq;
                    const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
                    V[(size_t)k * n + p] = c * vkp - sn * vkq;
                    V[(size_t)k * n + q] = sn * vkp + c * vkq;
                }
                __syncwarp();
                for (int k = lane; k < n; k += 32) { // rows p, q of A
                    const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * apk - sn * aqk;
                    A[(size_t)q * n + k] = sn * apk + c * aqk;
                }
                __syncwarp();
                if (lane == 0) {
                    A[(size_t)p * n + q] = 0.0;
                    A[(size_t)q * n + p] = 0.0;
                }
                __syncwarp();
            }
    }
    for (int col = 0, first = 0; col < n; first += n - col, ++col)
        for (int row = col + lane; row < n; row += 32) {
            double v = 0.0;
            for (int e = 0; e < n; ++e)
                v += fmax(A[(size_t)e * n + e], 0.0) * V[(size_t)row * n + e] * V[(size_t)col * n + e];
            out[first + row - col] = row == col ? v : v * R2;
        }
    __syncwarp(); // the scratch and out may be read by other lanes next
}

// Cone kinds an instantiation carries: SOC / RSOC (any S), the 3-slot
// exponential / power cones (S = 1 only; callers route those blocks there)
// and PSD blocks (psd: this block's scratch of 2 n^2 doubles).  Blocks with
// fixed slots (any type but PSD) are a launch class of their own,
// CONES_SECTION, projected by section.cuh.
enum ConeKinds { CONES_WIDE = 1, CONES_THREE = 2, CONES_PSD = 4, CONES_ALL = 7, CONES_SECTION = 8 };

template <int S, int KINDS = CONES_ALL>
__device__ __forceinline__ void warp_project(int type, WarpSlots<S> &sl, int L, int lane, bool uniform_unit,
                                             double *warm, double alpha = 0.0, double *psd = nullptr)
{
    if ((KINDS & CONES_WIDE) && type == 1) // CONE_STANDARD_SOC
        warp_project_soc<S>(sl, L, lane, uniform_unit, warm);
    else if ((KINDS & CONES_WIDE) && type == 0) // CONE_ROTATED_SOC
        warp_project_rsoc<S>(sl, L, lane, uniform_unit, warm);
    else if ((KINDS & CONES_THREE) && S == 1 && (type == 2 || type == 3)) // CONE_EXPONENTIAL, CONE_POWER
        warp_project3<S>(type, sl, lane, alpha);
    else if ((KINDS & CONES_PSD) && type == 4 && psd != nullptr) // CONE_PSD
        warp_project_psd<S>(sl, L, lane, psd);
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
