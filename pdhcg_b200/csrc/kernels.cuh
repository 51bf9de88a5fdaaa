// kernels.cuh -- the hot kernels of one PDHCG-B200 iteration.
//
// Layout in HBM (one solve, n variables, m rows):
//   A  : CSR, int32 row_ptr[m+1], int32 col[nnz], values T[nnz]
//   At : CSR of A^T (n rows), built on the device by a stable sort so each
//        row lists its entries in increasing row index (what the
//        reference's csr2csc produces, src/solver_state.cu:739-770)
//   vectors: problem data (c, bounds, diagonal Q, rescaling) and iterates
//        (x_init, x_cur, x_pdhg, x_refl; y_init, y_cur, y_pdhg), all of
//        storage type T.
// T = double is the plain FP64 iteration; T = float is the mixed-precision
// bulk phase: every load is widened to double, products are accumulated and
// the prox / projection arithmetic is done in double, and only the stores
// are rounded to FP32.
//
// One iteration (reference pdhg_update + halpern_update,
// src/pdhg_core_op.cu:705-845) is two launches:
//   primal_free_kernel / primal_cone_kernel : A^T y by row groups, diagonal-Q
//        prox, box clamp, cone projection (one warp per cone block), the
//        reflection and the Halpern average of x, all in registers
//   dual_kernel : A x_refl, dual prox, reflection and Halpern average of y
// Both are HBM-bandwidth bound: every matrix byte and every streamed vector
// byte is read once per iteration; the gathered vectors (y, x_refl) stay in
// L2.
#pragma once

#include "device.cuh"
#include "section.cuh"

namespace pdhcg {

constexpr int TPB = 256;
constexpr int WARPS = TPB / 32;

// Per-iteration parameters of the step kernels (passed by value).
struct StepParams {
    double tau, sigma; // primal / dual step sizes
    double w;          // Halpern weight (k+1)/(k+2)
    double rho;        // reflection coefficient
    int store_primal;  // write x_pdhg (and LP dual slack)
    int store_dual;    // write y_pdhg
    int want_fpe;      // write x_refl - x_cur into dx, y_refl - y_cur into dy
    int lp_slack;      // NON_Q: store (p - t)/tau in dual_slack
    int cone_box;      // some cone slot has a finite box bound (|bound| >= 1e30 passes validation)
};

template <typename T>
struct StepData {
    int n, m;
    const int *A_rp, *A_ci;
    const T *A_v;
    const int *At_rp, *At_ci;
    const T *At_v;
    const T *c, *l, *u, *q;
    const T *lc, *uc, *g;
    const T *vr; // variable rescaling (cone metric)
    const int *free_idx;
    int n_free; // variables outside cones (NULL: all)
    // the free variables as tiles of <= 32 consecutive rows {first, count}
    // (NULL: rows [32 t, 32 t + 32) of all n variables)
    const int2 *free_tiles;
    int n_free_tiles;
    const int *cone_start, *cone_len, *cone_type;
    const double *cone_alpha; // power-cone exponents (NULL: none)
    int n_cones;
    double *cone_warm; // per-cone multiplier warm start (may be NULL)
    // slots fixed by set_cone_fixed (NULL: none): mask over the variables
    const unsigned char *fixed;
    T *x0, *x, *xp, *xr, *dx, *dual_slack;
    T *y0, *y, *yp, *dy;
    LongRows A_long, At_long; // long rows of A (pass over x_refl) and of A^T (pass over y)
    double *psd_work;         // PSD blocks' projection scratch (NULL: no PSD blocks)
    const long long *psd_off; // per cone block: offset of its scratch in psd_work
    // affine cones F x + g in K over blocks of rows: the rows outside them as
    // tiles of <= 32 consecutive rows {first, count} (NULL: all rows in tiles
    // of 32), and the blocks themselves (projected with d = 1 / cr)
    const int2 *row_tiles;
    int n_row_tiles;
    const int *aff_start, *aff_len, *aff_type;
    const double *aff_alpha;
    const long long *aff_psd_off; // PSD scratch offsets of the affine blocks
    int n_aff;
    const double *cr; // constraint rescaling
};

// The step kernels are written as warp bodies (one tile or one cone block per
// call) so that the launch shape is chosen in one place; every body takes
// its warp's STREAM_CHUNK-double shared staging buffer.  The loads of each
// lane's own vector entries are issued before the row products, so they are
// in flight together with the matrix stream.

// Variables outside cones: one tile of <= 32 consecutive rows of A^T:
// A^T y by stream-mode products, then the prox step, box clamp, reflection
// and Halpern average of each row's variable in its lane.
template <typename T, bool HAS_Q, bool HAS_BOX>
__device__ __forceinline__ void primal_free_tile(const StepData<T> &D, const StepParams &P, int r0, int nr, int lane,
                                                 double *stage)
{
    const bool own = lane < nr;
    const int j = r0 + (own ? lane : 0);
    double xi = 0.0, c = 0.0, q = 0.0, lo = 0.0, hi = 0.0, x0 = 0.0;
    if (own) {
        xi = D.x[j];
        c = D.c[j];
        x0 = D.x0[j];
        if (HAS_Q)
            q = D.q[j];
        if (HAS_BOX) {
            lo = D.l[j];
            hi = D.u[j];
        }
    }
    double aty[1];
    warp_stream_rows<1>(D.At_rp, D.At_ci, D.At_v, D.y, r0, nr, lane, stage, aty, D.At_long);
    if (own) {
        double t = xi - P.tau * (c - aty[0]);
        if (HAS_Q)
            t /= (1.0 + P.tau * q);
        double p = HAS_BOX ? clampd(lo, t, hi) : t;
        double xr = 2.0 * p - xi;
        D.xr[j] = (T)xr;
        if (P.store_primal) {
            D.xp[j] = (T)p;
            if (P.lp_slack)
                D.dual_slack[j] = (T)((p - t) / P.tau);
        }
        if (P.want_fpe)
            D.dx[j] = (T)(xr - xi);
        double refl = P.rho * xr + (1.0 - P.rho) * xi;
        D.x[j] = (T)(P.w * refl + (1.0 - P.w) * x0);
    }
}

template <typename T, bool HAS_Q, bool HAS_BOX>
__global__ void __launch_bounds__(TPB) primal_free_kernel(StepData<T> D, StepParams P)
{
    __shared__ double stage_all[WARPS][STREAM_CHUNK];
    const int lane = threadIdx.x & 31;
    double *stage = stage_all[threadIdx.x >> 5];
    const int ntiles = D.free_tiles ? D.n_free_tiles : (D.n + 31) / 32;
    for (int t = blockIdx.x * WARPS + (threadIdx.x >> 5); t < ntiles; t += gridDim.x * WARPS) {
        int r0, nr;
        if (D.free_tiles) {
            const int2 ft = D.free_tiles[t];
            r0 = ft.x;
            nr = ft.y;
        } else {
            r0 = 32 * t;
            nr = min(32, D.n - r0);
        }
        primal_free_tile<T, HAS_Q, HAS_BOX>(D, P, r0, nr, lane, stage);
    }
}

// One cone block [st, st + L): A^T y for the block's rows by stream-mode
// products, the prox candidate of every slot, then the projection onto the
// cone in the (1 + tau q) d^2 metric (diagonal Q) or d^2 metric (LP).
template <int S, typename T, bool HAS_Q, int KINDS>
__device__ __forceinline__ void primal_cone_block(const StepData<T> &D, const StepParams &P, int cb, int lane,
                                                  double *stage)
{
    const int st = D.cone_start[cb], L = D.cone_len[cb], type = D.cone_type[cb];
    WarpSlots<S> sl;
    double xi[S], cc[S], x0[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        sl.x[s] = 0.0;
        sl.d[s] = 1.0;
        sl.w[s] = 1.0;
        xi[s] = cc[s] = x0[s] = 0.0;
        if (i < L) {
            const int j = st + i;
            xi[s] = D.x[j];
            cc[s] = D.c[j];
            x0[s] = D.x0[j];
            sl.d[s] = D.vr[j];
            if (HAS_Q)
                sl.w[s] = 1.0 + P.tau * (double)D.q[j];
        }
    }
    double aty[S];
    warp_stream_rows<S>(D.At_rp, D.At_ci, D.At_v, D.y, st, L, lane, stage, aty, D.At_long);
    double tt[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        tt[s] = 0.0;
        if (i < L) {
            const int j = st + i;
            double t = xi[s] - P.tau * (cc[s] - aty[s]);
            if (HAS_Q)
                t /= sl.w[s];
            tt[s] = t;
            sl.x[s] = P.cone_box ? clampd(D.l[j], t, D.u[j]) : t;
        }
    }
    // LP dual slack of the box step is recorded before the cone projection
    // (reference compute_lp_next_pdhg_primal_solution_major_kernel then
    // project_cone_runtime, src/pdhg_core_op.cu:426-455, 729-735)
    if (P.lp_slack) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int i = lane + 32 * s;
            if (i < L)
                D.dual_slack[st + i] = (T)((sl.x[s] - tt[s]) / P.tau);
        }
    }
    if constexpr ((KINDS & CONES_SECTION) != 0) { // blocks with fixed slots
        const unsigned fb = section_bits<S>(D.fixed, st, L, lane);
        warp_section_project<S>(type, sl, L, lane, fb, D.cone_warm ? D.cone_warm + cb : nullptr,
                                D.cone_alpha ? D.cone_alpha[cb] : 0.0);
    } else {
        bool uni = warp_uniform_unit<S>(sl, L, lane);
        warp_project<S, KINDS>(type, sl, L, lane, uni, D.cone_warm ? D.cone_warm + cb : nullptr,
                               D.cone_alpha ? D.cone_alpha[cb] : 0.0,
                               D.psd_work ? D.psd_work + D.psd_off[cb] : nullptr);
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        if (i < L) {
            const int j = st + i;
            double p = sl.x[s];
            double xr = 2.0 * p - xi[s];
            D.xr[j] = (T)xr;
            D.xp[j] = (T)p; // cones force the pdhg store (reference :428, :460)
            if (P.want_fpe)
                D.dx[j] = (T)(xr - xi[s]);
            double refl = P.rho * xr + (1.0 - P.rho) * xi[s];
            D.x[j] = (T)(P.w * refl + (1.0 - P.w) * x0[s]);
        }
    }
}

// A PSD block longer than the warp's registers hold (L > 32 S): the same
// step with the candidate staged in the block's scratch.  Chunks of 32 S
// rows of A^T y and prox, the projection in memory, then the reflection and
// Halpern average slot by slot.
template <int S, typename T, bool HAS_Q>
__device__ __noinline__ void primal_psd_long_block(const StepData<T> &D, const StepParams &P, int cb, int lane,
                                                   double *stage)
{
    const int st = D.cone_start[cb], L = D.cone_len[cb];
    const int n = psd_order(L);
    double *work = D.psd_work + D.psd_off[cb];
    double *sv = work + 2LL * n * n;
    for (int c0 = 0; c0 < L; c0 += 32 * S) {
        const int nr = min(32 * S, L - c0);
        double aty[S];
        warp_stream_rows<S>(D.At_rp, D.At_ci, D.At_v, D.y, st + c0, nr, lane, stage, aty, D.At_long);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int i = lane + 32 * s;
            if (i < nr) {
                const int j = st + c0 + i;
                double t = (double)D.x[j] - P.tau * ((double)D.c[j] - aty[s]);
                if (HAS_Q)
                    t /= 1.0 + P.tau * (double)D.q[j];
                const double xc = P.cone_box ? clampd(D.l[j], t, D.u[j]) : t;
                if (P.lp_slack)
                    D.dual_slack[j] = (T)((xc - t) / P.tau);
                sv[c0 + i] = xc;
            }
        }
    }
    __syncwarp();
    warp_project_psd_mem(sv, sv, L, lane, work);
    for (int i = lane; i < L; i += 32) {
        const int j = st + i;
        const double xi = D.x[j], p = sv[i];
        const double xr = 2.0 * p - xi;
        D.xr[j] = (T)xr;
        D.xp[j] = (T)p;
        if (P.want_fpe)
            D.dx[j] = (T)(xr - xi);
        const double refl = P.rho * xr + (1.0 - P.rho) * xi;
        D.x[j] = (T)(P.w * refl + (1.0 - P.w) * (double)D.x0[j]);
    }
    __syncwarp();
}

// One warp per cone block of the list ids (NULL: blocks 0 .. nids - 1);
// KINDS = CONES_WIDE for SOC / RSOC blocks, CONES_THREE (S = 1) for the
// 3-slot exponential and power blocks, CONES_PSD for PSD blocks (those
// longer than 32 S slots through their scratch).
template <int S, typename T, bool HAS_Q, int KINDS>
__global__ void __launch_bounds__(TPB) primal_cone_kernel(StepData<T> D, StepParams P, const int *ids, int nids)
{
    __shared__ double stage_all[WARPS][STREAM_CHUNK];
    const int lane = threadIdx.x & 31;
    const int warp = blockIdx.x * WARPS + (threadIdx.x >> 5);
    const int nwarps = gridDim.x * WARPS;
    double *stage = stage_all[threadIdx.x >> 5];
    for (int i = warp; i < nids; i += nwarps) {
        const int cb = ids ? ids[i] : i;
        if constexpr ((KINDS & CONES_PSD) != 0) {
            if (D.cone_len[cb] > 32 * S) {
                primal_psd_long_block<S, T, HAS_Q>(D, P, cb, lane, stage);
                continue;
            }
        }
        primal_cone_block<S, T, HAS_Q, KINDS>(D, P, cb, lane, stage);
    }
}

// One tile of 32 consecutive rows of A: A x_refl by stream-mode products,
// then the dual prox, reflection and Halpern average of y.
template <typename T, bool EQ_ROWS, bool HAS_G>
__device__ __forceinline__ void dual_tile(const StepData<T> &D, const StepParams &P, int r0, int nr, int lane,
                                          double *stage)
{
    const bool own = lane < nr;
    const int i = r0 + (own ? lane : 0);
    double yi = 0.0, y0 = 0.0, lc = 0.0, uc = 0.0, g = 0.0;
    if (own) {
        yi = D.y[i];
        y0 = D.y0[i];
        lc = D.lc[i];
        if (!EQ_ROWS)
            uc = D.uc[i];
        if (HAS_G)
            g = D.g[i];
    }
    double axr[1];
    warp_stream_rows<1>(D.A_rp, D.A_ci, D.A_v, D.xr, r0, nr, lane, stage, axr, D.A_long);
    if (own) {
        double v = HAS_G ? axr[0] + g : axr[0];
        double pr = EQ_ROWS ? lc : clampd(lc, v - yi / P.sigma, uc);
        double yn = yi - P.sigma * v + P.sigma * pr;
        if (P.store_dual)
            D.yp[i] = (T)yn;
        double yr = 2.0 * yn - yi;
        if (P.want_fpe)
            D.dy[i] = (T)(yr - yi);
        double refl = P.rho * yr + (1.0 - P.rho) * yi;
        D.y[i] = (T)(P.w * refl + (1.0 - P.w) * y0);
    }
}

template <typename T, bool EQ_ROWS, bool HAS_G>
__global__ void __launch_bounds__(TPB) dual_kernel(StepData<T> D, StepParams P)
{
    __shared__ double stage_all[WARPS][STREAM_CHUNK];
    const int lane = threadIdx.x & 31;
    double *stage = stage_all[threadIdx.x >> 5];
    const int ntiles = D.row_tiles ? D.n_row_tiles : (D.m + 31) / 32;
    for (int t = blockIdx.x * WARPS + (threadIdx.x >> 5); t < ntiles; t += gridDim.x * WARPS) {
        if (D.row_tiles) {
            const int2 rt = D.row_tiles[t];
            dual_tile<T, EQ_ROWS, HAS_G>(D, P, rt.x, rt.y, lane, stage);
        } else {
            const int r0 = 32 * t;
            dual_tile<T, EQ_ROWS, HAS_G>(D, P, r0, min(32, D.m - r0), lane, stage);
        }
    }
}

// One affine cone block of rows (reference pdhg_update with affine cones,
// src/pdhg_core_op.cu:810-829): A x_refl + g over the block's rows, the
// clamped point v - y / sigma projected onto the cone (unit metric of the
// scaled space, K on v / d with d = 1 / cr), then the dual update,
// reflection and Halpern average of the other rows.
template <int S, typename T>
__device__ __forceinline__ void dual_cone_block(const StepData<T> &D, const StepParams &P, int ab, int lane,
                                                double *stage)
{
    const int st = D.aff_start[ab], L = D.aff_len[ab], type = D.aff_type[ab];
    WarpSlots<S> sl;
    double yi[S], y0[S], gv[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        sl.x[s] = 0.0;
        sl.d[s] = 1.0;
        sl.w[s] = 1.0;
        yi[s] = y0[s] = gv[s] = 0.0;
        if (i < L) {
            const int j = st + i;
            yi[s] = D.y[j];
            y0[s] = D.y0[j];
            gv[s] = D.g ? (double)D.g[j] : 0.0;
            sl.d[s] = 1.0 / D.cr[j];
        }
    }
    double axr[S];
    warp_stream_rows<S>(D.A_rp, D.A_ci, D.A_v, D.xr, st, L, lane, stage, axr, D.A_long);
    double vv[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        vv[s] = axr[s] + gv[s];
        if (i < L) {
            const int j = st + i;
            sl.x[s] = clampd(D.lc[j], vv[s] - yi[s] / P.sigma, D.uc[j]);
        }
    }
    const bool uni = warp_uniform_unit<S>(sl, L, lane);
    warp_project<S>(type, sl, L, lane, uni, nullptr, D.aff_alpha ? D.aff_alpha[ab] : 0.0,
                    D.psd_work ? D.psd_work + D.aff_psd_off[ab] : nullptr);
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int i = lane + 32 * s;
        if (i < L) {
            const int j = st + i;
            const double yn = yi[s] - P.sigma * vv[s] + P.sigma * sl.x[s];
            if (P.store_dual)
                D.yp[j] = (T)yn;
            const double yr = 2.0 * yn - yi[s];
            if (P.want_fpe)
                D.dy[j] = (T)(yr - yi[s]);
            const double refl = P.rho * yr + (1.0 - P.rho) * yi[s];
            D.y[j] = (T)(P.w * refl + (1.0 - P.w) * y0[s]);
        }
    }
}

// One warp per affine cone block; 3-slot blocks (exponential, power) take
// the one-slot instantiation, which alone carries their projection.
template <int S, typename T>
__global__ void __launch_bounds__(TPB) dual_cone_kernel(StepData<T> D, StepParams P)
{
    __shared__ double stage_all[WARPS][STREAM_CHUNK];
    const int lane = threadIdx.x & 31;
    double *stage = stage_all[threadIdx.x >> 5];
    for (int ab = blockIdx.x * WARPS + (threadIdx.x >> 5); ab < D.n_aff; ab += gridDim.x * WARPS) {
        const int t = D.aff_type[ab];
        if (S > 1 && (t == 2 || t == 3))
            dual_cone_block<1, T>(D, P, ab, lane, stage);
        else
            dual_cone_block<S, T>(D, P, ab, lane, stage);
    }
}

// ---------------------------------------------------------------------------
// Deterministic reductions: each block writes NS partial values; a one-block
// kernel folds them in a fixed order.
// ---------------------------------------------------------------------------
enum ReduceOp { RSUM = 0, RMAX = 1 };

template <int NS>
__device__ __forceinline__ void block_reduce_store(double (&v)[NS], const int (&op)[NS], double *partials)
{
    __shared__ double sh[WARPS][NS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        double t = op[s] == RMAX ? warp_max(v[s]) : warp_sum(v[s]);
        if (lane == 0)
            sh[wid][s] = t;
    }
    __syncthreads();
    if (threadIdx.x < NS) {
        int s = threadIdx.x;
        double acc = sh[0][s];
        for (int w = 1; w < WARPS; ++w)
            acc = op[s] == RMAX ? fmax(acc, sh[w][s]) : acc + sh[w][s];
        partials[(size_t)blockIdx.x * NS + s] = acc;
    }
    __syncthreads();
}

// out[s] = fold over blocks of partials[b*NS+s]; one block of TPB threads.
__global__ void fold_partials_kernel(const double *partials, int nblocks, int ns, const int *ops, double *out)
{
    __shared__ double sh[TPB];
    for (int s = 0; s < ns; ++s) {
        int op = ops[s];
        double acc = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += TPB) {
            double v = partials[(size_t)b * ns + s];
            acc = op == RMAX ? fmax(acc, v) : acc + v;
        }
        sh[threadIdx.x] = acc;
        __syncthreads();
        for (int o = TPB / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o)
                sh[threadIdx.x] = op == RMAX ? fmax(sh[threadIdx.x], sh[threadIdx.x + o])
                                             : sh[threadIdx.x] + sh[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            out[s] = sh[0];
        __syncthreads();
    }
}

// y = M x, one warp per tile of 32 rows (stream-mode products); lr: M's
// long rows with the segment pass over this x done (or none)
__global__ void __launch_bounds__(TPB) spmv_kernel(int rows, const int *rp, const int *ci, const double *v,
                                                   const double *x, double *y, LongRows lr)
{
    __shared__ double stage_all[WARPS][STREAM_CHUNK];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int ntiles = (rows + 31) / 32;
    for (int tile = blockIdx.x * WARPS + wib; tile < ntiles; tile += gridDim.x * WARPS) {
        const int r0 = 32 * tile, nr = min(32, rows - r0);
        double a[1];
        warp_stream_rows<1>(rp, ci, v, x, r0, nr, lane, stage_all[wib], a, lr);
        if (lane < nr)
            y[r0 + lane] = a[0];
    }
}

__global__ void cone_len_kernel(int nc, const int *vdim, const int *type, int *len)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nc; b += gridDim.x * blockDim.x) {
        int t = type[b], v = vdim[b];
        len[b] = (t == 2 || t == 3) ? 3 : (t == 4 ? v * (v + 1) / 2 : v + 2);
    }
}

// element-wise precision conversion (phase switch of the mixed solve)
template <typename A, typename B>
__global__ void convert_kernel(const A *src, B *dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (B)src[i];
}

} // namespace pdhcg
