// mlp.cu -- the learned warm start: a small MLP from a parametric instance's
// parameters theta to a starting point (x, y) and a primal weight.
//
//   h1 = relu(W1 theta + b1)          (hidden)
//   h2 = relu(W2 h1 + b2)             (hidden)
//   z  = W3 h2 + b3                   (rank)      low-rank output head
//   o  = U z + bu                     (out_dim = n + m: x then y, normalised)
//   lw = wp . h2 + bp                 (log primal weight)
//
// Weights W are [out_features x in_features] row-major.  Every product runs
// on the tensor cores (mma.sync m16n8k16, BF16 operands, FP32
// accumulation).  The weights enter as their BF16 copy; FP32 master copies
// take the Adam updates.  Activations and gradients stay FP32: each such
// operand is staged as a BF16 pair hi = bf16(v), lo = bf16(v - hi) (16
// significant bits, ~8e-6 relative) and the products add hi.hi, hi.lo and
// lo.hi, so the network is the BF16-weight, FP32-activation one.  Products with a long reduction and few output tiles (the
// output head's dZ = dO U reduces over all n + m outputs) split K over the
// grid and fold the partial tiles in a fixed order.  The loss of a training
// run is accumulated on the device and read once at the end.  Every kernel
// here (products, bias/ReLU, loss, column sums, Adam) is written for this
// file.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "pdhcg_b200.h"

namespace {

#define MCK(call)                                                                                                      \
    do {                                                                                                               \
        cudaError_t e_ = (call);                                                                                       \
        if (e_ != cudaSuccess) {                                                                                       \
            std::fprintf(stderr, "[pdhcg_b200_mlp] %s: %s\n", #call, cudaGetErrorString(e_));                         \
            return -1;                                                                                                 \
        }                                                                                                              \
    } while (0)

using bf16 = __nv_bfloat16;

__device__ __forceinline__ float ld(const float *p) { return *p; }
__device__ __forceinline__ float ld(const bf16 *p) { return __bfloat162float(*p); }

// C[M x N] = alpha * op(A)[M x K] * op(B)[K x N] + beta * C on the tensor
// cores.  op(A)(i, k) = TA ? A[k * lda + i] : A[i * lda + k];
// op(B)(k, j) = TB ? B[j * ldb + k] : B[k * ldb + j].  A CTA of 4 warps owns
// a 64 x 64 tile and walks K in steps of 32 (its K range is
// [z kchunk, (z + 1) kchunk) for grid index z); each warp owns 32 x 32 as
// 2 x 4 mma tiles of 16 x 8.  Operands are staged in shared memory as BF16,
// FP32 ones as hi / lo pairs; rows of 32 + 8 elements (80 bytes: the
// fragment loads of a warp hit 32 different banks).  With part != NULL the
// CTA writes its FP32 tile to part[z] for splitk_fold_kernel instead of C.
constexpr int TM = 64, TN = 64, TK = 32, TKP = TK + 8;

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2])
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                 "{%8, %9}, {%0, %1, %2, %3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// v into its BF16 pair (hi, lo); a BF16 source is exact in hi alone
__device__ __forceinline__ void split_bf16(float v, bf16 &hi, bf16 &lo)
{
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

template <bool TA, bool TB, typename AT, typename BT>
__global__ void __launch_bounds__(128) mma_gemm_kernel(int M, int N, int K, int kchunk, const AT *A, int lda,
                                                       const BT *B, int ldb, float *C, int ldc, float alpha,
                                                       float beta, float *part)
{
    constexpr bool SA = !std::is_same<AT, bf16>::value, SB = !std::is_same<BT, bf16>::value; // FP32: hi / lo
    __shared__ __align__(16) bf16 As[SA ? 2 : 1][TM][TKP];
    __shared__ __align__(16) bf16 Bs[SB ? 2 : 1][TN][TKP];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int i0 = blockIdx.y * TM, j0 = blockIdx.x * TN;
    const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
    float acc[2][4][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q)
                acc[mt][nt][q] = 0.0f;
    for (int k0 = kb; k0 < ke; k0 += TK) {
        // stage op(A) and op(B)^T, the contiguous index of each source
        // varying fastest across the threads
        for (int e = threadIdx.x; e < TM * TK; e += 128) {
            const int ii = TA ? e % TM : e / TK, kk = TA ? e / TM : e % TK;
            const int i = i0 + ii, k = k0 + kk;
            const float v = (i < M && k < ke) ? ld(TA ? A + (size_t)k * lda + i : A + (size_t)i * lda + k) : 0.0f;
            bf16 hi, lo;
            split_bf16(v, hi, lo);
            As[0][ii][kk] = hi;
            if (SA)
                As[SA ? 1 : 0][ii][kk] = lo;
            const int jj = TB ? e / TK : e % TN, kb2 = TB ? e % TK : e / TN;
            const int j = j0 + jj, k2 = k0 + kb2;
            const float w = (j < N && k2 < ke) ? ld(TB ? B + (size_t)j * ldb + k2 : B + (size_t)k2 * ldb + j) : 0.0f;
            split_bf16(w, hi, lo);
            Bs[0][jj][kb2] = hi;
            if (SB)
                Bs[SB ? 1 : 0][jj][kb2] = lo;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < TK; ks += 16) {
            unsigned a[2][2][4], b[2][4][2]; // [hi / lo][tile][register]
#pragma unroll
            for (int h = 0; h < (SA ? 2 : 1); ++h)
#pragma unroll
                for (int mt = 0; mt < 2; ++mt) {
                    const int r = wm + mt * 16 + g;
                    a[h][mt][0] = *(const unsigned *)&As[h][r][ks + 2 * t];
                    a[h][mt][1] = *(const unsigned *)&As[h][r + 8][ks + 2 * t];
                    a[h][mt][2] = *(const unsigned *)&As[h][r][ks + 2 * t + 8];
                    a[h][mt][3] = *(const unsigned *)&As[h][r + 8][ks + 2 * t + 8];
                }
#pragma unroll
            for (int h = 0; h < (SB ? 2 : 1); ++h)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) {
                    const int c = wn + nt * 8 + g;
                    b[h][nt][0] = *(const unsigned *)&Bs[h][c][ks + 2 * t];
                    b[h][nt][1] = *(const unsigned *)&Bs[h][c][ks + 2 * t + 8];
                }
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) {
                    if (SA) // the small terms first
                        mma_bf16(acc[mt][nt], a[1][mt], b[0][nt]);
                    if (SB)
                        mma_bf16(acc[mt][nt], a[0][mt], b[1][nt]);
                    mma_bf16(acc[mt][nt], a[0][mt], b[0][nt]);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int i = i0 + wm + mt * 16 + g + 8 * (q >> 1), j = j0 + wn + nt * 8 + 2 * t + (q & 1);
                if (i < M && j < N) {
                    const float v = acc[mt][nt][q];
                    if (part)
                        part[((size_t)blockIdx.z * M + i) * N + j] = v;
                    else
                        C[(size_t)i * ldc + j] = beta == 0.0f ? alpha * v : alpha * v + beta * C[(size_t)i * ldc + j];
                }
            }
}

// C = alpha * sum_z part[z] + beta * C, the K slices added in order
__global__ void splitk_fold_kernel(int M, int N, int splits, const float *part, float *C, int ldc, float alpha,
                                   float beta)
{
    const long long MN = (long long)M * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < MN; e += (long long)gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int z = 0; z < splits; ++z)
            s += part[z * MN + e];
        const int i = (int)(e / N), j = (int)(e % N);
        float *c = C + (size_t)i * ldc + j;
        *c = beta == 0.0f ? alpha * s : alpha * s + beta * *c;
    }
}

// split-K workspace of the products (grown on demand, kept with the stream's owner)
struct SplitWs {
    float *p = nullptr;
    size_t cap = 0;
};

template <bool TA, bool TB, typename AT, typename BT>
int gemm(int M, int N, int K, const AT *A, int lda, const BT *B, int ldb, float *C, int ldc, float alpha, float beta,
         cudaStream_t s, SplitWs &ws)
{
    const int gm = (M + TM - 1) / TM, gn = (N + TN - 1) / TN;
    // few output tiles and a long reduction: split K so every SM has a slice
    int splits = 1;
    if (gm * gn < 74 && K >= 4 * TK * 8)
        splits = std::max(1, std::min(148 / (gm * gn), (K + 255) / 256));
    int kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + TK - 1) / TK * TK;
    splits = (K + kchunk - 1) / kchunk;
    if (splits > 1) {
        const size_t need = (size_t)splits * M * N;
        if (need > ws.cap) {
            if (ws.p)
                cudaFree(ws.p);
            ws.p = nullptr;
            ws.cap = 0;
            if (cudaMalloc((void **)&ws.p, need * sizeof(float)) != cudaSuccess)
                return -1;
            ws.cap = need;
        }
        mma_gemm_kernel<TA, TB, AT, BT><<<dim3(gn, gm, splits), 128, 0, s>>>(M, N, K, kchunk, A, lda, B, ldb, C, ldc,
                                                                            alpha, beta, ws.p);
        const long long MN = (long long)M * N;
        splitk_fold_kernel<<<(int)std::min<long long>((MN + 255) / 256, 148 * 8), 256, 0, s>>>(M, N, splits, ws.p, C,
                                                                                              ldc, alpha, beta);
    } else {
        mma_gemm_kernel<TA, TB, AT, BT><<<dim3(gn, gm, 1), 128, 0, s>>>(M, N, K, K, A, lda, B, ldb, C, ldc, alpha,
                                                                       beta, nullptr);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// Y[B x N] += bias, then ReLU if asked
__global__ void bias_act_kernel(int rows, int cols, float *Y, const float *bias, int relu)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)rows * cols;
         e += (long long)gridDim.x * blockDim.x) {
        float v = Y[e] + bias[e % cols];
        Y[e] = relu ? fmaxf(v, 0.0f) : v;
    }
}

// dH *= (H > 0)
__global__ void relu_back_kernel(long long n, float *dH, const float *H)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        if (!(H[e] > 0.0f))
            dH[e] = 0.0f;
}

// out[j] = sum_i Y[i][j] (column sums, rows summed in order)
__global__ void colsum_kernel(int rows, int cols, const float *Y, float *out)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < cols; j += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int i = 0; i < rows; ++i)
            s += Y[(size_t)i * cols + j];
        out[j] = s;
    }
}

// d = 2 (o - t) / (rows * cols); partial sums of (o - t)^2 per block
__global__ void mse_kernel(long long n, const float *o, const float *t, float scale, float *d, double *part)
{
    __shared__ double sh[256];
    double a = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        float r = o[e] - t[e];
        d[e] = 2.0f * r * scale;
        a += (double)r * (double)r;
    }
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        part[blockIdx.x] = sh[0];
}

// acc += (sum of the nb block partials, in order) / tot + the head's loss
__global__ void loss_fold_kernel(const double *part, int nb, double tot, const double *hloss, double *acc)
{
    __shared__ double sh[256];
    double a = 0.0;
    for (int b = threadIdx.x; b < nb; b += 256)
        a += part[b];
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        acc[0] += sh[0] / tot + hloss[0];
}

// log-weight head: lw[b] = wp . h2[b] + bp; dlw = 2 (lw - tl) / B; loss partial
__global__ void head_kernel(int B, int H, const float *h2, const float *wp, const float *bp, const float *tl, float *lw,
                            float *dlw, double *loss)
{
    __shared__ double sh[256];
    double a = 0.0;
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        float s = bp[0];
        for (int k = 0; k < H; ++k)
            s += wp[k] * h2[(size_t)b * H + k];
        lw[b] = s;
        if (tl) {
            float r = s - tl[b];
            dlw[b] = 2.0f * r / (float)B;
            a += (double)r * (double)r;
        }
    }
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        loss[0] = sh[0] / (double)B;
}

// dH2 += dlw (x) wp; gwp[k] = sum_b dlw[b] h2[b][k]; gbp = sum_b dlw[b]
__global__ void head_back_kernel(int B, int H, const float *h2, const float *wp, const float *dlw, float *dH2,
                                 float *gwp, float *gbp)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < H; k += gridDim.x * blockDim.x) {
        float g = 0.0f;
        for (int b = 0; b < B; ++b) {
            g += dlw[b] * h2[(size_t)b * H + k];
            dH2[(size_t)b * H + k] += dlw[b] * wp[k];
        }
        gwp[k] = g;
        if (k == 0) {
            float s = 0.0f;
            for (int b = 0; b < B; ++b)
                s += dlw[b];
            gbp[0] = s;
        }
    }
}

__global__ void to_bf16_kernel(long long n, const float *src, bf16 *dst)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        dst[e] = __float2bfloat16_rn(src[e]);
}

__global__ void adam_kernel(long long n, float *w, const float *g, float *mom, float *vel, float lr, float b1, float b2,
                            float c1, float c2, float eps)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        float gg = g[e];
        float mm = b1 * mom[e] + (1.0f - b1) * gg;
        float vv = b2 * vel[e] + (1.0f - b2) * gg * gg;
        mom[e] = mm;
        vel[e] = vv;
        w[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    }
}

int blocks_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 8); }

} // namespace

// Parameter block offsets (floats) in the packed order
// W1, b1, W2, b2, W3, b3, U, bu, wp, bp.
struct pdhcg_b200_mlp_s {
    int in, hid, rank, out;
    long long off[11], total;
    float *w = nullptr, *g = nullptr, *mom = nullptr, *vel = nullptr; // FP32 master, gradient, Adam
    bf16 *wb = nullptr;                                               // BF16 copy used by the products
    int step = 0;
    int cap = 0;                                                      // activations sized for this batch
    float *X = nullptr, *H1 = nullptr, *H2 = nullptr, *Z = nullptr, *O = nullptr, *LW = nullptr;
    float *T = nullptr, *TL = nullptr, *dO = nullptr, *dZ = nullptr, *dH2 = nullptr, *dH1 = nullptr, *dLW = nullptr;
    double *part = nullptr, *hloss = nullptr;
    double *acc = nullptr; // loss accumulated over the minibatches of a run (device)
    SplitWs ws;
    cudaStream_t s = nullptr;
};

namespace {

enum { P_W1 = 0, P_B1, P_W2, P_B2, P_W3, P_B3, P_U, P_BU, P_WP, P_BP, P_END };

void free_acts(pdhcg_b200_mlp_s *n)
{
    for (float *p : {n->X, n->H1, n->H2, n->Z, n->O, n->LW, n->T, n->TL, n->dO, n->dZ, n->dH2, n->dH1, n->dLW})
        if (p)
            cudaFree(p);
    n->X = n->H1 = n->H2 = n->Z = n->O = n->LW = n->T = n->TL = n->dO = n->dZ = n->dH2 = n->dH1 = n->dLW = nullptr;
    if (n->part)
        cudaFree(n->part);
    if (n->hloss)
        cudaFree(n->hloss);
    if (n->acc)
        cudaFree(n->acc);
    n->part = n->hloss = n->acc = nullptr;
    n->cap = 0;
}

int ensure_acts(pdhcg_b200_mlp_s *n, int B)
{
    if (B <= n->cap)
        return 0;
    free_acts(n);
    auto al = [&](float **p, long long k) { return cudaMalloc((void **)p, std::max<long long>(k, 1) * sizeof(float)); };
    if (al(&n->X, (long long)B * n->in) || al(&n->H1, (long long)B * n->hid) || al(&n->H2, (long long)B * n->hid) ||
        al(&n->Z, (long long)B * n->rank) || al(&n->O, (long long)B * n->out) || al(&n->LW, B) ||
        al(&n->T, (long long)B * n->out) || al(&n->TL, B) || al(&n->dO, (long long)B * n->out) ||
        al(&n->dZ, (long long)B * n->rank) || al(&n->dH2, (long long)B * n->hid) ||
        al(&n->dH1, (long long)B * n->hid) || al(&n->dLW, B) ||
        cudaMalloc((void **)&n->part, 148 * 8 * sizeof(double)) || cudaMalloc((void **)&n->hloss, sizeof(double)) ||
        cudaMalloc((void **)&n->acc, sizeof(double))) {
        std::fprintf(stderr, "[pdhcg_b200_mlp] activation allocation failed.\n");
        return -1;
    }
    n->cap = B;
    return 0;
}

// forward of B rows already in n->X; with targets (T, TL) also the loss and dO, dLW
int forward(pdhcg_b200_mlp_s *n, int B, bool with_loss)
{
    cudaStream_t s = n->s;
    const bf16 *W1 = n->wb + n->off[P_W1], *W2 = n->wb + n->off[P_W2], *W3 = n->wb + n->off[P_W3],
               *U = n->wb + n->off[P_U];
    const float *b1 = n->w + n->off[P_B1], *b2 = n->w + n->off[P_B2], *b3 = n->w + n->off[P_B3],
                *bu = n->w + n->off[P_BU], *wp = n->w + n->off[P_WP], *bp = n->w + n->off[P_BP];
    if (gemm<false, true>(B, n->hid, n->in, n->X, n->in, W1, n->in, n->H1, n->hid, 1.0f, 0.0f, s, n->ws))
        return -1;
    bias_act_kernel<<<blocks_for((long long)B * n->hid), 256, 0, s>>>(B, n->hid, n->H1, b1, 1);
    if (gemm<false, true>(B, n->hid, n->hid, n->H1, n->hid, W2, n->hid, n->H2, n->hid, 1.0f, 0.0f, s, n->ws))
        return -1;
    bias_act_kernel<<<blocks_for((long long)B * n->hid), 256, 0, s>>>(B, n->hid, n->H2, b2, 1);
    if (gemm<false, true>(B, n->rank, n->hid, n->H2, n->hid, W3, n->hid, n->Z, n->rank, 1.0f, 0.0f, s, n->ws))
        return -1;
    bias_act_kernel<<<blocks_for((long long)B * n->rank), 256, 0, s>>>(B, n->rank, n->Z, b3, 0);
    if (gemm<false, true>(B, n->out, n->rank, n->Z, n->rank, U, n->rank, n->O, n->out, 1.0f, 0.0f, s, n->ws))
        return -1;
    bias_act_kernel<<<blocks_for((long long)B * n->out), 256, 0, s>>>(B, n->out, n->O, bu, 0);
    head_kernel<<<1, 256, 0, s>>>(B, n->hid, n->H2, wp, bp, with_loss ? n->TL : nullptr, n->LW, n->dLW, n->hloss);
    if (with_loss) { // the minibatch's loss is added to n->acc on the device (no host wait)
        long long tot = (long long)B * n->out;
        int nb = blocks_for(tot);
        mse_kernel<<<nb, 256, 0, s>>>(tot, n->O, n->T, 1.0f / (float)tot, n->dO, n->part);
        loss_fold_kernel<<<1, 256, 0, s>>>(n->part, nb, (double)tot, n->hloss, n->acc);
    }
    MCK(cudaGetLastError());
    return 0;
}

// gradient of the loss of the last forward (with targets) into n->g
int backward(pdhcg_b200_mlp_s *n, int B)
{
    cudaStream_t s = n->s;
    const bf16 *W2 = n->wb + n->off[P_W2], *W3 = n->wb + n->off[P_W3], *U = n->wb + n->off[P_U];
    const float *wp = n->w + n->off[P_WP];
    float *g = n->g;
    // output head: dU = dO^T Z, dbu = colsum dO, dZ = dO U
    if (gemm<true, false>(n->out, n->rank, B, n->dO, n->out, n->Z, n->rank, g + n->off[P_U], n->rank, 1.0f, 0.0f, s, n->ws))
        return -1;
    colsum_kernel<<<blocks_for(n->out), 256, 0, s>>>(B, n->out, n->dO, g + n->off[P_BU]);
    if (gemm<false, false>(B, n->rank, n->out, n->dO, n->out, U, n->rank, n->dZ, n->rank, 1.0f, 0.0f, s, n->ws))
        return -1;
    // z = W3 h2 + b3
    if (gemm<true, false>(n->rank, n->hid, B, n->dZ, n->rank, n->H2, n->hid, g + n->off[P_W3], n->hid, 1.0f, 0.0f, s, n->ws))
        return -1;
    colsum_kernel<<<blocks_for(n->rank), 256, 0, s>>>(B, n->rank, n->dZ, g + n->off[P_B3]);
    if (gemm<false, false>(B, n->hid, n->rank, n->dZ, n->rank, W3, n->hid, n->dH2, n->hid, 1.0f, 0.0f, s, n->ws))
        return -1;
    // log-weight head
    head_back_kernel<<<blocks_for(n->hid), 256, 0, s>>>(B, n->hid, n->H2, wp, n->dLW, n->dH2, g + n->off[P_WP],
                                                         g + n->off[P_BP]);
    relu_back_kernel<<<blocks_for((long long)B * n->hid), 256, 0, s>>>((long long)B * n->hid, n->dH2, n->H2);
    // h2 = relu(W2 h1 + b2)
    if (gemm<true, false>(n->hid, n->hid, B, n->dH2, n->hid, n->H1, n->hid, g + n->off[P_W2], n->hid, 1.0f, 0.0f, s, n->ws))
        return -1;
    colsum_kernel<<<blocks_for(n->hid), 256, 0, s>>>(B, n->hid, n->dH2, g + n->off[P_B2]);
    if (gemm<false, false>(B, n->hid, n->hid, n->dH2, n->hid, W2, n->hid, n->dH1, n->hid, 1.0f, 0.0f, s, n->ws))
        return -1;
    relu_back_kernel<<<blocks_for((long long)B * n->hid), 256, 0, s>>>((long long)B * n->hid, n->dH1, n->H1);
    // h1 = relu(W1 x + b1)
    if (gemm<true, false>(n->hid, n->in, B, n->dH1, n->hid, n->X, n->in, g + n->off[P_W1], n->in, 1.0f, 0.0f, s, n->ws))
        return -1;
    colsum_kernel<<<blocks_for(n->hid), 256, 0, s>>>(B, n->hid, n->dH1, g + n->off[P_B1]);
    MCK(cudaGetLastError());
    return 0;
}

int refresh_bf16(pdhcg_b200_mlp_s *n)
{
    to_bf16_kernel<<<blocks_for(n->total), 256, 0, n->s>>>(n->total, n->w, n->wb);
    MCK(cudaGetLastError());
    return 0;
}

// splitmix64 -> uniform in [-1, 1)
double unif(unsigned long long &st)
{
    unsigned long long z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

} // namespace

extern "C" {

pdhcg_b200_mlp_t *pdhcg_b200_mlp_create(int in_dim, int hidden, int rank, int out_dim, unsigned long long seed)
{
    if (in_dim <= 0 || hidden <= 0 || rank <= 0 || out_dim <= 0) {
        std::fprintf(stderr, "[pdhcg_b200_mlp_create] invalid sizes.\n");
        return nullptr;
    }
    auto *n = new pdhcg_b200_mlp_s();
    n->in = in_dim;
    n->hid = hidden;
    n->rank = rank;
    n->out = out_dim;
    long long sz[P_END] = {(long long)hidden * in_dim, hidden, (long long)hidden * hidden, hidden,
                           (long long)rank * hidden, rank, (long long)out_dim * rank, out_dim, hidden, 1};
    long long o = 0;
    for (int i = 0; i < P_END; ++i) {
        n->off[i] = o;
        o += sz[i];
    }
    n->off[P_END] = o;
    n->total = o;
    // He-uniform weights for the ReLU layers, Glorot-uniform for the linear heads, zero biases
    std::vector<float> h(o, 0.0f);
    unsigned long long st = seed;
    auto fill = [&](int p, int fan_in, int fan_out, bool relu) {
        double a = relu ? std::sqrt(6.0 / fan_in) : std::sqrt(6.0 / (fan_in + fan_out));
        for (long long k = n->off[p]; k < n->off[p + 1]; ++k)
            h[k] = (float)(a * unif(st));
    };
    fill(P_W1, in_dim, hidden, true);
    fill(P_W2, hidden, hidden, true);
    fill(P_W3, hidden, rank, false);
    fill(P_U, rank, out_dim, false);
    fill(P_WP, hidden, 1, false);
    if (cudaStreamCreateWithFlags(&n->s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc((void **)&n->w, o * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&n->g, o * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&n->mom, o * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&n->vel, o * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&n->wb, o * sizeof(bf16)) != cudaSuccess ||
        cudaMemcpy(n->w, h.data(), o * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(n->mom, 0, o * sizeof(float)) != cudaSuccess ||
        cudaMemset(n->vel, 0, o * sizeof(float)) != cudaSuccess || refresh_bf16(n) != 0) {
        std::fprintf(stderr, "[pdhcg_b200_mlp_create] device allocation failed.\n");
        pdhcg_b200_mlp_free(n);
        return nullptr;
    }
    return n;
}

void pdhcg_b200_mlp_free(pdhcg_b200_mlp_t *n)
{
    if (!n)
        return;
    free_acts(n);
    if (n->ws.p)
        cudaFree(n->ws.p);
    for (void *p : {(void *)n->w, (void *)n->g, (void *)n->mom, (void *)n->vel, (void *)n->wb})
        if (p)
            cudaFree(p);
    if (n->s)
        cudaStreamDestroy(n->s);
    delete n;
}

long long pdhcg_b200_mlp_num_params(const pdhcg_b200_mlp_t *n) { return n ? n->total : -1; }

int pdhcg_b200_mlp_get_params(const pdhcg_b200_mlp_t *n, float *out)
{
    if (!n || !out)
        return -1;
    MCK(cudaMemcpy(out, n->w, n->total * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

int pdhcg_b200_mlp_set_params(pdhcg_b200_mlp_t *n, const float *in)
{
    if (!n || !in)
        return -1;
    MCK(cudaMemcpy(n->w, in, n->total * sizeof(float), cudaMemcpyHostToDevice));
    n->step = 0;
    MCK(cudaMemset(n->mom, 0, n->total * sizeof(float)));
    MCK(cudaMemset(n->vel, 0, n->total * sizeof(float)));
    return refresh_bf16(n);
}

int pdhcg_b200_mlp_predict(pdhcg_b200_mlp_t *n, int batch, const float *theta, float *out, float *logw)
{
    if (!n || batch <= 0 || !theta || !out)
        return -1;
    if (ensure_acts(n, batch))
        return -1;
    MCK(cudaMemcpyAsync(n->X, theta, (size_t)batch * n->in * sizeof(float), cudaMemcpyHostToDevice, n->s));
    if (forward(n, batch, false))
        return -1;
    MCK(cudaMemcpyAsync(out, n->O, (size_t)batch * n->out * sizeof(float), cudaMemcpyDeviceToHost, n->s));
    if (logw)
        MCK(cudaMemcpyAsync(logw, n->LW, batch * sizeof(float), cudaMemcpyDeviceToHost, n->s));
    MCK(cudaStreamSynchronize(n->s));
    return 0;
}

int pdhcg_b200_mlp_loss_grad(pdhcg_b200_mlp_t *n, int batch, const float *theta, const float *target,
                             const float *target_logw, double *loss, float *grad)
{
    if (!n || batch <= 0 || !theta || !target || !target_logw || !loss)
        return -1;
    if (ensure_acts(n, batch))
        return -1;
    MCK(cudaMemcpyAsync(n->X, theta, (size_t)batch * n->in * sizeof(float), cudaMemcpyHostToDevice, n->s));
    MCK(cudaMemcpyAsync(n->T, target, (size_t)batch * n->out * sizeof(float), cudaMemcpyHostToDevice, n->s));
    MCK(cudaMemcpyAsync(n->TL, target_logw, batch * sizeof(float), cudaMemcpyHostToDevice, n->s));
    MCK(cudaMemsetAsync(n->acc, 0, sizeof(double), n->s));
    if (forward(n, batch, true) || backward(n, batch))
        return -1;
    if (grad)
        MCK(cudaMemcpyAsync(grad, n->g, n->total * sizeof(float), cudaMemcpyDeviceToHost, n->s));
    MCK(cudaMemcpyAsync(loss, n->acc, sizeof(double), cudaMemcpyDeviceToHost, n->s));
    MCK(cudaStreamSynchronize(n->s));
    return 0;
}

int pdhcg_b200_mlp_train(pdhcg_b200_mlp_t *n, int count, const float *theta, const float *target,
                         const float *target_logw, int epochs, int batch, float lr, double *loss)
{
    if (!n || count <= 0 || batch <= 0 || !theta || !target || !target_logw)
        return -1;
    batch = std::min(batch, count);
    if (ensure_acts(n, batch))
        return -1;
    // the whole training set on the device once
    float *dth = nullptr, *dt = nullptr, *dtl = nullptr;
    MCK(cudaMalloc((void **)&dth, (size_t)count * n->in * sizeof(float)));
    MCK(cudaMalloc((void **)&dt, (size_t)count * n->out * sizeof(float)));
    MCK(cudaMalloc((void **)&dtl, count * sizeof(float)));
    MCK(cudaMemcpy(dth, theta, (size_t)count * n->in * sizeof(float), cudaMemcpyHostToDevice));
    MCK(cudaMemcpy(dt, target, (size_t)count * n->out * sizeof(float), cudaMemcpyHostToDevice));
    MCK(cudaMemcpy(dtl, target_logw, count * sizeof(float), cudaMemcpyHostToDevice));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    int rc = 0, nbat = 0;
    for (int ep = 0; ep < epochs && rc == 0; ++ep) {
        // the last epoch's mean minibatch loss is read once, after the run
        if (cudaMemsetAsync(n->acc, 0, sizeof(double), n->s) != cudaSuccess)
            rc = -1;
        nbat = 0;
        for (int b0 = 0; b0 + batch <= count && rc == 0; b0 += batch, ++nbat) { // full minibatches in order
            cudaMemcpyAsync(n->X, dth + (size_t)b0 * n->in, (size_t)batch * n->in * sizeof(float),
                            cudaMemcpyDeviceToDevice, n->s);
            cudaMemcpyAsync(n->T, dt + (size_t)b0 * n->out, (size_t)batch * n->out * sizeof(float),
                            cudaMemcpyDeviceToDevice, n->s);
            cudaMemcpyAsync(n->TL, dtl + b0, batch * sizeof(float), cudaMemcpyDeviceToDevice, n->s);
            rc = forward(n, batch, true);
            if (rc == 0)
                rc = backward(n, batch);
            if (rc == 0) {
                ++n->step;
                float c1 = 1.0f - std::pow(b1, (float)n->step), c2 = 1.0f - std::pow(b2, (float)n->step);
                adam_kernel<<<blocks_for(n->total), 256, 0, n->s>>>(n->total, n->w, n->g, n->mom, n->vel, lr, b1, b2,
                                                                    c1, c2, eps);
                rc = refresh_bf16(n);
            }
        }
    }
    double acc = 0.0;
    const cudaError_t e1 = cudaMemcpyAsync(&acc, n->acc, sizeof(double), cudaMemcpyDeviceToHost, n->s);
    const cudaError_t e2 = cudaStreamSynchronize(n->s);
    cudaFree(dth);
    cudaFree(dt);
    cudaFree(dtl);
    if (e1 != cudaSuccess || e2 != cudaSuccess)
        rc = -1;
    if (loss)
        *loss = nbat > 0 ? acc / nbat : 0.0;
    return rc;
}

} // extern "C"
