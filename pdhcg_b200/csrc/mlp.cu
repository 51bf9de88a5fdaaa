// mlp.cu -- the learned warm start: a small MLP from a parametric instance's
// parameters theta to a starting point (x, y) and a primal weight.
//
//   h1 = relu(W1 theta + b1)          (hidden)
//   h2 = relu(W2 h1 + b2)             (hidden)
//   z  = W3 h2 + b3                   (rank)      low-rank output head
//   o  = U z + bu                     (out_dim = n + m: x then y, normalised)
//   lw = wp . h2 + bp                 (log primal weight)
//
// Weights W are [out_features x in_features] row-major.  The products use
// BF16 copies of the weights with FP32 accumulation; FP32 master copies take
// the Adam updates.  Activations and gradients are FP32.  Every kernel here
// (products, bias/ReLU, loss, column sums, Adam) is written for this file;
// the products are tiled FP32-accumulate CUDA-core kernels: at these shapes
// (a batch of 64 against 512-wide layers and a rank-64 head) a step is a few
// microseconds of arithmetic and is bound by launch latency.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
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

// C[M x N] = alpha * op(A)[M x K] * op(B)[K x N] + beta * C, FP32 accumulation.
// op(A)(i, k) = TA ? A[k * lda + i] : A[i * lda + k]; op(B)(k, j) = TB ? B[j * ldb + k] : B[k * ldb + j].
// 64 x 64 tiles, 256 threads, 4 x 4 outputs per thread, K in steps of 16.
constexpr int GT = 64, GK = 16;
template <bool TA, bool TB, typename AT, typename BT>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const AT *A, int lda, const BT *B, int ldb,
                                                   float *C, int ldc, float alpha, float beta)
{
    __shared__ float As[GK][GT + 1];
    __shared__ float Bs[GK][GT + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int i0 = blockIdx.y * GT, j0 = blockIdx.x * GT;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += GK) {
        for (int e = threadIdx.x; e < GK * GT; e += 256) {
            int kk = e / GT, ii = e % GT;
            int i = i0 + ii, k = k0 + kk;
            As[kk][ii] = (i < M && k < K) ? ld(TA ? A + (size_t)k * lda + i : A + (size_t)i * lda + k) : 0.0f;
            int j = j0 + ii;
            Bs[kk][ii] = (j < N && k < K) ? ld(TB ? B + (size_t)j * ldb + k : B + (size_t)k * ldb + j) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                a[r] = As[kk][ty * 4 + r];
                b[r] = Bs[kk][tx * 4 + r];
            }
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    acc[r][q] = fmaf(a[r], b[q], acc[r][q]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int i = i0 + ty * 4 + r, j = j0 + tx * 4 + q;
            if (i < M && j < N) {
                float v = alpha * acc[r][q];
                C[(size_t)i * ldc + j] = beta == 0.0f ? v : v + beta * C[(size_t)i * ldc + j];
            }
        }
}

template <bool TA, bool TB, typename AT, typename BT>
void gemm(int M, int N, int K, const AT *A, int lda, const BT *B, int ldb, float *C, int ldc, float alpha, float beta,
          cudaStream_t s)
{
    dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT);
    gemm_kernel<TA, TB, AT, BT><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta);
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
    n->part = n->hloss = nullptr;
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
        cudaMalloc((void **)&n->part, 148 * 8 * sizeof(double)) || cudaMalloc((void **)&n->hloss, sizeof(double))) {
        std::fprintf(stderr, "[pdhcg_b200_mlp] activation allocation failed.\n");
        return -1;
    }
    n->cap = B;
    return 0;
}

// forward of B rows already in n->X; with targets (T, TL) also the loss and dO, dLW
int forward(pdhcg_b200_mlp_s *n, int B, bool with_loss, double *loss)
{
    cudaStream_t s = n->s;
    const bf16 *W1 = n->wb + n->off[P_W1], *W2 = n->wb + n->off[P_W2], *W3 = n->wb + n->off[P_W3],
               *U = n->wb + n->off[P_U];
    const float *b1 = n->w + n->off[P_B1], *b2 = n->w + n->off[P_B2], *b3 = n->w + n->off[P_B3],
                *bu = n->w + n->off[P_BU], *wp = n->w + n->off[P_WP], *bp = n->w + n->off[P_BP];
    gemm<false, true>(B, n->hid, n->in, n->X, n->in, W1, n->in, n->H1, n->hid, 1.0f, 0.0f, s);
    bias_act_kernel<<<blocks_for((long long)B * n->hid), 256, 0, s>>>(B, n->hid, n->H1, b1, 1);
    gemm<false, true>(B, n->hid, n->hid, n->H1, n->hid, W2, n->hid, n->H2, n->hid, 1.0f, 0.0f, s);
    bias_act_kernel<<<blocks_for((long long)B * n->hid), 256, 0, s>>>(B, n->hid, n->H2, b2, 1);
    gemm<false, true>(B, n->rank, n->hid, n->H2, n->hid, W3, n->hid, n->Z, n->rank, 1.0f, 0.0f, s);
    bias_act_kernel<<<blocks_for((long long)B * n->rank), 256, 0, s>>>(B, n->rank, n->Z, b3, 0);
    gemm<false, true>(B, n->out, n->rank, n->Z, n->rank, U, n->rank, n->O, n->out, 1.0f, 0.0f, s);
    bias_act_kernel<<<blocks_for((long long)B * n->out), 256, 0, s>>>(B, n->out, n->O, bu, 0);
    head_kernel<<<1, 256, 0, s>>>(B, n->hid, n->H2, wp, bp, with_loss ? n->TL : nullptr, n->LW, n->dLW, n->hloss);
    if (with_loss) {
        long long tot = (long long)B * n->out;
        int nb = blocks_for(tot);
        mse_kernel<<<nb, 256, 0, s>>>(tot, n->O, n->T, 1.0f / (float)tot, n->dO, n->part);
        std::vector<double> h(nb + 1);
        MCK(cudaMemcpyAsync(h.data(), n->part, nb * sizeof(double), cudaMemcpyDeviceToHost, s));
        MCK(cudaMemcpyAsync(h.data() + nb, n->hloss, sizeof(double), cudaMemcpyDeviceToHost, s));
        MCK(cudaStreamSynchronize(s));
        double a = 0.0;
        for (int b = 0; b < nb; ++b)
            a += h[b];
        *loss = a / (double)tot + h[nb];
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
    gemm<true, false>(n->out, n->rank, B, n->dO, n->out, n->Z, n->rank, g + n->off[P_U], n->rank, 1.0f, 0.0f, s);
    colsum_kernel<<<blocks_for(n->out), 256, 0, s>>>(B, n->out, n->dO, g + n->off[P_BU]);
    gemm<false, false>(B, n->rank, n->out, n->dO, n->out, U, n->rank, n->dZ, n->rank, 1.0f, 0.0f, s);
    // z = W3 h2 + b3
    gemm<true, false>(n->rank, n->hid, B, n->dZ, n->rank, n->H2, n->hid, g + n->off[P_W3], n->hid, 1.0f, 0.0f, s);
    colsum_kernel<<<blocks_for(n->rank), 256, 0, s>>>(B, n->rank, n->dZ, g + n->off[P_B3]);
    gemm<false, false>(B, n->hid, n->rank, n->dZ, n->rank, W3, n->hid, n->dH2, n->hid, 1.0f, 0.0f, s);
    // log-weight head
    head_back_kernel<<<blocks_for(n->hid), 256, 0, s>>>(B, n->hid, n->H2, wp, n->dLW, n->dH2, g + n->off[P_WP],
                                                         g + n->off[P_BP]);
    relu_back_kernel<<<blocks_for((long long)B * n->hid), 256, 0, s>>>((long long)B * n->hid, n->dH2, n->H2);
    // h2 = relu(W2 h1 + b2)
    gemm<true, false>(n->hid, n->hid, B, n->dH2, n->hid, n->H1, n->hid, g + n->off[P_W2], n->hid, 1.0f, 0.0f, s);
    colsum_kernel<<<blocks_for(n->hid), 256, 0, s>>>(B, n->hid, n->dH2, g + n->off[P_B2]);
    gemm<false, false>(B, n->hid, n->hid, n->dH2, n->hid, W2, n->hid, n->dH1, n->hid, 1.0f, 0.0f, s);
    relu_back_kernel<<<blocks_for((long long)B * n->hid), 256, 0, s>>>((long long)B * n->hid, n->dH1, n->H1);
    // h1 = relu(W1 x + b1)
    gemm<true, false>(n->hid, n->in, B, n->dH1, n->hid, n->X, n->in, g + n->off[P_W1], n->in, 1.0f, 0.0f, s);
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
    if (forward(n, batch, false, nullptr))
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
    if (forward(n, batch, true, loss) || backward(n, batch))
        return -1;
    if (grad)
        MCK(cudaMemcpyAsync(grad, n->g, n->total * sizeof(float), cudaMemcpyDeviceToHost, n->s));
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
    double epoch_loss = 0.0;
    int rc = 0;
    for (int ep = 0; ep < epochs && rc == 0; ++ep) {
        epoch_loss = 0.0;
        int nbat = 0;
        for (int b0 = 0; b0 + batch <= count && rc == 0; b0 += batch, ++nbat) { // full minibatches in order
            cudaMemcpyAsync(n->X, dth + (size_t)b0 * n->in, (size_t)batch * n->in * sizeof(float),
                            cudaMemcpyDeviceToDevice, n->s);
            cudaMemcpyAsync(n->T, dt + (size_t)b0 * n->out, (size_t)batch * n->out * sizeof(float),
                            cudaMemcpyDeviceToDevice, n->s);
            cudaMemcpyAsync(n->TL, dtl + b0, batch * sizeof(float), cudaMemcpyDeviceToDevice, n->s);
            double l = 0.0;
            rc = forward(n, batch, true, &l);
            if (rc == 0)
                rc = backward(n, batch);
            if (rc == 0) {
                ++n->step;
                float c1 = 1.0f - std::pow(b1, (float)n->step), c2 = 1.0f - std::pow(b2, (float)n->step);
                adam_kernel<<<blocks_for(n->total), 256, 0, n->s>>>(n->total, n->w, n->g, n->mom, n->vel, lr, b1, b2,
                                                                    c1, c2, eps);
                rc = refresh_bf16(n);
            }
            epoch_loss += l;
        }
        if (nbat > 0)
            epoch_loss /= nbat;
    }
    cudaFree(dth);
    cudaFree(dt);
    cudaFree(dtl);
    if (loss)
        *loss = epoch_loss;
    MCK(cudaStreamSynchronize(n->s));
    return rc;
}

} // extern "C"
