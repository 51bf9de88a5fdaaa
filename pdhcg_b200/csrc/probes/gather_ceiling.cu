// gather_ceiling.cu -- measurement probe (not part of the library): how fast
// can a B200 gather random 4- and 8-byte entries of a vector that lives in
// L2?  The hot products of the step (A x_refl, A^T y) are 5e6 such gathers
// each on the 1e6-variable SOC QP, so this rate bounds them.  Three ways:
//   - plain loads through L1TEX (__ldg / __ldcg), 8 independent per thread;
//   - TMA gather4 (cp.async.bulk.tensor.2d ... tile::gather4, rows of 16 or
//     32 bytes, each CTA for itself) into shared memory, waited on an mbarrier;
//   - distributed shared memory: the table spread over a cluster of 8 CTAs.
// Times are CUDA events, median of 20, after an L2 flush by a 512 MB read.
//
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 \
//        pdhcg_b200/csrc/probes/gather_ceiling.cu -o gather_ceiling -lcuda && ./gather_ceiling
#include <cooperative_groups.h>
#include <cuda.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

namespace cg = cooperative_groups;

#define CK(x)                                                                                                          \
    do {                                                                                                               \
        cudaError_t e_ = (x);                                                                                          \
        if (e_ != cudaSuccess) {                                                                                       \
            printf("CUDA %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__);                                 \
            exit(1);                                                                                                   \
        }                                                                                                              \
    } while (0)

__global__ void k_flush(const float4 *p, long long n, float *out)
{
    float a = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float4 v = __ldcs(p + i);
        a += v.x + v.y + v.z + v.w;
    }
    if (a == 12345.f)
        out[0] = a;
}

template <typename X, int MODE>
__global__ void k_gather(long long nnz, const int *ci, const X *x, double *out)
{
    double a = 0;
    const long long T = (long long)gridDim.x * blockDim.x;
    long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (; k + 7 * T < nnz; k += 8 * T) {
        int c[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            c[u] = __ldcs(ci + k + u * T);
#pragma unroll
        for (int u = 0; u < 8; ++u)
            a += MODE == 0 ? (double)__ldg(x + c[u]) : (double)__ldcg(x + c[u]);
    }
    for (; k < nnz; k += T)
        a += (double)__ldg(x + ci[k]);
    out[blockIdx.x * blockDim.x + threadIdx.x] = a;
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// TMA gather4: x viewed as rows of RW elements (RW * sizeof(X) = 16 or 32 bytes);
// each warp gathers 256 entries per chunk with 64 gather4 instructions (two per
// lane) into 128-byte slots, waits on its mbarrier, then reads its elements.
template <typename X, int RW>
__global__ void __launch_bounds__(256) k_gather_tma(long long nnz, const int *ci, const __grid_constant__ CUtensorMap tm,
                                                    double *out, int *err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *buf = smem + wib * (64 * 128);
    __shared__ __align__(8) unsigned long long bar[8];
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[wib])));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    __syncwarp();
    double a = 0;
    unsigned phase = 0;
    const long long nchunks = (nnz + 255) / 256;
    for (long long ch = blockIdx.x * 8LL + wib; ch < nchunks; ch += gridDim.x * 8LL) {
        const long long cb = ch * 256;
        // indices for this lane's two gather4 (entries 4 lane .. 4 lane + 3 and 128 + 4 lane ..)
        int r[8];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                long long k = cb + 128 * h + 4 * lane + j;
                r[4 * h + j] = k < nnz ? __ldcs(ci + k) / RW : 0;
            }
        if (lane == 0)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&bar[wib])),
                         "r"(64 * 4 * RW * (int)sizeof(X))
                         : "memory");
        __syncwarp();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            unsigned dst = smem_u32(buf + (32 * h + lane) * 128);
            asm volatile("cp.async.bulk.tensor.2d.shared::cta.global.tile::gather4.mbarrier::complete_tx::bytes [%0], "
                         "[%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
                         "l"(&tm), "r"(0), "r"(r[4 * h]), "r"(r[4 * h + 1]), "r"(r[4 * h + 2]), "r"(r[4 * h + 3]),
                         "r"(smem_u32(&bar[wib]))
                         : "memory");
        }
        // entries this lane reads: l + 32 u
        int cc[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            long long k = cb + 32 * u + lane;
            cc[u] = k < nnz ? __ldcs(ci + k) : -1;
        }
        unsigned done = 0;
        for (int it = 0; it < (1 << 22); ++it) {
            asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                         : "=r"(done)
                         : "r"(smem_u32(&bar[wib])), "r"(phase)
                         : "memory");
            if (done)
                break;
        }
        if (!done) {
            if (lane == 0)
                atomicExch(err, 1);
            for (int it = 0; it < (1 << 22) && !done; ++it)
                asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                             : "=r"(done)
                             : "r"(smem_u32(&bar[wib])), "r"(phase)
                             : "memory");
            return;
        }
        phase ^= 1;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = 32 * u + lane; // entry within chunk; its gather4 = e / 4 within half, slot row e % 4
            const int h = e >> 7, g = (e & 127) >> 2, j = e & 3;
            const X *row = (const X *)(buf + (32 * h + g) * 128) + j * RW;
            if (cc[u] >= 0)
                a += (double)row[cc[u] % RW];
        }
        __syncwarp();
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = a;
}

// Distributed shared memory: a cluster of CL CTAs holds a table of CL * TW
// floats (TW per CTA); gathers of table[ci[k] % (CL * TW)].
template <int CL>
__global__ void __launch_bounds__(256) k_gather_dsmem(long long nnz, const int *ci, const float *x, int TW, double *out)
{
    extern __shared__ __align__(16) float tab[];
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    for (int i = threadIdx.x; i < TW; i += blockDim.x)
        tab[i] = x[rank * TW + i];
    cl.sync();
    const int total = CL * TW;
    double a = 0;
    const long long T = (long long)gridDim.x * blockDim.x;
    long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (; k + 7 * T < nnz; k += 8 * T) {
        int c[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            c[u] = __ldcs(ci + k + u * T) % total;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const float *p = cl.map_shared_rank(tab, c[u] / TW);
            a += (double)p[c[u] % TW];
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = a;
    cl.sync(); // no CTA leaves while others read its table
}

static float4 *g_fl;
static const long long FLN = (512ll << 20) / 16;
static float *g_flo;

template <typename F>
float timeit(F &&launch, int reps = 20)
{
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    std::vector<float> t;
    for (int r = 0; r < reps + 3; ++r) {
        k_flush<<<148 * 8, 256>>>(g_fl, FLN, g_flo);
        CK(cudaEventRecord(a));
        launch();
        CK(cudaEventRecord(b));
        CK(cudaEventSynchronize(b));
        CK(cudaGetLastError());
        float ms;
        CK(cudaEventElapsedTime(&ms, a, b));
        if (r >= 3)
            t.push_back(ms * 1000.f);
    }
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

int main()
{
    const int n = 1000000;
    const long long nnz = 5000000;
    std::mt19937_64 rng(3);
    std::vector<int> ci(nnz);
    for (auto &c : ci)
        c = (int)(rng() % n);
    std::vector<float> xf(n);
    std::vector<double> xd(n);
    for (int i = 0; i < n; ++i)
        xf[i] = (float)(xd[i] = (double)(rng() % 1000) / 1000.0);
    double want = 0;
    for (auto c : ci)
        want += xd[c];
    int *dci;
    float *dxf;
    double *dxd, *out;
    int *err;
    CK(cudaMalloc(&dci, nnz * 4));
    CK(cudaMalloc(&dxf, n * 4 + 64));
    CK(cudaMalloc(&dxd, n * 8 + 64));
    CK(cudaMalloc(&out, 148 * 2048 * 8 * 8));
    CK(cudaMalloc(&err, 4));
    CK(cudaMemset(err, 0, 4));
    CK(cudaMalloc(&g_fl, FLN * 16));
    CK(cudaMemset(g_fl, 0, FLN * 16));
    CK(cudaMalloc(&g_flo, 16));
    CK(cudaMemcpy(dci, ci.data(), nnz * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dxf, xf.data(), n * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dxd, xd.data(), n * 8, cudaMemcpyHostToDevice));
    std::vector<double> hout(148 * 2048 * 8);
    auto check = [&](int threads, const char *what) {
        CK(cudaMemcpy(hout.data(), out, threads * 8, cudaMemcpyDeviceToHost));
        double s = 0;
        for (int i = 0; i < threads; ++i)
            s += hout[i];
        printf("    %s sum %.6f want %.6f (rel %.1e)\n", what, s, want, fabs(s - want) / want);
    };

    for (int g : {148 * 4, 148 * 8}) {
        float t0 = timeit([&] { k_gather<double, 0><<<g, 256>>>(nnz, dci, dxd, out); });
        check(g * 256, "ldg f64");
        float t1 = timeit([&] { k_gather<double, 1><<<g, 256>>>(nnz, dci, dxd, out); });
        float t2 = timeit([&] { k_gather<float, 0><<<g, 256>>>(nnz, dci, dxf, out); });
        float t3 = timeit([&] { k_gather<float, 1><<<g, 256>>>(nnz, dci, dxf, out); });
        printf("grid %d: ldg f64 %.2f us, ldcg f64 %.2f, ldg f32 %.2f, ldcg f32 %.2f  (%.0f / %.0f / %.0f / %.0f Gg/s)\n", g,
               t0, t1, t2, t3, nnz / t0 / 1e3, nnz / t1 / 1e3, nnz / t2 / 1e3, nnz / t3 / 1e3);
    }

    // tensor maps
    auto encode = [&](void *base, CUtensorMapDataType dt, int esize, int rw, long long rows) {
        CUtensorMap tm;
        cuuint64_t dims[2] = {(cuuint64_t)rw, (cuuint64_t)rows};
        cuuint64_t strides[1] = {(cuuint64_t)(rw * esize)};
        cuuint32_t box[2] = {(cuuint32_t)rw, 1};
        cuuint32_t es[2] = {1, 1};
        CUresult r = cuTensorMapEncodeTiled(&tm, dt, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            printf("encode failed %d\n", (int)r);
            exit(1);
        }
        return tm;
    };
    CUtensorMap tmf4 = encode(dxf, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, 4, n / 4);
    CUtensorMap tmf8 = encode(dxf, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, 8, n / 8);
    CUtensorMap tmd2 = encode(dxd, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, 2, n / 2);
    CUtensorMap tmd4 = encode(dxd, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, 4, n / 4);
    const int smem = 8 * 64 * 128;
    CK(cudaFuncSetAttribute(k_gather_tma<float, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CK(cudaFuncSetAttribute(k_gather_tma<float, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CK(cudaFuncSetAttribute(k_gather_tma<double, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CK(cudaFuncSetAttribute(k_gather_tma<double, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int hb = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&hb, k_gather_tma<float, 4>, 256, smem));
    printf("tma gather blocks/SM %d\n", hb);
    for (int g : {148 * hb}) {
        float t0 = timeit([&] { k_gather_tma<float, 4><<<g, 256, smem>>>(nnz, dci, tmf4, out, err); });
        int herr = 0;
        CK(cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost));
        check(g * 256, "tma f32 16B");
        float t1 = timeit([&] { k_gather_tma<float, 8><<<g, 256, smem>>>(nnz, dci, tmf8, out, err); });
        check(g * 256, "tma f32 32B");
        float t2 = timeit([&] { k_gather_tma<double, 2><<<g, 256, smem>>>(nnz, dci, tmd2, out, err); });
        check(g * 256, "tma f64 16B");
        float t3 = timeit([&] { k_gather_tma<double, 4><<<g, 256, smem>>>(nnz, dci, tmd4, out, err); });
        check(g * 256, "tma f64 32B");
        CK(cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost));
        printf("tma grid %d: f32/16B %.2f us, f32/32B %.2f, f64/16B %.2f, f64/32B %.2f  err %d\n", g, t0, t1, t2, t3,
               herr);
    }

    // DSMEM: clusters of 8, 48K floats per CTA (192 KB)
    {
        const int TW = 48 * 1024, CLN = 8;
        const int sm = TW * 4;
        CK(cudaFuncSetAttribute(k_gather_dsmem<CLN>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        for (int g : {144, 288}) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(g);
            cfg.blockDim = dim3(256);
            cfg.dynamicSmemBytes = sm;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = CLN;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            float t = timeit([&] { CK(cudaLaunchKernelEx(&cfg, k_gather_dsmem<CLN>, nnz, (const int *)dci, (const float *)dxf, TW, out)); });
            printf("dsmem cluster %d grid %d: %.2f us (%.0f Gg/s)\n", CLN, g, t, nnz / t / 1e3);
        }
    }
    CK(cudaDeviceSynchronize());
    printf("done\n");
    return 0;
}
