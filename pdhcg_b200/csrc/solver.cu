// solver.cu -- host driver of one PDHCG-B200 solve, plus the kernel-level
// C entry points.
//
// The control flow mirrors the reference's optimize() (src/solver.cu:35-210)
// decision for decision -- evaluation cadence, the (k+2) store rule for
// PDHG iterates, restart tests, PID primal weight -- because those
// decisions shape the iterate trajectory.  What differs is where the work
// runs: preprocessing (transpose, rescaling, power method) runs on the
// device, each iteration is two fused kernels, and the host synchronises
// only at evaluation points, reading one small block of scalars.

#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <atomic>
#include <chrono>
#include <cmath>
#include <csignal>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "internal.h"
#include "bb.cuh"
#include "residual.cuh"
#include "setup.cuh"

using namespace pdhcg;

namespace {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define CK(call)                                                                                                       \
    do {                                                                                                               \
        cudaError_t e_ = (call);                                                                                       \
        if (e_ != cudaSuccess)                                                                                         \
            throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " at " + __FILE__ + ":" +            \
                            std::to_string(__LINE__));                                                                 \
    } while (0)

thread_local pdhcg_b200_stats_t g_last_stats;

// pinned host mirror of a solve's scalar block, one per host thread, kept
// for the thread's lifetime (a solve runs on one thread)
double *pinned_scalars()
{
    struct Buf {
        double *p = nullptr;
        ~Buf()
        {
            if (p)
                cudaFreeHost(p);
        }
    };
    thread_local Buf b;
    if (!b.p)
        CK(cudaMallocHost(&b.p, 64 * sizeof(double)));
    return b.p;
}

// Host-to-device copy of a large host array through two page-locked chunks
// kept for the process: the host threads copy chunk i into one buffer while
// the DMA engine moves the previous chunk out of the other, so the copy runs
// at page-locked speed instead of through the driver's pageable staging.
// The source may be freed when this returns; the destination is written in
// stream order on s.  A chunk's buffer is reused once its copy has ended
// (its event), also across calls, which take turns on the buffers.
constexpr size_t STAGE_CHUNK = 32u << 20;
constexpr size_t STAGE_MIN = 16u << 20; // smaller copies go straight through

void staged_upload(void *dst, const void *src, size_t bytes, cudaStream_t s)
{
    static std::mutex mu;
    static char *buf[2] = {nullptr, nullptr};
    static cudaEvent_t ev[2] = {nullptr, nullptr};
    static bool pending[2] = {false, false};
    static int ev_dev = -1;
    static int b = 0;
    std::lock_guard<std::mutex> lock(mu);
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (!buf[0]) {
        void *p = nullptr;
        if (cudaHostAlloc(&p, 2 * STAGE_CHUNK, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
            CK(cudaStreamSynchronize(s));
            return;
        }
        buf[0] = (char *)p;
        buf[1] = (char *)p + STAGE_CHUNK;
    }
    if (ev_dev != dev) { // events are recorded on this device's streams
        for (int i = 0; i < 2; ++i) {
            if (ev[i]) {
                if (pending[i])
                    cudaEventSynchronize(ev[i]);
                cudaEventDestroy(ev[i]);
                ev[i] = nullptr;
            }
            pending[i] = false;
        }
        CK(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
        ev_dev = dev;
    }
    const int nt = (int)std::min<unsigned>(8u, std::max(1u, std::thread::hardware_concurrency()));
    const char *from = (const char *)src;
    char *to = (char *)dst;
    for (size_t off = 0; off < bytes; off += STAGE_CHUNK, b ^= 1) {
        const size_t len = std::min(STAGE_CHUNK, bytes - off);
        if (pending[b]) {
            CK(cudaEventSynchronize(ev[b]));
            pending[b] = false;
        }
        // the chunk's host copy, split over up to nt threads
        const size_t part = (len + nt - 1) / nt;
        char *chunk = buf[b];
        std::vector<std::thread> th;
        for (int t = 1; t < nt && (size_t)t * part < len; ++t) {
            const size_t a = (size_t)t * part, e = std::min(len, a + part);
            try {
                th.emplace_back([=]() { std::memcpy(chunk + a, from + off + a, e - a); });
            } catch (...) { // no thread to be had: this part here
                std::memcpy(chunk + a, from + off + a, e - a);
            }
        }
        std::memcpy(chunk, from + off, std::min(len, part));
        for (auto &x : th)
            x.join();
        CK(cudaMemcpyAsync(to + off, chunk, len, cudaMemcpyHostToDevice, s));
        CK(cudaEventRecord(ev[b], s));
        pending[b] = true;
    }
}

// f(begin, end) over [0, n) in up to 8 chunks on host threads, the calling
// thread taking the first (the problem checks of a device-problem build);
// chunks run at once, so f writes nothing that another chunk writes
template <typename F>
void host_chunks(long long n, F &&f)
{
    const int nt = n < (1 << 16) ? 1 : (int)std::min<unsigned>(8u, std::max(1u, std::thread::hardware_concurrency()));
    if (nt <= 1) {
        f(0LL, n);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) {
        const long long a = n * t / nt, e = n * (t + 1) / nt;
        try {
            th.emplace_back([&f, a, e]() { f(a, e); });
        } catch (...) { // no thread to be had: this chunk here
            f(a, e);
        }
    }
    f(0LL, n / nt);
    for (auto &x : th)
        x.join();
}

// The device's default memory pool keeps what solves free (no release
// threshold), so the allocations of the next solve are served from the pool
// instead of cudaMalloc; set once per device.
void keep_pool_memory()
{
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev])
        return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        unsigned long long keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done[dev] = true;
}

// Device allocations owned by one solve or one device problem: stream-ordered
// from the default pool on the owner's stream s, returned to the pool on the
// legacy stream when the owner (which has synchronised its streams by then)
// goes away.
struct Arena {
    std::vector<void *> ptrs;
    cudaStream_t s = nullptr;
    template <typename T>
    T *alloc(size_t count)
    {
        void *p = nullptr;
        keep_pool_memory();
        CK(cudaMallocAsync(&p, std::max<size_t>(count, 1) * sizeof(T), s));
        ptrs.push_back(p);
        return (T *)p;
    }
    template <typename T>
    T *upload(const T *h, size_t count, cudaStream_t s)
    {
        T *d = alloc<T>(count);
        if (count * sizeof(T) >= STAGE_MIN)
            staged_upload(d, h, count * sizeof(T), s);
        else if (count)
            CK(cudaMemcpyAsync(d, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
        return d;
    }
    ~Arena()
    {
        for (void *p : ptrs)
            cudaFreeAsync(p, 0);
    }
};

int grid_for(long long work, int per_block, int cap = 148 * 16)
{
    long long g = (work + per_block - 1) / per_block;
    if (g < 1)
        g = 1;
    if (g > cap)
        g = cap;
    return (int)g;
}

// Blocks of `kernel` (TPB threads, static shared memory) resident at once
// on the current device; cached per kernel and device.
int resident_blocks(const void *kernel)
{
    static std::mutex mu;
    static std::unordered_map<const void *, int> cache[64];
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    auto &c = cache[dev & 63];
    auto it = c.find(kernel);
    if (it != c.end())
        return it->second;
    int nsm = 0, per_sm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, TPB, 0));
    const int r = std::max(1, nsm * std::max(per_sm, 1));
    c.emplace(kernel, r);
    return r;
}

int print_frequency(int iter)
{
    int step = 10;
    long long threshold = 1000;
    while (iter >= threshold) {
        step *= 10;
        threshold *= 10;
    }
    return step;
}

// Runs of consecutive rows in a sorted index list, cut into tiles of at
// most 32 rows {first row, count} (one warp each in the step kernels).
std::vector<int2> row_tiles(const std::vector<int> &rows)
{
    std::vector<int2> t;
    for (size_t i = 0; i < rows.size();) {
        size_t j = i + 1;
        while (j < rows.size() && j - i < 32 && rows[j] == rows[j - 1] + 1)
            ++j;
        t.push_back(make_int2(rows[i], (int)(j - i)));
        i = j;
    }
    return t;
}

// The primal step launches the SOC / RSOC blocks and the 3-slot blocks
// (exponential, power) separately: the 3-slot projections would otherwise
// sit in the wide kernels' register allocation.  A list pointer stays null
// when its launch covers every block (all of one kind).
struct ConeSplit {
    std::vector<int> wide, three, psd, sect;
    int *wide_d = nullptr, *three_d = nullptr, *psd_d = nullptr, *sect_d = nullptr;
    int n_wide = 0, n_three = 0, n_psd = 0, n_sect = 0;

    // fixed (may be empty): per block, does it hold slots fixed by
    // set_cone_fixed?  Those blocks take the section projectors.
    void build(const std::vector<int> &types, const std::vector<char> &fixed = {})
    {
        wide.clear();
        three.clear();
        psd.clear();
        sect.clear();
        for (int b = 0; b < (int)types.size(); ++b) {
            if (!fixed.empty() && fixed[b])
                sect.push_back(b);
            else if (types[b] == CONE_EXPONENTIAL || types[b] == CONE_POWER)
                three.push_back(b);
            else if (types[b] == CONE_PSD)
                psd.push_back(b);
            else
                wide.push_back(b);
        }
        n_wide = (int)wide.size();
        n_three = (int)three.size();
        n_psd = (int)psd.size();
        n_sect = (int)sect.size();
    }
    // more than one launch: every launch takes its index list
    bool mixed() const { return (n_wide > 0) + (n_three > 0) + (n_psd > 0) + (n_sect > 0) > 1; }
    // the lists back to back in one device array of n_wide + n_three + n_psd + n_sect ints
    void place(int *ids)
    {
        wide_d = ids;
        three_d = ids + n_wide;
        psd_d = ids + n_wide + n_three;
        sect_d = ids + n_wide + n_three + n_psd;
    }
    std::vector<int> joined() const
    {
        std::vector<int> all(wide);
        all.insert(all.end(), three.begin(), three.end());
        all.insert(all.end(), psd.begin(), psd.end());
        all.insert(all.end(), sect.begin(), sect.end());
        return all;
    }
};

// lanes per row from the mean row length
int pick_group(long long nnz, int rows)
{
    double mean = rows > 0 ? (double)nnz / rows : 0.0;
    if (mean <= 1.5)
        return 1;
    if (mean <= 3)
        return 2;
    if (mean <= 6)
        return 4;
    if (mean <= 12)
        return 8;
    if (mean <= 24)
        return 16;
    return 32;
}

// slots per lane of the warp-per-cone kernels (cone blocks up to 256 slots)
int slots_class(int maxlen)
{
    int s = (maxlen + 31) / 32;
    if (s <= 1)
        return 1;
    if (s <= 2)
        return 2;
    if (s <= 4)
        return 4;
    if (s <= 8)
        return 8;
    return -1;
}

// lanes per row of the residual kernel (one kernel serves A and A^T rows)
int residual_group(int g)
{
    return g <= 2 ? 1 : (g <= 8 ? 4 : 32);
}

struct DevCsr {
    int rows = 0, cols = 0, nnz = 0;
    int *rp = nullptr, *ci = nullptr;
    double *v = nullptr;
    LongRows lr{}; // rows of more than LONG_ROW entries, cut into segments (n = 0: none)
    long long long_nnz = 0; // entries in those rows
};

// The long rows of M and their segments.  A count on the device decides
// whether the row pointer is read back at all (most problems have none).
void build_long_rows(DevCsr &M, Arena &ar, cudaStream_t s)
{
    M.lr = LongRows{};
    if (M.rows == 0 || M.nnz <= LONG_ROW)
        return;
    int *cnt = ar.alloc<int>(1);
    CK(cudaMemsetAsync(cnt, 0, sizeof(int), s));
    long_count_kernel<<<grid_for(M.rows, 256), 256, 0, s>>>(M.rows, M.rp, cnt);
    int count = 0;
    CK(cudaMemcpyAsync(&count, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (count == 0)
        return;
    std::vector<int> rp(M.rows + 1);
    CK(cudaMemcpyAsync(rp.data(), M.rp, rp.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::vector<int> rows, first{0};
    std::vector<int2> seg;
    M.long_nnz = 0;
    for (int r = 0; r < M.rows; ++r) {
        if (rp[r + 1] - rp[r] <= LONG_ROW)
            continue;
        M.long_nnz += rp[r + 1] - rp[r];
        rows.push_back(r);
        for (int b = rp[r]; b < rp[r + 1]; b += LONG_SEG)
            seg.push_back(make_int2(b, std::min(rp[r + 1], b + LONG_SEG)));
        first.push_back((int)seg.size());
    }
    M.lr.rows = ar.upload(rows.data(), rows.size(), s);
    M.lr.seg_first = ar.upload(first.data(), first.size(), s);
    M.lr.seg = ar.upload(seg.data(), seg.size(), s);
    M.lr.part = ar.alloc<double>(seg.size());
    M.lr.n = (int)rows.size();
    M.lr.nseg = (int)seg.size();
    CK(cudaStreamSynchronize(s)); // the host tables go out of scope
}

// stable transpose on the device (entries of each output row in increasing
// input-row order); M's long-row table, when it has one, is built first
DevCsr transpose(const DevCsr &M, Arena &ar, cudaStream_t s)
{
    DevCsr T;
    T.rows = M.cols;
    T.cols = M.rows;
    T.nnz = M.nnz;
    T.rp = ar.alloc<int>((size_t)T.rows + 1);
    T.ci = ar.alloc<int>(M.nnz);
    T.v = ar.alloc<double>(M.nnz);
    if (M.nnz == 0) {
        CK(cudaMemsetAsync(T.rp, 0, ((size_t)T.rows + 1) * sizeof(int), s));
        return T;
    }
    int *row_of = ar.alloc<int>(M.nnz), *idx = ar.alloc<int>(M.nnz), *keys_out = ar.alloc<int>(M.nnz),
        *perm = ar.alloc<int>(M.nnz);
    expand_rows_kernel<<<grid_for(M.rows, TPB), TPB, 0, s>>>(M.rp, M.rows, row_of, M.lr.n > 0);
    if (M.lr.n > 0)
        expand_long_rows_kernel<<<std::min(M.lr.n, 148 * 16), TPB, 0, s>>>(M.lr, M.rp, row_of);
    iota_kernel<<<grid_for(M.nnz, TPB), TPB, 0, s>>>(idx, M.nnz);
    size_t tmp_bytes = 0;
    int bits = 1;
    while ((1LL << bits) <= (long long)M.cols)
        ++bits;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, M.ci, keys_out, idx, perm, M.nnz, 0, bits, s);
    void *tmp = ar.alloc<char>(tmp_bytes);
    CK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, M.ci, keys_out, idx, perm, M.nnz, 0, bits, s));
    col_ptr_kernel<<<grid_for((long long)T.rows + 1, TPB), TPB, 0, s>>>(keys_out, M.nnz, T.rows, T.rp);
    gather_transpose_kernel<<<grid_for(M.nnz, TPB), TPB, 0, s>>>(perm, row_of, M.v, M.nnz, T.ci, T.v);
    return T;
}

struct HostScalars {
    double v[RS_COUNT + 2 * FP_COUNT];
};

// A problem resident in HBM: the raw (unscaled) arrays of a qp_problem_t
// plus the host-side metadata a solve needs.  solve_qp_problem builds a
// temporary one and lets the solve scale it in place; the handle API
// (pdhcg_b200_upload) keeps one and every solve works on copies.
struct DeviceProblem {
    int n = 0, m = 0, nnzA = 0, nnzQ = 0, qtype = PDHCG_NON_Q, S = 1;
    bool dummy = false, has_g = false, box_free = true, eq_rows = true, cone_box = false;
    std::vector<int> cone_start, cone_len, cone_type, cone_vdim, free_idx;
    std::vector<double> cone_alpha;
    double obj_const = 0.0;
    int orig_vars = 0, orig_cons = 0, orig_nnz = 0;
    std::string unsupported; // non-empty: reason the device path cannot solve it
    Arena ar;
    int *A_rp = nullptr, *A_ci = nullptr, *Q_rp = nullptr, *Q_ci = nullptr;
    double *A_v = nullptr, *Q_v = nullptr;
    // low-rank term R (k rows, CSR) and its middle matrix D
    int rank = 0, nnzR = 0, dkind = 0; // dkind 0 none (identity), 1 diagonal, 2 dense
    int *R_rp = nullptr, *R_ci = nullptr;
    double *R_v = nullptr, *Ddiag = nullptr, *Ddense = nullptr;
    double *c = nullptr, *l = nullptr, *u = nullptr, *lc = nullptr, *uc = nullptr, *g = nullptr;
    int *cst = nullptr, *clen = nullptr, *ctype = nullptr, *cvdim = nullptr, *free_d = nullptr;
    double *calpha = nullptr; // power-cone exponents per cone block
    ConeSplit split;            // cone blocks by launch (wide / 3-slot / PSD)
    bool has_psd = false;       // PSD blocks among the variable or affine cones (scratch needed)
    bool var_psd = false;       // PSD blocks among the variable cones
    // affine cones over blocks of rows (F x + g in K): blocks, their PSD
    // scratch offsets, and the rows outside them as tiles
    std::vector<int> aff_start, aff_len, aff_type, aff_vdim;
    std::vector<double> aff_alpha;
    std::vector<long long> aff_psd_off;
    int *ast = nullptr, *alen = nullptr, *atype = nullptr, *avdim = nullptr;
    double *aalpha = nullptr;
    long long *apsd_off_d = nullptr;
    int2 *row_tiles_d = nullptr;
    int n_row_tiles = 0, S_aff = 1;
    std::vector<long long> psd_off; // per cone block: offset of its PSD scratch (2 n^2 doubles)
    long long psd_total = 0;
    long long *psd_off_d = nullptr;
    int2 *free_tiles = nullptr; // free variables as tiles of consecutive rows
    int n_free_tiles = 0;
    double *pstart = nullptr, *dstart = nullptr;
    // slots fixed by set_cone_fixed: the mask over the variables, per block
    // whether it holds any, and the fixed slots with their values (pinned
    // into the scaled bounds after rescaling)
    bool has_fixed = false;
    std::vector<char> cone_fixed;
    unsigned char *fixed_d = nullptr, *cfix_d = nullptr;
    int n_fix = 0;
    int *fix_idx = nullptr;
    double *fix_val = nullptr;
    // solution kept on the device when a solve is asked to leave it there
    double *x_out = nullptr, *y_out = nullptr, *rc_out = nullptr;
};

// Classification (reference preprocess_qp_problem and detect_q_type,
// src/preconditioner.c:715-830, src/utils.cu:834-885) and upload.
std::unique_ptr<DeviceProblem> make_device_problem(const qp_problem_t *p, cudaStream_t s)
{
    auto dp = std::make_unique<DeviceProblem>();
    DeviceProblem &d = *dp;
    d.ar.s = s;
    d.n = p->num_variables;
    d.orig_vars = p->num_variables;
    d.orig_cons = p->num_constraints;
    d.orig_nnz = p->constraint_matrix_num_nonzeros;
    d.obj_const = p->objective_constant;
    d.dummy = p->num_constraints == 0 || p->constraint_matrix == nullptr;
    Arena &ar = d.ar;
    if (d.dummy) { // reference create_problem_with_dummy_constraint, src/utils.cu:80-135
        d.m = 1;
        d.nnzA = 1;
        const int rp[2] = {0, 1}, ci[1] = {0};
        const double v[1] = {1.0}, lo[1] = {-INFINITY}, up[1] = {INFINITY}, g0[1] = {0.0};
        d.A_rp = ar.upload(rp, 2, s);
        d.A_ci = ar.upload(ci, 1, s);
        d.A_v = ar.upload(v, 1, s);
        d.lc = ar.upload(lo, 1, s);
        d.uc = ar.upload(up, 1, s);
        d.g = ar.upload(g0, 1, s);
        CK(cudaStreamSynchronize(s)); // stack sources
        d.box_free = true;
        d.eq_rows = false;
    } else {
        d.m = p->num_constraints;
        d.nnzA = p->constraint_matrix_num_nonzeros;
        d.A_rp = ar.upload(p->constraint_matrix->row_ptr, (size_t)d.m + 1, s);
        d.A_ci = ar.upload(p->constraint_matrix->col_ind, d.nnzA, s);
        d.A_v = ar.upload(p->constraint_matrix->val, d.nnzA, s);
        d.lc = ar.upload(p->constraint_lower_bound, d.m, s);
        d.uc = ar.upload(p->constraint_upper_bound, d.m, s);
        d.g = ar.upload(p->affine_cone_offset, d.m, s);
        {
            const double *gg = p->affine_cone_offset, *lo = p->constraint_lower_bound,
                         *up = p->constraint_upper_bound;
            std::atomic<int> any_g{0}, unequal{0};
            host_chunks(d.m, [&](long long a, long long e) {
                int hg = 0, eq = 1;
                for (long long i = a; i < e; ++i) {
                    hg |= gg[i] != 0.0;
                    eq &= (lo[i] == up[i]) & (std::fabs(lo[i]) <= DBL_MAX); // equal and finite
                }
                if (hg)
                    any_g = 1;
                if (!eq)
                    unequal = 1;
            });
            d.has_g = d.has_g || any_g;
            d.eq_rows = d.eq_rows && !unequal;
        }
        if (p->dual_start)
            d.dstart = ar.upload(p->dual_start, d.m, s);
    }
    d.c = ar.upload(p->objective_vector, d.n, s);
    d.l = ar.upload(p->variable_lower_bound, d.n, s);
    d.u = ar.upload(p->variable_upper_bound, d.n, s);
    if (p->primal_start)
        d.pstart = ar.upload(p->primal_start, d.n, s);
    {
        const double *lo = p->variable_lower_bound, *up = p->variable_upper_bound;
        std::atomic<int> boxed{0};
        host_chunks(d.n, [&](long long a, long long e) {
            int fin = 0; // a finite bound
            for (long long i = a; i < e; ++i)
                fin |= (std::fabs(lo[i]) <= DBL_MAX) | (std::fabs(up[i]) <= DBL_MAX);
            if (fin)
                boxed = 1;
        });
        d.box_free = d.box_free && !boxed;
    }

    int nnzq = (p->objective_sparse_matrix && p->objective_sparse_matrix->row_ptr)
                   ? p->objective_sparse_matrix_num_nonzeros
                   : 0;
    int nnzr = (p->objective_lowrank_matrix && p->objective_lowrank_matrix->row_ptr && p->num_rank_lowrank_obj > 0)
                   ? p->objective_lowrank_matrix_num_nonzeros
                   : 0;
    if (nnzq == 0 && nnzr == 0)
        d.qtype = PDHCG_NON_Q;
    else if (nnzr > 0)
        d.qtype = nnzq > 0 ? PDHCG_LOW_RANK_PLUS_SPARSE_Q : PDHCG_LOW_RANK_Q;
    else {
        // diagonal unless some entry lies off the diagonal
        const int *qrp = p->objective_sparse_matrix->row_ptr, *qci = p->objective_sparse_matrix->col_ind;
        std::atomic<int> off{0};
        host_chunks(d.n, [&](long long a, long long e) {
            int o = 0;
            for (long long i = a; i < e; ++i)
                for (int k = qrp[i]; k < qrp[i + 1]; ++k)
                    o |= qci[k] != (int)i;
            if (o)
                off = 1;
        });
        d.qtype = off ? PDHCG_SPARSE_Q : PDHCG_DIAG_Q;
    }
    if (d.qtype != PDHCG_NON_Q && nnzq > 0) {
        const CsrComponent *Q = p->objective_sparse_matrix;
        d.nnzQ = p->objective_sparse_matrix_num_nonzeros;
        d.Q_rp = ar.upload(Q->row_ptr, (size_t)d.n + 1, s);
        d.Q_ci = ar.upload(Q->col_ind, d.nnzQ, s);
        d.Q_v = ar.upload(Q->val, d.nnzQ, s);
    }
    if (nnzr > 0) {
        const CsrComponent *R = p->objective_lowrank_matrix;
        d.rank = p->num_rank_lowrank_obj;
        d.nnzR = nnzr;
        d.R_rp = ar.upload(R->row_ptr, (size_t)d.rank + 1, s);
        d.R_ci = ar.upload(R->col_ind, d.nnzR, s);
        d.R_v = ar.upload(R->val, d.nnzR, s);
        // middle matrix kind (reference preprocess_qp_problem, src/preconditioner.c:742-791)
        const CsrComponent *Dm = p->objective_lowrank_middle_matrix;
        int k = d.rank;
        if (Dm && Dm->row_ptr && p->objective_lowrank_middle_matrix_num_nonzeros > 0) {
            bool diag_only = true;
            for (int r = 0; r < k && diag_only; ++r)
                for (int j = Dm->row_ptr[r]; j < Dm->row_ptr[r + 1]; ++j)
                    if (Dm->col_ind[j] != r) {
                        diag_only = false;
                        break;
                    }
            if (diag_only) {
                std::vector<double> dd(k, 0.0);
                for (int r = 0; r < k; ++r)
                    for (int j = Dm->row_ptr[r]; j < Dm->row_ptr[r + 1]; ++j)
                        dd[r] = Dm->val[j];
                d.dkind = 1;
                d.Ddiag = ar.upload(dd.data(), k, s);
                CK(cudaStreamSynchronize(s));
            } else {
                std::vector<double> dd((size_t)k * k, 0.0);
                for (int r = 0; r < k; ++r)
                    for (int j = Dm->row_ptr[r]; j < Dm->row_ptr[r + 1]; ++j)
                        dd[(size_t)r * k + Dm->col_ind[j]] = Dm->val[j];
                d.dkind = 2;
                d.Ddense = ar.upload(dd.data(), (size_t)k * k, s);
                CK(cudaStreamSynchronize(s));
            }
        }
        if (k > BB_MAX_RANK)
            d.unsupported = "low-rank terms of rank above 512 are not supported yet";
    }

    int maxlen = 0;
    std::vector<char> in_cone(d.n, 0);
    d.has_fixed = p->cones.is_fixed != nullptr && p->cones.num_cones > 0;
    for (int b = 0; b < p->cones.num_cones; ++b) {
        int len = pdhcg_b200_cone_length(p->cones.type[b], p->cones.v_dim[b]);
        if (d.has_fixed) {
            char any = 0;
            for (int i = 0; i < len; ++i)
                any |= p->cones.is_fixed[p->cones.start_idx[b] + i] != 0;
            d.cone_fixed.push_back(any);
        }
        d.cone_start.push_back(p->cones.start_idx[b]);
        d.cone_len.push_back(len);
        d.cone_type.push_back((int)p->cones.type[b]);
        d.cone_vdim.push_back(p->cones.v_dim[b]);
        // PSD blocks beyond the widest slot class take the memory path
        // (their length does not set the class)
        if (!(p->cones.type[b] == CONE_PSD && len > 32 * 8))
            maxlen = std::max(maxlen, len);
        {
            const int st = p->cones.start_idx[b];
            const double *lo = p->variable_lower_bound + st, *up = p->variable_upper_bound + st;
            std::fill(in_cone.begin() + st, in_cone.begin() + st + len, (char)1);
            int fin = 0;
            for (int i = 0; i < len; ++i)
                fin |= (std::fabs(lo[i]) <= DBL_MAX) | (std::fabs(up[i]) <= DBL_MAX);
            d.cone_box = d.cone_box || fin;
        }
        d.psd_off.push_back(d.psd_total);
        if (p->cones.type[b] == CONE_PSD) {
            // decomposition scratch, plus candidate staging for blocks the
            // registers of a warp do not hold (any order)
            d.has_psd = true;
            d.var_psd = true;
            d.psd_total += psd_scratch_doubles(p->cones.v_dim[b], len > 32);
        }
        d.cone_alpha.push_back(p->cones.power_alpha ? p->cones.power_alpha[b] : 0.0);
    }
    int nc = (int)d.cone_start.size();
    if (nc > 0) {
        size_t nfree = 0;
        for (int i = 0; i < d.n; ++i)
            nfree += !in_cone[i];
        d.free_idx.reserve(nfree);
        if (nfree > 0)
            for (int i = 0; i < d.n; ++i)
                if (!in_cone[i])
                    d.free_idx.push_back(i);
        d.S = slots_class(maxlen);
        d.cst = ar.upload(d.cone_start.data(), nc, s);
        d.clen = ar.upload(d.cone_len.data(), nc, s);
        d.ctype = ar.upload(d.cone_type.data(), nc, s);
        d.cvdim = ar.upload(d.cone_vdim.data(), nc, s);
        d.calpha = ar.upload(d.cone_alpha.data(), nc, s);
        d.split.build(d.cone_type, d.cone_fixed);
        if (d.has_fixed) {
            // fixed slots: bounds pinned after scaling, so the box step holds
            // them (reference pin_scaled_fixed_cone_bounds, src/preconditioner.c:311-327)
            d.cone_box = true;
            std::vector<unsigned char> mask(p->cones.is_fixed, p->cones.is_fixed + d.n);
            std::vector<unsigned char> cf(d.cone_fixed.begin(), d.cone_fixed.end());
            std::vector<int> fi;
            std::vector<double> fv;
            for (int j = 0; j < d.n; ++j)
                if (mask[j]) {
                    fi.push_back(j);
                    fv.push_back(p->primal_start ? p->primal_start[j] : 0.0);
                }
            d.n_fix = (int)fi.size();
            d.fixed_d = ar.upload(mask.data(), mask.size(), s);
            d.cfix_d = ar.upload(cf.data(), cf.size(), s);
            if (d.n_fix > 0) {
                d.fix_idx = ar.upload(fi.data(), fi.size(), s);
                d.fix_val = ar.upload(fv.data(), fv.size(), s);
            }
            CK(cudaStreamSynchronize(s));
        }
        if (d.split.mixed()) {
            std::vector<int> all = d.split.joined();
            d.split.place(ar.upload(all.data(), all.size(), s));
            CK(cudaStreamSynchronize(s));
        }
        if (d.has_psd) {
            d.psd_off_d = ar.upload(d.psd_off.data(), nc, s);
            CK(cudaStreamSynchronize(s));
        }
        if (!d.free_idx.empty()) {
            d.free_d = ar.upload(d.free_idx.data(), d.free_idx.size(), s);
            std::vector<int2> ft = row_tiles(d.free_idx);
            d.n_free_tiles = (int)ft.size();
            d.free_tiles = ar.upload(ft.data(), ft.size(), s);
            CK(cudaStreamSynchronize(s)); // ft goes out of scope
        }
    }
    // affine cones (reference initialize_affine_cones, src/pdhcg.c:332-370:
    // block starts already count the scalar rows before F)
    const int na = d.dummy ? 0 : p->affine_cones.num_cones;
    if (na > 0) {
        std::vector<char> in_aff(d.m, 0);
        int amax = 0;
        for (int b = 0; b < na; ++b) {
            const int t = (int)p->affine_cones.type[b], vd = p->affine_cones.v_dim[b];
            const int st = p->affine_cones.start_idx[b], len = pdhcg_b200_cone_length(p->affine_cones.type[b], vd);
            d.aff_start.push_back(st);
            d.aff_len.push_back(len);
            d.aff_type.push_back(t);
            d.aff_vdim.push_back(vd);
            d.aff_alpha.push_back(p->affine_cones.power_alpha ? p->affine_cones.power_alpha[b] : 0.0);
            d.aff_psd_off.push_back(d.psd_total);
            if (t == CONE_PSD) {
                if (vd > PSD_MAX_ORDER)
                    d.unsupported = "affine PSD blocks of order above 22 are not supported yet";
                d.has_psd = true;
                d.psd_total += 2LL * vd * vd;
            }
            amax = std::max(amax, len);
            for (int i = st; i < st + len && i < d.m; ++i)
                in_aff[i] = 1;
        }
        std::vector<int> free_rows;
        for (int i = 0; i < d.m; ++i)
            if (!in_aff[i])
                free_rows.push_back(i);
        std::vector<int2> rt = row_tiles(free_rows);
        d.n_row_tiles = (int)rt.size();
        if (rt.empty())
            rt.push_back(make_int2(0, 0)); // a non-NULL list of no tiles
        d.row_tiles_d = ar.upload(rt.data(), rt.size(), s);
        d.S_aff = slots_class(amax);
        if (d.S_aff < 0) {
            d.unsupported = "cone blocks longer than 256 slots are not supported yet";
            d.S_aff = 1;
        }
        d.ast = ar.upload(d.aff_start.data(), na, s);
        d.alen = ar.upload(d.aff_len.data(), na, s);
        d.atype = ar.upload(d.aff_type.data(), na, s);
        d.avdim = ar.upload(d.aff_vdim.data(), na, s);
        d.aalpha = ar.upload(d.aff_alpha.data(), na, s);
        d.apsd_off_d = ar.upload(d.aff_psd_off.data(), na, s);
        CK(cudaStreamSynchronize(s)); // host vectors go out of scope
    }
    if (d.S < 0)
        d.unsupported = "cone blocks longer than 256 slots are not supported yet";
    if (p->affine_cones.is_fixed)
        d.unsupported = "fixed slots of affine cones are not supported (the reference refuses them too)";
    if (p->num_quadratic_constraints > 0) // the solve entry points transform them first
        d.unsupported = "quadratic constraints must be transformed with qcqp_to_socp_qp first";
    CK(cudaStreamSynchronize(s)); // host sources of the uploads may go away
    return dp;
}

class Solve {
public:
    // own_inputs: the solve may scale dp's arrays in place (dp is temporary)
    Solve(DeviceProblem &dp, bool own_inputs, const pdhg_parameters_t &prm, const pdhcg_b200_options_t &opt)
        : dp_(dp), own_(own_inputs), prm_(prm), opt_(opt)
    {
    }
    ~Solve()
    {
        for (cudaEvent_t e : ev_pool_)
            cudaEventDestroy(e);
        if (st_) {
            cudaStreamSynchronize(st_); // the arena returns its memory on the legacy stream
            cudaStreamDestroy(st_);
            dp_.ar.s = nullptr;
        }
    }
    pdhcg_result_t *run();
    // the device rescaling only (upload, transpose, rescale), factors copied
    // to the host: con_rescale[orig rows], var_rescale[n], bound_obj[2]
    void rescaling(double *con_rescale, double *var_rescale, double *bound_obj);

private:
    void build_host();
    void setup_scratch();
    void check_finite();
    int *nonfinite_ = nullptr;
    void upload_and_preprocess();
    void rescale();
    void init_state();
    void step_size();
    void loop();
    void enqueue_step(bool store_primal, bool store_dual, bool want_fpe, double w);
    void enqueue_step_bb(bool store_dual, bool want_fpe, double w);
    template <typename T>
    void launch_dual(const StepData<T> &D, const StepParams &P);
    template <typename T>
    void enqueue_step_t(bool store_primal, bool store_dual, bool want_fpe, double w);
    template <typename T>
    StepData<T> step_data();
    double step_bytes(size_t s, bool store_primal, bool store_dual) const;
    double bb_inner_bytes(bool fp32) const;
    template <typename V, typename X>
    void long_pass(const DevCsr &M, const V *val, const X *x);
    void enqueue_residual(bool want_dist);
    template <typename VT>
    void enqueue_residual_t(bool want_dist);
    void enter_fp32();
    void leave_fp32();
    void enter_bb_fp32();
    void leave_bb_fp32();
    void read_residual();
    void enqueue_fpe(int slot);
    pdhcg_result_t *make_result();

    DeviceProblem &dp_;
    bool own_;
    pdhg_parameters_t prm_;
    pdhcg_b200_options_t opt_;
    cudaStream_t st_ = nullptr;
    Arena ar_;

    // working problem (dummy row added when m == 0)
    int n_ = 0, m_ = 0;
    int qtype_ = PDHCG_NON_Q;
    bool has_g_ = false, box_free_ = true, eq_rows_ = true, cone_box_ = false;
    std::vector<int> cone_start_, cone_len_, cone_type_, cone_vdim_, free_idx_;
    int S_ = 1;

    // device
    DevCsr A_, At_, Q_, R_, Rt_;
    int r_width_ = 0; // > 0: R dense over columns 0..r_width_-1 (row-major), Rt_ not built
    // inner BB solve (non-diagonal Q)
    bool bb_ = false;
    int bb_grid_ = 0, bb_limit_ = 1, GQ_ = 1;
    double *bb_aty_ = nullptr, *bb_grad_ = nullptr, *bb_dir_ = nullptr, *bb_qx_ = nullptr, *qx_res_ = nullptr;
    double *bb_part_ = nullptr, *bb_rxp_ = nullptr, *bb_rx_ = nullptr, *bb_tol_ = nullptr, *bb_tscale_ = nullptr;
    double *bb_diag_h_ = nullptr, *bb_m_ = nullptr, *bb_minv_ = nullptr;
    int *bb_inner_ = nullptr;
    double bb_cached_inv_tau_ = -1.0, bb_min_tol_ = 1e-9;
    // mixed precision on the inner-solve path: FP32 copies of Q's, R's and
    // R^T's values while bb_fp32_ (iterates and accumulation stay FP64)
    bool bb_fp32_ = false;
    float *Qf_ = nullptr, *Rf_ = nullptr, *Rtf_ = nullptr;
    float *Af_ = nullptr, *Atf_ = nullptr; // and of A's, A^T's values, read by the long-row passes
    long long bb_inner_fp32_ = 0;          // inner iterations taken with the FP32 values
    BBData bb_data() const;
    void setup_bb();
    void enqueue_q_apply(const double *v, double *qx);
    double *c_d_ = nullptr, *l_d_ = nullptr, *u_d_ = nullptr, *q_d_ = nullptr, *lc_d_ = nullptr, *uc_d_ = nullptr,
           *g_d_ = nullptr, *cr_d_ = nullptr, *vr_d_ = nullptr;
    int *free_d_ = nullptr, *cst_d_ = nullptr, *clen_d_ = nullptr, *ctype_d_ = nullptr, *cvdim_d_ = nullptr;
    double *cone_warm_ = nullptr, *warm_dual_ = nullptr, *warm_aug_ = nullptr; // per-cone multipliers
    double *psd_work_ = nullptr; // PSD blocks' eigen-decomposition scratch (2 n^2 doubles each)
    double *x0_, *x_, *xp_, *xr_, *dx_, *dslack_, *y0_, *y_, *yp_, *dy_;
    // FP32 mirrors of the matrices, problem vectors and iterates (mixed precision)
    struct {
        float *Av = nullptr, *Atv = nullptr, *c = nullptr, *l = nullptr, *u = nullptr, *q = nullptr, *lc = nullptr,
              *uc = nullptr, *g = nullptr, *vr = nullptr;
        float *x0 = nullptr, *x = nullptr, *xp = nullptr, *xr = nullptr, *dx = nullptr, *dslack = nullptr;
        float *y0 = nullptr, *y = nullptr, *yp = nullptr, *dy = nullptr;
    } f_;
    bool fp32_ = false;
    double step_bytes_sum_ = 0.0;
    double best_fp32_kkt_ = INFINITY;
    int fp32_stall_ = 0;
    double *partials_ = nullptr, *scal_d_ = nullptr, *h_scal_ = nullptr;
    int *res_ops_d_ = nullptr, *fpe_ops_d_ = nullptr, *norm_ops_d_ = nullptr;
    int *rayn_ops_d_ = nullptr, *ray_ops_d_ = nullptr;
    double *ray_d_ = nullptr; // [RN_COUNT + RY_COUNT] folded certificate scalars
    // infeasibility certificates of the last computation (zero until then)
    double p_ray_obj_ = 0.0, d_ray_obj_ = 0.0, max_p_ray_ = 0.0, max_d_ray_ = 0.0;
    void compute_infeasibility();
    int res_rows_blocks_ = 0, res_free_blocks_ = 0, res_cone_blocks_ = 0, res_aff_blocks_ = 0;
    int fpe_col_blocks_ = 0, fpe_row_blocks_ = 0;

    // scaling
    double sb_ = 1.0, sc_ = 1.0, cnorm_ = 0.0, bnorm_ = 0.0;

    // iteration state (host scalars, reference pdhg_solver_state_t)
    double step_ = 0.0, omega_ = 1.0, best_omega_ = 1.0, best_gap_ = INFINITY;
    double pw_err_sum_ = 0.0, pw_last_err_ = 0.0;
    int k_ = 0, inner_count_ = 0;
    long long inner_total_ = 0;
    bool is_major_ = false;
    double fpe_ = 0.0, fpe0_ = 0.0, fpe_last_ = INFINITY;
    double abs_p_ = 0, rel_p_ = 0, abs_d_ = 0, rel_d_ = 0, pobj_ = 0, dobj_ = 0, gap_ = 0, rel_gap_ = 0;
    double dist_x_ = 0, dist_y_ = 0;
    bool pending_fpe0_ = false;
    int pending_fpe_slot_ = -1;
    termination_reason_t reason_ = TERMINATION_REASON_UNSPECIFIED;
    double cum_time_ = 0.0;
    pdhcg_b200_stats_t stats_{};
    double nonconvexity_ = 0.0;

    // optional CUDA-event timing of the fused step kernels: pairs of events
    // recorded around each step, harvested at every host synchronisation
    std::vector<cudaEvent_t> ev_pool_;
    size_t ev_used_ = 0;
    void harvest_step_events();
};


template <typename F>
void dispatch_s(int S, F &&f)
{
    switch (S) {
    case 1: f(std::integral_constant<int, 1>{}); break;
    case 2: f(std::integral_constant<int, 2>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    default: f(std::integral_constant<int, 8>{}); break;
    }
}

// Primal step over the cone blocks: the SOC / RSOC blocks with S slots per
// lane, the 3-slot blocks with one; returns the number of launches.
template <typename T>
int launch_primal_cones(const StepData<T> &D, const StepParams &P, const ConeSplit &sp, int S, bool hasq,
                        cudaStream_t s)
{
    int launches = 0;
    if (sp.n_wide > 0) {
        // no more blocks than are resident at once: each warp then walks
        // several cone blocks and the warps drift apart, so one warp's
        // projection arithmetic overlaps other warps' loads (a full grid
        // starts every resident warp on its loads together); ~4 % of the
        // step on 20000 SOC blocks of 50
        dispatch_s(S, [&](auto SC) {
            if (hasq) {
                auto k = primal_cone_kernel<SC.value, T, true, CONES_WIDE>;
                int grid = std::min(grid_for(sp.n_wide, WARPS), resident_blocks((const void *)k));
                k<<<grid, TPB, 0, s>>>(D, P, sp.wide_d, sp.n_wide);
            } else {
                auto k = primal_cone_kernel<SC.value, T, false, CONES_WIDE>;
                int grid = std::min(grid_for(sp.n_wide, WARPS), resident_blocks((const void *)k));
                k<<<grid, TPB, 0, s>>>(D, P, sp.wide_d, sp.n_wide);
            }
        });
        ++launches;
    }
    if (sp.n_three > 0) {
        int grid = grid_for(sp.n_three, WARPS);
        if (hasq)
            primal_cone_kernel<1, T, true, CONES_THREE><<<grid, TPB, 0, s>>>(D, P, sp.three_d, sp.n_three);
        else
            primal_cone_kernel<1, T, false, CONES_THREE><<<grid, TPB, 0, s>>>(D, P, sp.three_d, sp.n_three);
        ++launches;
    }
    if (sp.n_psd > 0) { // LP path only: diagonal Q with PSD blocks takes the inner BB solve
        dispatch_s(S, [&](auto SC) {
            int grid = grid_for(sp.n_psd, WARPS);
            if (hasq)
                primal_cone_kernel<SC.value, T, true, CONES_PSD><<<grid, TPB, 0, s>>>(D, P, sp.psd_d, sp.n_psd);
            else
                primal_cone_kernel<SC.value, T, false, CONES_PSD><<<grid, TPB, 0, s>>>(D, P, sp.psd_d, sp.n_psd);
        });
        ++launches;
    }
    if (sp.n_sect > 0) { // blocks with fixed slots: section projectors, one slot class (any block length)
        int grid = grid_for(sp.n_sect, WARPS);
        if (hasq)
            primal_cone_kernel<8, T, true, CONES_SECTION><<<grid, TPB, 0, s>>>(D, P, sp.sect_d, sp.n_sect);
        else
            primal_cone_kernel<8, T, false, CONES_SECTION><<<grid, TPB, 0, s>>>(D, P, sp.sect_d, sp.n_sect);
        ++launches;
    }
    return launches;
}

template <typename F>
void dispatch_rg(int G, F &&f)
{
    switch (G) {
    case 1: f(std::integral_constant<int, 1>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    default: f(std::integral_constant<int, 32>{}); break;
    }
}

// ---- working copy on the device --------------------------------------------
void Solve::build_host()
{
    n_ = dp_.n;
    m_ = dp_.m;
    qtype_ = dp_.qtype;
    has_g_ = dp_.has_g;
    box_free_ = dp_.box_free;
    eq_rows_ = dp_.eq_rows;
    cone_box_ = dp_.cone_box;
    cone_start_ = dp_.cone_start;
    cone_len_ = dp_.cone_len;
    cone_type_ = dp_.cone_type;
    cone_vdim_ = dp_.cone_vdim;
    free_idx_ = dp_.free_idx;
    S_ = dp_.S;
}

void Solve::upload_and_preprocess()
{
    cudaStream_t s = st_;
    auto mut = [&](double *src, size_t k) -> double * { // arrays the solve rescales in place
        if (own_)
            return src;
        double *d = ar_.alloc<double>(k);
        if (k)
            CK(cudaMemcpyAsync(d, src, k * sizeof(double), cudaMemcpyDeviceToDevice, s));
        return d;
    };
    A_.rows = m_;
    A_.cols = n_;
    A_.nnz = dp_.nnzA;
    A_.rp = dp_.A_rp;
    A_.ci = dp_.A_ci;
    A_.v = mut(dp_.A_v, dp_.nnzA);
    build_long_rows(A_, ar_, s);
    At_ = transpose(A_, ar_, s);
    build_long_rows(At_, ar_, s);
    c_d_ = mut(dp_.c, n_);
    l_d_ = mut(dp_.l, n_);
    u_d_ = mut(dp_.u, n_);
    lc_d_ = mut(dp_.lc, m_);
    uc_d_ = mut(dp_.uc, m_);
    g_d_ = mut(dp_.g, m_);
    if (qtype_ != PDHCG_NON_Q) {
        Q_.rows = n_;
        Q_.cols = n_;
        Q_.nnz = dp_.nnzQ;
        Q_.rp = dp_.Q_rp;
        Q_.ci = dp_.Q_ci;
        Q_.v = mut(dp_.Q_v, dp_.nnzQ);
    }
    if (dp_.nnzR > 0) {
        R_.rows = dp_.rank;
        R_.cols = n_;
        R_.nnz = dp_.nnzR;
        R_.rp = dp_.R_rp;
        R_.ci = dp_.R_ci;
        R_.v = mut(dp_.R_v, dp_.nnzR);
        // an R whose rows all hold the same leading columns 0..w-1 in order
        // (a dense R, possibly zero on trailing auxiliary columns) is read
        // row-major by both products and needs no transpose
        r_width_ = 0;
        const int w = R_.rows > 0 ? R_.nnz / R_.rows : 0;
        if (w > 0 && w <= R_.cols && (long long)w * R_.rows == (long long)R_.nnz) {
            int *bad = ar_.alloc<int>(1);
            CK(cudaMemsetAsync(bad, 0, sizeof(int), s));
            dense_rows_check_kernel<<<grid_for(R_.nnz, TPB), TPB, 0, s>>>(R_.rows, w, R_.rp, R_.ci, bad);
            int h = 1;
            CK(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            r_width_ = h == 0 ? w : 0;
        }
        if (!r_width_) {
            build_long_rows(R_, ar_, s);
            Rt_ = transpose(R_, ar_, s);
        }
    }
    cst_d_ = dp_.cst;
    clen_d_ = dp_.clen;
    ctype_d_ = dp_.ctype;
    cvdim_d_ = dp_.cvdim;
    free_d_ = dp_.free_d;
}

// ---- rescaling (reference rescale_problem, src/preconditioner.c:654-713) --
void Solve::rescale()
{
    cudaStream_t s = st_;
    int n = n_, m = m_, nc = (int)cone_start_.size(), na = (int)dp_.aff_start.size();
    cr_d_ = ar_.alloc<double>(m);
    vr_d_ = ar_.alloc<double>(n);
    double *fcr = ar_.alloc<double>(m), *fvr = ar_.alloc<double>(n);
    std::vector<double> ones_n(n, 1.0), ones_m(m, 1.0);
    CK(cudaMemcpyAsync(cr_d_, ones_m.data(), m * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(vr_d_, ones_n.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    bool pres = prm_.use_cone_preserving_scaling;
    // scale the problem by (fcr, fvr) (reference scale_problem, src/preconditioner.c:231-332)
    auto apply_scaling = [&]() {
        scale_csr_kernel<<<grid_for(m, TPB), TPB, 0, s>>>(A_.rp, A_.ci, A_.v, m, fcr, fvr, 0, A_.lr.n > 0);
        scale_csr_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(At_.rp, At_.ci, At_.v, n, fvr, fcr, 1, At_.lr.n > 0);
        if (A_.lr.n > 0)
            long_scale_csr_kernel<<<std::min(A_.lr.n, 148 * 16), TPB, 0, s>>>(A_.lr, A_.rp, A_.ci, A_.v, fcr, fvr, 0);
        if (At_.lr.n > 0)
            long_scale_csr_kernel<<<std::min(At_.lr.n, 148 * 16), TPB, 0, s>>>(At_.lr, At_.rp, At_.ci, At_.v, fvr,
                                                                             fcr, 1);
        if (Q_.nnz > 0)
            scale_csr_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(Q_.rp, Q_.ci, Q_.v, n, fvr, fvr, 0, 0);
        if (R_.nnz > 0) { // R /= D_var by columns (reference scale_problem, src/preconditioner.c:295-307)
            scale_cols_kernel<<<grid_for(R_.nnz, TPB), TPB, 0, s>>>(R_.ci, R_.v, R_.nnz, fvr);
            if (Rt_.nnz > 0)
                scale_rows_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(Rt_.rp, Rt_.v, n, fvr);
        }
        scale_vectors_kernel<<<grid_for((long long)n + m, TPB), TPB, 0, s>>>(n, m, c_d_, l_d_, u_d_, fvr, lc_d_,
                                                                             uc_d_, g_d_, fcr, vr_d_, cr_d_);
        CK(cudaGetLastError());
    };
    // Ruiz / Pock-Chambolle factors: square roots, then the cone adjustment
    auto apply = [&](int ruiz_phase) {
        CK(cudaGetLastError());
        sqrt_or_one_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(fvr, n);
        sqrt_or_one_kernel<<<grid_for(m, TPB), TPB, 0, s>>>(fcr, m);
        if (nc > 0) {
            if (pres)
                cone_scaling_adjust_kernel<<<grid_for(nc, TPB), TPB, 0, s>>>(fvr, nc, cst_d_, clen_d_, ruiz_phase);
            else
                psd_scaling_kernel<<<grid_for(nc, TPB), TPB, 0, s>>>(fvr, nc, cst_d_, cvdim_d_, ctype_d_, 0);
        }
        if (na > 0) { // affine blocks: the same on the row factors
            if (pres)
                cone_scaling_adjust_kernel<<<grid_for(na, TPB), TPB, 0, s>>>(fcr, na, dp_.ast, dp_.alen, ruiz_phase);
            else
                psd_scaling_kernel<<<grid_for(na, TPB), TPB, 0, s>>>(fcr, na, dp_.ast, dp_.avdim, dp_.atype, 0);
        }
        apply_scaling();
    };
    if (prm_.curtis_reid_iterations > 0 && m > 0 && n > 0 && A_.nnz > 0) {
        // reference curtis_reid_rescaling, src/preconditioner.c:334-495
        double *rsum = ar_.alloc<double>(m), *csum = ar_.alloc<double>(n), *cs = ar_.alloc<double>(n);
        double *rs = ar_.alloc<double>(m); // row numerators before the division by the row count
        CK(cudaMemsetAsync(fvr, 0, n * sizeof(double), s)); // column log-scales start at 0
        cr_logsum_kernel<<<grid_for(m, TPB), TPB, 0, s>>>(A_.rp, A_.v, m, rsum);
        cr_logsum_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(At_.rp, At_.v, n, csum);
        for (int it = 0; it < prm_.curtis_reid_iterations; ++it) {
            cr_average_kernel<<<grid_for(m, TPB), TPB, 0, s>>>(A_.rp, A_.ci, m, rsum, fvr, fcr, rs);
            if (na > 0 && pres) // affine blocks averaged together, as the columns of a cone block
                cr_cone_average_kernel<<<grid_for(na, TPB), TPB, 0, s>>>(na, dp_.ast, dp_.alen, A_.rp, rs, fcr);
            else if (na > 0)
                psd_scaling_kernel<<<grid_for(na, TPB), TPB, 0, s>>>(fcr, na, dp_.ast, dp_.avdim, dp_.atype, 1);
            cr_average_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(At_.rp, At_.ci, n, csum, fcr, fvr, cs);
            if (nc > 0 && pres)
                cr_cone_average_kernel<<<grid_for(nc, TPB), TPB, 0, s>>>(nc, cst_d_, clen_d_, At_.rp, cs, fvr);
            else if (nc > 0)
                psd_scaling_kernel<<<grid_for(nc, TPB), TPB, 0, s>>>(fvr, nc, cst_d_, cvdim_d_, ctype_d_, 1);
        }
        cr_exp_kernel<<<grid_for(m, TPB), TPB, 0, s>>>(fcr, m);
        cr_exp_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(fvr, n);
        apply_scaling();
    }
    for (int it = 0; it < prm_.l_inf_ruiz_iterations; ++it) {
        row_absmax_kernel<<<grid_for(m, TPB), TPB, 0, s>>>(A_.rp, A_.v, m, fcr, A_.lr.n > 0);
        row_absmax_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(At_.rp, At_.v, n, fvr, At_.lr.n > 0);
        if (A_.lr.n > 0)
            long_row_absmax_kernel<<<std::min(A_.lr.n, 148 * 16), TPB, 0, s>>>(A_.lr, A_.rp, A_.v, fcr);
        if (At_.lr.n > 0)
            long_row_absmax_kernel<<<std::min(At_.lr.n, 148 * 16), TPB, 0, s>>>(At_.lr, At_.rp, At_.v, fvr);
        apply(1);
    }
    if (prm_.has_pock_chambolle_alpha) {
        double a = prm_.pock_chambolle_alpha;
        row_powsum_kernel<<<grid_for(m, TPB), TPB, 0, s>>>(A_.rp, A_.v, m, a, fcr, A_.lr.n > 0);
        row_powsum_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(At_.rp, At_.v, n, 2.0 - a, fvr, At_.lr.n > 0);
        if (A_.lr.n > 0)
            long_row_powsum_kernel<<<std::min(A_.lr.n, 148 * 16), TPB, 0, s>>>(A_.lr, A_.rp, A_.v, a, fcr);
        if (At_.lr.n > 0)
            long_row_powsum_kernel<<<std::min(At_.lr.n, 148 * 16), TPB, 0, s>>>(At_.lr, At_.rp, At_.v, 2.0 - a, fvr);
        apply(0);
    }
    if (prm_.bound_objective_rescaling) {
        int nb = grid_for((long long)n + m, TPB, 148 * 4);
        norms_kernel<<<nb, TPB, 0, s>>>(n, m, c_d_, lc_d_, uc_d_, g_d_, partials_);
        fold_partials_kernel<<<1, TPB, 0, s>>>(partials_, nb, NS_COUNT, norm_ops_d_, scal_d_);
        double h[NS_COUNT];
        CK(cudaMemcpyAsync(h, scal_d_, sizeof(h), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        sb_ = 1.0 / (std::sqrt(h[NS_B2]) + 1.0);
        sc_ = 1.0 / (std::sqrt(h[NS_C2]) + 1.0);
        bound_obj_scale_kernel<<<grid_for((long long)n + m, TPB), TPB, 0, s>>>(n, m, sb_, sc_, c_d_, l_d_, u_d_,
                                                                               lc_d_, uc_d_, g_d_);
        if (Q_.nnz > 0)
            mul_scalar_kernel<<<grid_for(Q_.nnz, TPB), TPB, 0, s>>>(Q_.v, Q_.nnz, sc_ / sb_);
        if (R_.nnz > 0) {
            double f = std::sqrt(sc_ / sb_);
            mul_scalar_kernel<<<grid_for(R_.nnz, TPB), TPB, 0, s>>>(R_.v, R_.nnz, f);
            if (Rt_.nnz > 0)
                mul_scalar_kernel<<<grid_for(Rt_.nnz, TPB), TPB, 0, s>>>(Rt_.v, Rt_.nnz, f);
        }
    }
    if (dp_.n_fix > 0) // fixed cone slots: scaled bounds pinned at the scaled value
        pin_fixed_kernel<<<grid_for(dp_.n_fix, TPB), TPB, 0, s>>>(dp_.n_fix, dp_.fix_idx, dp_.fix_val, vr_d_, sb_,
                                                                  l_d_, u_d_);
    CK(cudaGetLastError());
}

void Solve::init_state()
{
    cudaStream_t s = st_;
    int n = n_, m = m_, nc = (int)cone_start_.size();
    x0_ = ar_.alloc<double>(n);
    x_ = ar_.alloc<double>(n);
    xp_ = ar_.alloc<double>(n);
    xr_ = ar_.alloc<double>(n);
    dx_ = ar_.alloc<double>(n);
    dslack_ = ar_.alloc<double>(n);
    y0_ = ar_.alloc<double>(m);
    y_ = ar_.alloc<double>(m);
    yp_ = ar_.alloc<double>(m);
    dy_ = ar_.alloc<double>(m);
    CK(cudaMemsetAsync(x0_, 0, n * sizeof(double), s));
    CK(cudaMemsetAsync(dslack_, 0, n * sizeof(double), s));
    if (dp_.pstart)
        scale_start_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(n, dp_.pstart, vr_d_, sb_, x0_);
    const double *ds = dp_.dstart;
    dual_start_kernel<<<grid_for(m, TPB), TPB, 0, s>>>(m, ds, cr_d_, sc_, y0_, y_, yp_);
    if (dp_.has_psd) // variable and affine PSD blocks
        psd_work_ = ar_.alloc<double>((size_t)dp_.psd_total);
    if (nc > 0) {
        cone_warm_ = ar_.alloc<double>(3 * (size_t)nc);
        warm_dual_ = cone_warm_ + nc;
        warm_aug_ = cone_warm_ + 2 * (size_t)nc;
        CK(cudaMemsetAsync(cone_warm_, 0, 3 * (size_t)nc * sizeof(double), s)); // 0 = no warm start
        cone_aux_init_kernel<<<grid_for(nc, TPB), TPB, 0, s>>>(nc, cst_d_, cvdim_d_, ctype_d_, vr_d_, sb_, x0_,
                                                               dp_.fixed_d);
        dispatch_s(S_, [&](auto SC) {
            project_cones_kernel<SC.value><<<grid_for(nc, WARPS), TPB, 0, s>>>(
                nc, cst_d_, clen_d_, ctype_d_, dp_.calpha, x0_, vr_d_, nullptr, 0.0, psd_work_, dp_.psd_off_d,
                dp_.fixed_d, dp_.cfix_d, cone_warm_);
        });
    }
    box_clamp_copy_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(n, l_d_, u_d_, x0_, x_, xp_, xr_);
    if (qtype_ == PDHCG_DIAG_Q) {
        q_d_ = ar_.alloc<double>(n);
        CK(cudaMemsetAsync(q_d_, 0, n * sizeof(double), s));
        q_diag_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(Q_.rp, Q_.ci, Q_.v, n, q_d_);
        std::vector<double> qh(n);
        CK(cudaMemcpyAsync(qh.data(), q_d_, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        double mn = 0.0;
        for (double v : qh)
            mn = std::fmin(mn, v);
        nonconvexity_ = mn; // reference initialize_quadratic_term_information, src/solver_state.cu:400-418
    }
    CK(cudaGetLastError());
}

// ---- inner BB solve set-up (reference initialize_inner_solver and
// initialize_quadratic_term_information, src/solver_state.cu:280-420) -------
BBData Solve::bb_data() const
{
    BBData D{};
    D.n = n_;
    D.c = c_d_;
    D.l = l_d_;
    D.u = u_d_;
    D.aty = bb_aty_;
    D.sparse = Q_.nnz > 0;
    D.Q_rp = Q_.rp;
    D.Q_ci = Q_.ci;
    D.Q_v = Q_.v;
    D.k = R_.nnz > 0 ? R_.rows : 0;
    D.R_rp = R_.rp;
    D.R_ci = R_.ci;
    D.R_v = R_.v;
    D.Rt_rp = Rt_.rp;
    D.Rt_ci = Rt_.ci;
    D.Rt_v = Rt_.v;
    D.r_width = r_width_;
    D.dkind = dp_.dkind;
    D.Ddiag = dp_.Ddiag;
    D.Ddense = dp_.Ddense;
    D.Q_vf = bb_fp32_ && Q_.nnz > 0 ? Qf_ : nullptr;
    D.R_vf = bb_fp32_ && R_.nnz > 0 ? Rf_ : nullptr;
    D.Rt_vf = bb_fp32_ && Rt_.nnz > 0 && !r_width_ ? Rtf_ : nullptr;
    D.m_diag = bb_m_;
    D.m_inv = bb_minv_;
    D.tol_scale = bb_tscale_;
    D.free_idx = free_d_;
    D.n_free = (int)free_idx_.size();
    D.cone_start = cst_d_;
    D.cone_len = clen_d_;
    D.cone_type = ctype_d_;
    D.cone_alpha = dp_.calpha;
    D.psd_work = psd_work_;
    D.psd_off = dp_.psd_off_d;
    D.n_cones = (int)cone_start_.size();
    D.vr = vr_d_;
    D.cone_warm = cone_warm_;
    D.fixed = dp_.fixed_d;
    D.cone_fixed = dp_.cfix_d;
    D.x0 = x0_;
    D.x = x_;
    D.xp = xp_;
    D.xr = xr_;
    D.dx = dx_;
    D.grad = bb_grad_;
    D.dir = bb_dir_;
    D.qx = bb_qx_;
    D.part = bb_part_;
    D.rx_part = bb_rxp_;
    D.rx = bb_rx_;
    D.tol = bb_tol_;
    D.limit = bb_limit_;
    D.inner_total = bb_inner_;
    return D;
}

void Solve::setup_bb()
{
    cudaStream_t s = st_;
    int n = n_;
    // a dense R is read by columns, one thread per variable (coalesced over
    // the threads of a warp); otherwise lanes per row from the mean row length
    GQ_ = r_width_ ? 1 : residual_group(pick_group((long long)Q_.nnz + Rt_.nnz, n));
    // cooperative grid: every block resident at once
    int dev = 0, nsm = 0, per_sm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    // problems with fixed cone slots take the widest slot class (one
    // instantiation per row group serves every block length)
    dispatch_rg(GQ_, [&](auto GC) {
        if (dp_.has_fixed)
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bb_kernel<GC.value, 8, true>, TPB, 0));
        else
            dispatch_s(S_, [&](auto SC) {
                CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bb_kernel<GC.value, SC.value, false>, TPB,
                                                                 0));
            });
    });
    int q_per_sm = 0;
    dispatch_rg(GQ_, [&](auto GC) {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&q_per_sm, q_apply_kernel<GC.value>, TPB, 0));
    });
    per_sm = std::min(per_sm, q_per_sm);
    if (per_sm < 1)
        throw CudaError("inner BB kernel cannot be made resident");
    bb_grid_ = nsm * std::min(per_sm, 4);
    int k = R_.nnz > 0 ? R_.rows : 0;
    bb_aty_ = ar_.alloc<double>(n);
    bb_grad_ = ar_.alloc<double>(n);
    bb_dir_ = ar_.alloc<double>(n);
    bb_qx_ = ar_.alloc<double>(n);
    qx_res_ = ar_.alloc<double>(n);
    bb_part_ = ar_.alloc<double>((size_t)4 * bb_grid_);
    bb_rxp_ = ar_.alloc<double>((size_t)bb_grid_ * std::max(k, 1));
    bb_rx_ = ar_.alloc<double>(std::max(k, 1));
    bb_tol_ = ar_.alloc<double>(2);
    bb_tscale_ = bb_tol_ + 1;
    bb_inner_ = ar_.alloc<int>(1);
    CK(cudaMemsetAsync(bb_inner_, 0, sizeof(int), s));
    int lim = prm_.inner_solver_parameters.iteration_limit;
    double it0 = prm_.inner_solver_parameters.initial_tolerance;
    double mt = prm_.inner_solver_parameters.min_tolerance;
    if (lim < 1)
        lim = 1;
    if (it0 <= 0.0)
        it0 = 1e-3;
    if (mt <= 0.0)
        mt = 1e-9;
    bb_limit_ = lim;
    bb_min_tol_ = mt;
    double init[2] = {it0, 1.0};
    CK(cudaMemcpyAsync(bb_tol_, init, sizeof(init), cudaMemcpyHostToDevice, s));
    if (prm_.diag_jacobi_precond && !dp_.var_psd) { // the reference runs PSD models unpreconditioned
        bb_diag_h_ = ar_.alloc<double>(n);
        bb_m_ = ar_.alloc<double>(n);
        bb_minv_ = ar_.alloc<double>(n);
        bb_diag_h_kernel<<<grid_for(n, TPB), TPB, 0, s>>>(n, Q_.nnz > 0, Q_.rp, Q_.ci, Q_.v, k, Rt_.rp, Rt_.ci,
                                                          Rt_.v, r_width_ ? R_.v : nullptr, r_width_, dp_.dkind,
                                                          dp_.Ddiag, dp_.Ddense, bb_diag_h_);
    }
    // eigenvalues of a sparse Q (the reference computes them for SPARSE_Q only)
    if (qtype_ == PDHCG_SPARSE_Q) {
        std::vector<double> v0(n);
        unsigned int seed = 1234;
        for (int i = 0; i < n; ++i)
            v0[i] = (double)rand_r(&seed) / RAND_MAX;
        double *v = ar_.alloc<double>(n), *av = ar_.alloc<double>(n), *out = ar_.alloc<double>(2);
        double *part = ar_.alloc<double>((size_t)2 * bb_grid_);
        int eper = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&eper, power_eig_kernel, TPB, 0));
        int eg = std::max(1, std::min(bb_grid_, nsm * std::max(eper, 1)));
        double lmax = 0.0;
        for (int shifted = 0; shifted < 2; ++shifted) {
            CK(cudaMemcpyAsync(v, v0.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
            int maxit = prm_.sv_max_iter;
            double tol = prm_.sv_tol;
            void *args[] = {&n, &Q_.rp, &Q_.ci, &Q_.v, &v, &av, &part, &maxit, &tol, &shifted, &lmax, &out};
            CK(cudaLaunchCooperativeKernel((void *)power_eig_kernel, eg, TPB, args, 0, s));
            double h[2];
            CK(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (shifted)
                nonconvexity_ = h[0];
            else
                lmax = h[0];
        }
    }
    if (nonconvexity_ < 0)
        bb_limit_ = 1; // reference optimize, src/solver.cu:109-112
    CK(cudaGetLastError());
}

void Solve::enqueue_q_apply(const double *v, double *qx)
{
    BBData D = bb_data();
    int grid = bb_grid_;
    dispatch_rg(GQ_, [&](auto GC) {
        void *args[] = {&D, (void *)&v, &qx};
        CK(cudaLaunchCooperativeKernel((void *)q_apply_kernel<GC.value>, grid, TPB, args, 0, st_));
    });
    stats_.kernel_launches++;
}

// ---- step size (reference initialize_step_size_and_primal_weight,
// src/pdhg_core_op.cu:933-971) -------------------------------------------
void Solve::step_size()
{
    cudaStream_t s = st_;
    if (A_.nnz == 0) {
        step_ = 1.0;
    } else if (opt_.has_initial_step_size && opt_.initial_step_size > 0.0) {
        step_ = opt_.initial_step_size; // from a previous solve with the same scaled A
    } else {
        int m = m_, n = n_;
        std::vector<double> v0(m);
        unsigned int seed = 1234;
        for (int i = 0; i < m; ++i)
            v0[i] = ((double)rand_r(&seed) / (double)RAND_MAX) * 2.0 - 1.0;
        double *v = ar_.upload(v0.data(), m, s), *nv = ar_.alloc<double>(m), *dp = ar_.alloc<double>(n);
        double *out = ar_.alloc<double>(2);
        int dev = 0, nsm = 0, per_sm = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, power_sigma_kernel<double>, TPB, 0));
        int grid = std::max(1, std::min(nsm * std::max(per_sm, 1), nsm * 4));
        double *part = ar_.alloc<double>((size_t)4 * grid);
        int max_iter = prm_.sv_max_iter;
        double tol = prm_.sv_tol;
        LongRows al = A_.lr, atl = At_.lr;
        void *args[] = {&m, &n, &A_.rp, &A_.ci, &A_.v, &At_.rp, &At_.ci, &At_.v, &v, &nv, &dp, &part, &max_iter,
                        &tol, &out, &al, &atl};
        CK(cudaLaunchCooperativeKernel((void *)power_sigma_kernel<double>, grid, TPB, args, 0, s));
        double h[2];
        CK(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        double sv = h[0];
        step_ = sv < 1e-12 ? 1.0 : 0.998 / sv;
    }
    omega_ = prm_.bound_objective_rescaling ? 1.0 : (cnorm_ + 1.0) / (bnorm_ + 1.0);
    if (opt_.has_initial_primal_weight && opt_.initial_primal_weight > 0.0)
        omega_ = opt_.initial_primal_weight;
    best_omega_ = omega_;
}

void Solve::harvest_step_events()
{
    for (size_t i = 0; i + 1 < ev_used_; i += 2) {
        float ms = 0.0f;
        CK(cudaEventSynchronize(ev_pool_[i + 1]));
        CK(cudaEventElapsedTime(&ms, ev_pool_[i], ev_pool_[i + 1]));
        stats_.step_kernel_ms += ms;
    }
    ev_used_ = 0;
}

template <typename T>
StepData<T> Solve::step_data()
{
    StepData<T> D{};
    D.row_tiles = dp_.aff_start.empty() ? nullptr : dp_.row_tiles_d; // rows outside the affine blocks
    D.n_row_tiles = dp_.n_row_tiles;
    D.aff_start = dp_.ast;
    D.aff_len = dp_.alen;
    D.aff_type = dp_.atype;
    D.aff_alpha = dp_.aalpha;
    D.aff_psd_off = dp_.apsd_off_d;
    D.n_aff = (int)dp_.aff_start.size();
    D.cr = cr_d_;
    D.A_long = A_.lr;
    D.At_long = At_.lr;
    D.cone_warm = cone_warm_;
    D.fixed = dp_.fixed_d;
    D.n = n_;
    D.m = m_;
    D.A_rp = A_.rp;
    D.A_ci = A_.ci;
    D.At_rp = At_.rp;
    D.At_ci = At_.ci;
    D.free_idx = free_d_;
    D.n_free = (int)free_idx_.size();
    D.free_tiles = dp_.free_tiles;
    D.n_free_tiles = dp_.n_free_tiles;
    D.cone_start = cst_d_;
    D.cone_len = clen_d_;
    D.cone_type = ctype_d_;
    D.cone_alpha = dp_.calpha;
    D.psd_work = psd_work_;
    D.psd_off = dp_.psd_off_d;
    D.n_cones = (int)cone_start_.size();
    if constexpr (std::is_same<T, double>::value) {
        D.A_v = A_.v;
        D.At_v = At_.v;
        D.c = c_d_;
        D.l = l_d_;
        D.u = u_d_;
        D.q = q_d_;
        D.lc = lc_d_;
        D.uc = uc_d_;
        D.g = g_d_;
        D.vr = vr_d_;
        D.x0 = x0_;
        D.x = x_;
        D.xp = xp_;
        D.xr = xr_;
        D.dx = dx_;
        D.dual_slack = dslack_;
        D.y0 = y0_;
        D.y = y_;
        D.yp = yp_;
        D.dy = dy_;
    } else {
        D.A_v = f_.Av;
        D.At_v = f_.Atv;
        D.c = f_.c;
        D.l = f_.l;
        D.u = f_.u;
        D.q = f_.q;
        D.lc = f_.lc;
        D.uc = f_.uc;
        D.g = f_.g;
        D.vr = f_.vr;
        D.x0 = f_.x0;
        D.x = f_.x;
        D.xp = f_.xp;
        D.xr = f_.xr;
        D.dx = f_.dx;
        D.dual_slack = f_.dslack;
        D.y0 = f_.y0;
        D.y = f_.y;
        D.yp = f_.yp;
        D.dy = f_.dy;
    }
    return D;
}

template <typename T>
void Solve::launch_dual(const StepData<T> &D, const StepParams &P)
{
    cudaStream_t s = st_;
    if constexpr (std::is_same<T, double>::value) {
        if (bb_fp32_ && Af_)
            long_pass(A_, (const float *)Af_, D.xr);
        else
            long_pass(A_, D.A_v, D.xr);
    } else {
        long_pass(A_, D.A_v, D.xr);
    }
    if (D.n_aff > 0) { // affine cone blocks: one warp each
        dispatch_s(dp_.S_aff, [&](auto SC) {
            dual_cone_kernel<SC.value, T><<<grid_for(D.n_aff, WARPS), TPB, 0, s>>>(D, P);
        });
        stats_.kernel_launches++;
        if (D.n_row_tiles == 0)
            return;
    }
    int grid = grid_for(D.row_tiles ? (long long)D.n_row_tiles : ((long long)m_ + 31) / 32, WARPS);
    if (eq_rows_) {
        if (has_g_)
            dual_kernel<T, true, true><<<grid, TPB, 0, s>>>(D, P);
        else
            dual_kernel<T, true, false><<<grid, TPB, 0, s>>>(D, P);
    } else {
        if (has_g_)
            dual_kernel<T, false, true><<<grid, TPB, 0, s>>>(D, P);
        else
            dual_kernel<T, false, false><<<grid, TPB, 0, s>>>(D, P);
    }
    stats_.kernel_launches++;
}

// BB path: A^T y, preconditioner refresh when tau changed, the cooperative
// inner solve (which also writes x_refl and the Halpern x), then the dual step.
void Solve::enqueue_step_bb(bool store_dual, bool want_fpe, double w)
{
    cudaStream_t s = st_;
    if (opt_.time_steps) {
        if (ev_used_ + 2 > ev_pool_.size()) {
            for (int i = 0; i < 64; ++i) {
                cudaEvent_t e;
                CK(cudaEventCreate(&e));
                ev_pool_.push_back(e);
            }
        }
        CK(cudaEventRecord(ev_pool_[ev_used_++], s));
    }
    double tau = step_ / omega_;
    if (nonconvexity_ < 0) {
        tau = std::fmax(tau, -1.01 * std::fmin(0.0, nonconvexity_));
        tau /= 100;
    }
    if (bb_fp32_ && Atf_)
        long_pass(At_, (const float *)Atf_, y_);
    else
        long_pass(At_, At_.v, y_);
    spmv_kernel<<<grid_for(((long long)n_ + 31) / 32, WARPS), TPB, 0, s>>>(n_, At_.rp, At_.ci, At_.v, y_, bb_aty_,
                                                                          At_.lr);
    double inv_tau = 1.0 / tau;
    if (bb_m_ && inv_tau != bb_cached_inv_tau_) {
        int nb = grid_for(n_, TPB, 148 * 4);
        bb_precond_kernel<<<nb, TPB, 0, s>>>(n_, bb_diag_h_, inv_tau, bb_m_, bb_minv_, partials_);
        fold_partials_kernel<<<1, TPB, 0, s>>>(partials_, nb, 1, fpe_ops_d_, bb_part_);
        bb_tol_scale_kernel<<<1, 1, 0, s>>>(bb_part_, n_, bb_tscale_);
        bb_cached_inv_tau_ = inv_tau;
        stats_.kernel_launches += 3;
    }
    BBData D = bb_data();
    BBParams BP{tau, w, prm_.reflection_coefficient, want_fpe ? 1 : 0};
    dispatch_rg(GQ_, [&](auto GC) {
        dispatch_s(S_, [&](auto SC) {
            void *args[] = {&D, &BP};
            void *k = dp_.has_fixed ? (void *)bb_kernel<GC.value, 8, true> : (void *)bb_kernel<GC.value, SC.value, false>;
            CK(cudaLaunchCooperativeKernel(k, bb_grid_, TPB, args, 0, s));
        });
    });
    StepParams P{};
    P.tau = tau;
    P.sigma = step_ * omega_;
    P.w = w;
    P.rho = prm_.reflection_coefficient;
    P.store_primal = 1;
    P.store_dual = store_dual;
    P.want_fpe = want_fpe;
    P.lp_slack = 0;
    P.cone_box = cone_box_;
    StepData<double> SD = step_data<double>();
    launch_dual<double>(SD, P);
    stats_.kernel_launches += 2;
    stats_.step_kernel_launches++;
    if (bb_fp32_)
        stats_.fp32_iterations++;
    {
        // entries of long rows read as FP32 values in the mixed bulk phase
        const double f32 = bb_fp32_ ? (double)((Af_ ? A_.long_nnz : 0) + (Atf_ ? At_.long_nnz : 0)) : 0.0;
        step_bytes_sum_ += step_bytes(sizeof(double), true, store_dual) - 4.0 * f32;
    }
    if (opt_.time_steps)
        CK(cudaEventRecord(ev_pool_[ev_used_++], s));
}

void Solve::enqueue_step(bool store_primal, bool store_dual, bool want_fpe, double w)
{
    if (bb_) {
        enqueue_step_bb(store_dual, want_fpe, w);
        return;
    }
    if (fp32_)
        enqueue_step_t<float>(store_primal, store_dual, want_fpe, w);
    else
        enqueue_step_t<double>(store_primal, store_dual, want_fpe, w);
}

template <typename T>
void Solve::enqueue_step_t(bool store_primal, bool store_dual, bool want_fpe, double w)
{
    cudaStream_t s = st_;
    if (opt_.time_steps) {
        if (ev_used_ + 2 > ev_pool_.size()) {
            for (int i = 0; i < 64; ++i) {
                cudaEvent_t e;
                CK(cudaEventCreate(&e));
                ev_pool_.push_back(e);
            }
        }
        CK(cudaEventRecord(ev_pool_[ev_used_++], s));
    }
    StepParams P;
    P.tau = step_ / omega_;
    if (nonconvexity_ < 0) {
        P.tau = std::fmax(P.tau, -1.01 * std::fmin(0.0, nonconvexity_));
        P.tau /= 100;
    }
    P.sigma = step_ * omega_;
    P.w = w;
    P.rho = prm_.reflection_coefficient;
    P.store_primal = store_primal;
    P.store_dual = store_dual;
    P.want_fpe = want_fpe;
    P.lp_slack = qtype_ == PDHCG_NON_Q;
    P.cone_box = cone_box_;
    StepData<T> D = step_data<T>();
    long_pass(At_, D.At_v, D.y); // A^T y of both primal kernels
    bool hasq = qtype_ == PDHCG_DIAG_Q;
    int nfree = D.n_cones > 0 ? D.n_free : n_;
    if (nfree > 0) {
        int ntiles = D.free_tiles ? D.n_free_tiles : (n_ + 31) / 32;
        int grid = grid_for(ntiles, WARPS);
        if (hasq) {
            if (box_free_)
                primal_free_kernel<T, true, false><<<grid, TPB, 0, s>>>(D, P);
            else
                primal_free_kernel<T, true, true><<<grid, TPB, 0, s>>>(D, P);
        } else {
            if (box_free_)
                primal_free_kernel<T, false, false><<<grid, TPB, 0, s>>>(D, P);
            else
                primal_free_kernel<T, false, true><<<grid, TPB, 0, s>>>(D, P);
        }
        stats_.kernel_launches++;
    }
    if (D.n_cones > 0)
        stats_.kernel_launches += launch_primal_cones(D, P, dp_.split, S_, hasq, s);
    launch_dual<T>(D, P);
    stats_.step_kernel_launches++;
    step_bytes_sum_ += step_bytes(sizeof(T), store_primal || !cone_start_.empty(), store_dual);
    if (fp32_)
        stats_.fp32_iterations++;
    if (opt_.time_steps)
        CK(cudaEventRecord(ev_pool_[ev_used_++], s));
}

// Algorithmic HBM bytes of one step as the kernels above move them: each
// matrix byte and each streamed vector once, each gathered vector once.
double Solve::step_bytes(size_t s, bool store_primal, bool store_dual) const
{
    double n = n_, m = m_, nnz = A_.nnz, nc = (double)cone_start_.size();
    double ncs = 0.0; // slots in cones
    for (int L : cone_len_)
        ncs += L;
    double nf = n - ncs;
    bool hasq = qtype_ == PDHCG_DIAG_Q;
    // primal: A^T (values + indices + row pointers), y gathered once,
    // x_cur, x_init, c (+ q) (+ box) read; x_refl, x_cur (+ x_pdhg) written
    double primal = nnz * (s + 4) + (n + 1) * 4 + m * s + n * s * (3 + (hasq ? 1 : 0)) +
                    (box_free_ ? 0.0 : 2 * nf * s) + (cone_box_ ? 2 * ncs * s : 0.0) /* box on cone slots */ + ncs * s /* d */ +
                    (nc > 0 ? nf * 4 + nc * (3 * 4 + 2 * 8) : 0.0) + n * s * (2 + (store_primal ? 1 : 0));
    // dual: A, x_refl gathered once, y_cur, y_init, bounds (+ offset) read;
    // y_cur (+ y_pdhg) written
    double dual = nnz * (s + 4) + (m + 1) * 4 + n * s + m * s * (2 + (eq_rows_ ? 1 : 2) + (has_g_ ? 1 : 0)) +
                  m * s * (1 + (store_dual ? 1 : 0));
    return primal + dual;
}

// Algorithmic bytes of one inner BB iteration (bb_kernel): the rows of Q
// with x_p gathered once, two passes over R (R x_p, then R^T (D R x_p))
// with x_p gathered once, and fifteen n-vectors of the gradient and
// projection phases (grad phase: c, A^T y, x_p, x, grad, dir read, grad,
// Q x written; var phase: grad, x_p, l, u, M^-1 read, x_p, dir written).
double Solve::bb_inner_bytes(bool fp32) const
{
    double n = n_;
    const double vb = fp32 ? 4.0 : 8.0; // bytes of a value of Q, R, R^T
    double q = Q_.nnz > 0 ? Q_.nnz * (4.0 + vb) + (n + 1) * 4 + n * 8 : 0.0;
    double r = R_.nnz == 0 ? 0.0
               : r_width_ ? 2.0 * R_.nnz * vb + r_width_ * 8.0 // values only, x_p read contiguously
                          : 2.0 * R_.nnz * (4.0 + vb) + (R_.rows + 1) * 4.0 + (n + 1) * 4 + n * 8;
    return q + r + 15.0 * n * 8;
}

// Segment pass of M's long rows over x, ahead of a product that reads them.
template <typename V, typename X>
void Solve::long_pass(const DevCsr &M, const V *val, const X *x)
{
    if (M.lr.n == 0)
        return;
    // at most what is resident at once: warps walk their segments
    // grid-stride, the next one's bounds in flight
    const int grid = std::min(grid_for(M.lr.nseg, WARPS), resident_blocks((const void *)long_partials_kernel<V, X>));
    long_partials_kernel<V, X><<<grid, TPB, 0, st_>>>(M.lr, M.ci, val, x);
    stats_.kernel_launches++;
}

void Solve::enqueue_residual(bool want_dist)
{
    if (fp32_)
        enqueue_residual_t<float>(want_dist);
    else
        enqueue_residual_t<double>(want_dist);
}

template <typename VT>
void Solve::enqueue_residual_t(bool want_dist)
{
    cudaStream_t s = st_;
    ResidualData<VT> D{};
    D.warm_dual = warm_dual_;
    D.warm_aug = warm_aug_;
    D.fixed = dp_.fixed_d;
    D.cone_fixed = dp_.cfix_d;
    D.n = n_;
    D.m = m_;
    D.A_rp = A_.rp;
    D.A_ci = A_.ci;
    D.A_v = A_.v;
    D.At_rp = At_.rp;
    D.At_ci = At_.ci;
    D.At_v = At_.v;
    D.c = c_d_;
    D.l = l_d_;
    D.u = u_d_;
    D.q = q_d_;
    D.qx = nullptr;
    D.lc = lc_d_;
    D.uc = uc_d_;
    D.g = g_d_;
    D.cr = cr_d_;
    D.vr = vr_d_;
    if constexpr (std::is_same<VT, double>::value) {
        D.xp = xp_;
        D.yp = yp_;
        D.x0 = x0_;
        D.y0 = y0_;
        D.dual_slack = dslack_;
    } else {
        D.xp = f_.xp;
        D.yp = f_.yp;
        D.x0 = f_.x0;
        D.y0 = f_.y0;
        D.dual_slack = f_.dslack;
    }
    D.free_idx = free_d_;
    D.n_free = (int)free_idx_.size();
    D.free_tiles = dp_.free_tiles;
    D.n_free_tiles = dp_.n_free_tiles;
    D.cone_start = cst_d_;
    D.cone_len = clen_d_;
    D.cone_type = ctype_d_;
    D.cone_alpha = dp_.calpha;
    D.psd_work = psd_work_;
    D.psd_off = dp_.psd_off_d;
    D.n_cones = (int)cone_start_.size();
    D.partials = partials_;
    D.rows_blocks = res_rows_blocks_;
    D.free_blocks = res_free_blocks_;
    D.cone_blocks = res_cone_blocks_;
    D.row_tiles = dp_.aff_start.empty() ? nullptr : dp_.row_tiles_d;
    D.n_row_tiles = dp_.n_row_tiles;
    D.aff_start = dp_.ast;
    D.aff_len = dp_.alen;
    D.aff_type = dp_.atype;
    D.aff_alpha = dp_.aalpha;
    D.aff_psd_off = dp_.apsd_off_d;
    D.n_aff = (int)dp_.aff_start.size();
    D.aff_blocks = res_aff_blocks_;
    D.A_long = A_.lr;
    D.At_long = At_.lr;
    long_pass(A_, A_.v, D.xp);
    long_pass(At_, At_.v, D.yp);
    ResidualParams P;
    P.l2 = prm_.optimality_norm == NORM_TYPE_L2;
    P.is_lp = qtype_ == PDHCG_NON_Q;
    P.qmode = qtype_ == PDHCG_DIAG_Q ? 1 : 0;
    if (bb_) { // Q x_pdhg for the residual (reference update_obj_product in compute_residual)
        if constexpr (std::is_same<VT, double>::value)
            enqueue_q_apply(xp_, qx_res_);
        D.qx = qx_res_;
        P.qmode = 2;
    }
    P.has_cones = D.n_cones > 0;
    P.want_dist = want_dist;
    P.tau = step_ / omega_;
    double sa = step_ / omega_;
    if (!(sa > 0.0) || !std::isfinite(sa))
        sa = 1.0;
    P.s_aug = sa;
    P.sb = sb_;
    int nb = D.rows_blocks + D.free_blocks + D.cone_blocks + D.aff_blocks;
    if (dp_.has_fixed) // one slot class for problems with fixed cone slots
        residual_kernel<8, VT, true><<<nb, TPB, 0, s>>>(D, P);
    else
        dispatch_s(std::max(S_, dp_.S_aff), [&](auto SC) { residual_kernel<SC.value, VT, false><<<nb, TPB, 0, s>>>(D, P); });
    fold_partials_kernel<<<1, TPB, 0, s>>>(partials_, nb, RS_COUNT, res_ops_d_, scal_d_);
    stats_.kernel_launches += 2;
    stats_.evaluations++;
}

void Solve::enqueue_fpe(int slot)
{
    cudaStream_t s = st_;
    int nb = fpe_col_blocks_ + fpe_row_blocks_;
    double *part = partials_; // stream order serialises every user of the partials buffer
    if (fp32_) {
        long_pass(At_, At_.v, f_.dy);
        fpe_kernel<float><<<nb, TPB, 0, s>>>(n_, m_, At_.rp, At_.ci, At_.v, f_.dx, f_.dy, part, fpe_col_blocks_,
                                             At_.lr);
    } else {
        long_pass(At_, At_.v, dy_);
        fpe_kernel<double><<<nb, TPB, 0, s>>>(n_, m_, At_.rp, At_.ci, At_.v, dx_, dy_, part, fpe_col_blocks_,
                                              At_.lr);
    }
    fold_partials_kernel<<<1, TPB, 0, s>>>(part, nb, FP_COUNT, fpe_ops_d_, scal_d_ + RS_COUNT + slot * FP_COUNT);
    stats_.kernel_launches += 2;
    if (bb_) {
        bb_tol_update_kernel<<<1, 1, 0, s>>>(scal_d_ + RS_COUNT + slot * FP_COUNT + FP_DX2, step_, omega_, bb_min_tol_,
                                             bb_tol_);
        stats_.kernel_launches++;
    }
}

// Infeasibility certificates from the differences of the last major step
// (reference compute_infeasibility_information, src/pdhg_core_op.cu:1296-1429;
// called, like there, only without cones, at major iterations before
// 3 * termination_evaluation_frequency).  dx and dy are modified in place,
// as the reference modifies delta_primal/dual_solution.
void Solve::compute_infeasibility()
{
    cudaStream_t s = st_;
    int nb = grid_for((long long)n_ + m_, TPB, 148 * 4);
    if (fp32_)
        ray_project_kernel<float><<<nb, TPB, 0, s>>>(n_, m_, f_.dx, f_.dy, l_d_, u_d_, lc_d_, uc_d_, partials_);
    else
        ray_project_kernel<double><<<nb, TPB, 0, s>>>(n_, m_, dx_, dy_, l_d_, u_d_, lc_d_, uc_d_, partials_);
    fold_partials_kernel<<<1, TPB, 0, s>>>(partials_, nb, RN_COUNT, rayn_ops_d_, ray_d_);
    if (fp32_)
        ray_scale_kernel<float><<<grid_for(n_, TPB), TPB, 0, s>>>(n_, f_.dx, ray_d_);
    else
        ray_scale_kernel<double><<<grid_for(n_, TPB), TPB, 0, s>>>(n_, dx_, ray_d_);
    RayData D{};
    D.n = n_;
    D.m = m_;
    D.A_rp = A_.rp;
    D.A_ci = A_.ci;
    D.A_v = A_.v;
    D.At_rp = At_.rp;
    D.At_ci = At_.ci;
    D.At_v = At_.v;
    D.c = c_d_;
    D.l = l_d_;
    D.u = u_d_;
    D.q = q_d_;
    D.lc = lc_d_;
    D.uc = uc_d_;
    D.g = g_d_;
    D.cr = cr_d_;
    D.vr = vr_d_;
    D.qmode = (qtype_ == PDHCG_NON_Q) ? 0 : (qtype_ == PDHCG_DIAG_Q ? 1 : 2);
    if (D.qmode == 2) { // Q dx through the BB apply (FP64 only)
        enqueue_q_apply(dx_, qx_res_);
        D.qx = qx_res_;
    }
    D.rows_blocks = res_rows_blocks_;
    D.partials = partials_;
    D.A_long = A_.lr;
    D.At_long = At_.lr;
    int grid = res_rows_blocks_ + fpe_col_blocks_;
    if (fp32_) {
        long_pass(A_, A_.v, f_.dx);
        long_pass(At_, At_.v, f_.dy);
        ray_kernel<float><<<grid, TPB, 0, s>>>(D, f_.dx, f_.dy);
    } else {
        long_pass(A_, A_.v, dx_);
        long_pass(At_, At_.v, dy_);
        ray_kernel<double><<<grid, TPB, 0, s>>>(D, dx_, dy_);
    }
    fold_partials_kernel<<<1, TPB, 0, s>>>(partials_, grid, RY_COUNT, ray_ops_d_, ray_d_ + RN_COUNT);
    stats_.kernel_launches += 6;
    double h[RN_COUNT + RY_COUNT];
    CK(cudaMemcpyAsync(h, ray_d_, sizeof(h), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const double *r = h + RN_COUNT;
    p_ray_obj_ = r[RY_CDX] / (sb_ * sc_);
    d_ray_obj_ = (r[RY_PSLACK] + r[RY_DSLACK]) / (sb_ * sc_);
    max_p_ray_ = r[RY_PINF];
    if (qtype_ != PDHCG_NON_Q)
        max_p_ray_ = std::fmax(max_p_ray_, r[RY_QDX] / sc_);
    max_d_ray_ = r[RY_DINF];
    double f = std::fmax(h[RN_DY], r[RY_DINF]);
    if (f > 0.0) {
        max_d_ray_ /= f;
        d_ray_obj_ /= f;
    } else {
        max_d_ray_ = 0.0;
        d_ray_obj_ = 0.0;
    }
}

// ---- mixed precision (FP32 bulk phase, then FP64 polish) ----------------
void Solve::enter_fp32()
{
    cudaStream_t s = st_;
    long long n = n_, m = m_, nnz = A_.nnz;
    auto mk = [&](long long k) { return ar_.alloc<float>((size_t)std::max(k, 1LL)); };
    auto cv = [&](const double *src, float *dst, long long k) {
        if (k > 0 && src)
            convert_kernel<double, float><<<grid_for(k, TPB), TPB, 0, s>>>(src, dst, k);
    };
    f_.Av = mk(nnz);
    f_.Atv = mk(nnz);
    cv(A_.v, f_.Av, nnz);
    cv(At_.v, f_.Atv, nnz);
    float **vecs_n[] = {&f_.c, &f_.l, &f_.u, &f_.vr, &f_.x0, &f_.x, &f_.xp, &f_.xr, &f_.dx, &f_.dslack};
    for (float **p : vecs_n)
        *p = mk(n);
    float **vecs_m[] = {&f_.lc, &f_.uc, &f_.g, &f_.y0, &f_.y, &f_.yp, &f_.dy};
    for (float **p : vecs_m)
        *p = mk(m);
    cv(c_d_, f_.c, n);
    cv(l_d_, f_.l, n);
    cv(u_d_, f_.u, n);
    cv(vr_d_, f_.vr, n);
    cv(lc_d_, f_.lc, m);
    cv(uc_d_, f_.uc, m);
    cv(g_d_, f_.g, m);
    if (q_d_) {
        f_.q = mk(n);
        cv(q_d_, f_.q, n);
    }
    cv(x0_, f_.x0, n);
    cv(x_, f_.x, n);
    cv(xp_, f_.xp, n);
    cv(xr_, f_.xr, n);
    cv(dslack_, f_.dslack, n);
    cv(y0_, f_.y0, m);
    cv(y_, f_.y, m);
    cv(yp_, f_.yp, m);
    CK(cudaGetLastError());
    fp32_ = true;
}

// the inner-solve path: FP32 copies of the quadratic term's values and of
// the values of A's and A^T's long rows (the products keep FP64 iterates and
// accumulation); leaving only switches the pointers back, since the
// iterates never left FP64
void Solve::enter_bb_fp32()
{
    cudaStream_t s = st_;
    auto mk = [&](long long k) { return ar_.alloc<float>((size_t)std::max(k, 1LL)); };
    auto cv = [&](const double *src, float *dst, long long k) {
        if (k > 0 && src)
            convert_kernel<double, float><<<grid_for(k, TPB), TPB, 0, s>>>(src, dst, k);
    };
    if (Q_.nnz > 0) {
        Qf_ = mk(Q_.nnz);
        cv(Q_.v, Qf_, Q_.nnz);
    }
    if (R_.nnz > 0) {
        Rf_ = mk(R_.nnz);
        cv(R_.v, Rf_, R_.nnz);
    }
    if (Rt_.nnz > 0 && !r_width_) {
        Rtf_ = mk(Rt_.nnz);
        cv(Rt_.v, Rtf_, Rt_.nnz);
    }
    // the long rows of A and A^T (segment passes ahead of the products) read
    // FP32 values too; the products' other rows keep FP64 values
    if (A_.lr.n > 0) {
        Af_ = mk(A_.nnz);
        cv(A_.v, Af_, A_.nnz);
    }
    if (At_.lr.n > 0) {
        Atf_ = mk(At_.nnz);
        cv(At_.v, Atf_, At_.nnz);
    }
    CK(cudaGetLastError());
    bb_fp32_ = true;
}

void Solve::leave_bb_fp32()
{
    int inner = 0;
    CK(cudaMemcpyAsync(&inner, bb_inner_, sizeof(int), cudaMemcpyDeviceToHost, st_));
    CK(cudaStreamSynchronize(st_));
    bb_inner_fp32_ = inner_total_ + inner; // first passes counted here, further ones on the device
    bb_fp32_ = false;
}

void Solve::leave_fp32()
{
    cudaStream_t s = st_;
    long long n = n_, m = m_;
    auto cv = [&](const float *src, double *dst, long long k) {
        if (k > 0)
            convert_kernel<float, double><<<grid_for(k, TPB), TPB, 0, s>>>(src, dst, k);
    };
    cv(f_.x0, x0_, n);
    cv(f_.x, x_, n);
    cv(f_.xp, xp_, n);
    cv(f_.xr, xr_, n);
    cv(f_.dslack, dslack_, n);
    cv(f_.y0, y0_, m);
    cv(f_.y, y_, m);
    cv(f_.yp, yp_, m);
    CK(cudaGetLastError());
    fp32_ = false;
}

// ---- main loop (reference optimize, src/solver.cu:121-170) ---------------
void Solve::read_residual()
{
    cudaStream_t s = st_;
    CK(cudaMemcpyAsync(h_scal_, scal_d_, (RS_COUNT + 2 * FP_COUNT) * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    harvest_step_events();
    const double *r = h_scal_;
    bool l2 = prm_.optimality_norm == NORM_TYPE_L2;
    auto nrm = [&](double v) { return l2 ? std::sqrt(v) : v; };
    // pending fixed-point errors computed since the previous read
    auto fpe_of = [&](const double *f) {
        double pn2 = f[FP_DX2], dn2 = f[FP_DY2], cross = f[FP_CROSS];
        double movement = pn2 * omega_ + dn2 / omega_;
        return std::sqrt(movement + 2 * step_ * cross);
    };
    if (pending_fpe0_) {
        fpe0_ = fpe_of(r + RS_COUNT);
        pending_fpe0_ = false;
    }
    if (pending_fpe_slot_ >= 0) {
        fpe_ = fpe_of(r + RS_COUNT + pending_fpe_slot_ * FP_COUNT);
        pending_fpe_slot_ = -1;
    }
    // compute_residual scalars (reference src/pdhg_core_op.cu:1169-1293)
    abs_p_ = nrm(r[RS_PRIMAL_RES]) / sb_;
    double lin_abs_p = abs_p_;
    // power-cone primal violation joins the primal residual
    // (reference src/pdhg_core_op.cu:1156-1163 and 1235-1239)
    const bool cones = !cone_type_.empty();
    const double pv_abs = nrm(r[RS_POW_ABS]), pv_rel = nrm(r[RS_POW_REL]);
    auto join = [&](double a, double b) { return l2 ? std::hypot(a, b) : std::fmax(a, b); };
    if (cones)
        abs_p_ = join(abs_p_, pv_abs);
    // the cone complementarity (nonzero on power blocks with fixed slots
    // only, reference compute_cone_complementarity_norm,
    // src/pdhg_core_op.cu:92-100) and, with affine cones, their dual
    // membership and complementarity join the dual residual (reference
    // compute_residual, src/pdhg_core_op.cu:1166-1190); all are 0 when absent
    abs_d_ = (l2 ? std::sqrt(r[RS_DUAL_RES] + r[RS_CONE_COMPL] + r[RS_AFF_MEM] + r[RS_AFF_COMPL])
                 : std::fmax(std::fmax(r[RS_DUAL_RES], r[RS_CONE_COMPL]), std::fmax(r[RS_AFF_MEM], r[RS_AFF_COMPL]))) /
             sc_;
    double half_xqx = qtype_ == PDHCG_NON_Q ? 0.0 : 0.5 * r[RS_XQX];
    pobj_ = (r[RS_CX] + half_xqx) / (sb_ * sc_) + dp_.obj_const;
    dobj_ = (r[RS_SLACKX] + r[RS_PRIMAL_SLACK] - half_xqx) / (sb_ * sc_) + dp_.obj_const;
    rel_p_ = lin_abs_p / (1.0 + bnorm_);
    if (cones)
        rel_p_ = join(rel_p_, pv_rel);
    double den;
    if (qtype_ == PDHCG_NON_Q)
        den = 1.0 + cnorm_;
    else
        den = 1.0 + std::fmax(cnorm_, std::fmax(nrm(r[RS_QX_NORM]) / sc_, nrm(r[RS_ATY_NORM]) / sc_));
    rel_d_ = abs_d_ / den;
    gap_ = std::fabs(pobj_ - dobj_);
    rel_gap_ = gap_ / (1.0 + std::fabs(pobj_) + std::fabs(dobj_));
    dist_x_ = std::sqrt(r[RS_DIST_X]);
    dist_y_ = std::sqrt(r[RS_DIST_Y]);
}

void Solve::loop()
{
    const termination_criteria_t &tc = prm_.termination_criteria;
    const restart_parameters_t &rp = prm_.restart_params;
    int freq = prm_.termination_evaluation_frequency;
    bool do_restart = false;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, st_));
    auto t0 = std::chrono::steady_clock::now();
    while (k_ < tc.iteration_limit) {
        if (is_major_ || k_ == 0 || (k_ % print_frequency(k_)) == 0) {
            bool restart_check = is_major_ || k_ == 0;
            enqueue_residual(restart_check);
            read_residual();
            // reference src/solver.cu:127-131
            if (cone_start_.empty() && dp_.aff_start.empty() && is_major_ && k_ < 3 * freq)
                compute_infeasibility();
            cum_time_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            // check_termination_criteria (reference src/utils.cu:250-289)
            if (pdhcg_b200_cancel_requested())
                reason_ = TERMINATION_REASON_USER_INTERRUPT;
            else if (rel_d_ < tc.eps_feasible_relative && rel_p_ < tc.eps_feasible_relative &&
                     rel_gap_ < tc.eps_optimal_relative)
                reason_ = TERMINATION_REASON_OPTIMAL;
            else if (cone_start_.empty() && d_ray_obj_ > 0.0 && max_d_ray_ / d_ray_obj_ <= tc.eps_infeasible)
                reason_ = TERMINATION_REASON_PRIMAL_INFEASIBLE;
            else if (cone_start_.empty() && p_ray_obj_ < 0.0 && max_p_ray_ / (-p_ray_obj_) <= tc.eps_infeasible)
                reason_ = TERMINATION_REASON_DUAL_INFEASIBLE;
            else if (k_ >= tc.iteration_limit)
                reason_ = TERMINATION_REASON_ITERATION_LIMIT;
            else if (cum_time_ >= tc.time_sec_limit)
                reason_ = TERMINATION_REASON_TIME_LIMIT;
            if (reason_ != TERMINATION_REASON_UNSPECIFIED)
                break;
            if (fp32_ || bb_fp32_) {
                // FP32 bulk phase hands over to FP64 once the relative KKT error
                // is below the polish threshold, or when it stops improving
                double kkt = std::fmax(rel_p_, std::fmax(rel_d_, rel_gap_));
                if (kkt < best_fp32_kkt_ * 0.9) {
                    best_fp32_kkt_ = kkt;
                    fp32_stall_ = 0;
                } else {
                    ++fp32_stall_;
                }
                if (kkt < opt_.polish_threshold || fp32_stall_ >= 30) {
                    if (fp32_)
                        leave_fp32();
                    else
                        leave_bb_fp32();
                }
            }
        }
        if (is_major_ || k_ == 0) {
            // should_do_adaptive_restart (reference src/utils.cu:291-322)
            do_restart = false;
            if (k_ == freq)
                do_restart = true;
            else if (k_ > freq) {
                if (fpe_ <= rp.sufficient_reduction_for_restart * fpe0_)
                    do_restart = true;
                if (fpe_ <= rp.necessary_reduction_for_restart * fpe0_ && fpe_ > fpe_last_)
                    do_restart = true;
                if (inner_count_ >= rp.artificial_restart_threshold * k_)
                    do_restart = true;
            }
            fpe_last_ = fpe_;
            if (do_restart) {
                // perform_restart (reference src/pdhg_core_op.cu:859-931)
                double pd = dist_x_, dd = dist_y_, ratio = rel_d_ / rel_p_;
                if (pd > 1e-16 && dd > 1e-16 && pd < 1e12 && dd < 1e12 && ratio > 1e-8 && ratio < 1e8) {
                    double err = std::log(dd) - std::log(pd) - std::log(omega_);
                    pw_err_sum_ *= rp.i_smooth;
                    pw_err_sum_ += err;
                    double derr = err - pw_last_err_;
                    omega_ *= std::exp(rp.k_p * err + rp.k_i * pw_err_sum_ + rp.k_d * derr);
                    pw_last_err_ = err;
                } else {
                    omega_ = best_omega_;
                    pw_err_sum_ = 0.0;
                    pw_last_err_ = 0.0;
                }
                double g = std::fabs(std::log10(rel_d_ / rel_p_));
                if (g < best_gap_) {
                    best_gap_ = g;
                    best_omega_ = omega_;
                }
                if (fp32_)
                    restart_copy_kernel<float><<<grid_for((long long)n_ + m_, TPB), TPB, 0, st_>>>(
                        n_, m_, f_.xp, f_.x0, f_.x, f_.yp, f_.y0, f_.y);
                else
                    restart_copy_kernel<double><<<grid_for((long long)n_ + m_, TPB), TPB, 0, st_>>>(
                        n_, m_, xp_, x0_, x_, yp_, y0_, y_);
                stats_.kernel_launches++;
                stats_.restarts++;
                inner_count_ = 0;
                fpe_last_ = INFINITY;
            }
        }
        is_major_ = ((k_ + 1) % freq) == 0;
        bool store_rule = ((k_ + 2) % print_frequency(k_ + 2)) == 0;
        bool store_primal = is_major_ || store_rule || !cone_start_.empty();
        bool store_dual = is_major_ || store_rule;
        bool want_fpe = is_major_ || do_restart;
        double w = (double)(inner_count_ + 1) / (inner_count_ + 2);
        enqueue_step(store_primal, store_dual, want_fpe, w);
        inner_total_++;
        if (want_fpe) {
            // The error of this iteration becomes fixed_point_error, and on a
            // restart also initial_fixed_point_error.  Slot 0 holds a
            // restart's error, slot 1 a later major iteration's, so both
            // survive until the next read.
            int slot = do_restart ? 0 : 1;
            enqueue_fpe(slot);
            if (do_restart)
                pending_fpe0_ = true;
            pending_fpe_slot_ = slot;
            do_restart = false;
        }
        inner_count_++;
        k_++;
        CK(cudaGetLastError());
    }
    if (reason_ == TERMINATION_REASON_UNSPECIFIED) {
        reason_ = TERMINATION_REASON_ITERATION_LIMIT;
        enqueue_residual(false);
        read_residual();
    }
    CK(cudaEventRecord(e1, st_));
    CK(cudaEventSynchronize(e1));
    harvest_step_events();
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    stats_.loop_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    stats_.iterations = k_;
}

pdhcg_result_t *Solve::make_result()
{
    cudaStream_t s = st_;
    int n = n_, m = m_;
    bool on_dev = opt_.solution_on_device != 0;
    double *xo, *yo, *rco;
    if (on_dev) { // kept with the device problem for pdhcg_b200_device_solution
        if (!dp_.x_out) {
            dp_.x_out = dp_.ar.alloc<double>(n);
            dp_.y_out = dp_.ar.alloc<double>(m);
            dp_.rc_out = dp_.ar.alloc<double>(n);
        }
        xo = dp_.x_out;
        yo = dp_.y_out;
        rco = dp_.rc_out;
    } else {
        xo = ar_.alloc<double>(n);
        yo = ar_.alloc<double>(m);
        rco = ar_.alloc<double>(n);
    }
    if (bb_) {
        enqueue_q_apply(xp_, qx_res_);
        result_kernel<double><<<grid_for((long long)n + m, TPB), TPB, 0, s>>>(
            n, m, At_.rp, At_.ci, At_.v, c_d_, q_d_, qx_res_, 2, l_d_, u_d_, vr_d_, cr_d_, sb_, sc_, xp_, yp_, xo, yo,
            rco);
    } else if (fp32_)
        result_kernel<float><<<grid_for((long long)n + m, TPB), TPB, 0, s>>>(
            n, m, At_.rp, At_.ci, At_.v, c_d_, q_d_, nullptr, qtype_ == PDHCG_DIAG_Q ? 1 : 0, l_d_, u_d_, vr_d_,
            cr_d_, sb_, sc_, f_.xp, f_.yp, xo, yo, rco);
    else
        result_kernel<double><<<grid_for((long long)n + m, TPB), TPB, 0, s>>>(
            n, m, At_.rp, At_.ci, At_.v, c_d_, q_d_, nullptr, qtype_ == PDHCG_DIAG_Q ? 1 : 0, l_d_, u_d_, vr_d_,
            cr_d_, sb_, sc_, xp_, yp_, xo, yo, rco);
    pdhcg_result_t *r = (pdhcg_result_t *)std::calloc(1, sizeof(pdhcg_result_t));
    if (!on_dev) {
        r->primal_solution = (double *)std::malloc(std::max(n, 1) * sizeof(double));
        r->dual_solution = (double *)std::malloc(std::max(m, 1) * sizeof(double));
        r->reduced_cost = (double *)std::malloc(std::max(n, 1) * sizeof(double));
        CK(cudaMemcpyAsync(r->primal_solution, xo, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(r->dual_solution, yo, m * sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(r->reduced_cost, rco, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    r->num_variables = dp_.orig_vars;
    r->num_constraints = dp_.orig_cons;
    r->num_nonzeros = dp_.orig_nnz;
    r->total_count = k_;
    r->total_inner_count = (int)inner_total_;
    r->cumulative_time_sec = cum_time_;
    r->relative_primal_residual = rel_p_;
    r->relative_dual_residual = rel_d_;
    r->absolute_primal_residual = abs_p_;
    r->absolute_dual_residual = abs_d_;
    r->primal_objective_value = pobj_;
    r->dual_objective_value = dobj_;
    r->objective_gap = gap_;
    r->relative_objective_gap = rel_gap_;
    r->termination_reason = reason_;
    r->max_primal_ray_infeasibility = max_p_ray_;
    r->max_dual_ray_infeasibility = max_d_ray_;
    r->primal_ray_linear_objective = p_ray_obj_;
    r->dual_ray_objective = d_ray_obj_;
    return r;
}

// Reduction scratch (block partials sized for the widest user, folded
// scalars, the pinned host mirror) and the fold operators.
void Solve::setup_scratch()
{
    // reduction scratch sized for the widest user
    // residual ranges: one warp per tile of 32 rows / per cone block
    res_rows_blocks_ = grid_for(dp_.aff_start.empty() ? ((long long)m_ + 31) / 32 : (long long)dp_.n_row_tiles, WARPS,
                                148 * 8);
    res_aff_blocks_ = dp_.aff_start.empty() ? 0 : grid_for((long long)dp_.aff_start.size(), WARPS, 148 * 8);
    res_free_blocks_ = grid_for(cone_start_.empty() ? ((long long)n_ + 31) / 32 : (long long)dp_.n_free_tiles, WARPS,
                                148 * 8);
    if (!cone_start_.empty() && free_idx_.empty())
        res_free_blocks_ = 0;
    res_cone_blocks_ = cone_start_.empty() ? 0 : grid_for((long long)cone_start_.size(), WARPS, 148 * 8);
    fpe_col_blocks_ = grid_for(((long long)n_ + 31) / 32, WARPS, 148 * 8);
    fpe_row_blocks_ = grid_for(m_, TPB, 148 * 4);
    int maxb = std::max({res_rows_blocks_ + res_free_blocks_ + res_cone_blocks_ + res_aff_blocks_,
                         fpe_col_blocks_ + fpe_row_blocks_,
                         res_rows_blocks_ + fpe_col_blocks_, 148 * 4});
    partials_ = ar_.alloc<double>((size_t)maxb * RS_COUNT);
    scal_d_ = ar_.alloc<double>(RS_COUNT + 2 * FP_COUNT);
    CK(cudaMemsetAsync(scal_d_, 0, (RS_COUNT + 2 * FP_COUNT) * sizeof(double), st_));
    h_scal_ = pinned_scalars();
    {
        int nop = prm_.optimality_norm == NORM_TYPE_L2 ? RSUM : RMAX;
        int res_ops[RS_COUNT] = {nop, RSUM, nop, RSUM, RSUM, RSUM, nop, nop, RSUM, RSUM, nop, nop, nop, nop, nop};
        int fpe_ops[FP_COUNT] = {RSUM, RSUM, RSUM};
        int norm_ops[NS_COUNT] = {RSUM, RSUM, RMAX, RMAX};
        res_ops_d_ = ar_.upload(res_ops, RS_COUNT, st_);
        fpe_ops_d_ = ar_.upload(fpe_ops, FP_COUNT, st_);
        norm_ops_d_ = ar_.upload(norm_ops, NS_COUNT, st_);
        int rayn_ops[RN_COUNT] = {RMAX, RMAX};
        int ray_ops[RY_COUNT] = {RSUM, RSUM, RSUM, RMAX, RMAX, RMAX};
        rayn_ops_d_ = ar_.upload(rayn_ops, RN_COUNT, st_);
        ray_ops_d_ = ar_.upload(ray_ops, RY_COUNT, st_);
        ray_d_ = ar_.alloc<double>(RN_COUNT + RY_COUNT);
        CK(cudaStreamSynchronize(st_)); // the uploads above read stack arrays
    }
}

// A NaN in c, the bounds or the matrix values, or an infinite entry of c
// or of a matrix, would only be noticed as a NaN residual at the first
// evaluation and then iterated on until a limit: refuse the problem.
void Solve::check_finite()
{
    cudaStream_t s = st_;
    nonfinite_ = ar_.alloc<int>(1);
    CK(cudaMemsetAsync(nonfinite_, 0, sizeof(int), s));
    nonfinite_kernel<<<grid_for(n_, TPB, 148 * 4), TPB, 0, s>>>(c_d_, n_, 1, nonfinite_);
    nonfinite_kernel<<<grid_for(n_, TPB, 148 * 4), TPB, 0, s>>>(l_d_, n_, 0, nonfinite_);
    nonfinite_kernel<<<grid_for(n_, TPB, 148 * 4), TPB, 0, s>>>(u_d_, n_, 0, nonfinite_);
    nonfinite_kernel<<<grid_for(m_, TPB, 148 * 4), TPB, 0, s>>>(lc_d_, m_, 0, nonfinite_);
    nonfinite_kernel<<<grid_for(m_, TPB, 148 * 4), TPB, 0, s>>>(uc_d_, m_, 0, nonfinite_);
    nonfinite_kernel<<<grid_for(A_.nnz, TPB, 148 * 8), TPB, 0, s>>>(A_.v, A_.nnz, 1, nonfinite_);
    if (Q_.nnz > 0)
        nonfinite_kernel<<<grid_for(Q_.nnz, TPB, 148 * 8), TPB, 0, s>>>(Q_.v, Q_.nnz, 1, nonfinite_);
    if (R_.nnz > 0)
        nonfinite_kernel<<<grid_for(R_.nnz, TPB, 148 * 8), TPB, 0, s>>>(R_.v, R_.nnz, 1, nonfinite_);
    int bad = 0;
    CK(cudaMemcpyAsync(&bad, nonfinite_, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (bad)
        throw CudaError("the problem holds NaN values, or infinite objective or matrix entries");
}

void Solve::rescaling(double *con_rescale, double *var_rescale, double *bound_obj)
{
    CK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    ar_.s = st_;
    dp_.ar.s = st_;
    build_host();
    if (!dp_.unsupported.empty())
        throw CudaError(dp_.unsupported);
    upload_and_preprocess();
    check_finite();
    setup_scratch();
    rescale();
    const int rows = dp_.dummy ? 0 : m_;
    if (rows > 0)
        CK(cudaMemcpyAsync(con_rescale, cr_d_, rows * sizeof(double), cudaMemcpyDeviceToHost, st_));
    CK(cudaMemcpyAsync(var_rescale, vr_d_, n_ * sizeof(double), cudaMemcpyDeviceToHost, st_));
    CK(cudaStreamSynchronize(st_));
    bound_obj[0] = sb_;
    bound_obj[1] = sc_;
}

pdhcg_result_t *Solve::run()
{
    auto t_setup = std::chrono::steady_clock::now();
    CK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    ar_.s = st_;
    dp_.ar.s = st_; // outputs kept with the device problem are allocated in this solve's order
    build_host();
    auto t_host = std::chrono::steady_clock::now();
    stats_.host_copy_ms = std::chrono::duration<double, std::milli>(t_host - t_setup).count();
    if (!dp_.unsupported.empty())
        throw CudaError(dp_.unsupported);
    upload_and_preprocess();
    check_finite();
    stats_.upload_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host).count();
    setup_scratch();
    // unscaled norms for the relative errors (reference src/solver_state.cu:854-934)
    {
        int nb = grid_for((long long)n_ + m_, TPB, 148 * 4);
        norms_kernel<<<nb, TPB, 0, st_>>>(n_, m_, c_d_, lc_d_, uc_d_, g_d_, partials_);
        fold_partials_kernel<<<1, TPB, 0, st_>>>(partials_, nb, NS_COUNT, norm_ops_d_, scal_d_);
        double h[NS_COUNT];
        CK(cudaMemcpyAsync(h, scal_d_, sizeof(h), cudaMemcpyDeviceToHost, st_));
        CK(cudaStreamSynchronize(st_));
        if (prm_.optimality_norm == NORM_TYPE_L_INF) {
            cnorm_ = h[NS_CMAX];
            bnorm_ = h[NS_BMAX];
        } else {
            cnorm_ = std::sqrt(h[NS_C2]);
            bnorm_ = std::sqrt(h[NS_B2]);
        }
        if (dp_.dummy)
            bnorm_ = 0.0; // the dummy row has infinite bounds and no offset
    }
    rescale();
    init_state();
    step_size();
    CK(cudaStreamSynchronize(st_));
    // diagonal Q with PSD blocks takes the inner BB solve, as the reference
    // does (a nonuniform diagonal metric has no one-decomposition PSD prox)
    bb_ = qtype_ != PDHCG_NON_Q && (qtype_ != PDHCG_DIAG_Q || dp_.var_psd);
    if (bb_)
        setup_bb();
    if (opt_.precision == PDHCG_B200_MIXED) {
        if (bb_)
            enter_bb_fp32();
        else
            enter_fp32();
    }
    stats_.setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_setup).count();
    loop();
    if (bb_) {
        int inner = 0;
        CK(cudaMemcpyAsync(&inner, bb_inner_, sizeof(int), cudaMemcpyDeviceToHost, st_));
        CK(cudaStreamSynchronize(st_));
        inner_total_ += inner;
    }
    auto t_res = std::chrono::steady_clock::now();
    pdhcg_result_t *r = make_result();
    stats_.result_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_res).count();
    r->rescaling_time_sec = stats_.setup_ms * 1e-3;
    double nnz = (double)A_.nnz;
    stats_.spmv_bytes = 2.0 * nnz * (8 + 4) + 4.0 * ((double)n_ + m_ + 2) + 8.0 * ((double)n_ + m_);
    double bytes = step_bytes_sum_;
    if (bb_) { // the inner solve: one first pass per step plus every further inner iteration
        const long long in32 = std::min(bb_inner_fp32_, inner_total_);
        bytes += (double)(inner_total_ - in32) * bb_inner_bytes(false) + (double)in32 * bb_inner_bytes(true);
    }
    stats_.step_bytes = stats_.step_kernel_launches > 0 ? bytes / stats_.step_kernel_launches : 0.0;
    stats_.primal_weight = omega_;
    stats_.step_size = step_;
    g_last_stats = stats_;
    return r;
}

// Kernel-level step: the solver's fused kernels on caller-owned arrays.
int step_impl(StepData<double> D, StepParams P, const pdhcg_b200_step_t *t, cudaStream_t s)
{
    int n = t->n, nc = t->num_cones;
    int *len_d = nullptr, *free_d = nullptr, *ids_d = nullptr;
    int2 *tiles_d = nullptr;
    int S = 1;
    ConeSplit split;
    if (nc > 0) {
        std::vector<int> st(nc), vd(nc), tp(nc), len(nc);
        CK(cudaMemcpyAsync(st.data(), t->cone_start, nc * sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(vd.data(), t->cone_vdim, nc * sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(tp.data(), t->cone_type, nc * sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        std::vector<char> in(n, 0);
        int maxlen = 0;
        for (int b = 0; b < nc; ++b) {
            len[b] = pdhcg_b200_cone_length((cone_type_t)tp[b], vd[b]);
            maxlen = std::max(maxlen, len[b]);
            for (int i = 0; i < len[b]; ++i)
                in[st[b] + i] = 1;
        }
        std::vector<int> fr;
        for (int i = 0; i < n; ++i)
            if (!in[i])
                fr.push_back(i);
        S = slots_class(maxlen);
        if (S < 0)
            return -2;
        std::vector<int2> ft = row_tiles(fr);
        split.build(tp);
        if (split.n_psd > 0) { // the kernel-level step keeps no PSD scratch
            std::fprintf(stderr, "[pdhcg_b200_pdhg_step] PSD blocks are not supported by the kernel-level step.\n");
            return -3;
        }
        if (split.mixed()) {
            std::vector<int> all = split.joined();
            CK(cudaMallocAsync((void **)&ids_d, nc * sizeof(int), s));
            CK(cudaMemcpyAsync(ids_d, all.data(), nc * sizeof(int), cudaMemcpyHostToDevice, s));
            CK(cudaStreamSynchronize(s)); // all goes out of scope
            split.place(ids_d);
        }
        CK(cudaMallocAsync((void **)&len_d, nc * sizeof(int), s));
        CK(cudaMallocAsync((void **)&free_d, std::max<size_t>(fr.size(), 1) * sizeof(int), s));
        CK(cudaMallocAsync((void **)&tiles_d, std::max<size_t>(ft.size(), 1) * sizeof(int2), s));
        CK(cudaMemcpyAsync(len_d, len.data(), nc * sizeof(int), cudaMemcpyHostToDevice, s));
        if (!fr.empty()) {
            CK(cudaMemcpyAsync(free_d, fr.data(), fr.size() * sizeof(int), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(tiles_d, ft.data(), ft.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
        }
        CK(cudaStreamSynchronize(s)); // host vectors go out of scope
        D.free_idx = free_d;
        D.n_free = (int)fr.size();
        D.free_tiles = tiles_d;
        D.n_free_tiles = (int)ft.size();
        D.cone_start = t->cone_start;
        D.cone_len = len_d;
        D.cone_type = t->cone_type;
        D.cone_alpha = t->cone_alpha;
        D.n_cones = nc;
    }
    bool hasq = t->q_diag != nullptr;
    int nfree = nc > 0 ? D.n_free : n;
    if (nfree > 0) {
        int ntiles = nc > 0 ? D.n_free_tiles : (n + 31) / 32;
        int grid = grid_for(ntiles, WARPS);
        if (hasq)
            primal_free_kernel<double, true, true><<<grid, TPB, 0, s>>>(D, P);
        else
            primal_free_kernel<double, false, true><<<grid, TPB, 0, s>>>(D, P);
    }
    if (nc > 0)
        launch_primal_cones(D, P, split, S, hasq, s);
    int dgrid = grid_for(((long long)t->m + 31) / 32, WARPS);
    if (t->affine_offset)
        dual_kernel<double, false, true><<<dgrid, TPB, 0, s>>>(D, P);
    else
        dual_kernel<double, false, false><<<dgrid, TPB, 0, s>>>(D, P);
    CK(cudaGetLastError());
    if (len_d)
        CK(cudaFreeAsync(len_d, s));
    if (free_d)
        CK(cudaFreeAsync(free_d, s));
    if (tiles_d)
        CK(cudaFreeAsync(tiles_d, s));
    if (ids_d)
        CK(cudaFreeAsync(ids_d, s));
    return 0;
}

// ---- scratch of pdhcg_b200_project_cones_noalloc ---------------------------
// A file-scope device array replaces the stream-ordered temporary of
// pdhcg_b200_project_cones: [0, nc) the block lengths, then the longest
// length and a flag for a cone type without a projection.  Every call
// writes all of them before reading any, so nothing has to start at zero.
constexpr int NOALLOC_MAX_CONES = PDHCG_B200_NOALLOC_MAX_CONES;
static __device__ __align__(256) int g_noalloc_scratch[NOALLOC_MAX_CONES + 2];

__global__ void __launch_bounds__(TPB) noalloc_len_kernel(int nc, const int *vdim, const int *type, int has_alpha,
                                                          int *scratch)
{
    __shared__ int sh_max[TPB], sh_bad[TPB];
    int mx = 0, bad = 0;
    for (int b = threadIdx.x; b < nc; b += TPB) {
        const int t = type[b], v = vdim[b];
        const int len = (t == 2 || t == 3) ? 3 : (t == 4 ? v * (v + 1) / 2 : v + 2);
        scratch[b] = len;
        mx = max(mx, len);
        bad |= !(t == CONE_STANDARD_SOC || t == CONE_ROTATED_SOC || t == CONE_EXPONENTIAL ||
                 (t == CONE_POWER && has_alpha));
    }
    sh_max[threadIdx.x] = mx;
    sh_bad[threadIdx.x] = bad;
    __syncthreads();
    for (int o = TPB / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sh_max[threadIdx.x] = max(sh_max[threadIdx.x], sh_max[threadIdx.x + o]);
            sh_bad[threadIdx.x] |= sh_bad[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        scratch[NOALLOC_MAX_CONES] = sh_max[0];
        scratch[NOALLOC_MAX_CONES + 1] = sh_bad[0];
    }
}

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (cudaGetSymbolAddress with that device current) and cached.
int *noalloc_scratch()
{
    constexpr int MAX_DEVICES = 64;
    static std::mutex mu;
    static int *addr[MAX_DEVICES] = {};
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "[pdhcg_b200_project_cones_noalloc] cudaGetSymbolAddress: %s\n",
                         cudaGetErrorString(e));
            return nullptr;
        }
        addr[dev] = (int *)p;
    }
    return addr[dev];
}

} // namespace

// ---------------------------------------------------------------------------
// C entry points
// ---------------------------------------------------------------------------

extern "C" {

// The reference's cancellation flag (reference src/pdhcg.c:31), written by
// its Python binding's SIGINT handler (reference
// python_bindings/_core_bindings.cpp:41-47) and read at every evaluation.
volatile std::sig_atomic_t g_pdhcg_cancel_request = 0;

int pdhcg_b200_cancel_requested(void) { return g_pdhcg_cancel_request != 0; }

void pdhcg_b200_request_cancel(int on) { g_pdhcg_cancel_request = on ? 1 : 0; }

void pdhcg_b200_default_options(pdhcg_b200_options_t *o)
{
    std::memset(o, 0, sizeof(*o));
    o->precision = PDHCG_B200_FP64;
    o->polish_threshold = 1e-5;
}

static pdhcg_result_t *solve_on_device(const qp_problem_t *prob, const pdhg_parameters_t &prm,
                                       pdhcg_b200_options_t opt);

pdhcg_result_t *pdhcg_b200_solve(const qp_problem_t *prob, const pdhg_parameters_t *params,
                                 const pdhcg_b200_options_t *opts)
{
    if (!prob) {
        std::fprintf(stderr, "[interface] solve_qp_problem: invalid arguments.\n");
        return nullptr;
    }
    // fixed cone slots are checked on the problem as given, before any
    // rewrite (reference solve_qp_problem, src/pdhcg.c:894-902)
    if (pdhcg_b200_validate_fixed_sections(prob) != 0)
        return nullptr;
    pdhg_parameters_t prm;
    if (params)
        prm = *params;
    else
        set_default_parameters(&prm);
    pdhcg_b200_options_t opt;
    if (opts)
        opt = *opts;
    else
        pdhcg_b200_default_options(&opt);
    if (prob->num_quadratic_constraints > 0) {
        // quadratic constraints become cone blocks, as the reference's
        // optimize does (src/solver.cu:43-66, 199), and the result is trimmed
        // back to the original sizes
        qp_problem_t *ext = qcqp_to_socp_qp(prob, prm.default_cone_type);
        if (!ext) {
            std::fprintf(stderr, "Error: QCQP -> SOCP transformation failed; cannot solve.\n");
            return nullptr;
        }
        pdhcg_result_t *r = solve_on_device(ext, prm, opt);
        pdhcg_b200_restore_qcqp_result(r, prob);
        qp_problem_free(ext);
        return r;
    }
    return solve_on_device(prob, prm, opt);
}

static pdhcg_result_t *solve_on_device(const qp_problem_t *prob, const pdhg_parameters_t &prm,
                                       pdhcg_b200_options_t opt)
{
    try {
        auto t0 = std::chrono::steady_clock::now();
        pdhcg_result_t *r = nullptr;
        {
            cudaStream_t us = nullptr;
            CK(cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking));
            std::unique_ptr<DeviceProblem> dp;
            try {
                dp = make_device_problem(prob, us);
            } catch (...) {
                cudaStreamDestroy(us);
                throw;
            }
            cudaStreamDestroy(us);
            const double build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            opt.solution_on_device = 0; // the temporary device problem dies with this call
            Solve s(*dp, true, prm, opt);
            r = s.run();
            g_last_stats.upload_ms += build_ms; // the problem's copies to the device (ended by a synchronise)
        }
        g_last_stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (r && prm.verbose >= 1) {
            std::printf("Solution Summary\n");
            std::printf("  Status             : %d\n", (int)r->termination_reason);
            std::printf("  Solve time         : %.3g sec\n", r->cumulative_time_sec);
            std::printf("  Iterations         : %d\n", r->total_count);
            std::printf("  Primal objective   : %.10g\n", r->primal_objective_value);
            std::printf("  Dual objective     : %.10g\n", r->dual_objective_value);
            std::printf("  Objective gap      : %.3e\n", r->relative_objective_gap);
            std::printf("  Primal infeas      : %.3e\n", r->relative_primal_residual);
            std::printf("  Dual infeas        : %.3e\n", r->relative_dual_residual);
        }
        return r;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "[pdhcg_b200] solve failed: %s\n", e.what());
        return nullptr;
    }
}

struct pdhcg_b200_device_problem_s {
    std::unique_ptr<DeviceProblem> dp;
};

pdhcg_b200_device_problem_t *pdhcg_b200_upload(const qp_problem_t *prob)
{
    if (!prob) {
        std::fprintf(stderr, "[pdhcg_b200_upload] prob is NULL\n");
        return nullptr;
    }
    if (pdhcg_b200_validate_fixed_sections(prob) != 0)
        return nullptr;
    cudaStream_t us = nullptr;
    try {
        CK(cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking));
        auto h = new pdhcg_b200_device_problem_s;
        h->dp = make_device_problem(prob, us);
        cudaStreamDestroy(us);
        return h;
    } catch (const std::exception &e) {
        if (us)
            cudaStreamDestroy(us);
        std::fprintf(stderr, "[pdhcg_b200_upload] failed: %s\n", e.what());
        return nullptr;
    }
}

pdhcg_result_t *pdhcg_b200_solve_device(pdhcg_b200_device_problem_t *h, const pdhg_parameters_t *params,
                                        const pdhcg_b200_options_t *opts)
{
    if (!h || !h->dp) {
        std::fprintf(stderr, "[pdhcg_b200_solve_device] invalid handle\n");
        return nullptr;
    }
    pdhg_parameters_t prm;
    if (params)
        prm = *params;
    else
        set_default_parameters(&prm);
    pdhcg_b200_options_t opt;
    if (opts)
        opt = *opts;
    else
        pdhcg_b200_default_options(&opt);
    try {
        auto t0 = std::chrono::steady_clock::now();
        pdhcg_result_t *r = nullptr;
        {
            Solve s(*h->dp, false, prm, opt);
            r = s.run();
        }
        g_last_stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return r;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "[pdhcg_b200] solve failed: %s\n", e.what());
        return nullptr;
    }
}

int pdhcg_b200_device_solution(const pdhcg_b200_device_problem_t *h, const double **x, const double **y,
                               const double **reduced_cost)
{
    if (!h || !h->dp || !h->dp->x_out)
        return -1;
    if (x)
        *x = h->dp->x_out;
    if (y)
        *y = h->dp->y_out;
    if (reduced_cost)
        *reduced_cost = h->dp->rc_out;
    return 0;
}

void pdhcg_b200_device_problem_free(pdhcg_b200_device_problem_t *h)
{
    delete h;
}

pdhcg_result_t *solve_qp_problem(const qp_problem_t *prob, const pdhg_parameters_t *params)
{
    return pdhcg_b200_solve(prob, params, nullptr);
}

int pdhcg_b200_last_stats(pdhcg_b200_stats_t *out)
{
    if (!out)
        return -1;
    *out = g_last_stats;
    return 0;
}

int pdhcg_b200_rescaling(const qp_problem_t *prob, const pdhg_parameters_t *params, double *con_rescale,
                         double *var_rescale, double *bound_obj)
{
    if (!prob || !var_rescale || !bound_obj || (prob->num_constraints > 0 && !con_rescale)) {
        std::fprintf(stderr, "[pdhcg_b200_rescaling] invalid arguments\n");
        return -1;
    }
    pdhg_parameters_t prm;
    if (params)
        prm = *params;
    else
        set_default_parameters(&prm);
    try {
        cudaStream_t us = nullptr;
        CK(cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking));
        std::unique_ptr<DeviceProblem> dp;
        try {
            dp = make_device_problem(prob, us);
        } catch (...) {
            cudaStreamDestroy(us);
            throw;
        }
        cudaStreamDestroy(us);
        pdhcg_b200_options_t opt;
        pdhcg_b200_default_options(&opt);
        Solve s(*dp, true, prm, opt);
        s.rescaling(con_rescale, var_rescale, bound_obj);
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "[pdhcg_b200_rescaling] %s\n", e.what());
        return -1;
    }
}

int pdhcg_b200_csr_spmv(int rows, const int *row_ptr, const int *col_ind, const double *val, const double *x,
                        double *y, void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    spmv_kernel<<<grid_for(((long long)rows + 31) / 32, WARPS), TPB, 0, s>>>(rows, row_ptr, col_ind, val, x, y,
                                                                            LongRows{});
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int pdhcg_b200_project_cones(int num_cones, const int *cone_start, const int *cone_vdim, const int *cone_type,
                             const double *cone_alpha, double *x, const double *d, const double *q, double tau,
                             void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    if (num_cones <= 0)
        return 0;
    // cone lengths from v_dim (SOC / RSOC: v_dim + 2) on the device
    int *len = nullptr;
    if (cudaMallocAsync((void **)&len, num_cones * sizeof(int), s) != cudaSuccess)
        return -1;
    cone_len_kernel<<<grid_for(num_cones, TPB), TPB, 0, s>>>(num_cones, cone_vdim, cone_type, len);
    int maxlen = 0;
    bool types_ok = true;
    std::vector<long long> psd_off(num_cones, 0);
    long long psd_total = 0;
    {
        std::vector<int> h(num_cones), t(num_cones), vd(num_cones);
        // a failed enqueue would leave h and t unset: check every call
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(h.data(), len, num_cones * sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(t.data(), cone_type, num_cones * sizeof(int), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            cudaFreeAsync(len, s);
            return -1;
        }
        if (cudaMemcpyAsync(vd.data(), cone_vdim, num_cones * sizeof(int), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            cudaFreeAsync(len, s);
            return -1;
        }
        for (int i = 0; i < num_cones; ++i) {
            if (!(t[i] == CONE_PSD && h[i] > 32 * 8)) // long PSD blocks: projected in memory, in place
                maxlen = std::max(maxlen, h[i]);
            types_ok = types_ok && (t[i] == CONE_STANDARD_SOC || t[i] == CONE_ROTATED_SOC ||
                                    t[i] == CONE_EXPONENTIAL || (t[i] == CONE_POWER && cone_alpha) ||
                                    t[i] == CONE_PSD);
            if (t[i] == CONE_PSD) {
                psd_off[i] = psd_total;
                psd_total += 2LL * vd[i] * vd[i];
            }
        }
    }
    if (!types_ok) { // a power block needs its exponent
        std::fprintf(stderr, "[pdhcg_b200_project_cones] only SOC, rotated-SOC, exponential, power (with "
                             "cone_alpha) and PSD blocks are supported.\n");
        cudaFreeAsync(len, s);
        return -3;
    }
    int S = slots_class(maxlen);
    if (S < 0) {
        cudaFreeAsync(len, s);
        return -2;
    }
    double *psd_work = nullptr;
    long long *psd_off_d = nullptr;
    if (psd_total > 0) {
        if (cudaMallocAsync((void **)&psd_work, psd_total * sizeof(double), s) != cudaSuccess ||
            cudaMallocAsync((void **)&psd_off_d, num_cones * sizeof(long long), s) != cudaSuccess ||
            cudaMemcpyAsync(psd_off_d, psd_off.data(), num_cones * sizeof(long long), cudaMemcpyHostToDevice, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) { // psd_off goes out of scope
            cudaFreeAsync(len, s);
            return -1;
        }
    }
    dispatch_s(S, [&](auto SC) {
        project_cones_kernel<SC.value><<<grid_for(num_cones, WARPS), TPB, 0, s>>>(num_cones, cone_start, len,
                                                                                 cone_type, cone_alpha, x, d, q,
                                                                                 tau, psd_work, psd_off_d);
    });
    cudaFreeAsync(len, s);
    if (psd_work) {
        cudaFreeAsync(psd_work, s);
        cudaFreeAsync(psd_off_d, s);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int pdhcg_b200_project_cone_sections(int num_cones, const int *cone_start, const int *cone_vdim,
                                     const int *cone_type, const double *cone_alpha, const unsigned char *fixed,
                                     double *x, const double *d, const double *q, double tau, double *warm,
                                     void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    if (num_cones <= 0)
        return 0;
    if (!fixed)
        return -3;
    int *len = nullptr;
    if (cudaMallocAsync((void **)&len, num_cones * sizeof(int), s) != cudaSuccess)
        return -1;
    cone_len_kernel<<<grid_for(num_cones, TPB), TPB, 0, s>>>(num_cones, cone_vdim, cone_type, len);
    std::vector<int> h(num_cones), t(num_cones);
    if (cudaMemcpyAsync(h.data(), len, num_cones * sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(t.data(), cone_type, num_cones * sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaFreeAsync(len, s);
        return -1;
    }
    int maxlen = 0;
    bool types_ok = true;
    for (int i = 0; i < num_cones; ++i) {
        maxlen = std::max(maxlen, h[i]);
        types_ok = types_ok && (t[i] == CONE_STANDARD_SOC || t[i] == CONE_ROTATED_SOC || t[i] == CONE_EXPONENTIAL ||
                                (t[i] == CONE_POWER && cone_alpha));
    }
    if (!types_ok) {
        std::fprintf(stderr, "[pdhcg_b200_project_cone_sections] only SOC, rotated-SOC, exponential and power "
                             "(with cone_alpha) blocks have fixed sections.\n");
        cudaFreeAsync(len, s);
        return -3;
    }
    int S = slots_class(maxlen);
    if (S < 0) {
        cudaFreeAsync(len, s);
        return -2;
    }
    dispatch_s(S, [&](auto SC) {
        project_sections_kernel<SC.value><<<grid_for(num_cones, WARPS), TPB, 0, s>>>(
            num_cones, cone_start, len, cone_type, cone_alpha, x, d, q, tau, fixed, warm);
    });
    cudaFreeAsync(len, s);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int pdhcg_b200_project_cones_noalloc(int num_cones, const int *cone_start, const int *cone_vdim,
                                     const int *cone_type, const double *cone_alpha, double *x, const double *d,
                                     const double *q, double tau, void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    if (num_cones <= 0)
        return 0;
    if (num_cones > NOALLOC_MAX_CONES) {
        std::fprintf(stderr,
                     "[pdhcg_b200_project_cones_noalloc] %d cone blocks exceed the limit of %d "
                     "(use pdhcg_b200_project_cones)\n",
                     num_cones, NOALLOC_MAX_CONES);
        return -4;
    }
    int *scratch = noalloc_scratch();
    if (!scratch)
        return -1;
    noalloc_len_kernel<<<1, TPB, 0, s>>>(num_cones, cone_vdim, cone_type, cone_alpha != nullptr, scratch);
    int info[2] = {0, 0}; // longest block, unsupported-type flag
    if (cudaMemcpyAsync(info, scratch + NOALLOC_MAX_CONES, sizeof(info), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return -1;
    if (info[1]) {
        std::fprintf(stderr, "[pdhcg_b200_project_cones_noalloc] only SOC, rotated-SOC, exponential and power "
                             "blocks (with cone_alpha) are supported.\n");
        return -3;
    }
    int S = slots_class(info[0]);
    if (S < 0)
        return -2;
    dispatch_s(S, [&](auto SC) {
        project_cones_kernel<SC.value><<<grid_for(num_cones, WARPS), TPB, 0, s>>>(num_cones, cone_start, scratch,
                                                                                 cone_type, cone_alpha, x, d, q,
                                                                                 tau, nullptr, nullptr);
    });
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int pdhcg_b200_pdhg_step(const pdhcg_b200_step_t *t, void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    StepData<double> D{};
    D.n = t->n;
    D.m = t->m;
    D.A_rp = t->A_row_ptr;
    D.A_ci = t->A_col_ind;
    D.A_v = t->A_val;
    D.At_rp = t->At_row_ptr;
    D.At_ci = t->At_col_ind;
    D.At_v = t->At_val;
    D.c = t->c;
    D.l = t->var_lb;
    D.u = t->var_ub;
    D.q = t->q_diag;
    D.lc = t->con_lb;
    D.uc = t->con_ub;
    D.g = t->affine_offset;
    D.vr = t->var_rescale;
    D.free_idx = nullptr;
    D.n_free = 0;
    D.n_cones = 0;
    D.x0 = t->x_init;
    D.x = t->x_cur;
    D.xp = t->x_pdhg;
    D.xr = t->x_refl;
    D.dx = t->x_refl; // unused (want_fpe = 0)
    D.dual_slack = nullptr;
    D.y0 = t->y_init;
    D.y = t->y_cur;
    D.yp = t->y_pdhg;
    D.dy = nullptr;
    StepParams P{t->tau, t->sigma, t->halpern_weight, t->reflection, 1, 1, 0, 0, 1};
    // the kernel-level step keeps cone handling separate: free kernel over all
    // variables, then project + re-reflect cone blocks, then the dual kernel.
    // Halpern is applied at the end so the cone correction sees x_cur.
    try {
        return step_impl(D, P, t, s);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "[pdhcg_b200] step failed: %s\n", e.what());
        return -1;
    }
}

} // extern "C"
