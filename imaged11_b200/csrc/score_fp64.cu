// Exact FP64 scoring kernels: the reference's arithmetic on the GPU.
//
// score, score_and_refine, refine_assigned, score_and_assign and
// verify_rounding, one UBI per call, bit-exact in every decision with
// ImageD11 src/closest.c (no FMA, left-to-right sums, magic-constant
// rounding, strict drlv2 < tol^2).  Least-squares sums are reduced in a fixed
// tree (per-thread partials -> warp butterfly -> CTA -> one finishing CTA), so
// a call is reproducible run to run; the refined UBI differs from the
// reference's sequential sum only by the rounding of that order (<1e-12
// relative on the test sets).
//
// Also the plain batched FP64 scorer (many UBIs x many g, one launch per
// tolerance set), the baseline against which the batched FP32 kernels are
// measured.
#include <cuda.h>

#include <mutex>

#include "common.cuh"

namespace id11b {

constexpr int kThreads = 256;
constexpr int kLsqMaxBlocks = 1024;
constexpr int64_t kLsqSingleMax = 16384;  // peaks scored by one CTA in one launch

struct LsqPartial {
    double r[9];   // sum ih_j * g_i       (R, row-major)
    double h[6];   // sum ih_i * ih_j      (H upper triangle: 00 01 02 11 12 22)
    double ss;     // sum drlv2
    long long n;   // accepted peaks
};

__device__ __forceinline__ void load_ubi(const double* __restrict__ p, double u[9]) {
#pragma unroll
    for (int i = 0; i < 9; i++) u[i] = __ldg(p + i);
}

// ---------------------------------------------------------------- score ----
__global__ void __launch_bounds__(kThreads)
k_score(const double* __restrict__ ubi, const double* __restrict__ gv, double tolsq,
        int64_t ng, int* __restrict__ count) {
    double u[9];
    load_ubi(ubi, u);
    int n = 0;
    for (int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x; k < ng;
         k += (int64_t)gridDim.x * kThreads) {
        double ih[3];
        double s = drlv2_exact(u, __ldg(gv + 3 * k), __ldg(gv + 3 * k + 1),
                               __ldg(gv + 3 * k + 2), ih);
        n += (s < tolsq);
    }
    n = warp_sum(n);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(count, n);
}

// ------------------------------------------------------ LSQ (two stages) ----
// Stage 1: per-CTA partial sums.  MODE 0 = score_and_refine (accept by tol),
// MODE 1 = refine_assigned (accept by label).
template <int MODE>
__device__ __forceinline__ void lsq_partials_body(const double* __restrict__ ubi,
                                                  const double* __restrict__ gv, double tolsq,
                                                  const int* __restrict__ labels, int label,
                                                  int64_t ng, LsqPartial* __restrict__ part,
                                                  int blk, int nblk) {
    double u[9];
    load_ubi(ubi, u);
    double r[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double h[6] = {0, 0, 0, 0, 0, 0};
    double ss = 0.;
    long long n = 0;
    for (int64_t k = (int64_t)blk * kThreads + threadIdx.x; k < ng;
         k += (int64_t)nblk * kThreads) {
        if (MODE == 1 && __ldg(labels + k) != label) continue;
        double g0 = __ldg(gv + 3 * k), g1 = __ldg(gv + 3 * k + 1), g2 = __ldg(gv + 3 * k + 2);
        double ih[3];
        double s = drlv2_exact(u, g0, g1, g2, ih);
        if (MODE == 0 && !(s < tolsq)) continue;
        n++;
        ss = dadd(ss, s);
        const double g[3] = {g0, g1, g2};
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) r[3 * i + j] = dadd(r[3 * i + j], dmul(ih[j], g[i]));
        h[0] = dadd(h[0], dmul(ih[0], ih[0]));
        h[1] = dadd(h[1], dmul(ih[1], ih[0]));
        h[2] = dadd(h[2], dmul(ih[2], ih[0]));
        h[3] = dadd(h[3], dmul(ih[1], ih[1]));
        h[4] = dadd(h[4], dmul(ih[2], ih[1]));
        h[5] = dadd(h[5], dmul(ih[2], ih[2]));
    }
    // warp butterfly, then CTA in warp order
#pragma unroll
    for (int i = 0; i < 9; i++) r[i] = warp_sum(r[i]);
#pragma unroll
    for (int i = 0; i < 6; i++) h[i] = warp_sum(h[i]);
    ss = warp_sum(ss);
    n = warp_sum(n);
    __shared__ LsqPartial s_w[kThreads / 32];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int i = 0; i < 9; i++) s_w[w].r[i] = r[i];
#pragma unroll
        for (int i = 0; i < 6; i++) s_w[w].h[i] = h[i];
        s_w[w].ss = ss;
        s_w[w].n = n;
    }
    __syncthreads();
    if (threadIdx.x < 17) {
        const int f = threadIdx.x;
        if (f < 16) {
            double acc = 0.;
            for (int q = 0; q < kThreads / 32; q++) {
                const double* src = f < 9 ? s_w[q].r + f : (f < 15 ? s_w[q].h + (f - 9) : &s_w[q].ss);
                acc += *src;
            }
            double* dst = f < 9 ? part[blk].r + f : (f < 15 ? part[blk].h + (f - 9) : &part[blk].ss);
            *dst = acc;
        } else {
            long long acc = 0;
            for (int q = 0; q < kThreads / 32; q++) acc += s_w[q].n;
            part[blk].n = acc;
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads)
k_lsq_partials(const double* __restrict__ ubi, const double* __restrict__ gv, double tolsq,
               const int* __restrict__ labels, int label, int64_t ng,
               LsqPartial* __restrict__ part) {
    lsq_partials_body<MODE>(ubi, gv, tolsq, labels, label, ng, part, blockIdx.x, gridDim.x);
}

// Stage 2: one CTA sums the partials in a fixed order and applies the
// reference's least-squares update (ImageD11 src/closest.c:326-344).
__device__ __forceinline__ void lsq_finish_body(const LsqPartial* __restrict__ part, int nparts,
                                                double* __restrict__ ubi, int* __restrict__ n_out,
                                                double* __restrict__ mean_out) {
    __shared__ double s_acc[kThreads / 32][16];
    __shared__ long long s_n[kThreads / 32];
    double acc[16];
    long long n = 0;
#pragma unroll
    for (int f = 0; f < 16; f++) acc[f] = 0.;
    for (int p = threadIdx.x; p < nparts; p += kThreads) {
#pragma unroll
        for (int i = 0; i < 9; i++) acc[i] += part[p].r[i];
#pragma unroll
        for (int i = 0; i < 6; i++) acc[9 + i] += part[p].h[i];
        acc[15] += part[p].ss;
        n += part[p].n;
    }
#pragma unroll
    for (int f = 0; f < 16; f++) acc[f] = warp_sum(acc[f]);
    n = warp_sum(n);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int f = 0; f < 16; f++) s_acc[w][f] = acc[f];
        s_n[w] = n;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[16];
        long long nn = 0;
        for (int f = 0; f < 16; f++) t[f] = 0.;
        for (int q = 0; q < kThreads / 32; q++) {
            for (int f = 0; f < 16; f++) t[f] += s_acc[q][f];
            nn += s_n[q];
        }
        double R[9], H[9];
        for (int i = 0; i < 9; i++) R[i] = t[i];
        H[0] = t[9];  H[1] = t[10]; H[2] = t[11];
        H[3] = t[10]; H[4] = t[12]; H[5] = t[13];
        H[6] = t[11]; H[7] = t[13]; H[8] = t[14];
        double u[9];
        for (int i = 0; i < 9; i++) u[i] = ubi[i];
        lsq_update_exact(R, H, u);
        for (int i = 0; i < 9; i++) ubi[i] = u[i];
        *n_out = (int)nn;
        *mean_out = nn > 0 ? ddiv(t[15], (double)nn) : 0.;
    }
}

__global__ void __launch_bounds__(kThreads)
k_lsq_finish(const LsqPartial* __restrict__ part, int nparts, double* __restrict__ ubi,
             int* __restrict__ n_out, double* __restrict__ mean_out) {
    lsq_finish_body(part, nparts, ubi, n_out, mean_out);
}

// Small inputs: both stages in one CTA and one launch (the partial sums of
// one CTA, then the finish), so that a small call pays one kernel launch.
template <int MODE>
__global__ void __launch_bounds__(kThreads)
k_lsq_single(double* __restrict__ ubi, const double* __restrict__ gv, double tolsq,
             const int* __restrict__ labels, int label, int64_t ng, LsqPartial* __restrict__ part,
             int* __restrict__ n_out, double* __restrict__ mean_out) {
    lsq_partials_body<MODE>(ubi, gv, tolsq, labels, label, ng, part, 0, 1);
    __syncthreads();  // part[0] written by this CTA
    lsq_finish_body(part, 1, ubi, n_out, mean_out);
}

// ------------------------------------------------------- score_and_assign ----
// ImageD11 src/closest.c:366-397, elementwise and bit-exact.
__global__ void __launch_bounds__(kThreads)
k_score_and_assign(const double* __restrict__ ubi, const double* __restrict__ gv,
                   double tolsq, double* __restrict__ drlv2, int* __restrict__ labels,
                   int label, int64_t ng, int* __restrict__ count) {
    double u[9];
    load_ubi(ubi, u);
    int n = 0;
    for (int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x; k < ng;
         k += (int64_t)gridDim.x * kThreads) {
        double ih[3];
        double s = drlv2_exact(u, __ldg(gv + 3 * k), __ldg(gv + 3 * k + 1),
                               __ldg(gv + 3 * k + 2), ih);
        if ((s < tolsq) && (s < drlv2[k])) {
            labels[k] = label;
            drlv2[k] = s;
            n++;
        } else if (labels[k] == label) {
            labels[k] = -1;
        }
    }
    n = warp_sum(n);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(count, n);
}

// -------------------------------------------------------- verify_rounding ----
// ImageD11 src/closest.c:100-119 with the device's rounding.
__global__ void k_verify_rounding(int n, int* __restrict__ bad) {
    int b = 0;
    for (int i = threadIdx.x; i < 600; i += blockDim.x) {
        int pass = i / 300, ii = i % 300 - 100;
        double v = dadd((double)(pass == 0 ? n : -n), dmul((double)ii, 50.0));
        int fast = (int)dround(v);
        int slow = (int)floor(dadd(v, 0.5));
        b += (fast != slow);
    }
    b = warp_sum(b);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(bad, b);
}

// ------------------------------------------ plain batched FP64 (baseline) ----
// counts[m*ntol + j] += #{k : drlv2(ubis[m], g_k) < tolsq[j]}.  CTA b handles
// UBI b / chunks and g range (b % chunks); one thread per g, grid-stride over
// the range; warp sums + one atomic per warp.  The straightforward GPU port of
// a loop of reference score() calls; all decisions bit-exact.
struct TolSq {
    double t[ID11B_MAX_TOLS];
};

__global__ void __launch_bounds__(kThreads)
k_score_many_fp64(const double* __restrict__ ubis, int64_t m, const double* __restrict__ gv,
                  int64_t ng, TolSq tolsq, int ntol, int chunks, int* __restrict__ counts) {
    const int64_t ui = blockIdx.x / chunks;
    const int c = blockIdx.x % chunks;
    if (ui >= m) return;
    const int64_t per = (ng + chunks - 1) / chunks;
    const int64_t k0 = c * per, k1 = min(ng, k0 + per);
    double u[9];
    load_ubi(ubis + 9 * ui, u);
    int cnt[ID11B_MAX_TOLS] = {0, 0, 0, 0};
    for (int64_t k = k0 + threadIdx.x; k < k1; k += kThreads) {
        double ih[3];
        double s = drlv2_exact(u, __ldg(gv + 3 * k), __ldg(gv + 3 * k + 1),
                               __ldg(gv + 3 * k + 2), ih);
#pragma unroll
        for (int j = 0; j < ID11B_MAX_TOLS; j++)
            if (j < ntol) cnt[j] += (s < tolsq.t[j]);
    }
#pragma unroll
    for (int j = 0; j < ID11B_MAX_TOLS; j++) {
        if (j >= ntol) break;
        int v = warp_sum(cnt[j]);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(counts + ui * ntol + j, v);
    }
}

static int sm_count() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

static int stream_grid(int64_t ng, int per_sm) {
    int64_t b = (ng + kThreads - 1) / kThreads;
    int64_t cap = (int64_t)sm_count() * per_sm;
    if (b > cap) b = cap;
    return (int)(b > 0 ? b : 1);
}

// LSQ partial CTAs: a deterministic function of ng only (not of the device),
// so a given input always reduces in the same order.
static int lsq_blocks(int64_t ng) {
    int64_t b = (ng + 4 * kThreads - 1) / (4 * kThreads);
    if (b > kLsqMaxBlocks) b = kLsqMaxBlocks;
    return (int)(b > 0 ? b : 1);
}

}  // namespace id11b

using namespace id11b;

extern "C" int64_t id11b_lsq_workspace_bytes(int64_t ng) {
    (void)ng;
    return (int64_t)kLsqMaxBlocks * (int64_t)sizeof(LsqPartial);
}

extern "C" int id11b_dev_score(const double* ubi, const double* gv, double tol, int64_t ng,
                               int32_t* count, void* stream) {
    if (ng < 0 || !ubi || !count || (ng > 0 && !gv)) return ID11B_ERR_ARG;
    if (ng > INT32_MAX) return ID11B_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    ID11B_CHECK(cudaMemsetAsync(count, 0, sizeof(int32_t), st));
    if (ng == 0) return ID11B_OK;
    k_score<<<stream_grid(ng, 8), kThreads, 0, st>>>(ubi, gv, tol * tol, ng, count);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

static int lsq_launch(int mode, double* ubi, const double* gv, double tol,
                      const int32_t* labels, int label, int64_t ng, int32_t* n,
                      double* mean, void* ws, int64_t ws_bytes, void* stream) {
    if (ng < 0 || !ubi || !n || !mean || !ws || (ng > 0 && !gv)) return ID11B_ERR_ARG;
    if (mode == 1 && ng > 0 && !labels) return ID11B_ERR_ARG;
    if (ng > INT32_MAX) return ID11B_ERR_SIZE;
    if (ws_bytes < id11b_lsq_workspace_bytes(ng)) return ID11B_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    LsqPartial* part = (LsqPartial*)ws;
    int nb = lsq_blocks(ng);
    if (ng > 0 && ng <= kLsqSingleMax) {
        if (mode == 0)
            k_lsq_single<0><<<1, kThreads, 0, st>>>(ubi, gv, tol * tol, nullptr, 0, ng, part, n,
                                                    mean);
        else
            k_lsq_single<1><<<1, kThreads, 0, st>>>(ubi, gv, 0., labels, label, ng, part, n,
                                                    mean);
        ID11B_CHECK_LAUNCH();
        return ID11B_OK;
    }
    if (ng == 0) {
        ID11B_CHECK(cudaMemsetAsync(part, 0, sizeof(LsqPartial), st));
    } else if (mode == 0) {
        k_lsq_partials<0><<<nb, kThreads, 0, st>>>(ubi, gv, tol * tol, nullptr, 0, ng, part);
    } else {
        k_lsq_partials<1><<<nb, kThreads, 0, st>>>(ubi, gv, 0., labels, label, ng, part);
    }
    ID11B_CHECK_LAUNCH();
    k_lsq_finish<<<1, kThreads, 0, st>>>(part, ng == 0 ? 1 : nb, ubi, n, mean);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_score_and_refine(double* ubi, const double* gv, double tol,
                                          int64_t ng, int32_t* n, double* mean_drlv2,
                                          void* workspace, int64_t workspace_bytes,
                                          void* stream) {
    return lsq_launch(0, ubi, gv, tol, nullptr, 0, ng, n, mean_drlv2, workspace,
                      workspace_bytes, stream);
}

extern "C" int id11b_dev_refine_assigned(double* ubi, const double* gv,
                                         const int32_t* labels, int label, int64_t ng,
                                         int32_t* npk, double* mean_drlv2, void* workspace,
                                         int64_t workspace_bytes, void* stream) {
    return lsq_launch(1, ubi, gv, 0., labels, label, ng, npk, mean_drlv2, workspace,
                      workspace_bytes, stream);
}

extern "C" int id11b_dev_score_and_assign(const double* ubi, const double* gv, double tol,
                                          double* drlv2, int32_t* labels, int label,
                                          int64_t ng, int32_t* count, void* stream) {
    if (ng < 0 || !ubi || !count || (ng > 0 && (!gv || !drlv2 || !labels)))
        return ID11B_ERR_ARG;
    if (ng > INT32_MAX) return ID11B_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    ID11B_CHECK(cudaMemsetAsync(count, 0, sizeof(int32_t), st));
    if (ng == 0) return ID11B_OK;
    k_score_and_assign<<<stream_grid(ng, 8), kThreads, 0, st>>>(ubi, gv, tol * tol, drlv2,
                                                                 labels, label, ng, count);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_verify_rounding(int n, int32_t* bad, void* stream) {
    if (!bad) return ID11B_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    ID11B_CHECK(cudaMemsetAsync(bad, 0, sizeof(int32_t), st));
    k_verify_rounding<<<1, 320, 0, st>>>(n, bad);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_score_many_fp64(const double* ubis, int64_t m, const double* gv,
                                         int64_t ng, const double* tols_host, int ntol,
                                         int32_t* counts, void* stream) {
    if (m < 0 || ng < 0 || ntol < 1 || ntol > ID11B_MAX_TOLS || !tols_host)
        return ID11B_ERR_ARG;
    if ((m > 0 && (!ubis || !counts)) || (ng > 0 && !gv)) return ID11B_ERR_ARG;
    if (m == 0) return ID11B_OK;
    cudaStream_t st = (cudaStream_t)stream;
    ID11B_CHECK(cudaMemsetAsync(counts, 0, sizeof(int32_t) * m * ntol, st));
    if (ng == 0) return ID11B_OK;
    TolSq ts;
    for (int j = 0; j < ID11B_MAX_TOLS; j++) ts.t[j] = j < ntol ? tols_host[j] * tols_host[j] : 0.;
    // g range per CTA: 64 g per thread, so CTA start-up stays a small part of
    // each CTA's time, and M x chunks CTAs fill every SM many times over.
    int64_t chunks = (ng + 64 * kThreads - 1) / (64 * kThreads);
    if (chunks < 1) chunks = 1;
    if (m * chunks > INT32_MAX) return ID11B_ERR_SIZE;
    k_score_many_fp64<<<(unsigned)(m * chunks), kThreads, 0, st>>>(ubis, m, gv, ng, ts, ntol,
                                                                  (int)chunks, counts);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

// ------------------------------------------------ allocation-free variant ----
// score_and_refine for callers that must not allocate device memory: a
// process that reserves the GPU's memory up front for detector frame buffers
// and forbids later allocations (to keep acquisition latency predictable), or
// a host that runs this code inside another framework's memory pool with a
// hard cap.  The least-squares partial sums live in this file-scope device
// array (kLsqMaxBlocks x 136 bytes = 136 KiB, held by every GPU that loads the
// library until the process exits) instead of caller- or pool-provided memory.
//
// CUDA loads modules lazily (the default since CUDA 12.2): the module holding
// this array and the kernels below is loaded, and its memory taken, on the
// first call in each context.  A caller that reserves memory or caps a pool
// afterwards makes one warm-up call per device first (one g-vector is enough;
// it launches both kernels).
//
// Every call on a device shares the array.  Each partial-sum CTA writes its own
// slot before the finishing CTA reads it, so the previous call's contents never
// leak into a result (the empty-input case zeroes slot 0 itself); calls that
// overlap on the GPU -- on different streams, or from different host threads
// without ordering -- race on the array and must be serialised by the caller.
static __device__ __align__(256) LsqPartial g_lsq_scratch[kLsqMaxBlocks];

namespace {
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// The array's device address belongs to the context the module was loaded
// in: a driver-API caller's own context, or a primary context recreated after
// cudaDeviceReset, holds it elsewhere.  So the cache is keyed by the unique id
// of the current context (cuCtxGetId), never by the device ordinal.
constexpr int kMaxContexts = 64;
struct ScratchEntry {
    unsigned long long ctx_id;
    void* ptr;
};
std::mutex g_lsq_scratch_mu;
ScratchEntry g_lsq_scratch_cache[kMaxContexts] = {};
int g_lsq_scratch_used = 0;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

int driver_entry_points() {  // under g_lsq_scratch_mu
    if (g_ctx_get_current && g_ctx_get_id) return ID11B_OK;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q);
    if (e != cudaSuccess) return id11b_record_cuda(e);
    if (q != cudaDriverEntryPointSuccess || !f) return ID11B_ERR_CUDA;
    g_ctx_get_current = (CtxGetCurrentFn)f;
    f = nullptr;
    e = cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q);
    if (e != cudaSuccess) return id11b_record_cuda(e);
    if (q != cudaDriverEntryPointSuccess || !f) return ID11B_ERR_CUDA;
    g_ctx_get_id = (CtxGetIdFn)f;
    return ID11B_OK;
}

// The name g_lsq_scratch is only a host-side stand-in: a kernel must be given
// the device address, looked up with the context current in which it runs.
int lsq_scratch_address(void** out) {
    std::lock_guard<std::mutex> lock(g_lsq_scratch_mu);
    int rc = driver_entry_points();
    if (rc) return rc;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    void* p = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) return ID11B_ERR_CUDA;
    if (ctx) {
        if (g_ctx_get_id(ctx, &id) != CUDA_SUCCESS) return ID11B_ERR_CUDA;
        for (int i = 0; i < g_lsq_scratch_used; i++)
            if (g_lsq_scratch_cache[i].ctx_id == id) {
                *out = g_lsq_scratch_cache[i].ptr;
                return ID11B_OK;
            }
    }
    // with no context current yet, this runtime call makes the current
    // device's primary context current first
    cudaError_t e = cudaGetSymbolAddress(&p, g_lsq_scratch);
    if (e != cudaSuccess) return id11b_record_cuda(e);
    if (!ctx) {
        if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return ID11B_ERR_CUDA;
        if (g_ctx_get_id(ctx, &id) != CUDA_SUCCESS) return ID11B_ERR_CUDA;
    }
    // context ids are never reused; past kMaxContexts the oldest slot is replaced
    const int slot = g_lsq_scratch_used < kMaxContexts ? g_lsq_scratch_used++
                                                       : (int)(id % kMaxContexts);
    g_lsq_scratch_cache[slot] = ScratchEntry{id, p};
    *out = p;
    return ID11B_OK;
}
}  // namespace

extern "C" int64_t id11b_noalloc_scratch_bytes(void) { return (int64_t)sizeof(g_lsq_scratch); }

extern "C" int id11b_dev_score_and_refine_noalloc(double* ubi, const double* gv, double tol,
                                                  int64_t ng, int32_t* n, double* mean_drlv2,
                                                  void* stream) {
    if (ng < 0) return ID11B_ERR_ARG;
    if (ng > INT32_MAX) return ID11B_ERR_SIZE;  // the reference's int peak count
    void* scratch = nullptr;
    int rc = lsq_scratch_address(&scratch);
    if (rc) return rc;
    return lsq_launch(0, ubi, gv, tol, nullptr, 0, ng, n, mean_drlv2, scratch,
                      (int64_t)sizeof(g_lsq_scratch), stream);
}
