// Batched per-grain refinement over CSR peak lists (score_and_refine x iters).
//
// Grain g owns the g-vectors gv[off[g] : off[g+1]] (20 .. 2000 peaks each in
// the uneven workload) and `iters` rounds of the reference's score_and_refine
// (ImageD11 src/closest.c:267-345) are applied to its UBI.  One CTA (128,
// 256 or 512 threads, chosen from the largest grain) refines one grain at a
// time and runs all rounds itself: per round, every thread tests its peaks
// with the reference's exact FP64 arithmetic and accumulates the accepted
// peaks' normal-equation terms, the CTA reduces them in a fixed tree (warp
// butterfly, then warps in order),
// and nine threads apply the reference's update (one cofactor / one UB element
// each; the same expressions as inverse3x3, so the result equals the
// single-thread update bit for bit).
//
// Persistent mode (queue != null): a grid sized to the GPU pulls grains from
// an atomic work counter in the caller's order -- largest grains first (LPT)
// keeps the tail short.  No CTA ever waits on another, so there is nothing to
// time out.  Plain mode (queue == null): CTA b refines grain order[b]; used
// one launch per round as the straightforward baseline.
//
// Peaks are evaluated in exact FP64 here: refinement segments are a grain's
// own peaks, nearly all accepted, and every accepted pair needs its FP64
// g-vector and exact drlv2 anyway, so an FP32 pre-screen would only add work.
#include "common.cuh"

namespace id11b {

// Element idx of the cofactor inverse, as inverse3x3 (src/closest.c:38-76).
__device__ __forceinline__ double inv3_elem(const double* a, double det, int idx) {
    const double a00 = a[0], a01 = a[1], a02 = a[2], a10 = a[3], a11 = a[4], a12 = a[5],
                 a20 = a[6], a21 = a[7], a22 = a[8];
    switch (idx) {
        case 0: return ddiv(dsub(dmul(a22, a11), dmul(a21, a12)), det);
        case 1: return ddiv(-dsub(dmul(a22, a01), dmul(a21, a02)), det);
        case 2: return ddiv(dsub(dmul(a12, a01), dmul(a11, a02)), det);
        case 3: return ddiv(-dsub(dmul(a22, a10), dmul(a20, a12)), det);
        case 4: return ddiv(dsub(dmul(a22, a00), dmul(a20, a02)), det);
        case 5: return ddiv(-dsub(dmul(a12, a00), dmul(a10, a02)), det);
        case 6: return ddiv(dsub(dmul(a21, a10), dmul(a20, a11)), det);
        case 7: return ddiv(-dsub(dmul(a21, a00), dmul(a20, a01)), det);
        default: return ddiv(dsub(dmul(a11, a00), dmul(a10, a01)), det);
    }
}

__device__ __forceinline__ double det3_exact(const double* a) {
    return dadd(dsub(dmul(a[0], dsub(dmul(a[8], a[4]), dmul(a[7], a[5]))),
                     dmul(a[3], dsub(dmul(a[8], a[1]), dmul(a[7], a[2])))),
                dmul(a[6], dsub(dmul(a[5], a[1]), dmul(a[4], a[2]))));
}

template <int NT>
struct RefineSmem {
    double red[NT / 32][17];  // per-warp partial sums
    double R[9], H[9], Hi[9], UB[9], UBI[9], ubi[9];
    long long n;
    double ss;
    int ok, ok2;
    int grain;
};

// H upper-triangle slot (00 01 02 11 12 22) -> row, column
__constant__ int c_hrow[6] = {0, 0, 0, 1, 1, 2};
__constant__ int c_hcol[6] = {0, 1, 2, 1, 2, 2};

template <int NT>
__global__ void __launch_bounds__(NT)
k_refine_csr(double* __restrict__ ubis, const double* __restrict__ gv,
             const int64_t* __restrict__ off, const int* __restrict__ order, int ngrains,
             double tolsq, int iters, int* __restrict__ queue, int* __restrict__ npk,
             double* __restrict__ mean) {
    __shared__ RefineSmem<NT> sm;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int slot = blockIdx.x;; slot += gridDim.x) {
        if (queue) {
            if (tid == 0) sm.grain = atomicAdd(queue, 1);
            __syncthreads();
            slot = sm.grain;
        }
        if (slot >= ngrains) break;
        const int g = order ? order[slot] : slot;
        const int64_t k0 = off[g], k1 = off[g + 1];
        if (tid < 9) sm.ubi[tid] = ubis[9 * (int64_t)g + tid];
        __syncthreads();
        for (int it = 0; it < iters; it++) {
            double u[9];
#pragma unroll
            for (int e = 0; e < 9; e++) u[e] = sm.ubi[e];
            double acc[17];
#pragma unroll
            for (int f = 0; f < 17; f++) acc[f] = 0.;
            // kU peaks per lane per step: all their loads are issued before any
            // is used, so one memory latency covers kU peaks (the segment is
            // read-only and re-read every round, so later rounds hit L1)
            constexpr int kU = 4;
            for (int64_t kb = k0 + tid; kb < k1; kb += kU * NT) {
                double gg[kU][3];
#pragma unroll
                for (int q = 0; q < kU; q++) {
                    const int64_t k = kb + (int64_t)q * NT;
                    if (k < k1) {
                        gg[q][0] = __ldg(gv + 3 * k);
                        gg[q][1] = __ldg(gv + 3 * k + 1);
                        gg[q][2] = __ldg(gv + 3 * k + 2);
                    }
                }
#pragma unroll
                for (int q = 0; q < kU; q++) {
                    if (kb + (int64_t)q * NT >= k1) break;
                    double ih[3];
                    const double s = drlv2_exact(u, gg[q][0], gg[q][1], gg[q][2], ih);
                    if (!(s < tolsq)) continue;
                    // normal equations with fused multiply-adds: H (products of
                    // integers) is exact either way; each R term is rounded once
                    // instead of twice -- R is order-dependent against the
                    // reference's sequential sum in any case
#pragma unroll
                    for (int i = 0; i < 3; i++)
#pragma unroll
                        for (int j = 0; j < 3; j++)
                            acc[3 * i + j] = fma(ih[j], gg[q][i], acc[3 * i + j]);
                    acc[9] = fma(ih[0], ih[0], acc[9]);
                    acc[10] = fma(ih[1], ih[0], acc[10]);
                    acc[11] = fma(ih[2], ih[0], acc[11]);
                    acc[12] = fma(ih[1], ih[1], acc[12]);
                    acc[13] = fma(ih[2], ih[1], acc[13]);
                    acc[14] = fma(ih[2], ih[2], acc[14]);
                    acc[15] = dadd(acc[15], s);
                    acc[16] += 1.0;
                }
            }
#pragma unroll
            for (int f = 0; f < 17; f++) acc[f] = warp_sum(acc[f]);
            if (lane == 0)
#pragma unroll
                for (int f = 0; f < 17; f++) sm.red[w][f] = acc[f];
            __syncthreads();
            if (tid < 17) {
                double t = 0.;
                for (int q = 0; q < NT / 32; q++) t += sm.red[q][tid];
                if (tid < 9) {
                    sm.R[tid] = t;
                } else if (tid < 15) {
                    const int i = c_hrow[tid - 9], j = c_hcol[tid - 9];
                    sm.H[3 * i + j] = t;  // identical sums for (i,j) and (j,i)
                    sm.H[3 * j + i] = t;
                } else if (tid == 15) {
                    sm.ss = t;
                } else {
                    sm.n = (long long)t;
                }
            }
            __syncthreads();
            // UB = R . inv(H); UBI = inv(UB); keep ubi unless both inverses exist
            if (tid < 9) {
                const double det = det3_exact(sm.H);
                if (tid == 0) sm.ok = det != 0.;
                if (det != 0.) sm.Hi[tid] = inv3_elem(sm.H, det, tid);
            }
            __syncthreads();
            if (tid < 9 && sm.ok) {
                const int i = tid / 3, j = tid % 3;
                double s = 0.;
                s = dadd(s, dmul(sm.R[3 * i + 0], sm.Hi[0 + j]));
                s = dadd(s, dmul(sm.R[3 * i + 1], sm.Hi[3 + j]));
                s = dadd(s, dmul(sm.R[3 * i + 2], sm.Hi[6 + j]));
                sm.UB[tid] = s;
            }
            __syncthreads();
            if (tid < 9 && sm.ok) {
                const double det = det3_exact(sm.UB);
                if (tid == 0) sm.ok2 = det != 0.;
                if (det != 0.) sm.UBI[tid] = inv3_elem(sm.UB, det, tid);
            }
            __syncthreads();
            if (tid < 9 && sm.ok && sm.ok2) sm.ubi[tid] = sm.UBI[tid];
            if (tid == 0 && it == iters - 1) {
                if (npk) npk[g] = (int)sm.n;
                if (mean) mean[g] = sm.n > 0 ? ddiv(sm.ss, (double)sm.n) : 0.;
            }
            __syncthreads();
        }
        if (tid < 9) ubis[9 * (int64_t)g + tid] = sm.ubi[tid];
        __syncthreads();
        if (!queue && slot + (int)gridDim.x >= ngrains) break;  // plain: one grain per CTA
    }
}

static int sm_count_rc() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

}  // namespace id11b

using namespace id11b;

template <int NT>
static int launch_refine(double* ubis, const double* gv, const int64_t* offsets,
                         const int32_t* order, int32_t ngrains, double tolsq, int iters,
                         int* queue, int32_t* npk, double* mean, cudaStream_t st) {
    int grid = ngrains;
    if (queue) {
        static int occ = 0;
        if (!occ) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_refine_csr<NT>, NT, 0);
            if (occ < 1) occ = 1;
        }
        const int cap = sm_count_rc() * occ;
        grid = ngrains < cap ? ngrains : cap;
    }
    k_refine_csr<NT><<<grid, NT, 0, st>>>(ubis, gv, offsets, order, ngrains, tolsq, iters,
                                          queue, npk, mean);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int64_t id11b_refine_csr_workspace_bytes(void) { return 256; }

extern "C" int id11b_dev_refine_csr(double* ubis, const double* gv, const int64_t* offsets,
                                    const int32_t* order, int32_t ngrains, double tol,
                                    int iters, int persistent, int threads, int32_t* npk,
                                    double* mean_drlv2, void* workspace, int64_t ws_bytes,
                                    void* stream) {
    if (ngrains < 0 || iters < 0) return ID11B_ERR_ARG;
    if (ngrains > 0 && (!ubis || !offsets)) return ID11B_ERR_ARG;
    if (persistent && (!workspace || ws_bytes < id11b_refine_csr_workspace_bytes()))
        return ID11B_ERR_ARG;
    if (threads != 0 && threads != 32 && threads != 64 && threads != 128 && threads != 256 &&
        threads != 512)
        return ID11B_ERR_ARG;
    if (ngrains == 0 || iters == 0) return ID11B_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int* queue = nullptr;
    if (persistent) {
        queue = (int*)workspace;
        ID11B_CHECK(cudaMemsetAsync(queue, 0, sizeof(int), st));
    }
    const double tolsq = tol * tol;
    switch (threads) {
        case 32: return launch_refine<32>(ubis, gv, offsets, order, ngrains, tolsq, iters, queue, npk, mean_drlv2, st);
        case 64: return launch_refine<64>(ubis, gv, offsets, order, ngrains, tolsq, iters, queue, npk, mean_drlv2, st);
        case 256: return launch_refine<256>(ubis, gv, offsets, order, ngrains, tolsq, iters, queue, npk, mean_drlv2, st);
        case 512: return launch_refine<512>(ubis, gv, offsets, order, ngrains, tolsq, iters, queue, npk, mean_drlv2, st);
        default: return launch_refine<128>(ubis, gv, offsets, order, ngrains, tolsq, iters, queue, npk, mean_drlv2, st);
    }
}
