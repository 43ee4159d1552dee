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

// Compensated FP32 accumulation (the F32C variant): a sum kept as s + c with
// every addition's rounding error recovered exactly (TwoSum) and every
// product's by an FMA (TwoProduct), Ogita, Rump and Oishi, "Accurate sum and
// dot product", SIAM J. Sci. Comput. 26 (2005) -- as accurate as a sum in
// twice the working precision.
__device__ __forceinline__ void comp_add(float& s, float& c, float x) {
    const float t = s + x;
    const float bp = t - s;
    c += (s - (t - bp)) + (x - bp);
    s = t;
}

template <int NT, bool F32C = false>
__global__ void __launch_bounds__(NT)
k_refine_csr(double* __restrict__ ubis, const double* __restrict__ gv,
             const int64_t* __restrict__ off, const int* __restrict__ order, int ngrains,
             double tolsq, int iters, int* __restrict__ queue, int* __restrict__ npk,
             double* __restrict__ mean, double gmax) {
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
            // F32C: screening thresholds of the proven band (score_batch.cu) for
            // this UBI, FP32 copy of the UBI, compensated R and drlv2 sums,
            // exact integer H
            float lo32 = 0.f, hi32 = 0.f, u32[9], rs[9], rc[9], ss32 = 0.f, sc32 = 0.f;
            int hint[6] = {0, 0, 0, 0, 0, 0}, nacc = 0;
            if (F32C) {
                double S = 0.;
#pragma unroll
                for (int r = 0; r < 3; r++)
                    S = fmax(S, fabs(u[3 * r]) + fabs(u[3 * r + 1]) + fabs(u[3 * r + 2]));
                const double E = 6.0 * 5.9604644775390625e-08 * S * (1. + 1e-15) * gmax;
                const double t = sqrt(tolsq);
                const double band = 1.25 * (3.0 * E * (2.0 * (t + 1e-3) + E) +
                                            4.0 * 5.9604644775390625e-08 * (tolsq + 0.01));
                lo32 = __double2float_rd(tolsq - band);
                hi32 = __double2float_ru(tolsq + band);
#pragma unroll
                for (int e = 0; e < 9; e++) {
                    u32[e] = __double2float_rn(u[e]);
                    rs[e] = rc[e] = 0.f;
                }
            }
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
                    if (F32C) {
                        // g split exactly enough into hi + lo floats
                        float gh[3], gl[3], ihf[3], t[3];
#pragma unroll
                        for (int i = 0; i < 3; i++) {
                            gh[i] = __double2float_rn(gg[q][i]);
                            gl[i] = __double2float_rn(gg[q][i] - (double)gh[i]);
                        }
                        const float M = 12582912.0f;  // 1.5 * 2^23
#pragma unroll
                        for (int r = 0; r < 3; r++) {
                            const float h = fmaf(u32[3 * r + 2], gh[2],
                                                 fmaf(u32[3 * r + 1], gh[1], u32[3 * r] * gh[0]));
                            ihf[r] = __fsub_rn(__fadd_rn(h, M), M);
                            t[r] = h - ihf[r];
                        }
                        float s32 = fmaf(t[2], t[2], fmaf(t[1], t[1], t[0] * t[0]));
                        if (!(s32 < hi32)) continue;
                        if (!(s32 < lo32)) {  // inside the band: the exact decision
                            double ih[3];
                            const double s = drlv2_exact(u, gg[q][0], gg[q][1], gg[q][2], ih);
                            if (!(s < tolsq)) continue;
#pragma unroll
                            for (int r = 0; r < 3; r++) ihf[r] = (float)ih[r];
                            s32 = (float)s;
                        }
#pragma unroll
                        for (int i = 0; i < 3; i++)
#pragma unroll
                            for (int j = 0; j < 3; j++) {
                                // ih_j * g_i = ih_j * gh_i (TwoProduct) + ih_j * gl_i
                                const float p = ihf[j] * gh[i];
                                const float pe = fmaf(ihf[j], gh[i], -p);
                                comp_add(rs[3 * i + j], rc[3 * i + j], p);
                                rc[3 * i + j] += pe + ihf[j] * gl[i];
                            }
                        const int a = (int)ihf[0], b = (int)ihf[1], c = (int)ihf[2];
                        hint[0] += a * a;
                        hint[1] += b * a;
                        hint[2] += c * a;
                        hint[3] += b * b;
                        hint[4] += c * b;
                        hint[5] += c * c;
                        comp_add(ss32, sc32, s32);
                        nacc++;
                        continue;
                    }
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
            if (F32C) {  // to FP64 for the fixed reduction: s + c, exact integers
#pragma unroll
                for (int e = 0; e < 9; e++) acc[e] = (double)rs[e] + (double)rc[e];
#pragma unroll
                for (int e = 0; e < 6; e++) acc[9 + e] = (double)hint[e];
                acc[15] = (double)ss32 + (double)sc32;
                acc[16] = (double)nacc;
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

template <int NT, bool F32C = false>
static int launch_refine(double* ubis, const double* gv, const int64_t* offsets,
                         const int32_t* order, int32_t ngrains, double tolsq, int iters,
                         int* queue, int32_t* npk, double* mean, cudaStream_t st,
                         double gmax = 0.) {
    int grid = ngrains;
    if (queue) {
        static int occ = 0;
        if (!occ) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_refine_csr<NT, F32C>, NT, 0);
            if (occ < 1) occ = 1;
        }
        const int cap = sm_count_rc() * occ;
        grid = ngrains < cap ? ngrains : cap;
    }
    k_refine_csr<NT, F32C><<<grid, NT, 0, st>>>(ubis, gv, offsets, order, ngrains, tolsq, iters,
                                                queue, npk, mean, gmax);
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

// The same rounds with FP32 screening (the proven band, FP64 inside it) and
// compensated FP32 normal-equation sums (integer H), FP64 3x3 solves: the
// accumulation the batched design could use instead of FP64 sums.  gmax:
// bound on every |g_j| of the segments (the band's input); g-vectors beyond
// 1024 or non-finite are not supported by this variant (ID11B_ERR_ARG).
extern "C" int id11b_dev_refine_csr_f32c(double* ubis, const double* gv, const int64_t* offsets,
                                         const int32_t* order, int32_t ngrains, double tol,
                                         int iters, double gmax, int32_t* npk,
                                         double* mean_drlv2, void* workspace, int64_t ws_bytes,
                                         void* stream) {
    if (ngrains < 0 || iters < 0 || !(gmax >= 0.) || !(gmax <= 1024.) || !(tol >= 0.) ||
        !(tol < 0.4))
        return ID11B_ERR_ARG;
    if (ngrains > 0 && (!ubis || !offsets)) return ID11B_ERR_ARG;
    if (!workspace || ws_bytes < id11b_refine_csr_workspace_bytes()) return ID11B_ERR_ARG;
    if (ngrains == 0 || iters == 0) return ID11B_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int* queue = (int*)workspace;
    ID11B_CHECK(cudaMemsetAsync(queue, 0, sizeof(int), st));
    return launch_refine<64, true>(ubis, gv, offsets, order, ngrains, tol * tol, iters, queue,
                                   npk, mean_drlv2, st, gmax);
}
