// Batched scoring and dense refinement: FP32 screening, exact FP64 recheck.
//
// Work: M trial UBIs x N g-vectors x T tolerances.  Each CTA owns 256*R UBIs
// (R per thread, in registers) and one g range; g tiles (float4, 16 KB) are
// staged into shared memory by 1-D TMA bulk copies on a two-stage mbarrier
// ring and read by every lane (broadcast).  Per (UBI, g) pair (computed for
// two UBIs at a time with packed f32x2 instructions):
//
//   h   = UBI32 . g32             3 FFMA chains            (9 FMA-pipe ops)
//   t   = h - rint(h)             magic-constant rounding  (9)
//   s   = t.t                                              (3)
//   s < hi_max ?  -> rare path                             (1)
//
// The rare path (s near or below the largest tol^2) counts the pair for every
// tolerance it clears by more than a proven error band, and re-evaluates it
// with the reference's exact FP64 arithmetic (common.cuh) when s lies inside
// the band.  The band: for FP32 inputs rounded from FP64 and an FMA chain,
//   |h32 - h64| <= E = 6 * 2^-24 * S * gmax,
// S = max over UBIs and rows of sum_j |u_ij|, gmax = max |g_j| (Higham,
// Accuracy and Stability of Numerical Algorithms, 2nd ed., sections 2-3);
// hence |s32 - s64| <= 3E(2 tol + E) + 4 * 2^-24 * s.  For tol < 0.45 every
// pair that can be counted has all |t| < 0.5 - E, so FP32 and FP64 round h to
// the same integers; counts are therefore identical to the reference's.
// UBIs whose S * gmax is too large for that argument (or with non-finite
// elements), and g-vectors with non-finite or |g_j| > 1024 components, are
// evaluated entirely in exact FP64 by k_exact_lists.
//
// MODE_REFINE (dense score_and_refine over many UBIs): every candidate below
// hi_max is evaluated exactly in FP64 and accepted pairs accumulate the
// reference's normal equations (R = sum ih g^T, H = sum ih ih^T, n, sum s) in
// FP64, per CTA and UBI, into scratch; k_refine_finish sums the CTA partials
// of each UBI in a fixed order and applies the reference's update.
#include <float.h>
#include <stdio.h>
#include <stdlib.h>

#include "common.cuh"
#include "tma.cuh"

namespace id11b {

constexpr int kBT = 256;            // threads per CTA
// UBIs held per thread by the screening kernel (even: screened in packed
// pairs).  The default; id11b_dev_score_batch_tiled also offers 2.
#ifndef ID11B_SCORE_UBIS_PER_THREAD
#define ID11B_SCORE_UBIS_PER_THREAD 4
#endif
constexpr int kScoreR = ID11B_SCORE_UBIS_PER_THREAD;
// g-vectors per unrolled step of the screening loop (20,000 UBIs x 1.1M g on
// B200, autotuned tiles: 17.97 / 17.33 / 16.86-17.03 / 27.6 ms at 1 / 2 / 4 / 8)
#ifndef ID11B_SCORE_UNROLL
#define ID11B_SCORE_UNROLL 4
#endif
constexpr int kScoreUnroll = ID11B_SCORE_UNROLL;
// counts-only screening with register counters where a CTA's g range allows
// (20,000 UBIs x 1.1M g on B200: 16.4 ms against 16.9 ms with shared counters)
#ifndef ID11B_SCORE_REGCOUNT
#define ID11B_SCORE_REGCOUNT 1
#endif
// resident CTAs per SM the screening kernel is compiled for (register budget)
__host__ __device__ constexpr int score_ctas_per_sm(int r) { return r <= 2 ? 4 : r <= 4 ? 3 : 2; }
constexpr int kTile = 1024;         // g per TMA tile (16 KB of float4)
constexpr float kGLimit = 1024.f;   // larger |g_j| -> exact FP64 only
constexpr double kEps32 = 5.9604644775390625e-08;  // 2^-24
constexpr double kSGLimit = 16384.0;  // S * gmax above this -> exact FP64 only
constexpr double kTolLimit = 0.45;    // tolerances at or above -> exact FP64 only

enum { MODE_SCORE = 0, MODE_REFINE = 1 };

struct GvecInfo {
    unsigned int gmax_bits;  // max |g_j| over regular g, float bits (rounded up)
    int nspecial;            // g-vectors evaluated in FP64 only
    int pad[2];
};

struct UbiInfo {
    unsigned int smax_bits;        // max row sum |u_i.| over FP32-path UBIs
    int nfallback;                 // UBIs evaluated in FP64 only
    unsigned long long nrecheck;   // pairs re-evaluated in FP64
    int error;                     // ID11B_ERR_TIMEOUT if a bounded wait gave up
    int pad[3];
};

struct Tols {
    double t[ID11B_MAX_TOLS];
    double fix;  // fixed-point scale of the sums (fixsum_scale)
};

struct LsqAcc {  // one UBI's normal-equation sums (same layout as the single-call path)
    double r[9];
    double h[6];
    double ss;
    long long n;
};

__device__ __forceinline__ unsigned int fbits(float x) { return __float_as_uint(x); }

// ------------------------------------------------------------ preparation --
__global__ void __launch_bounds__(kBT)
k_prepare_gvecs(const double* __restrict__ gv, int64_t n, float4* __restrict__ g4,
                GvecInfo* __restrict__ info, int* __restrict__ special) {
    float gm = 0.f;
    for (int64_t k = (int64_t)blockIdx.x * kBT + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * kBT) {
        double a = gv[3 * k], b = gv[3 * k + 1], c = gv[3 * k + 2];
        double m = fmax(fabs(a), fmax(fabs(b), fabs(c)));
        bool reg = isfinite(a) && isfinite(b) && isfinite(c) && m <= (double)kGLimit;
        if (reg) {
            g4[k] = make_float4(__double2float_rn(a), __double2float_rn(b),
                                __double2float_rn(c), 0.f);
            gm = fmaxf(gm, __double2float_ru(m));
        } else {
            g4[k] = make_float4(__int_as_float(0x7fc00000), __int_as_float(0x7fc00000),
                                __int_as_float(0x7fc00000), 0.f);
            int slot = atomicAdd(&info->nspecial, 1);
            special[slot] = (int)k;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) gm = fmaxf(gm, __shfl_xor_sync(0xffffffffu, gm, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&info->gmax_bits, fbits(gm));
}

__global__ void __launch_bounds__(kBT)
k_prepare_ubis(const double* __restrict__ ubis, int64_t m, const GvecInfo* __restrict__ gi,
               UbiInfo* __restrict__ ui, float4* __restrict__ packs, int* __restrict__ fallback,
               int force_fallback) {
    const double gmax = (double)__uint_as_float(gi->gmax_bits);
    float sm = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * kBT + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * kBT) {
        double u[9];
        bool fin = true;
#pragma unroll
        for (int e = 0; e < 9; e++) {
            u[e] = ubis[9 * i + e];
            fin = fin && isfinite(u[e]);
        }
        double s = 0.;
#pragma unroll
        for (int r = 0; r < 3; r++)
            s = fmax(s, fabs(u[3 * r]) + fabs(u[3 * r + 1]) + fabs(u[3 * r + 2]));
        s = s * (1. + 1e-15);
        bool fb = force_fallback || !fin || s * gmax >= kSGLimit;
        float4* p = packs + 3 * i;
        if (fb) {
            float nan = __int_as_float(0x7fc00000);
            p[0] = p[1] = p[2] = make_float4(nan, nan, nan, nan);
            int slot = atomicAdd(&ui->nfallback, 1);
            fallback[slot] = (int)i;
        } else {
            p[0] = make_float4(__double2float_rn(u[0]), __double2float_rn(u[1]),
                               __double2float_rn(u[2]), __double2float_rn(u[3]));
            p[1] = make_float4(__double2float_rn(u[4]), __double2float_rn(u[5]),
                               __double2float_rn(u[6]), __double2float_rn(u[7]));
            p[2] = make_float4(__double2float_rn(u[8]), 0.f, 0.f, 0.f);
            sm = fmaxf(sm, __double2float_ru(s));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sm = fmaxf(sm, __shfl_xor_sync(0xffffffffu, sm, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&ui->smax_bits, fbits(sm));
}

// Thresholds shared by every UBI of a launch (uniform: computed from gmax and
// smax, identical in every thread).
template <int NT>
struct Band {
    float lo[NT], hi[NT];
    float hmax;
};

template <int NT>
__device__ __forceinline__ Band<NT> make_band(const Tols& tols, const GvecInfo* gi,
                                              const UbiInfo* ui) {
    Band<NT> b;
    const double gmax = (double)__uint_as_float(gi->gmax_bits);
    const double smax = (double)__uint_as_float(ui->smax_bits);
    const double E = 6.0 * kEps32 * smax * gmax;
    b.hmax = 0.f;
#pragma unroll
    for (int j = 0; j < NT; j++) {
        double t = tols.t[j];
        double T = t * t;
        double band = 1.25 * (3.0 * E * (2.0 * (t + 1e-3) + E) + 4.0 * kEps32 * (T + 0.01));
        b.lo[j] = __double2float_rd(T - band);
        b.hi[j] = __double2float_ru(T + band);
        b.hmax = fmaxf(b.hmax, b.hi[j]);
    }
    return b;
}

__device__ __forceinline__ float drlv2_f32(const float u[9], float4 g, float ih[3]) {
    const float M = 12582912.0f;  // 1.5 * 2^23: x + M - M rounds |x| < 2^22 to nearest even
    float h0 = fmaf(u[2], g.z, fmaf(u[1], g.y, u[0] * g.x));
    float h1 = fmaf(u[5], g.z, fmaf(u[4], g.y, u[3] * g.x));
    float h2 = fmaf(u[8], g.z, fmaf(u[7], g.y, u[6] * g.x));
    ih[0] = __fsub_rn(__fadd_rn(h0, M), M);
    ih[1] = __fsub_rn(__fadd_rn(h1, M), M);
    ih[2] = __fsub_rn(__fadd_rn(h2, M), M);
    float t0 = h0 - ih[0], t1 = h1 - ih[1], t2 = h2 - ih[2];
    return fmaf(t2, t2, fmaf(t1, t1, t0 * t0));
}

// Two UBIs at once with packed FP32x2 arithmetic (sm_100: add/sub/mul/fma
// .f32x2).  B200's FP32 pipe does no more lane-operations per cycle with the
// packed forms, but each instruction issues two of them, which frees issue
// slots for the loads, compares and loop control that otherwise compete with
// the FMA pipe.  Every lane performs exactly the scalar drlv2_f32 operations
// (same order, round-to-nearest), so the screening values are bit-identical.
__device__ __forceinline__ uint64_t pk2(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk2(uint64_t v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// drlv2_f32 for the UBI pair packed in up[9] against one g (gx, gy, gz each
// duplicated into both halves); returns both drlv2 values packed.
__device__ __forceinline__ uint64_t drlv2_pair(const uint64_t up[9], uint64_t gx, uint64_t gy,
                                               uint64_t gz) {
    const uint64_t M2 = 0x4B4000004B400000ull;  // (1.5 * 2^23, 1.5 * 2^23)
    const uint64_t h0 = fma2(up[2], gz, fma2(up[1], gy, mul2(up[0], gx)));
    const uint64_t h1 = fma2(up[5], gz, fma2(up[4], gy, mul2(up[3], gx)));
    const uint64_t h2 = fma2(up[8], gz, fma2(up[7], gy, mul2(up[6], gx)));
    const uint64_t t0 = sub2(h0, sub2(add2(h0, M2), M2));
    const uint64_t t1 = sub2(h1, sub2(add2(h1, M2), M2));
    const uint64_t t2 = sub2(h2, sub2(add2(h2, M2), M2));
    return fma2(t2, t2, fma2(t1, t1, mul2(t0, t0)));
}

// ------------------------------------------------------------ main kernel --
// SUMS = false (MODE_SCORE without a sums output): the rare path counts only
// and the float sums are not even allocated.  REGC (with SUMS = false, when a
// CTA's g range is below 65,536): the counts live in registers, two 16-bit
// counters per 32-bit register, instead of shared memory.
template <int R, int NT, int MODE, bool SUMS = true, bool REGC = false>
__global__ void __launch_bounds__(kBT, MODE == MODE_SCORE ? score_ctas_per_sm(R) : 2)
k_batch(const float4* __restrict__ packs, int64_t m, const float4* __restrict__ g4,
        const double* __restrict__ gv, const double* __restrict__ ubis, int64_t n, int gsplit,
        Tols tols, const GvecInfo* __restrict__ gi, UbiInfo* __restrict__ ui,
        int* __restrict__ counts, double* __restrict__ sums, LsqAcc* __restrict__ part) {
    __shared__ __align__(128) float4 s_g[2][kTile];
    __shared__ __align__(8) uint64_t s_bar[2];
    extern __shared__ double s_acc[];  // MODE_REFINE: [17][kBT*R]

    const int tid = threadIdx.x;
    const int64_t ub = blockIdx.x / gsplit;
    const int gs = blockIdx.x % gsplit;
    const int64_t per = (((n + gsplit - 1) / gsplit) + 3) & ~(int64_t)3;
    const int64_t k0 = min(n, gs * per), k1 = min(n, k0 + per);
    const int ntiles = (int)((k1 - k0 + kTile - 1) / kTile);

    const Band<NT> band = make_band<NT>(tols, gi, ui);

    static_assert(R % 2 == 0, "UBIs are screened in packed pairs");
    uint64_t up[R / 2][9];  // UBI pairs (2p, 2p+1), element-wise packed
    int64_t mi[R];
#pragma unroll
    for (int p = 0; p < R / 2; p++) {
        float u[2][9];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int r = 2 * p + h;
            mi[r] = ub * (kBT * R) + r * kBT + tid;
            if (mi[r] < m) {
                float4 a = packs[3 * mi[r]], b = packs[3 * mi[r] + 1], c = packs[3 * mi[r] + 2];
                u[h][0] = a.x; u[h][1] = a.y; u[h][2] = a.z; u[h][3] = a.w;
                u[h][4] = b.x; u[h][5] = b.y; u[h][6] = b.z; u[h][7] = b.w; u[h][8] = c.x;
            } else {
#pragma unroll
                for (int e = 0; e < 9; e++) u[h][e] = __int_as_float(0x7fc00000);
            }
        }
#pragma unroll
        for (int e = 0; e < 9; e++) up[p][e] = pk2(u[0][e], u[1][e]);
    }
    // rare-path accumulators in shared memory, [field][kBT*R] so that lanes hit
    // consecutive words: MODE_SCORE int counts [NT] + float sums [NT]
    int* s_cnt = reinterpret_cast<int*>(s_acc);
    float* s_sum = reinterpret_cast<float*>(s_cnt + NT * kBT * R);
    static_assert(!REGC || (MODE == MODE_SCORE && !SUMS), "register counts: counts only");
    unsigned pc[R][(NT + 1) / 2];
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
        for (int q = 0; q < (NT + 1) / 2; q++) pc[r][q] = 0u;
    if (MODE == MODE_SCORE && !REGC) {
        for (int j = 0; j < NT; j++)
#pragma unroll
            for (int r = 0; r < R; r++) {
                s_cnt[j * (kBT * R) + r * kBT + tid] = 0;
                if (SUMS) s_sum[j * (kBT * R) + r * kBT + tid] = 0.f;  // absent otherwise
            }
    } else if (MODE == MODE_REFINE) {  // (REGC allocates no shared accumulators at all)
        for (int f = 0; f < 17; f++)
#pragma unroll
            for (int r = 0; r < R; r++) s_acc[f * (kBT * R) + r * kBT + tid] = 0.;
    }

    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        for (int t = 0; t < 2 && t < ntiles; t++) {
            int64_t a = k0 + (int64_t)t * kTile;
            uint32_t bytes = (uint32_t)(min((int64_t)kTile, k1 - a) * 16);
            mbar_arrive_expect_tx(&s_bar[t], bytes);
            tma_load_1d(s_g[t], g4 + a, bytes, &s_bar[t]);
        }
    }

    int failed_tile = -1;
    for (int t = 0; t < ntiles; t++) {
        const int buf = t & 1;
        const uint32_t parity = (t >> 1) & 1;
        // every thread waits; the CTA leaves together if any wait gave up
        if (!__syncthreads_and(mbar_wait_bounded(&s_bar[buf], parity))) {
            failed_tile = t;
            break;
        }
        const int64_t a = k0 + (int64_t)t * kTile;
        const int cntg = (int)min((int64_t)kTile, k1 - a);
#pragma unroll kScoreUnroll
        for (int k = 0; k < cntg; k++) {
            const float4 g = s_g[buf][k];
            const uint64_t gx = pk2(g.x, g.x), gy = pk2(g.y, g.y), gz = pk2(g.z, g.z);
            float s[R];
            bool any = false;
#pragma unroll
            for (int p = 0; p < R / 2; p++) {
                upk2(drlv2_pair(up[p], gx, gy, gz), s[2 * p], s[2 * p + 1]);
                any |= (s[2 * p] < band.hmax) | (s[2 * p + 1] < band.hmax);
            }
            if (any) {
#pragma unroll
                for (int r = 0; r < R; r++) {
                    if (!(s[r] < band.hmax)) continue;
                    const int64_t gk = a + k;
                    if (MODE == MODE_SCORE) {
#pragma unroll
                        for (int j = 0; j < NT; j++) {
                            const int slot = j * (kBT * R) + r * kBT + tid;
                            if (s[r] < band.lo[j]) {
                                if (REGC) {
                                    pc[r][j >> 1] += 1u << ((j & 1) * 16);
                                } else {
                                    s_cnt[slot]++;
                                    if (SUMS) s_sum[slot] += s[r];
                                }
                            } else if (s[r] < band.hi[j]) {
                                double uu[9], ihd[3];
#pragma unroll
                                for (int e = 0; e < 9; e++) uu[e] = ubis[9 * mi[r] + e];
                                double s64 = drlv2_exact(uu, gv[3 * gk], gv[3 * gk + 1],
                                                         gv[3 * gk + 2], ihd);
                                atomicAdd(&ui->nrecheck, 1ull);
                                if (s64 < tols.t[j] * tols.t[j]) {
                                    if (REGC) {
                                        pc[r][j >> 1] += 1u << ((j & 1) * 16);
                                    } else {
                                        s_cnt[slot]++;
                                        if (SUMS) s_sum[slot] += (float)s64;
                                    }
                                }
                            }
                        }
                    } else {
                        double uu[9], ihd[3];
#pragma unroll
                        for (int e = 0; e < 9; e++) uu[e] = ubis[9 * mi[r] + e];
                        const double g0 = gv[3 * gk], g1 = gv[3 * gk + 1], g2 = gv[3 * gk + 2];
                        double s64 = drlv2_exact(uu, g0, g1, g2, ihd);
                        atomicAdd(&ui->nrecheck, 1ull);
                        if (s64 < tols.t[0] * tols.t[0]) {
                            double* acc = s_acc + r * kBT + tid;
                            const int st = kBT * R;
                            const double gg[3] = {g0, g1, g2};
#pragma unroll
                            for (int i = 0; i < 3; i++)
#pragma unroll
                                for (int jj = 0; jj < 3; jj++)
                                    acc[(3 * i + jj) * st] =
                                        dadd(acc[(3 * i + jj) * st], dmul(ihd[jj], gg[i]));
                            acc[9 * st] = dadd(acc[9 * st], dmul(ihd[0], ihd[0]));
                            acc[10 * st] = dadd(acc[10 * st], dmul(ihd[1], ihd[0]));
                            acc[11 * st] = dadd(acc[11 * st], dmul(ihd[2], ihd[0]));
                            acc[12 * st] = dadd(acc[12 * st], dmul(ihd[1], ihd[1]));
                            acc[13 * st] = dadd(acc[13 * st], dmul(ihd[2], ihd[1]));
                            acc[14 * st] = dadd(acc[14 * st], dmul(ihd[2], ihd[2]));
                            acc[15 * st] = dadd(acc[15 * st], s64);
                            acc[16 * st] += 1.0;
                        }
                    }
                }
            }
        }
        __syncthreads();  // every lane is done with s_g[buf]
        if (tid == 0 && t + 2 < ntiles) {
            fence_proxy_async_smem();
            int64_t a2 = k0 + (int64_t)(t + 2) * kTile;
            uint32_t bytes = (uint32_t)(min((int64_t)kTile, k1 - a2) * 16);
            mbar_arrive_expect_tx(&s_bar[buf], bytes);
            tma_load_1d(s_g[buf], g4 + a2, bytes, &s_bar[buf]);
        }
    }
    if (failed_tile >= 0) {
        // A wait gave up: record it, then wait (bounded) for the copies this
        // CTA still has in flight (tiles failed_tile and failed_tile + 1)
        // before its shared memory goes away.
        if (tid == 0) {
            atomicExch(&ui->error, (int)ID11B_ERR_TIMEOUT);
            for (int t = failed_tile; t < failed_tile + 2 && t < ntiles; t++)
                mbar_wait_bounded(&s_bar[t & 1], (t >> 1) & 1, 1u << 16);
        }
        return;
    }

    if (REGC) {
#pragma unroll
        for (int r = 0; r < R; r++) {
            if (mi[r] >= m) continue;
#pragma unroll
            for (int j = 0; j < NT; j++) {
                const int c = (int)((pc[r][j >> 1] >> ((j & 1) * 16)) & 0xffffu);
                if (c) atomicAdd(counts + mi[r] * NT + j, c);
            }
        }
    } else if (MODE == MODE_SCORE) {
#pragma unroll
        for (int r = 0; r < R; r++) {
            if (mi[r] >= m) continue;
#pragma unroll
            for (int j = 0; j < NT; j++) {
                const int slot = j * (kBT * R) + r * kBT + tid;
                if (s_cnt[slot]) {
                    atomicAdd(counts + mi[r] * NT + j, s_cnt[slot]);
                    if (SUMS && sums) fixsum_add(sums + mi[r] * NT + j, (double)s_sum[slot], tols.fix);
                }
            }
        }
    } else {
#pragma unroll
        for (int r = 0; r < R; r++) {
            if (mi[r] >= m) continue;
            LsqAcc* p = part + (int64_t)gs * m + mi[r];
            const double* acc = s_acc + r * kBT + tid;
            const int st = kBT * R;
#pragma unroll
            for (int i = 0; i < 9; i++) p->r[i] = acc[i * st];
#pragma unroll
            for (int i = 0; i < 6; i++) p->h[i] = acc[(9 + i) * st];
            p->ss = acc[15 * st];
            p->n = (long long)acc[16 * st];
        }
    }
}

// ------------------------------------------- exact FP64 for the lists ------
// Items: (fallback UBI x every g) then (every non-fallback UBI x special g).
template <int MODE>
__global__ void __launch_bounds__(kBT)
k_exact_lists(const double* __restrict__ ubis, int64_t m, const double* __restrict__ gv,
              int64_t n, const GvecInfo* __restrict__ gi, const UbiInfo* __restrict__ ui,
              const int* __restrict__ special, const int* __restrict__ fallback,
              const float4* __restrict__ packs, Tols tols, int ntol, int* __restrict__ counts,
              double* __restrict__ sums, LsqAcc* __restrict__ extra) {
    const int64_t nf = ui->nfallback, ns = gi->nspecial;
    const int64_t items = nf * n + m * ns;
    for (int64_t it = (int64_t)blockIdx.x * kBT + threadIdx.x; it < items;
         it += (int64_t)gridDim.x * kBT) {
        int64_t ui_idx, k;
        if (it < nf * n) {
            ui_idx = fallback[it / n];
            k = it % n;
        } else {
            // every UBI x special g; fallback UBIs (NaN packs) were covered above
            int64_t q = it - nf * n;
            ui_idx = q / ns;
            k = special[q % ns];
            if (isnan(packs[3 * ui_idx].x)) continue;  // already covered as a fallback UBI
        }
        double uu[9], ih[3];
#pragma unroll
        for (int e = 0; e < 9; e++) uu[e] = ubis[9 * ui_idx + e];
        const double g0 = gv[3 * k], g1 = gv[3 * k + 1], g2 = gv[3 * k + 2];
        double s = drlv2_exact(uu, g0, g1, g2, ih);
        if (MODE == MODE_SCORE) {
            for (int j = 0; j < ntol; j++)
                if (s < tols.t[j] * tols.t[j]) {
                    atomicAdd(counts + ui_idx * ntol + j, 1);
                    if (sums) fixsum_add(sums + ui_idx * ntol + j, s, tols.fix);
                }
        } else if (s < tols.t[0] * tols.t[0]) {
            LsqAcc* p = extra + ui_idx;
            const double gg[3] = {g0, g1, g2};
            for (int i = 0; i < 3; i++)
                for (int jj = 0; jj < 3; jj++) atomicAdd(&p->r[3 * i + jj], dmul(ih[jj], gg[i]));
            atomicAdd(&p->h[0], dmul(ih[0], ih[0]));
            atomicAdd(&p->h[1], dmul(ih[1], ih[0]));
            atomicAdd(&p->h[2], dmul(ih[2], ih[0]));
            atomicAdd(&p->h[3], dmul(ih[1], ih[1]));
            atomicAdd(&p->h[4], dmul(ih[2], ih[1]));
            atomicAdd(&p->h[5], dmul(ih[2], ih[2]));
            atomicAdd(&p->ss, s);
            atomicAdd((unsigned long long*)&p->n, 1ull);
        }
    }
}

// ------------------------------------------------- refinement finishing ----
// One thread per UBI: sum the gsplit CTA partials (+ the exact-list slot) in
// a fixed order, apply the reference's update, record n and mean drlv2.
__global__ void __launch_bounds__(kBT)
k_refine_finish(const LsqAcc* __restrict__ part, int gsplit, int64_t m, double* __restrict__ ubis,
                int* __restrict__ npk, double* __restrict__ mean) {
    const int64_t i = (int64_t)blockIdx.x * kBT + threadIdx.x;
    if (i >= m) return;
    double t[15], ss = 0.;
    long long n = 0;
    for (int f = 0; f < 15; f++) t[f] = 0.;
    for (int g = 0; g <= gsplit; g++) {  // slot gsplit holds the exact-list sums
        const LsqAcc& p = part[(int64_t)g * m + i];
        for (int f = 0; f < 9; f++) t[f] += p.r[f];
        for (int f = 0; f < 6; f++) t[9 + f] += p.h[f];
        ss += p.ss;
        n += p.n;
    }
    double R[9], H[9], u[9];
    for (int f = 0; f < 9; f++) R[f] = t[f];
    H[0] = t[9];  H[1] = t[10]; H[2] = t[11];
    H[3] = t[10]; H[4] = t[12]; H[5] = t[13];
    H[6] = t[11]; H[7] = t[13]; H[8] = t[14];
    for (int f = 0; f < 9; f++) u[f] = ubis[9 * i + f];
    lsq_update_exact(R, H, u);
    for (int f = 0; f < 9; f++) ubis[9 * i + f] = u[f];
    if (npk) npk[i] = (int)n;
    if (mean) mean[i] = n > 0 ? ddiv(ss, (double)n) : 0.;
}

// ------------------------------------------------------------------ host ----
static int num_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct UbiWs {  // layout of the per-call workspace
    UbiInfo* info;
    int* fallback;
    float4* packs;
    LsqAcc* part;
    size_t bytes;
};

// g ranges per block of UBIs: about sixteen waves of CTAs (short CTAs balance
// the tail; 20,000 UBIs x 1.1M g on B200: 17.8 ms vs 19.3 ms at four waves),
// at least one g tile each
static int choose_gsplit(int64_t m, int64_t n, int mode, int r) {
    const int per_cta = kBT * r;
    int64_t ublocks = (m + per_cta - 1) / per_cta;
    int64_t target = (int64_t)num_sms() * (mode == MODE_SCORE ? score_ctas_per_sm(r) : 2) *
                     (mode == MODE_SCORE ? 16 : 4);
    int64_t gs = (target + ublocks - 1) / ublocks;
    int64_t maxgs = (n + kTile - 1) / kTile;  // at least one tile per CTA
    if (gs > maxgs) gs = maxgs;
    if (gs < 1) gs = 1;
    return (int)gs;
}

static UbiWs ubi_ws_layout(void* base, int64_t m, int64_t n, int mode) {
    UbiWs w;
    size_t off = 0;
    char* b = (char*)base;
    w.info = (UbiInfo*)(b + off);
    off = align256(off + sizeof(UbiInfo));
    w.fallback = (int*)(b + off);
    off = align256(off + sizeof(int) * (size_t)(m > 0 ? m : 1));
    w.packs = (float4*)(b + off);
    off = align256(off + sizeof(float4) * 3 * (size_t)(m > 0 ? m : 1));
    w.part = (LsqAcc*)(b + off);
    if (mode == MODE_REFINE) {
        int gs = choose_gsplit(m, n, mode, 2);
        off = align256(off + sizeof(LsqAcc) * (size_t)(gs + 1) * (size_t)(m > 0 ? m : 1));
    }
    w.bytes = off;
    return w;
}

template <int R, int NT, int MODE, bool SUMS = true, bool REGC = false>
static void launch_batch(int64_t m, int64_t n, int gsplit, const float4* packs, const float4* g4,
                         const double* gv, const double* ubis, const Tols& tols,
                         const GvecInfo* gi, UbiInfo* ui, int* counts, double* sums,
                         LsqAcc* part, cudaStream_t st) {
    static_assert(MODE == MODE_SCORE || R == 2, "refinement keeps two UBIs per thread");
    const int64_t ublocks = (m + kBT * R - 1) / (kBT * R);
    size_t dyn = MODE == MODE_REFINE ? sizeof(double) * 17 * kBT * R
                 : REGC ? 0
                        : (sizeof(int) + (SUMS ? sizeof(float) : 0)) * NT * kBT * R;
    auto kern = k_batch<R, NT, MODE, SUMS, REGC>;
    // static (32 KB of tiles) + dynamic exceeds the 48 KB default: opt in once
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)dyn);
        if (getenv("ID11B_DEBUG"))
            fprintf(stderr, "id11b: set max dynamic smem %zu -> %s\n", dyn, cudaGetErrorString(e));
        attr_set = true;
    }
    if (getenv("ID11B_DEBUG")) {
        cudaFuncAttributes fa;
        cudaError_t e = cudaFuncGetAttributes(&fa, kern);
        fprintf(stderr,
                "id11b: k_batch<%d,%d,%d> grid %lld x %d dyn %zu | attr %s: static %zu maxdyn %d "
                "regs %d maxthreads %d\n",
                R, NT, MODE, (long long)(ublocks * gsplit), kBT, dyn, cudaGetErrorString(e),
                fa.sharedSizeBytes, fa.maxDynamicSharedSizeBytes, fa.numRegs,
                fa.maxThreadsPerBlock);
    }
    kern<<<(unsigned)(ublocks * gsplit), kBT, dyn, st>>>(packs, m, g4, gv, ubis, n, gsplit, tols,
                                                         gi, ui, counts, sums, part);
}

}  // namespace id11b

using namespace id11b;

extern "C" int64_t id11b_gvec_workspace_bytes(int64_t n) {
    return (int64_t)(align256(sizeof(GvecInfo)) + align256(sizeof(int) * (size_t)(n > 0 ? n : 1)));
}

extern "C" int id11b_dev_prepare_gvecs(const double* gv, int64_t n, float* g4, void* gws,
                                       int64_t gws_bytes, void* stream) {
    if (n < 0 || !g4 || !gws || (n > 0 && !gv)) return ID11B_ERR_ARG;
    if (((uintptr_t)g4 & 15) || ((uintptr_t)gws & 255)) return ID11B_ERR_ALIGN;
    if (n > INT32_MAX) return ID11B_ERR_SIZE;
    if (gws_bytes < id11b_gvec_workspace_bytes(n)) return ID11B_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    GvecInfo* gi = (GvecInfo*)gws;
    int* special = (int*)((char*)gws + align256(sizeof(GvecInfo)));
    ID11B_CHECK(cudaMemsetAsync(gi, 0, sizeof(GvecInfo), st));
    if (n == 0) return ID11B_OK;
    int64_t blocks = (n + kBT - 1) / kBT;
    if (blocks > (int64_t)num_sms() * 8) blocks = (int64_t)num_sms() * 8;
    k_prepare_gvecs<<<(unsigned)blocks, kBT, 0, st>>>(gv, n, (float4*)g4, gi, special);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int64_t id11b_batch_workspace_bytes(int64_t m, int64_t n, int refine) {
    return (int64_t)ubi_ws_layout(nullptr, m, n, refine ? MODE_REFINE : MODE_SCORE).bytes;
}

static int check_tols(const double* tols, int ntol, Tols& T) {
    if (!tols || ntol < 1 || ntol > ID11B_MAX_TOLS) return ID11B_ERR_ARG;
    for (int j = 0; j < ID11B_MAX_TOLS; j++) T.t[j] = j < ntol ? tols[j] : 0.;
    T.fix = 0.;  // set where sums are accumulated
    for (int j = 0; j < ntol; j++)
        if (!(tols[j] >= 0.)) return ID11B_ERR_ARG;
    return ID11B_OK;
}

static int prepare_ubis(const double* ubis, int64_t m, const void* gws, UbiWs& w, bool force,
                        cudaStream_t st) {
    ID11B_CHECK(cudaMemsetAsync(w.info, 0, sizeof(UbiInfo), st));
    if (m == 0) return ID11B_OK;
    int64_t blocks = (m + kBT - 1) / kBT;
    if (blocks > (int64_t)num_sms() * 8) blocks = (int64_t)num_sms() * 8;
    k_prepare_ubis<<<(unsigned)blocks, kBT, 0, st>>>(ubis, m, (const GvecInfo*)gws, w.info,
                                                     w.packs, w.fallback, force ? 1 : 0);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

static int exact_lists(int mode, const double* ubis, int64_t m, const double* gv, int64_t n,
                       const void* gws, const UbiWs& w, const Tols& T, int ntol, int* counts,
                       double* sums, LsqAcc* extra, cudaStream_t st) {
    const GvecInfo* gi = (const GvecInfo*)gws;
    const int* special = (const int*)((const char*)gws + align256(sizeof(GvecInfo)));
    unsigned blocks = (unsigned)num_sms() * 4;
    if (mode == MODE_SCORE)
        k_exact_lists<MODE_SCORE><<<blocks, kBT, 0, st>>>(ubis, m, gv, n, gi, w.info, special,
                                                          w.fallback, w.packs, T, ntol, counts,
                                                          sums, extra);
    else
        k_exact_lists<MODE_REFINE><<<blocks, kBT, 0, st>>>(ubis, m, gv, n, gi, w.info, special,
                                                           w.fallback, w.packs, T, ntol, counts,
                                                           sums, extra);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

template <int R>
static void launch_score(int ntol, int64_t m, int64_t n, int gsplit, const UbiWs& w,
                         const float4* g4, const double* gv, const double* ubis, const Tols& T,
                         const GvecInfo* gi, int* counts, double* sums, cudaStream_t st) {
    if (sums) {
        switch (ntol) {
            case 1: launch_batch<R, 1, MODE_SCORE, true>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, sums, nullptr, st); break;
            case 2: launch_batch<R, 2, MODE_SCORE, true>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, sums, nullptr, st); break;
            case 3: launch_batch<R, 3, MODE_SCORE, true>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, sums, nullptr, st); break;
            default: launch_batch<R, 4, MODE_SCORE, true>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, sums, nullptr, st); break;
        }
    } else if (ID11B_SCORE_REGCOUNT && ((((n + gsplit - 1) / gsplit) + 3) & ~(int64_t)3) < 65536) {
        switch (ntol) {  // a CTA counts below 65,536 g: 16-bit register counters suffice
            case 1: launch_batch<R, 1, MODE_SCORE, false, true>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, nullptr, nullptr, st); break;
            case 2: launch_batch<R, 2, MODE_SCORE, false, true>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, nullptr, nullptr, st); break;
            case 3: launch_batch<R, 3, MODE_SCORE, false, true>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, nullptr, nullptr, st); break;
            default: launch_batch<R, 4, MODE_SCORE, false, true>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, nullptr, nullptr, st); break;
        }
    } else {
        switch (ntol) {
            case 1: launch_batch<R, 1, MODE_SCORE, false>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, nullptr, nullptr, st); break;
            case 2: launch_batch<R, 2, MODE_SCORE, false>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, nullptr, nullptr, st); break;
            case 3: launch_batch<R, 3, MODE_SCORE, false>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, nullptr, nullptr, st); break;
            default: launch_batch<R, 4, MODE_SCORE, false>(m, n, gsplit, w.packs, g4, gv, ubis, T, gi, w.info, counts, nullptr, nullptr, st); break;
        }
    }
}

extern "C" int id11b_score_tile_default(int64_t m, int64_t n, int* ubis_per_thread, int* gsplit) {
    if (m < 0 || n < 0 || !ubis_per_thread || !gsplit) return ID11B_ERR_ARG;
    *ubis_per_thread = kScoreR;
    *gsplit = choose_gsplit(m, n, MODE_SCORE, kScoreR);
    return ID11B_OK;
}

extern "C" int id11b_dev_score_batch_tiled(const double* ubis, int64_t m, const double* gv,
                                           const float* g4, int64_t n, const void* gws,
                                           const double* tols_host, int ntol, int32_t* counts,
                                           double* sums, int ubis_per_thread, int gsplit,
                                           void* ws, int64_t ws_bytes, void* stream) {
    Tols T;
    int rc = check_tols(tols_host, ntol, T);
    if (rc) return rc;
    if (m < 0 || n < 0 || !ws || !gws || (m > 0 && (!ubis || !counts)) ||
        (n > 0 && (!gv || !g4)))
        return ID11B_ERR_ARG;
    const int r = ubis_per_thread ? ubis_per_thread : kScoreR;
    if ((r != 2 && r != 4 && r != kScoreR) || gsplit < 0) return ID11B_ERR_ARG;
    if (((uintptr_t)g4 & 15) || ((uintptr_t)ws & 255) || ((uintptr_t)gws & 255))
        return ID11B_ERR_ALIGN;
    if (ws_bytes < id11b_batch_workspace_bytes(m, n, 0)) return ID11B_ERR_SIZE;
    if (n > INT32_MAX || m > INT32_MAX) return ID11B_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    UbiWs w = ubi_ws_layout(ws, m, n, MODE_SCORE);
    if (m > 0) ID11B_CHECK(cudaMemsetAsync(counts, 0, sizeof(int32_t) * (size_t)m * ntol, st));
    if (sums && m > 0) ID11B_CHECK(cudaMemsetAsync(sums, 0, sizeof(double) * (size_t)m * ntol, st));
    double tmax = 0.;
    for (int j = 0; j < ntol; j++) tmax = tols_host[j] > tmax ? tols_host[j] : tmax;
    T.fix = fixsum_scale(n, tmax);
    bool force = tmax >= kTolLimit;  // too close to the rounding half-point: all FP64
    rc = prepare_ubis(ubis, m, gws, w, force, st);
    if (rc) return rc;
    if (m == 0 || n == 0) return ID11B_OK;
    const GvecInfo* gi = (const GvecInfo*)gws;
    const int64_t maxgs = (n + kTile - 1) / kTile;  // every CTA streams at least one tile
    int gs = gsplit ? (int)(gsplit < maxgs ? gsplit : maxgs) : choose_gsplit(m, n, MODE_SCORE, r);
    if (r == 2)
        launch_score<2>(ntol, m, n, gs, w, (const float4*)g4, gv, ubis, T, gi, counts, sums, st);
    else if (r == 4)
        launch_score<4>(ntol, m, n, gs, w, (const float4*)g4, gv, ubis, T, gi, counts, sums, st);
#if ID11B_SCORE_UBIS_PER_THREAD != 2 && ID11B_SCORE_UBIS_PER_THREAD != 4
    else
        launch_score<kScoreR>(ntol, m, n, gs, w, (const float4*)g4, gv, ubis, T, gi, counts,
                              sums, st);
#endif
    ID11B_CHECK_LAUNCH();
    rc = exact_lists(MODE_SCORE, ubis, m, gv, n, gws, w, T, ntol, counts, sums, nullptr, st);
    if (rc) return rc;
    return id11b_fixsum_finish(sums, m * ntol, T.fix, st);
}

extern "C" int id11b_dev_score_batch(const double* ubis, int64_t m, const double* gv,
                                     const float* g4, int64_t n, const void* gws,
                                     const double* tols_host, int ntol, int32_t* counts,
                                     double* sums, void* ws, int64_t ws_bytes, void* stream) {
    return id11b_dev_score_batch_tiled(ubis, m, gv, g4, n, gws, tols_host, ntol, counts, sums, 0,
                                       0, ws, ws_bytes, stream);
}

extern "C" int id11b_dev_refine_batch(double* ubis, int64_t m, const double* gv, const float* g4,
                                      int64_t n, const void* gws, double tol, int iters,
                                      int32_t* npk, double* mean_drlv2, void* ws,
                                      int64_t ws_bytes, void* stream) {
    Tols T;
    int rc = check_tols(&tol, 1, T);
    if (rc) return rc;
    if (m < 0 || n < 0 || iters < 0 || !ws || !gws || (m > 0 && !ubis) ||
        (n > 0 && (!gv || !g4)))
        return ID11B_ERR_ARG;
    if (((uintptr_t)g4 & 15) || ((uintptr_t)ws & 255) || ((uintptr_t)gws & 255))
        return ID11B_ERR_ALIGN;
    if (ws_bytes < id11b_batch_workspace_bytes(m, n, 1)) return ID11B_ERR_SIZE;
    if (n > INT32_MAX || m > INT32_MAX) return ID11B_ERR_SIZE;
    if (m == 0) return ID11B_OK;
    cudaStream_t st = (cudaStream_t)stream;
    UbiWs w = ubi_ws_layout(ws, m, n, MODE_REFINE);
    const int gsplit = choose_gsplit(m, n, MODE_REFINE, 2);
    const GvecInfo* gi = (const GvecInfo*)gws;
    for (int it = 0; it < iters; it++) {
        rc = prepare_ubis(ubis, m, gws, w, tol >= kTolLimit, st);
        if (rc) return rc;
        // only the exact-list slot needs zeroing: every CTA writes its own slots
        ID11B_CHECK(cudaMemsetAsync(w.part + (int64_t)gsplit * m, 0, sizeof(LsqAcc) * m, st));
        if (n > 0) {
            launch_batch<2, 1, MODE_REFINE>(m, n, gsplit, w.packs, (const float4*)g4, gv, ubis, T,
                                         gi, w.info, nullptr, nullptr, w.part, st);
            ID11B_CHECK_LAUNCH();
            rc = exact_lists(MODE_REFINE, ubis, m, gv, n, gws, w, T, 1, nullptr, nullptr,
                             w.part + (int64_t)gsplit * m, st);
            if (rc) return rc;
        } else {
            ID11B_CHECK(cudaMemsetAsync(w.part, 0, sizeof(LsqAcc) * m * gsplit, st));
        }
        k_refine_finish<<<(unsigned)((m + kBT - 1) / kBT), kBT, 0, st>>>(
            w.part, gsplit, m, ubis, it == iters - 1 ? npk : nullptr,
            it == iters - 1 ? mean_drlv2 : nullptr);
        ID11B_CHECK_LAUNCH();
    }
    return ID11B_OK;
}

// Statistics and status of the last batch call that used workspace `ws`.
extern "C" int id11b_batch_stats(const void* ws, int64_t m, int64_t n, int refine,
                                 int64_t* nrecheck, int32_t* nfallback, int32_t* error,
                                 void* stream) {
    if (!ws) return ID11B_ERR_ARG;
    UbiWs w = ubi_ws_layout((void*)ws, m, n, refine ? MODE_REFINE : MODE_SCORE);
    UbiInfo h;
    cudaStream_t st = (cudaStream_t)stream;
    ID11B_CHECK(cudaMemcpyAsync(&h, w.info, sizeof(h), cudaMemcpyDeviceToHost, st));
    ID11B_CHECK(cudaStreamSynchronize(st));
    if (nrecheck) *nrecheck = (int64_t)h.nrecheck;
    if (nfallback) *nfallback = h.nfallback;
    if (error) *error = h.error;
    return h.error ? h.error : ID11B_OK;
}
