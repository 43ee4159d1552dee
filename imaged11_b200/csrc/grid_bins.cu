// Binned scoring through the reciprocal-space cell index: a spatial join of
// (UBI, hkl) boxes with the g-vectors.
//
// score() (ImageD11 src/closest.c:227-248) counts, for one UBI, the g with
// |UBI.g - round(UBI.g)|^2 < tol^2.  Such a g lies in the box
// [UB.hkl - w, UB.hkl + w] of its own hkl = round(UBI.g) (grid.cuh: the half
// widths w are conservative).  Here every box that can reach the data is
// enumerated once per UBI (the lookup scorer's enumeration, its per-candidate
// work in FP32 with the rounding folded into w) and the boxes are sorted by
// the row of grid cells holding their centre (fixed y and z cell): counts per
// block of 16 rows in shared memory per CTA, a scan, a second enumeration that
// writes each CTA's boxes of a block as one sequential stream, and a split of
// each block into its rows.  One CTA then takes one
// row: it sorts the row's boxes by x cell in shared memory, stages the
// g-vectors of the row's region (its y/z cell widened by the largest half
// width W, all x cells the boxes need) sorted by x cell, and every run of 32
// boxes (a warp, one box per lane) is tested against the contiguous range of
// staged g whose x cells its boxes can reach.  Each lane holds its box's UBI
// in FP32 registers, duplicated into packed pairs, and its hkl; two staged g
// are read by all lanes at once (broadcast) and tested with packed f32x2
// instructions.
//
// Per (box, g), the screening kernel's FP32 arithmetic (score_batch.cu), with
// the subtraction of hkl folded into the first FMA of each chain:
//   d = UBI32 . g32 - hkl (one FMA chain from -hkl),  s = d.d;
//   s < lo_j           -> counted for tolerance j,
//   lo_j <= s < hi_j   -> re-evaluated with the reference's exact FP64
//                         arithmetic, counted when drlv2 < tol_j^2 and the
//                         rounded h is the box's hkl,
//   s >= hi_j          -> not counted for j.
// The band [lo_j, hi_j) is the screening kernel's proven one with the folded
// chain's bound |d32 - d64| <= E = 2^-24 * S * (8 gmax + 3 W) (S = largest row
// sum of |UBI|; partial sums stay below |hkl| + S gmax <= S (2 gmax + W)).
// With every tolerance below 0.4 and S * gmax < 16384, a pair with s < hi_j
// has all |d| < 0.5 - E, and for s < lo_j the rounded h64
// is hkl and drlv2 < tol_j^2: the pair is counted under its own hkl exactly
// when the reference counts it.  A pair tested against a box of another hkl
// has some |d| >= 0.5 - E, so s >= 0.2 > hi_j: never counted.  A staged tile
// holds each g once, so no pair is tested twice in a tile, and every g of a
// row's region lies in exactly one tile.
//
// UBIs outside the limits (the lookup plan's caps, hkl beyond -256..255,
// S * gmax too large) are scored by an exact FP64 scan of every regular g, and
// the g-vectors outside the regular range by an exact FP64 scan of their list.
// Counts go to the output with integer atomics (exact); the optional sums of
// the counted drlv2 are added in fixed point (each term rounded to one step,
// then integer atomics), so they repeat bit for bit.
//
// The same pipeline serves the batched assignment (score_and_assign over many
// grains, k_assign's two passes in gvec_grid.cu): the join's AS modes send
// every pair the screen cannot exclude from tol^2 to the exact FP64 path and
// apply the assignment's atomic minima there.
#include <math.h>
#include <string.h>
#include <algorithm>
#include <vector>

#include "grid.cuh"

namespace id11b {
namespace grid {
namespace bins {

// warps per enumeration CTA, and CTAs per SM (ID11B_ENUM_MINB): every CTA
// writes one stream of box records per block, so fewer, larger CTAs mean fewer
// streams, each filling its L2 sectors sooner.  Binned scoring of 20,000 UBIs x
// 1.1M g: 2.96 ms at 8 warps x 3 CTAs (444 CTAs), 2.88 at 12 x 2, 2.87 at
// 16 x 1 (104 registers), 2.79 at 24 x 1 (80 registers).
#ifndef ID11B_ENUM_WARPS
#define ID11B_ENUM_WARPS 24
#endif
constexpr int kEW = ID11B_ENUM_WARPS;
constexpr int kET = 32 * kEW;
constexpr int kJT = 256;            // threads per join CTA (one row at a time)
constexpr int kJW = kJT / 32;
#ifndef ID11B_JOIN_FOLD
#define ID11B_JOIN_FOLD 1
#endif
#ifndef ID11B_JOIN_RANKED
#define ID11B_JOIN_RANKED 1
#endif
#ifndef ID11B_JOIN_BMAX
#define ID11B_JOIN_BMAX 4096
#endif
#ifndef ID11B_JOIN_GMAX
#define ID11B_JOIN_GMAX 1536
#endif
constexpr int kBMax = ID11B_JOIN_BMAX;  // boxes of a row sorted in shared memory at a time
constexpr int kGMax = ID11B_JOIN_GMAX;  // g staged at a time (one tile)
// rows per block: 2^ID11B_ROW_BITS (blocks of 32 rows halve the streams but
// were slower: 2.83 against 2.79 ms with 24-warp enumeration CTAs)
#ifndef ID11B_ROW_BITS
#define ID11B_ROW_BITS 4
#endif
constexpr int kRowBits = ID11B_ROW_BITS;
constexpr int kRowBlock = 1 << kRowBits;  // rows of cells per block of the enumeration's streams
constexpr int kMaxBlocks = 4096;    // blocks the enumeration's counters hold (nx^2 <= 65536)
constexpr int kMaxNxx = 8191;       // x cells per row (13-bit field of a box record)
constexpr int kMaxHalo = 1024;      // rows of cells around a row (the halo R: (2R+1)^2)
constexpr int kMaxEnumCtas = 512;
constexpr double kTolLimit = 0.4;
constexpr double kSGLimit = 16384.0;
constexpr double kEps32 = 5.9604644775390625e-08;  // 2^-24
constexpr int kHklOff = 256;        // hkl in 9-bit fields: -256 .. 255
// box record fields above the 13-bit x cell: the row within its block, l, k,
// h, then the UBI (within a range of UBIs) in what is left of the 64 bits
constexpr int kLShift = 13 + kRowBits, kKShift = kLShift + 9, kHShift = kKShift + 9,
              kUShift = kHShift + 9;
constexpr int kUbiBits = 64 - kUShift;
constexpr int kFallbackParts = 128; // warps per plainly scanned UBI
constexpr int kBT = 128;            // threads per CTA of the exact scans
constexpr int kBW = kBT / 32;
#ifndef ID11B_JOIN_MINB
#define ID11B_JOIN_MINB 3
#endif
constexpr int kJoinMinBlocks = ID11B_JOIN_MINB;  // resident join CTAs per SM compiled for

struct BinInfo {
    unsigned long long wmax_bits;  // largest (widened) box half width (positive doubles order as integers)
    unsigned long long total;      // boxes enumerated by the first counting pass
    unsigned int smax_bits;        // largest row sum of |UBI| over binned UBIs (float, rounded up)
    int nfallback;                 // UBIs scored by the plain scan
    int next_row;                  // row counter of the join
    int pad;
};

// Everything the join needs that is uniform over the launch, computed on the
// host after the counting pass (kernel parameters: no registers).
struct JoinParams {
    // thresholds in ascending order of tolerance; ord[j]: the caller's index
    // of the j-th (where its count and sum are written)
    float lo[ID11B_MAX_TOLS], hi[ID11B_MAX_TOLS];
    double t2[ID11B_MAX_TOLS];
    int ord[ID11B_MAX_TOLS];
    double fix;                    // fixed-point scale of the sums (fixsum_scale)
    float hmax;
    // y/z region of row (iy, iz): [rlo + iy * cs, rhi + (iy + 1) * cs] (the
    // cell widened by W + eps; eps covers the FP32 rounding of the box
    // centres' cells and of these bounds); the halo in whole cells
    float rlo, rhi, cs;
    int R, Rx, nx, nxx;
    int64_t i0;                    // first UBI of the range (box records are relative to it)
    // assignment (k_join's AS modes): sorted position -> g index, each g's
    // drlv2 on entry, the smallest drlv2 bits and the lowest grain reaching it
    const int* gidx;
    const double* d0;
    unsigned long long* best;
    int* lab;
};

// box record (64 bits): UBI (kUbiBits, relative to the range) | h + 256 (9) |
// k + 256 (9) | l + 256 (9) | row within its block (kRowBits) | x cell (13)
__device__ __forceinline__ uint64_t pack_box(int64_t u, int h, int k, int l, int rowlo, int fx) {
    return ((uint64_t)u << kUShift) | ((uint64_t)(h + kHklOff) << kHShift) |
           ((uint64_t)(k + kHklOff) << kKShift) | ((uint64_t)(l + kHklOff) << kLShift) |
           ((uint64_t)rowlo << 13) | (uint64_t)fx;
}
__device__ __forceinline__ int box_fx(uint64_t r) { return (int)(r & 8191u); }
__device__ __forceinline__ int box_rowlo(uint64_t r) {
    return (int)((r >> 13) & (uint64_t)(kRowBlock - 1));
}

struct BinLayout {
    size_t info, packs, cnt_ubi, fallback, cta_blk, blktot, blkstart, rstart, tot, tmp, recs,
        bytes;
};

// workspace: info | packs (m x 3 float4) | per-UBI box counts | fallback list |
// per-CTA block counts / offsets | block totals | block starts | row starts |
// scan totals | boxes by block | boxes by row
inline BinLayout bin_layout(int64_t m, int64_t nrows, int64_t cap) {
    BinLayout L;
    const size_t mm = (size_t)(m > 0 ? m : 1);
    const int64_t nblk = (nrows + kRowBlock - 1) / kRowBlock;
    const size_t cc = (size_t)(cap > 0 ? cap : 1);
    size_t o = 0;
    L.info = o;     o = al256(o + sizeof(BinInfo));
    L.packs = o;    o = al256(o + 3 * sizeof(float4) * mm);
    L.cnt_ubi = o;  o = al256(o + sizeof(int) * mm);
    L.fallback = o; o = al256(o + sizeof(int) * mm);
    L.cta_blk = o;  o = al256(o + sizeof(int) * (size_t)kMaxEnumCtas * (size_t)nblk);
    L.blktot = o;   o = al256(o + sizeof(int) * (size_t)(nblk + 1));
    L.blkstart = o; o = al256(o + sizeof(int) * (size_t)(nblk + 1));
    L.rstart = o;   o = al256(o + sizeof(int) * (size_t)(nrows + 1));
    L.tot = o;      o = al256(o + sizeof(int) * (size_t)((nblk + 1 + kScanPer - 1) / kScanPer + 1));
    L.tmp = o;      o = al256(o + sizeof(uint64_t) * cc);
    L.recs = o;     o = al256(o + sizeof(uint64_t) * cc);
    L.bytes = o;
    return L;
}

// packed FP32 pairs (sm_100 f32x2): every lane does exactly the scalar operation
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
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// FP32 form of a UBI's plan for the candidate work of the enumeration.  The
// half widths are widened by a bound on the FP32 error of the box centre:
// c = fma(l, ub_r2, fma(k, ub_r1, h * ub_r0)) with ub rounded to FP32 is
// within 4 * 2^-24 * max|hkl| * sum_j |ub_rj| of UB.hkl (input rounding plus
// three roundings of partial sums no larger than that sum), so every box
// [c - w', c + w'] holds the exact one, and every test on it is conservative.
struct Plan32 {
    float ub[9], w[3];
    float G, rmax2;       // cube half side and squared radius, rounded up
};

__device__ __forceinline__ void make_plan32(const volatile WarpPlan* wp, const Header& H,
                                            volatile Plan32* p, double* wmax) {
    double hm = 0.;
#pragma unroll
    for (int r = 0; r < 3; r++)
        hm = fmax(hm, fmax(fabs((double)wp->lo[r]), fabs((double)(wp->lo[r] + wp->nh[r] - 1))));
    double wm = 0.;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const double us = fabs(wp->ub[3 * r]) + fabs(wp->ub[3 * r + 1]) + fabs(wp->ub[3 * r + 2]);
        const double err = 4.0 * kEps32 * hm * us * (1. + 1e-6);
        const float wr = __double2float_ru(wp->w[r] + err);
        p->w[r] = wr;
        wm = fmax(wm, (double)wr);
#pragma unroll
        for (int j = 0; j < 3; j++) p->ub[3 * r + j] = __double2float_rn(wp->ub[3 * r + j]);
    }
    p->G = __double2float_ru(-H.lo * (1. + 1e-6));
    p->rmax2 = __double2float_ru(H.rmax * H.rmax * (1. + 1e-5));
    *wmax = wm;
}

// mode 0 counts the boxes per block of kRowBlock rows of cells (and, in the
// first pass, writes the plans' FP32 packs, the largest widened half width and
// row sum, the per-UBI box counts and the fallback list); mode 1 writes every
// box.  CTA c takes UBIs i0 + [c * per, (c + 1) * per), its warps one UBI at
// a time in a fixed order, and keeps one counter per block in shared memory:
// mode 0 stores them in cta_blk[c][block]; mode 1 starts them at
// blkstart[block] + cta_blk[c][block] (the CTA's offset inside the block) and
// writes each box at its counter.  So every CTA writes one sequential stream
// per block (few enough streams that L2 fills their lines before it evicts
// them).  The mode is a run-time argument of one kernel, so both passes run
// the same machine code and put every box in the same block; each write is
// still bounded by the capacity of the box array.
#ifndef ID11B_ENUM_MINB
#define ID11B_ENUM_MINB 1
#endif
__global__ void __launch_bounds__(kET, ID11B_ENUM_MINB)
k_enum(int mode, const double* __restrict__ ubis, int64_t i0, int64_t mc, int64_t per,
       const Header* __restrict__ Hp, const int* __restrict__ start, double tmax, int first,
       int nblk, BinInfo* __restrict__ info, float4* __restrict__ packs,
       int* __restrict__ cnt_ubi, int* __restrict__ fallback, int* __restrict__ cta_blk,
       const int* __restrict__ blkstart, uint64_t* __restrict__ tmp, int64_t cap) {
    __shared__ int s_blk[kMaxBlocks];
    __shared__ WarpPlan s_plan[kEW];
    __shared__ Plan32 s_p32[kEW];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int* my = cta_blk + (int64_t)blockIdx.x * nblk;
    for (int b = threadIdx.x; b < nblk; b += kET) s_blk[b] = mode == 0 ? 0 : blkstart[b] + my[b];
    __syncthreads();
    const Header H = *Hp;
    const int64_t nreg = start[H.ncells];
    const float flo = (float)H.lo, inv_cs = (float)H.inv_cs, inv_csx = (float)H.inv_csx;
    const int64_t u1 = min((int64_t)(blockIdx.x + 1) * per, mc);
    volatile WarpPlan* wp = s_plan + w;
    volatile Plan32* p32 = s_p32 + w;
    for (int64_t u = (int64_t)blockIdx.x * per + w; u < u1; u += kEW) {
        const int64_t i = i0 + u;
        bool ok = setup_plan(wp, ubis, i, tmax, H, nreg, lane);
        double smax = 0.;
#pragma unroll
        for (int r = 0; r < 3; r++) {
            smax = fmax(smax, fabs(wp->u[3 * r]) + fabs(wp->u[3 * r + 1]) + fabs(wp->u[3 * r + 2]));
            ok = ok && wp->lo[r] >= -kHklOff && wp->lo[r] + wp->nh[r] - 1 < kHklOff;
        }
        smax *= 1. + 1e-15;
        ok = ok && smax * (-H.lo) < kSGLimit;
        const bool lead = mode == 0 && first && lane == 0;
        if (!ok) {
            if (lead) {
                const int slot = atomicAdd(&info->nfallback, 1);
                fallback[slot] = (int)i;
            }
            __syncwarp();
            continue;
        }
        if (lane == 0) {
            double wm;
            make_plan32(wp, H, p32, &wm);
            if (lead) {
                float4* p = packs + 3 * i;
                p[0] = make_float4(__double2float_rn(wp->u[0]), __double2float_rn(wp->u[1]),
                                   __double2float_rn(wp->u[2]), __double2float_rn(wp->u[3]));
                p[1] = make_float4(__double2float_rn(wp->u[4]), __double2float_rn(wp->u[5]),
                                   __double2float_rn(wp->u[6]), __double2float_rn(wp->u[7]));
                p[2] = make_float4(__double2float_rn(wp->u[8]), 0.f, 0.f, 0.f);
                atomicMax(&info->smax_bits, __float_as_uint(__double2float_ru(smax)));
                atomicMax(&info->wmax_bits, (unsigned long long)__double_as_longlong(wm));
            }
        }
        __syncwarp();
        // the FP32 plan in registers for the candidate loop
        float ub[9], wr[3];
#pragma unroll
        for (int e = 0; e < 9; e++) ub[e] = p32->ub[e];
#pragma unroll
        for (int r = 0; r < 3; r++) wr[r] = p32->w[r];
        const float G = p32->G, rmax2 = p32->rmax2;
        int nbox = 0;
        // the lookup enumeration's columns (FP64, flattened across the warp)
        const int nh0 = wp->nh[0];
        const int64_t nhk = (int64_t)nh0 * wp->nh[1];
        const double R = (H.rmax + sqrt((double)wr[0] * wr[0] + (double)wr[1] * wr[1] +
                                        (double)wr[2] * wr[2])) * (1. + 1e-9) + 1e-12;
        double n0, n1;
        ub_column_norms(wp, n0, n1);
        for (int64_t hb = 0; hb < nhk; hb += 32) {
            const int64_t hk = hb + lane;
            int len = 0, l0 = 0, h = 0, k = 0;
            if (hk < nhk) {
                h = wp->lo[0] + (int)(hk % nh0);
                k = wp->lo[1] + (int)(hk / nh0);
                column_l_range(wp, n0, n1, h, k, R, l0, len);
            }
            int total;
            const int excl = warp_excl_scan(len, lane, total);
            for (int f0 = 0; f0 < total; f0 += 32) {
                const int f = f0 + lane;
                const int j = owner(excl, f);
                const int hj = __shfl_sync(0xffffffffu, h, j);
                const int kj = __shfl_sync(0xffffffffu, k, j);
                const int lj = __shfl_sync(0xffffffffu, l0, j) + f - __shfl_sync(0xffffffffu, excl, j);
                if (f < total) {
                    const float fh = (float)hj, fk = (float)kj, fl = (float)lj;
                    float c[3], d2 = 0.f;
                    bool in = true;
#pragma unroll
                    for (int r = 0; r < 3; r++) {
                        c[r] = fmaf(fl, ub[3 * r + 2], fmaf(fk, ub[3 * r + 1], fh * ub[3 * r]));
                        in = in && (c[r] - wr[r] <= G) && (c[r] + wr[r] >= -G);
                        const float e = fmaxf(fabsf(c[r]) - wr[r], 0.f);
                        d2 = fmaf(e, e, d2);
                    }
                    if (in && d2 <= rmax2) {
                        const int cx = min(max(__float2int_rd((c[0] - flo) * inv_csx), 0), H.nxx - 1);
                        const int cy = min(max(__float2int_rd((c[1] - flo) * inv_cs), 0), H.nx - 1);
                        const int cz = min(max(__float2int_rd((c[2] - flo) * inv_cs), 0), H.nx - 1);
                        const int row = cz * H.nx + cy;
                        const int slot = atomicAdd(s_blk + row / kRowBlock, 1);
                        if (mode == 0) {
                            nbox++;
                        } else if (slot < cap) {
                            tmp[slot] = pack_box(u, hj, kj, lj, row % kRowBlock, cx);
                        }
                    }
                }
            }
        }
        if (mode == 0 && first) {
            const int nb = warp_sum(nbox);
            if (lane == 0) {
                cnt_ubi[i] = nb;
                if (nb) atomicAdd(&info->total, (unsigned long long)nb);
            }
        }
    }
    __syncthreads();
    if (mode == 0)
        for (int b = threadIdx.x; b < nblk; b += kET) my[b] = s_blk[b];
}

// Per block: the CTAs' counts turned into exclusive offsets inside the block
// (in place), and the block's total.  One warp per block.
__global__ void __launch_bounds__(kGT)
k_blk_offsets(int* __restrict__ cta_blk, int nctas, int nblk, int* __restrict__ blktot) {
    const int lane = threadIdx.x & 31;
    for (int64_t b = ((int64_t)blockIdx.x * kGT + threadIdx.x) >> 5; b < nblk;
         b += ((int64_t)gridDim.x * kGT) >> 5) {
        int run = 0;
        for (int c0 = 0; c0 < nctas; c0 += 32) {
            const int c = c0 + lane;
            const int v = c < nctas ? cta_blk[(int64_t)c * nblk + b] : 0;
            int tot;
            const int ex = warp_excl_scan(v, lane, tot);
            if (c < nctas) cta_blk[(int64_t)c * nblk + b] = run + ex;
            run += tot;
        }
        if (lane == 0) blktot[b] = run;
    }
}

// The boxes of each block split into its kRowBlock rows (any order within a
// row): one CTA per block, each thread taking kRK boxes at a time (loads in
// flight), counts and then cursors per (warp, row) in shared memory, so each
// warp writes one sequential stream per row.  Both passes give each box to the
// same thread.  Writes each row's start to rstart.
// threads per row-split CTA and records each thread loads at a time: binned
// scoring of 20,000 UBIs x 1.1M g took 2.79 ms at 512 x 8, 2.76 at 512 x 16
// (24 and 32 the same), 2.79 at 1024 x 16, 2.80 at 1024 x 8
#ifndef ID11B_RS_T
#define ID11B_RS_T 512
#endif
constexpr int kRS = ID11B_RS_T;
constexpr int kRSW = kRS / 32;
#ifndef ID11B_RS_K
#define ID11B_RS_K 16
#endif
constexpr int kRK = ID11B_RS_K;
#ifndef ID11B_RS_PER_SM
#define ID11B_RS_PER_SM 1
#endif
// row-split CTAs per SM: one block (~340 KB on the headline) in flight per SM
// keeps every block in L2 between its counting and placing reads (one per
// SM: 3.12 ms per headline step; four: 3.23 ms)
constexpr int kRSPerSM = ID11B_RS_PER_SM;

__global__ void __launch_bounds__(kRS)
k_rowsplit(const uint64_t* __restrict__ tmp, const int* __restrict__ blkstart, int nblk,
           int nrows, int* __restrict__ rstart, uint64_t* __restrict__ recs) {
    __shared__ int s_wh[kRSW][kRowBlock];
    const int w = threadIdx.x >> 5;
    for (int b = blockIdx.x; b < nblk; b += gridDim.x) {
        const int p0 = blkstart[b], p1 = blkstart[b + 1];
        if (threadIdx.x < kRSW * kRowBlock) s_wh[threadIdx.x / kRowBlock][threadIdx.x % kRowBlock] = 0;
        __syncthreads();
        for (int i0 = p0; i0 < p1; i0 += kRS * kRK) {
            uint64_t r[kRK];
#pragma unroll
            for (int k = 0; k < kRK; k++) {
                const int i = i0 + k * kRS + threadIdx.x;
                r[k] = i < p1 ? __ldg(tmp + i) : 0;
            }
#pragma unroll
            for (int k = 0; k < kRK; k++)
                if (i0 + k * kRS + (int)threadIdx.x < p1) atomicAdd(&s_wh[w][box_rowlo(r[k])], 1);
        }
        __syncthreads();
        if (threadIdx.x == 0) {  // per-warp cursors: rows in order, warps in order inside a row
            int run = p0;
            for (int v = 0; v < kRowBlock; v++) {
                const int row = b * kRowBlock + v;
                if (row < nrows) rstart[row] = run;
                for (int q = 0; q < kRSW; q++) {
                    const int c = s_wh[q][v];
                    s_wh[q][v] = run;
                    run += c;
                }
            }
            if (b == nblk - 1) rstart[nrows] = run;
        }
        __syncthreads();
        for (int i0 = p0; i0 < p1; i0 += kRS * kRK) {
            uint64_t r[kRK];
#pragma unroll
            for (int k = 0; k < kRK; k++) {
                const int i = i0 + k * kRS + threadIdx.x;
                r[k] = i < p1 ? __ldg(tmp + i) : 0;
            }
#pragma unroll
            for (int k = 0; k < kRK; k++)
                if (i0 + k * kRS + (int)threadIdx.x < p1)
                    recs[atomicAdd(&s_wh[w][box_rowlo(r[k])], 1)] = r[k];
        }
        __syncthreads();
    }
}

// A pair inside a band (or, with sums, any pair below hmax): the reference's
// exact FP64 drlv2 and whether it belongs to the box's hkl, by value.  Out of
// line: rare, and its registers would otherwise weigh on the whole join.
struct Exact {
    double s;   // drlv2
    bool own;   // the rounded h is the box's hkl
};

__device__ __noinline__ Exact exact_pair(const double* __restrict__ ubis, int64_t ubi,
                                         const double* __restrict__ gs, int pos, float hk0,
                                         float hk1, float hk2) {
    double u[9], ih[3];
#pragma unroll
    for (int e = 0; e < 9; e++) u[e] = __ldg(ubis + 9 * ubi + e);
    Exact r;
    r.s = drlv2_exact(u, __ldg(gs + 3 * (int64_t)pos), __ldg(gs + 3 * (int64_t)pos + 1),
                      __ldg(gs + 3 * (int64_t)pos + 2), ih);
    r.own = ih[0] == (double)hk0 && ih[1] == (double)hk1 && ih[2] == (double)hk2;
    return r;
}

// A pair inside a band (or, with sums, any pair below hmax), evaluated
// exactly: counted for the tolerances its FP64 drlv2 clears under its own hkl
// (those it cleared in FP32 by more than the band were counted already).
//
// AS 1 and 2 (assignment, NT 1, SUMS): the two passes of k_assign
// (gvec_grid.cu) on the pair -- below tol^2 and below the g's drlv2 on entry,
// pass 1 takes the smallest drlv2 bits per g, pass 2 the lowest UBI index
// reaching them.
template <int NT, bool SUMS, int AS>
__device__ __forceinline__ void rare_pair(float s, int pos, const JoinParams& P,
                                          const double* __restrict__ ubis, int64_t ubi,
                                          const double* __restrict__ gs, const float* hkf,
                                          int cnt[NT], unsigned long long sum[NT]) {
    const Exact e = exact_pair(ubis, ubi, gs, pos, hkf[0], hkf[1], hkf[2]);
    if (!e.own) return;
    if (AS) {
        if (!(e.s < P.t2[0])) return;
        const int k = __ldg(P.gidx + pos);
        if (!(e.s < __ldg(P.d0 + k))) return;
        const unsigned long long b = (unsigned long long)__double_as_longlong(e.s);
        if (AS == 1)
            atomicMin(P.best + k, b);
        else if (P.best[k] == b)
            atomicMin(P.lab + k, (int)ubi);
        return;
    }
#pragma unroll
    for (int j = 0; j < NT; j++) {
        if (!(e.s < P.t2[j])) continue;
        if (SUMS) {
            cnt[j]++;
            sum[j] += __double2ull_rn(e.s * P.fix);  // per term: order-free
        } else if (!(s < P.lo[j])) {
            cnt[j]++;
        }
    }
}

struct Staged {  // the tile of staged g, structure of arrays (pairs read as 64 bits)
    const float *x, *y, *z;
    const int* pos;
};

// The box of one lane against staged g [ga, gb), two at a time with packed
// f32x2 instructions (lane by lane the operations of drlv2_f32, so every
// screening value is the scalar one).  The range is widened to even bounds
// (an odd tile ends with a NaN g): testing g beyond a run's range is harmless,
// every g of a tile being tested at most once per box.  Counting is free of
// branches; one branch per pair of g catches the rare band cases.
//
// RANKED (lo and hi both non-decreasing in j): a value below lo_j is below
// every later lo, so the only band it can lie in is that of the largest lo_j
// not above it -- one select chain and one compare instead of a test per
// tolerance.  (If s lies in band i <= J, J the largest j with lo_j <= s, then
// s < hi_i <= hi_J.)
template <int NT, bool SUMS, bool RANKED, int AS>
__device__ __forceinline__ void test_range(const Staged& t, int ga, int gb, const uint64_t uu[9],
                                           const uint64_t hh[3], const float* hkf,
                                           const JoinParams& P, const double* __restrict__ ubis,
                                           int64_t ubi, const double* __restrict__ gs, int cnt[NT],
                                           unsigned long long sum[NT], unsigned& ntest) {
    for (int q = ga & ~1; q < gb; q += 2) {
        const uint64_t gx = *reinterpret_cast<const uint64_t*>(t.x + q);
        const uint64_t gy = *reinterpret_cast<const uint64_t*>(t.y + q);
        const uint64_t gz = *reinterpret_cast<const uint64_t*>(t.z + q);
#if ID11B_JOIN_FOLD
        // UBI.g - hkl with the subtraction folded into the first FMA (hh holds
        // -hkl): three roundings of partial sums below |hkl| + S gmax
        const uint64_t d0 = fma2(uu[2], gz, fma2(uu[1], gy, fma2(uu[0], gx, hh[0])));
        const uint64_t d1 = fma2(uu[5], gz, fma2(uu[4], gy, fma2(uu[3], gx, hh[1])));
        const uint64_t d2 = fma2(uu[8], gz, fma2(uu[7], gy, fma2(uu[6], gx, hh[2])));
#else
        const uint64_t h0 = fma2(uu[2], gz, fma2(uu[1], gy, mul2(uu[0], gx)));
        const uint64_t h1 = fma2(uu[5], gz, fma2(uu[4], gy, mul2(uu[3], gx)));
        const uint64_t h2 = fma2(uu[8], gz, fma2(uu[7], gy, mul2(uu[6], gx)));
        const uint64_t d0 = sub2(h0, hh[0]), d1 = sub2(h1, hh[1]), d2 = sub2(h2, hh[2]);
#endif
        float sa, sb;
        upk2(fma2(d2, d2, fma2(d1, d1, mul2(d0, d0))), sa, sb);
        bool ra, rb;
        if (SUMS) {
            ra = sa < P.hmax;
            rb = sb < P.hmax;
        } else if (RANKED) {
            bool ia[NT], ib[NT];
#pragma unroll
            for (int j = 0; j < NT; j++) {
                ia[j] = sa < P.lo[j];
                ib[j] = sb < P.lo[j];
                cnt[j] += (int)ia[j] + (int)ib[j];
            }
            float ha = P.hi[NT - 1], hb = P.hi[NT - 1];
#pragma unroll
            for (int j = NT - 2; j >= 0; j--) {
                ha = ia[j + 1] ? P.hi[j] : ha;
                hb = ib[j + 1] ? P.hi[j] : hb;
            }
            ra = !ia[0] && sa < ha;
            rb = !ib[0] && sb < hb;
        } else {
            ra = rb = false;
#pragma unroll
            for (int j = 0; j < NT; j++) {
                const bool ia = sa < P.lo[j], ib = sb < P.lo[j];
                cnt[j] += (int)ia + (int)ib;
                ra |= !ia && sa < P.hi[j];
                rb |= !ib && sb < P.hi[j];
            }
        }
        if (ra || rb) {
            ntest += (unsigned)ra + (unsigned)rb;
            if (ra) rare_pair<NT, SUMS, AS>(sa, t.pos[q], P, ubis, ubi, gs, hkf, cnt, sum);
            if (rb) rare_pair<NT, SUMS, AS>(sb, t.pos[q + 1], P, ubis, ubi, gs, hkf, cnt, sum);
        }
    }
}

// Exclusive scan of a[0 .. len) into b (block-wide; ends with a barrier).
__device__ __forceinline__ void block_scan(const int* a, int* b, int len, int* s_w) {
    const int per = (len + kJT - 1) / kJT;
    const int b0 = threadIdx.x * per, b1 = min(b0 + per, len);
    int sum = 0;
    for (int i = b0; i < b1; i++) sum += a[i];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int tot;
    const int ex = warp_excl_scan(sum, lane, tot);
    if (lane == 0) s_w[w] = tot;
    __syncthreads();
    int base = 0;
    for (int k = 0; k < w; k++) base += s_w[k];
    int run = base + ex;
    for (int i = b0; i < b1; i++) {
        const int v = a[i];
        b[i] = run;
        run += v;
    }
    __syncthreads();
}

// Persistent CTAs, each taking one row of cells at a time (a counter).  The
// row's boxes are counted per x cell, the row is cut into windows of x cells
// holding at most kBMax boxes (a cell with more is taken alone, in pieces of
// kBMax boxes in storage order), and each window's boxes are placed in shared
// memory sorted by x cell.  The g-vectors of the window's region are staged in
// tiles of at most kGMax, each sorted by x cell, and every run of 32 sorted
// boxes (one warp) is tested against the staged g in the x cells its boxes
// can reach.
template <int NT, bool SUMS, bool RANKED, int AS = 0>
__global__ void __launch_bounds__(kJT, kJoinMinBlocks)
k_join(const uint64_t* __restrict__ recs, const int* __restrict__ rstart, int nrows,
       int nhalo, BinInfo* __restrict__ info, const float4* __restrict__ packs,
       const double* __restrict__ ubis, Header* __restrict__ Hp, const int* __restrict__ start,
       const double* __restrict__ gs, const float4* __restrict__ g4, const JoinParams P,
       int* __restrict__ counts, double* __restrict__ sums) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* s_box = reinterpret_cast<uint64_t*>(smem);        // kBMax sorted boxes
    float* s_gx = reinterpret_cast<float*>(s_box + kBMax);      // kGMax staged g
    float* s_gy = s_gx + kGMax;
    float* s_gz = s_gy + kGMax;
    int* s_gp = reinterpret_cast<int*>(s_gz + kGMax);
    const int nh1 = max(P.nxx, nhalo) + 1;
    int* s_bs = s_gp + kGMax;        // boxes of the row before each x cell (nxx + 1)
    int* s_bc = s_bs + nh1;          // box counts, then cursors
    int* s_gh = s_bc + nh1;          // halo row lengths; g counts / cursors
    int* s_gs = s_gh + nh1;          // staged g before each x cell of the tile
    int* s_rp = s_gs + nh1;          // halo rows: candidate prefix (nhalo + 1)
    int* s_rs = s_rp + (nhalo + 1);  // halo rows: first g
    __shared__ int s_row, s_w[kJW], s_base;
    const Staged T{s_gx, s_gy, s_gz, s_gp};
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned ntest = 0;
    unsigned long long npairs = 0;  // lane 0: (box, g) pairs screened
    for (;;) {
        if (threadIdx.x == 0) s_row = atomicAdd(&info->next_row, 1);
        __syncthreads();
        const int r = s_row;
        __syncthreads();
        if (r >= nrows) break;
        const int b0 = rstart[r], b1 = rstart[r + 1];
        if (b0 == b1) continue;
        const int iy = r % P.nx, iz = r / P.nx;
        const float ylo = fmaf((float)iy, P.cs, P.rlo), yhi = fmaf((float)(iy + 1), P.cs, P.rhi);
        const float zlo = fmaf((float)iz, P.cs, P.rlo), zhi = fmaf((float)(iz + 1), P.cs, P.rhi);
        const int ry0 = max(iy - P.R, 0), rz0 = max(iz - P.R, 0);
        const int ny = min(iy + P.R, P.nx - 1) - ry0 + 1;
        const int nhr = ny * (min(iz + P.R, P.nx - 1) - rz0 + 1);
        // the row's boxes per x cell
        for (int x = threadIdx.x; x <= P.nxx; x += kJT) s_bc[x] = 0;
        __syncthreads();
        for (int i = b0 + threadIdx.x; i < b1; i += kJT) atomicAdd(s_bc + box_fx(recs[i]), 1);
        __syncthreads();
        block_scan(s_bc, s_bs, P.nxx + 1, s_w);
        int wa = 0, piece = 0;
        while (wa < P.nxx) {  // uniform over the CTA
            int lo = wa, hi = P.nxx;  // the largest wb with s_bs[wb] - s_bs[wa] <= kBMax
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (s_bs[mid] - s_bs[wa] <= kBMax) lo = mid; else hi = mid - 1;
            }
            const bool big = lo == wa;  // cell wa alone holds more than kBMax boxes
            const int wb = big ? wa + 1 : lo;
            const int skip = big ? piece * kBMax : 0;
            const int ncell = s_bs[wb] - s_bs[wa];
            const int nb = big ? min(kBMax, ncell - skip) : ncell;
            const int cur_wa = wa;
            if (big && skip + nb < ncell) {
                piece++;
            } else {
                piece = 0;
                wa = wb;
            }
            if (nb == 0) continue;
            // the window's boxes in shared memory, sorted by x cell
            if (!big) {
                for (int x = cur_wa + threadIdx.x; x < wb; x += kJT) s_bc[x] = 0;
                __syncthreads();
                for (int i = b0 + threadIdx.x; i < b1; i += kJT) {
                    const uint64_t rec = recs[i];
                    const int fx = box_fx(rec);
                    if (fx >= cur_wa && fx < wb)
                        s_box[s_bs[fx] - s_bs[cur_wa] + atomicAdd(s_bc + fx, 1)] = rec;
                }
            } else {  // boxes skip .. skip + nb - 1 of cell cur_wa, in storage order
                if (threadIdx.x == 0) s_base = 0;
                __syncthreads();
                for (int i0 = b0; i0 < b1; i0 += kJT) {
                    const int i = i0 + threadIdx.x;
                    uint64_t rec = 0;
                    const bool mine = i < b1 && box_fx(rec = recs[i]) == cur_wa;
                    const unsigned bal = __ballot_sync(0xffffffffu, mine);
                    if (lane == 0) s_w[w] = __popc(bal);
                    __syncthreads();
                    int rank = s_base + __popc(bal & ((1u << lane) - 1u));
                    for (int k = 0; k < w; k++) rank += s_w[k];
                    if (mine && rank >= skip && rank < skip + nb) s_box[rank - skip] = rec;
                    __syncthreads();
                    if (threadIdx.x == 0)
                        for (int k = 0; k < kJW; k++) s_base += s_w[k];
                    __syncthreads();
                }
            }
            __syncthreads();
            // x cells the window's boxes can reach, and the halo rows' g in them
            const int gxa = max(box_fx(s_box[0]) - P.Rx, 0);
            const int gxb = min(box_fx(s_box[nb - 1]) + P.Rx, P.nxx - 1);
            const int gw = gxb - gxa + 1;
            for (int j = threadIdx.x; j <= nhr; j += kJT) {
                int len = 0;
                if (j < nhr) {
                    const int zq = j / ny;
                    const int64_t base = ((int64_t)(rz0 + zq) * P.nx + (ry0 + j - zq * ny)) * P.nxx;
                    const int st = start[base + gxa];
                    s_rs[j] = st;
                    len = start[base + gxb + 1] - st;
                }
                s_gh[j] = len;
            }
            __syncthreads();
            block_scan(s_gh, s_rp, nhr + 1, s_w);
            const int ncand = s_rp[nhr];
            // candidate q: its g (w: its x cell) and position; true when inside
            // the row's y/z region
            auto candidate = [&](int q, float4& v, int& pos) {
                int a = 0, c = nhr - 1;  // the last halo row with s_rp <= q
                while (a < c) {
                    const int mid = (a + c + 1) >> 1;
                    if (s_rp[mid] <= q) a = mid; else c = mid - 1;
                }
                pos = s_rs[a] + (q - s_rp[a]);
                v = __ldg(g4 + pos);
                return v.y >= ylo && v.y <= yhi && v.z >= zlo && v.z <= zhi;
            };
            // tiles of at most kGMax staged g, each sorted by x cell
            for (int c0 = 0; c0 < ncand;) {
                for (int x = threadIdx.x; x <= gw; x += kJT) s_gh[x] = 0;
                __syncthreads();
                int cend = c0, tot = 0;
                while (cend < ncand && tot <= kGMax - kJT) {
                    const int q = cend + threadIdx.x;
                    bool in = false;
                    if (q < ncand) {
                        float4 v;
                        int pos;
                        in = candidate(q, v, pos);
                        if (in) atomicAdd(s_gh + (__float_as_int(v.w) - gxa), 1);
                    }
                    tot += __syncthreads_count(in);
                    cend = min(cend + kJT, ncand);
                }
                block_scan(s_gh, s_gs, gw + 1, s_w);
                for (int x = threadIdx.x; x <= gw; x += kJT) s_gh[x] = 0;
                __syncthreads();
                for (int q = c0 + threadIdx.x; q < cend; q += kJT) {
                    float4 v;
                    int pos;
                    if (candidate(q, v, pos)) {
                        const int cx = __float_as_int(v.w) - gxa;
                        const int slot = s_gs[cx] + atomicAdd(s_gh + cx, 1);
                        s_gx[slot] = v.x;
                        s_gy[slot] = v.y;
                        s_gz[slot] = v.z;
                        s_gp[slot] = pos;
                    }
                }
                if (threadIdx.x == 0 && (s_gs[gw] & 1)) {  // pad an odd tile with a NaN g
                    const float nan = __int_as_float(0x7fc00000);
                    s_gx[s_gs[gw]] = nan;
                    s_gy[s_gs[gw]] = nan;
                    s_gz[s_gs[gw]] = nan;
                    s_gp[s_gs[gw]] = 0;
                }
                __syncthreads();
                // runs of 32 sorted boxes, one warp each
                for (int k0 = 32 * w; k0 < nb; k0 += 32 * kJW) {
                    const int nrun = min(32, nb - k0);
                    const int ga = s_gs[max(box_fx(s_box[k0]) - P.Rx, gxa) - gxa];
                    const int gb = s_gs[min(box_fx(s_box[k0 + nrun - 1]) + P.Rx, gxb) - gxa + 1];
                    if (lane == 0 && ga < gb)
                        npairs += (unsigned long long)nrun * (unsigned)(((gb + 1) & ~1) - (ga & ~1));
                    if (lane < nrun && ga < gb) {
                        const uint64_t rec = s_box[k0 + lane];
                        const int64_t ubi = P.i0 + (int64_t)(rec >> kUShift);
                        const float hkf[3] = {(float)((int)((rec >> kHShift) & 511) - kHklOff),
                                              (float)((int)((rec >> kKShift) & 511) - kHklOff),
                                              (float)((int)((rec >> kLShift) & 511) - kHklOff)};
                        const float4 p0 = __ldg(packs + 3 * ubi);
                        const float4 p1 = __ldg(packs + 3 * ubi + 1);
                        const float4 p2 = __ldg(packs + 3 * ubi + 2);
                        const float u[9] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w, p2.x};
                        uint64_t uu[9], hh[3];
#pragma unroll
                        for (int e = 0; e < 9; e++) uu[e] = pk2(u[e], u[e]);
#pragma unroll
                        for (int e = 0; e < 3; e++)
                            hh[e] = ID11B_JOIN_FOLD ? pk2(-hkf[e], -hkf[e]) : pk2(hkf[e], hkf[e]);
                        int cnt[NT];
                        unsigned long long sum[NT];
#pragma unroll
                        for (int j = 0; j < NT; j++) {
                            cnt[j] = 0;
                            sum[j] = 0ull;
                        }
                        test_range<NT, SUMS, RANKED, AS>(T, ga, gb, uu, hh, hkf, P, ubis, ubi,
                                                         gs, cnt, sum, ntest);
#pragma unroll
                        for (int j = 0; j < NT && !AS; j++) {
                            if (cnt[j]) atomicAdd(counts + ubi * NT + P.ord[j], cnt[j]);
                            if (SUMS && sum[j])
                                atomicAdd(reinterpret_cast<unsigned long long*>(
                                              sums + ubi * NT + P.ord[j]), sum[j]);
                        }
                    }
                }
                __syncthreads();
                c0 = cend;
            }
        }
    }
    const long long tt = warp_sum((long long)ntest);
    if (lane == 0 && tt) atomicAdd(&Hp->ntested, (unsigned long long)tt);
    if (lane == 0 && npairs) atomicAdd(&Hp->npairs, npairs);
}

// UBIs outside the binned path's limits: exact FP64 over every regular g, one
// warp per (listed UBI, part).
template <int NT, bool SUMS>
__global__ void __launch_bounds__(kBT)
k_fallback(const double* __restrict__ ubis, const int* __restrict__ list, int nlist,
           Header* __restrict__ Hp, const int* __restrict__ start, const double* __restrict__ gs,
           Tols tols, int* __restrict__ counts, double* __restrict__ sums) {
    const int lane = threadIdx.x & 31;
    const int64_t wk = ((int64_t)blockIdx.x * kBT + threadIdx.x) >> 5;
    if (wk >= (int64_t)nlist * kFallbackParts) return;  // uniform per warp
    const int i = list[wk / kFallbackParts];
    const int part = (int)(wk % kFallbackParts);
    const int64_t nreg = start[Hp->ncells];
    double u[9];
#pragma unroll
    for (int e = 0; e < 9; e++) u[e] = ubis[9 * (int64_t)i + e];
    int cnt[NT];
    double sum[NT];
#pragma unroll
    for (int j = 0; j < NT; j++) {
        cnt[j] = 0;
        sum[j] = 0.;
    }
    for (int64_t f = (int64_t)part * 32 + lane; f < nreg; f += 32 * (int64_t)kFallbackParts) {
        double ih[3];
        const double s = drlv2_exact(u, gs[3 * f], gs[3 * f + 1], gs[3 * f + 2], ih);
#pragma unroll
        for (int j = 0; j < NT; j++)
            if (s < tols.t[j] * tols.t[j]) {
                cnt[j]++;
                sum[j] += s;
            }
    }
#pragma unroll
    for (int j = 0; j < NT; j++) {
        const int c = warp_sum(cnt[j]);
        const double sm = warp_sum(sum[j]);
        if (lane == 0 && c) {
            atomicAdd(counts + (int64_t)i * NT + j, c);
            if (SUMS) fixsum_add(sums + (int64_t)i * NT + j, sm, tols.fix);
        }
    }
    if (part == 0 && lane == 0) atomicAdd(&Hp->nfallback, 1ull);
}

// The g-vectors outside the regular range, for every UBI: one warp per UBI.
template <int NT, bool SUMS>
__global__ void __launch_bounds__(kBT)
k_special(const double* __restrict__ ubis, int64_t m, const double* __restrict__ gv,
          const int* __restrict__ special, const int* __restrict__ nspecial, Tols tols,
          int* __restrict__ counts, double* __restrict__ sums) {
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * kBT + threadIdx.x) >> 5;
    if (i >= m) return;  // uniform per warp
    const int ns = *nspecial;
    double u[9];
#pragma unroll
    for (int e = 0; e < 9; e++) u[e] = ubis[9 * i + e];
    int cnt[NT];
    double sum[NT];
#pragma unroll
    for (int j = 0; j < NT; j++) {
        cnt[j] = 0;
        sum[j] = 0.;
    }
    for (int q = lane; q < ns; q += 32) {
        const int64_t k = special[q];
        double ih[3];
        const double s = drlv2_exact(u, gv[3 * k], gv[3 * k + 1], gv[3 * k + 2], ih);
#pragma unroll
        for (int j = 0; j < NT; j++)
            if (s < tols.t[j] * tols.t[j]) {
                cnt[j]++;
                sum[j] += s;
            }
    }
#pragma unroll
    for (int j = 0; j < NT; j++) {
        const int c = warp_sum(cnt[j]);
        const double sm = warp_sum(sum[j]);
        if (lane == 0 && c) {
            atomicAdd(counts + i * NT + j, c);
            if (SUMS) fixsum_add(sums + i * NT + j, sm, tols.fix);
        }
    }
}

// The assignment's rules (k_assign, gvec_grid.cu) for the UBIs outside the
// binned path's limits: exact FP64 over every regular g, one warp per
// (listed UBI, part); PASS 0 the smallest drlv2 bits, PASS 1 the lowest UBI.
template <int PASS>
__global__ void __launch_bounds__(kBT)
k_assign_fallback(const double* __restrict__ ubis, const int* __restrict__ list, int nlist,
                  const Header* __restrict__ Hp, const int* __restrict__ start,
                  const double* __restrict__ gs, const int* __restrict__ gidx, double tol,
                  const double* __restrict__ d0, unsigned long long* __restrict__ best,
                  int* __restrict__ lab) {
    const int lane = threadIdx.x & 31;
    const int64_t wk = ((int64_t)blockIdx.x * kBT + threadIdx.x) >> 5;
    if (wk >= (int64_t)nlist * kFallbackParts) return;  // uniform per warp
    const int i = list[wk / kFallbackParts];
    const int part = (int)(wk % kFallbackParts);
    const int64_t nreg = start[Hp->ncells];
    const double t2 = tol * tol;
    double u[9];
#pragma unroll
    for (int e = 0; e < 9; e++) u[e] = ubis[9 * (int64_t)i + e];
    for (int64_t f = (int64_t)part * 32 + lane; f < nreg; f += 32 * (int64_t)kFallbackParts) {
        double ih[3];
        const double s = drlv2_exact(u, gs[3 * f], gs[3 * f + 1], gs[3 * f + 2], ih);
        if (!(s < t2)) continue;
        const int k = gidx[f];
        if (!(s < d0[k])) continue;
        const unsigned long long b = (unsigned long long)__double_as_longlong(s);
        if (PASS == 0)
            atomicMin(best + k, b);
        else if (best[k] == b)
            atomicMin(lab + k, i);
    }
}

template <int NT, bool SUMS, bool RANKED, int AS = 0>
int launch_join_k(int grid, size_t smem, const uint64_t* recs, const int* rstart, int nrows,
                  int nhalo, BinInfo* info, const float4* packs, const double* ubis, Header* H,
                  const int* start, const double* gs, const float4* g4, const JoinParams& P,
                  int* counts, double* sums, cudaStream_t st) {
    ID11B_CHECK(cudaFuncSetAttribute(k_join<NT, SUMS, RANKED, AS>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_join<NT, SUMS, RANKED, AS><<<grid, kJT, smem, st>>>(recs, rstart, nrows, nhalo, info, packs,
                                                          ubis, H, start, gs, g4, P, counts,
                                                          sums);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

// the ranked test where it applies (no sums, at least two tolerances, the
// thresholds monotone); the per-tolerance test otherwise
template <int NT, bool SUMS>
int launch_join(int grid, size_t smem, bool ranked, const uint64_t* recs, const int* rstart,
                int nrows, int nhalo, BinInfo* info, const float4* packs, const double* ubis,
                Header* H, const int* start, const double* gs, const float4* g4,
                const JoinParams& P, int* counts, double* sums, cudaStream_t st) {
    if (!SUMS && NT > 1 && ranked)
        return launch_join_k<NT, SUMS, !SUMS && NT != 1>(grid, smem, recs, rstart, nrows, nhalo,
                                                         info, packs, ubis, H, start, gs, g4, P,
                                                         counts, sums, st);
    return launch_join_k<NT, SUMS, false>(grid, smem, recs, rstart, nrows, nhalo, info, packs,
                                          ubis, H, start, gs, g4, P, counts, sums, st);
}

template <int NT, bool SUMS>
int launch_rest(const double* ubis, int64_t m, const int* fallback, int nfallback, Header* H,
                const int* start, const double* gs, const double* gv, const int* special,
                const int* nspecial, int has_special, const Tols& T, int* counts, double* sums,
                cudaStream_t st) {
    if (nfallback > 0) {
        const int64_t warps = (int64_t)nfallback * kFallbackParts;
        k_fallback<NT, SUMS><<<(unsigned)((warps + kBW - 1) / kBW), kBT, 0, st>>>(
            ubis, fallback, nfallback, H, start, gs, T, counts, sums);
        ID11B_CHECK_LAUNCH();
    }
    if (has_special) {
        k_special<NT, SUMS><<<(unsigned)((m + kBW - 1) / kBW), kBT, 0, st>>>(
            ubis, m, gv, special, nspecial, T, counts, sums);
        ID11B_CHECK_LAUNCH();
    }
    return ID11B_OK;
}

// resident CTAs per SM of a kernel with the given dynamic shared memory
template <class K>
int ctas_per_sm(K kernel, int threads, size_t smem) {
    int per = 0;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) !=
            cudaSuccess || per < 1)
        per = 1;
    return per;
}

template <int NT, bool SUMS>
int join_ctas(size_t smem, bool ranked) {
    if (!SUMS && NT > 1 && ranked)
        return ctas_per_sm(k_join<NT, SUMS, !SUMS && NT != 1>, kJT, smem);
    return ctas_per_sm(k_join<NT, SUMS, false>, kJT, smem);
}

// float nearest to x in the given direction (x itself when representable)
float float_rd(double x) {
    float f = (float)x;
    if ((double)f > x) f = nextafterf(f, -INFINITY);
    return f;
}
float float_ru(double x) {
    float f = (float)x;
    if ((double)f < x) f = nextafterf(f, INFINITY);
    return f;
}


}  // namespace bins
}  // namespace grid
}  // namespace id11b

using namespace id11b::grid;
using namespace id11b::grid::bins;

namespace {
// events that bracket the join launches of the calling thread's next binned
// call (a measurement hook; cleared by that call)
thread_local cudaEvent_t t_join_start = nullptr, t_join_stop = nullptr;
}  // namespace

extern "C" int id11b_grid_bins_time_join(void* start_event, void* stop_event) {
    if ((start_event == nullptr) != (stop_event == nullptr)) return ID11B_ERR_ARG;
    t_join_start = (cudaEvent_t)start_event;
    t_join_stop = (cudaEvent_t)stop_event;
    return ID11B_OK;
}

extern "C" int64_t id11b_grid_bins_workspace_bytes(int64_t m, int32_t nx, int32_t xsub,
                                                   int64_t boxes) {
    if (m < 0 || !grid_dims_ok(nx, xsub) || boxes < 0) return -1;
    return (int64_t)bin_layout(m, (int64_t)nx * nx, boxes).bytes;
}

#define ID11B_BINS_DISPATCH(FN, ...)                                                        \
    (sums ? (ntol == 1   ? FN<1, true>(__VA_ARGS__)                                         \
             : ntol == 2 ? FN<2, true>(__VA_ARGS__)                                         \
             : ntol == 3 ? FN<3, true>(__VA_ARGS__)                                         \
                         : FN<4, true>(__VA_ARGS__))                                        \
          : (ntol == 1   ? FN<1, false>(__VA_ARGS__)                                        \
             : ntol == 2 ? FN<2, false>(__VA_ARGS__)                                        \
             : ntol == 3 ? FN<3, false>(__VA_ARGS__)                                        \
                         : FN<4, false>(__VA_ARGS__)))

// What a join launch of the binned pipeline needs (one range of UBIs).
struct JoinLaunch {
    int grid;
    size_t smem;
    bool ranked;
    const uint64_t* recs;
    const int* rstart;
    int nrows, nhalo;
    BinInfo* info;
    const float4* packs;
    Header* H;
    const int* start;
    const double* gs;
    const float4* g4;
    const JoinParams* P;
};

// The binned pipeline shared by scoring and assignment: the counting
// enumeration, the UBI ranges that fit the workspace, the join's band and
// region; then for each pass, for each range, the box records (written again
// only when there are several ranges) and join(pass, launch), and after the
// ranges after(pass, fallback list, its length, g outside the regular range,
// ...).  ctas(smem, ranked): resident join CTAs per SM.  P.fix is T.fix; the
// assignment's fields of P are set by the caller's P0.
template <class Ctas, class Join, class After>
static int bins_pipeline(const double* ubis, int64_t m, int64_t n, int32_t nx, int32_t xsub,
                         const void* gridbuf, const Tols& T, int ntol, double tmax, void* ws,
                         int64_t ws_bytes, cudaStream_t st, int passes, const JoinParams& P0,
                         Ctas ctas, Join join, After after) {
    const int nrows = nx * nx;
    const int nxx = nx * xsub;
    const int nblk = (nrows + kRowBlock - 1) / kRowBlock;
    if (nblk > kMaxBlocks || nxx > kMaxNxx) return ID11B_ERR_SIZE;  // use id11b_dev_score_grid
    // the largest box capacity the workspace holds
    const BinLayout L0 = bin_layout(m, nrows, 0);
    if (ws_bytes < (int64_t)L0.bytes) return ID11B_ERR_SIZE;
    int64_t cap = (ws_bytes - (int64_t)L0.bytes) / (int64_t)(2 * sizeof(uint64_t));
    while (cap > 0 && (int64_t)bin_layout(m, nrows, cap).bytes > ws_bytes) cap -= 1 + cap / 1024;
    if (cap > INT32_MAX - 1) cap = INT32_MAX - 1;
    const BinLayout B = bin_layout(m, nrows, cap);
    const Layout L = layout(n, (int64_t)nrows * nxx);
    char* g = (char*)gridbuf;
    Header* H = (Header*)g;
    const int* start = (const int*)(g + L.start);
    const double* gs = (const double*)(g + L.g);
    const float4* g4 = (const float4*)(g + L.g4);
    char* w = (char*)ws;
    BinInfo* info = (BinInfo*)(w + B.info);
    float4* packs = (float4*)(w + B.packs);
    int* cnt_ubi = (int*)(w + B.cnt_ubi);
    int* fallback = (int*)(w + B.fallback);
    int* cta_blk = (int*)(w + B.cta_blk);
    int* blktot = (int*)(w + B.blktot);
    int* blkstart = (int*)(w + B.blkstart);
    int* rstart = (int*)(w + B.rstart);
    int* tot = (int*)(w + B.tot);
    uint64_t* tmp = (uint64_t*)(w + B.tmp);
    uint64_t* recs = (uint64_t*)(w + B.recs);
    ID11B_CHECK(cudaMemsetAsync(&H->nfallback, 0, 3 * sizeof(unsigned long long), st));
    if (m == 0) return ID11B_OK;
    ID11B_CHECK(cudaMemsetAsync(info, 0, sizeof(BinInfo), st));
    // the enumeration's CTAs (same count and UBI ranges in both passes)
    static thread_local int enum_per_sm = 0;
    if (!enum_per_sm) enum_per_sm = ctas_per_sm(k_enum, kET, 0);
    const int nctas = (int)std::min<int64_t>(kMaxEnumCtas, (int64_t)num_sms() * enum_per_sm);
    auto enumerate = [&](int mode, int64_t i0, int64_t mc, int first) {
        const int64_t per = (mc + nctas - 1) / nctas;
        const int grid = (int)std::min<int64_t>(nctas, (mc + per - 1) / per);
        k_enum<<<grid, kET, 0, st>>>(mode, ubis, i0, mc, per, H, start, tmax, first, nblk, info,
                                     packs, cnt_ubi, fallback, cta_blk, blkstart, tmp, cap);
        return grid;
    };
    int egrid = enumerate(0, 0, m, 1);
    ID11B_CHECK_LAUNCH();
    // small reads back to the host: the box total (for the capacity), the
    // band's inputs, the grid header and the number of g outside the regular range
    BinInfo bi;
    Header hh;
    int nspecial = 0;
    ID11B_CHECK(cudaMemcpyAsync(&bi, info, sizeof(BinInfo), cudaMemcpyDeviceToHost, st));
    ID11B_CHECK(cudaMemcpyAsync(&hh, H, sizeof(Header), cudaMemcpyDeviceToHost, st));
    ID11B_CHECK(cudaMemcpyAsync(&nspecial, g + L.spos + sizeof(int) * (size_t)n, sizeof(int),
                                cudaMemcpyDeviceToHost, st));
    ID11B_CHECK(cudaStreamSynchronize(st));
    // UBI ranges whose boxes fit the capacity and whose indices fit a record
    std::vector<int64_t> cuts{0};
    if ((int64_t)bi.total > cap || m > (int64_t(1) << kUbiBits)) {
        std::vector<int> cu((size_t)m);
        ID11B_CHECK(cudaMemcpyAsync(cu.data(), cnt_ubi, sizeof(int) * (size_t)m,
                                    cudaMemcpyDeviceToHost, st));
        ID11B_CHECK(cudaStreamSynchronize(st));
        int64_t acc = 0;
        for (int64_t i = 0; i < m; i++) {
            if (cu[i] > cap) return ID11B_ERR_SIZE;
            if (acc + cu[i] > cap || i - cuts.back() >= (int64_t(1) << kUbiBits)) {
                cuts.push_back(i);
                acc = 0;
            }
            acc += cu[i];
        }
    }
    cuts.push_back(m);
    // the screening kernel's band (score_batch.cu) for gmax = G and the largest
    // row sum of the binned UBIs; the region geometry
    JoinParams P = P0;
    P.fix = T.fix;
    bool ranked = false;
    {
        const double G = -hh.lo;
        float smax;
        memcpy(&smax, &bi.smax_bits, sizeof(smax));
        double W;
        memcpy(&W, &bi.wmax_bits, sizeof(W));
        // the FP32 error of the screened UBI.g - hkl per component: inputs
        // rounded (2 eps S G) and three roundings, of partial sums below S G
        // (h; the subtraction of hkl is then exact where it matters) or, folded,
        // below |hkl| + S G <= S (2 G + W) (a box's centre c lies within G + W of
        // the origin in every component, and hkl = UBI.c)
        const double E = ID11B_JOIN_FOLD
                             ? kEps32 * (double)smax * (8.0 * G + 3.0 * W) * (1. + 1e-6)
                             : 6.0 * kEps32 * (double)smax * G;
        P.hmax = 0.f;
        // ascending order of tolerance (stable), unused slots last
        int ord[ID11B_MAX_TOLS];
        for (int j = 0; j < ID11B_MAX_TOLS; j++) ord[j] = j;
        std::stable_sort(ord, ord + ntol, [&](int a, int b) { return T.t[a] < T.t[b]; });
        for (int j = 0; j < ID11B_MAX_TOLS; j++) {
            const double t = T.t[ord[j]], TT = t * t;
            const double band = 1.25 * (3.0 * E * (2.0 * (t + 1e-3) + E) +
                                        4.0 * kEps32 * (TT + 0.01));
            P.lo[j] = float_rd(TT - band);
            P.hi[j] = float_ru(TT + band);
            P.t2[j] = TT;
            P.ord[j] = ord[j];
            if (j < ntol) P.hmax = fmaxf(P.hmax, P.hi[j]);
        }
        ranked = ID11B_JOIN_RANKED != 0;
        for (int j = 1; j < ntol; j++)
            ranked = ranked && P.lo[j] >= P.lo[j - 1] && P.hi[j] >= P.hi[j - 1];
        // eps: far above the FP32 rounding of the box centres' cells (about
        // 2^-23 of |c| + |lo|) and of the FP32 region bounds
        const double eps = 2e-5 * (1. + G);
        const double csx = 1.0 / hh.inv_csx;
        P.rlo = float_rd(hh.lo - W - eps);
        P.rhi = float_ru(hh.lo + W + eps);
        P.cs = (float)hh.cs;
        P.R = (int)ceil((W + 2. * eps) / hh.cs);
        P.Rx = (int)ceil((W + 2. * eps) / csx);
        P.nx = hh.nx;
        P.nxx = hh.nxx;
    }
    const int nhalo = (2 * P.R + 1) * (2 * P.R + 1);
    if (bi.total > 0 && nhalo > kMaxHalo) return ID11B_ERR_SIZE;  // cells far smaller than W
    const size_t jsmem = sizeof(uint64_t) * kBMax + 4 * sizeof(float) * kGMax +
                         4 * sizeof(int) * (size_t)(std::max(nxx, nhalo) + 1) +
                         2 * sizeof(int) * (size_t)(nhalo + 1);
    const int jgrid = num_sms() * ctas(jsmem, ranked);
    cudaEvent_t ev0 = t_join_start, ev1 = t_join_stop;
    t_join_start = t_join_stop = nullptr;
    bool ev0_done = false;
    for (int pass = 0; pass < passes; pass++) {
        for (size_t c = 0; c + 1 < cuts.size() && bi.total > 0; c++) {
            const int64_t i0 = cuts[c], mc = cuts[c + 1] - cuts[c];
            // one range keeps its records from pass to pass
            if (pass == 0 || cuts.size() > 2) {
                if (cuts.size() > 2) {
                    egrid = enumerate(0, i0, mc, 0);
                    ID11B_CHECK_LAUNCH();
                }
                k_blk_offsets<<<grid_for((int64_t)nblk * 32, kGT), kGT, 0, st>>>(cta_blk, egrid,
                                                                                nblk, blktot);
                ID11B_CHECK_LAUNCH();
                ID11B_CHECK(cudaMemsetAsync(blktot + nblk, 0, sizeof(int), st));
                int rc = scan(blktot, nblk + 1, blkstart, tot, st);
                if (rc) return rc;
                enumerate(1, i0, mc, 0);
                ID11B_CHECK_LAUNCH();
                k_rowsplit<<<(unsigned)std::min(nblk, num_sms() * kRSPerSM), kRS, 0, st>>>(
                    tmp, blkstart, nblk, nrows, rstart, recs);
                ID11B_CHECK_LAUNCH();
            }
            ID11B_CHECK(cudaMemsetAsync(&info->next_row, 0, sizeof(int), st));
            P.i0 = i0;
            if (ev0 && !ev0_done) {
                ID11B_CHECK(cudaEventRecord(ev0, st));
                ev0_done = true;
            }
            const int rc = join(pass, JoinLaunch{jgrid, jsmem, ranked, recs, rstart, nrows, nhalo,
                                                 info, packs, H, start, gs, g4, &P});
            if (rc) return rc;
        }
        if (ev1 && pass == passes - 1) {
            if (!ev0_done) ID11B_CHECK(cudaEventRecord(ev0, st));
            ID11B_CHECK(cudaEventRecord(ev1, st));
        }
        const int rc = after(pass, fallback, (int)bi.nfallback, nspecial, H, start, gs,
                             (const int*)(g + L.spec), (const int*)(g + L.spos) + n);
        if (rc) return rc;
    }
    return ID11B_OK;
}

extern "C" int id11b_dev_score_grid_bins(const double* ubis, int64_t m, const double* gv,
                                         int64_t n, int32_t nx, int32_t xsub,
                                         const void* gridbuf, const double* tols_host, int ntol,
                                         int32_t* counts, double* sums, void* ws,
                                         int64_t ws_bytes, void* stream) {
    if (!tols_host || ntol < 1 || ntol > ID11B_MAX_TOLS || m < 0 || n < 0 ||
        !grid_dims_ok(nx, xsub) || !gridbuf || !ws || (m > 0 && (!ubis || !counts)) ||
        (n > 0 && !gv))
        return ID11B_ERR_ARG;
    Tols T;
    double tmax = 0.;
    for (int j = 0; j < ID11B_MAX_TOLS; j++) T.t[j] = j < ntol ? tols_host[j] : 0.;
    for (int j = 0; j < ntol; j++) {
        if (!(tols_host[j] >= 0.) || !(tols_host[j] < kTolLimit)) return ID11B_ERR_ARG;
        tmax = fmax(tmax, tols_host[j]);
    }
    T.fix = id11b::fixsum_scale(n, tmax);
    if (((uintptr_t)gridbuf & 255) || ((uintptr_t)ws & 255)) return ID11B_ERR_ALIGN;
    if (m > INT32_MAX - 1) return ID11B_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    if (m > 0) {
        ID11B_CHECK(cudaMemsetAsync(counts, 0, sizeof(int32_t) * (size_t)(m * ntol), st));
        if (sums) ID11B_CHECK(cudaMemsetAsync(sums, 0, sizeof(double) * (size_t)(m * ntol), st));
    }
    JoinParams P0 = {};
    const int rc = bins_pipeline(
        ubis, m, n, nx, xsub, gridbuf, T, ntol, tmax, ws, ws_bytes, st, 1, P0,
        [&](size_t smem, bool ranked) { return ID11B_BINS_DISPATCH(join_ctas, smem, ranked); },
        [&](int, const JoinLaunch& J) {
            return ID11B_BINS_DISPATCH(launch_join, J.grid, J.smem, J.ranked, J.recs, J.rstart,
                                       J.nrows, J.nhalo, J.info, J.packs, ubis, J.H, J.start,
                                       J.gs, J.g4, *J.P, counts, sums, st);
        },
        [&](int, const int* fallback, int nfallback, int nspecial, Header* H, const int* start,
            const double* gs, const int* special, const int* nspec) {
            return ID11B_BINS_DISPATCH(launch_rest, ubis, m, fallback, nfallback, H, start, gs,
                                       gv, special, nspec, nspecial > 0, T, counts, sums, st);
        });
    if (rc) return rc;
    if (m == 0) return ID11B_OK;
    return id11b_fixsum_finish(sums, m * ntol, T.fix, st);
}

// Both passes of the batched assignment (id11b_dev_assign_grid_pass 0 and 1
// over all m grains) through the binned join.  best and lab as pass -1 leaves
// them; apply id11b_dev_assign_grid_final afterwards (winners, resets and the
// g outside the regular range).  Every (grain, g) pair the FP32 screen cannot
// exclude from tol^2 is evaluated in the reference's FP64 arithmetic under
// the g's own rounded hkl, so best and lab end as the lookup passes leave them.
extern "C" int id11b_dev_assign_grid_bins(const double* ubis, int64_t m, const double* gv,
                                          int64_t n, int32_t nx, int32_t xsub,
                                          const void* gridbuf, double tol, const double* drlv2,
                                          uint64_t* best, int32_t* lab, void* ws,
                                          int64_t ws_bytes, void* stream) {
    if (m < 0 || n < 0 || !grid_dims_ok(nx, xsub) || !gridbuf || !ws || !best || !lab ||
        (m > 0 && !ubis) || (n > 0 && (!gv || !drlv2)) || !(tol >= 0.) || !(tol < kTolLimit))
        return ID11B_ERR_ARG;
    if (((uintptr_t)gridbuf & 255) || ((uintptr_t)ws & 255)) return ID11B_ERR_ALIGN;
    if (m > INT32_MAX - 1) return ID11B_ERR_SIZE;
    if (m == 0 || n == 0) return ID11B_OK;
    Tols T;
    for (int j = 0; j < ID11B_MAX_TOLS; j++) T.t[j] = j == 0 ? tol : 0.;
    T.fix = 0.;
    cudaStream_t st = (cudaStream_t)stream;
    const Layout L = layout(n, (int64_t)nx * nx * nx * xsub);
    const int* gidx = (const int*)((const char*)gridbuf + L.idx);
    unsigned long long* bst = (unsigned long long*)best;
    JoinParams P0 = {};
    P0.gidx = gidx;
    P0.d0 = drlv2;
    P0.best = bst;
    P0.lab = lab;
    return bins_pipeline(
        ubis, m, n, nx, xsub, gridbuf, T, 1, tol, ws, ws_bytes, st, 2, P0,
        [&](size_t smem, bool) { return ctas_per_sm(k_join<1, true, false, 1>, kJT, smem); },
        [&](int pass, const JoinLaunch& J) {
            if (pass == 0)
                return launch_join_k<1, true, false, 1>(J.grid, J.smem, J.recs, J.rstart, J.nrows,
                                                        J.nhalo, J.info, J.packs, ubis, J.H,
                                                        J.start, J.gs, J.g4, *J.P, nullptr,
                                                        nullptr, st);
            return launch_join_k<1, true, false, 2>(J.grid, J.smem, J.recs, J.rstart, J.nrows,
                                                    J.nhalo, J.info, J.packs, ubis, J.H, J.start,
                                                    J.gs, J.g4, *J.P, nullptr, nullptr, st);
        },
        [&](int pass, const int* fallback, int nfallback, int, Header* H, const int* start,
            const double* gs, const int*, const int*) {
            if (nfallback > 0) {
                const int64_t warps = (int64_t)nfallback * kFallbackParts;
                const unsigned blocks = (unsigned)((warps + kBW - 1) / kBW);
                if (pass == 0)
                    k_assign_fallback<0><<<blocks, kBT, 0, st>>>(
                        ubis, fallback, nfallback, H, start, gs, gidx, tol, drlv2, bst, lab);
                else
                    k_assign_fallback<1><<<blocks, kBT, 0, st>>>(
                        ubis, fallback, nfallback, H, start, gs, gidx, tol, drlv2, bst, lab);
                ID11B_CHECK_LAUNCH();
            }
            return ID11B_OK;
        });
}
