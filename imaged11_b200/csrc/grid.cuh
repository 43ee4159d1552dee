// Reciprocal-space cell index over the g-vectors: layout, cell coordinates
// and the per-UBI query plan, shared by the lookup scorer (gvec_grid.cu) and
// the binned scorer (grid_bins.cu).
#pragma once
#include <math.h>
#include <limits.h>
#include <stdint.h>

#include "common.cuh"

namespace id11b {
namespace grid {

constexpr int kGT = 256;           // threads per CTA of the build kernels
constexpr int kScanT = 1024;       // scan CTA
constexpr int kScanPer = 4 * kScanT;
constexpr double kGLimit = 1024.0;  // regular g: finite, every |g_j| <= 1024
constexpr double kHklMargin = 1e-6;
constexpr double kMaxCond = 1e6;
constexpr int kMaxParts = 64;

struct Header {
    double lo, cs, inv_cs;  // cube [lo, lo + nx*cs)^3; y and z cells of side cs
    double inv_csx;         // x cells: side cs / xsub (nxx = nx * xsub of them)
    double rmax;            // max |g| over regular g (rounded up)
    int64_t ncells;
    int64_t n;
    int32_t nx;
    int32_t nxx;
    unsigned long long nfallback;  // UBIs scored by the plain scan (last call)
    unsigned long long ntested;    // (UBI, g) pairs evaluated in FP64 (last call)
    unsigned long long npairs;     // (box, g) pairs screened in FP32 (last binned call)
};

struct Tols {
    double t[ID11B_MAX_TOLS];
    double fix;  // fixed-point scale of order-free sums (fixsum_scale)
};

__host__ __device__ inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// Grid buffer: header | cnt[ncells+1] | start[ncells+1] | g[n][3] | gidx[n] |
// flag[n+1] | spos[n+1] | spec[n] | scan totals
struct Layout {
    size_t header, cnt, start, g, idx, flag, spos, spec, tot, g4, bytes;
};

__host__ __device__ inline Layout layout(int64_t n, int64_t ncells) {
    Layout L;
    const size_t nn = (size_t)(n > 0 ? n : 1);
    const int64_t big = ncells + 1 > n + 1 ? ncells + 1 : n + 1;
    size_t o = 0;
    L.header = o; o = al256(o + sizeof(Header));
    L.cnt = o;    o = al256(o + sizeof(int) * (size_t)(ncells + 1));
    L.start = o;  o = al256(o + sizeof(int) * (size_t)(ncells + 1));
    L.g = o;      o = al256(o + sizeof(double) * 3 * nn);
    L.idx = o;    o = al256(o + sizeof(int) * nn);
    L.flag = o;   o = al256(o + sizeof(int) * (nn + 1));
    L.spos = o;   o = al256(o + sizeof(int) * (nn + 1));
    L.spec = o;   o = al256(o + sizeof(int) * nn);
    L.tot = o;    o = al256(o + sizeof(int) * (size_t)((big + kScanPer - 1) / kScanPer + 1));
    L.g4 = o;     o = al256(o + sizeof(float) * 4 * nn);  // FP32 copy of the sorted g
    L.bytes = o;
    return L;
}

__device__ __forceinline__ bool regular(double a, double b, double c) {
    double m = fmax(fabs(a), fmax(fabs(b), fabs(c)));
    return isfinite(a) && isfinite(b) && isfinite(c) && m <= kGLimit;
}

// A g the index holds in a cell: regular, inside the cube [lo, -lo]^3 and
// within rmax of the origin.  Every scorer enumerates the boxes that meet that
// cube and that ball only, so a g outside the bounds the index was built for
// (a caller's smaller gmax or rmax, or g moved before a rebuild into the same
// shape) joins the list of g scored by a plain scan instead of a cell no box
// reaches.  The bounds of id11b_dev_gvec_bounds are rounded up, so they hold
// every regular g they were taken from.
__device__ __forceinline__ bool indexed(double a, double b, double c, const Header& H) {
    return regular(a, b, c) && fmax(fabs(a), fmax(fabs(b), fabs(c))) <= -H.lo &&
           a * a + b * b + c * c <= H.rmax * H.rmax;
}

// Monotone in x (RN subtraction and multiplication by a positive constant,
// clamp, truncation of a non-negative value); NaN must not reach it.
__device__ __forceinline__ int coord(double x, const Header& H) {
    double f = __dmul_rn(__dsub_rn(x, H.lo), H.inv_cs);
    f = fmin(fmax(f, 0.0), (double)(H.nx - 1));
    return (int)f;
}

// x is cut finer (a row of cells is one contiguous range whatever its length,
// so finer x cells cost memory, not lookups)
__device__ __forceinline__ int coord_x(double x, const Header& H) {
    double f = __dmul_rn(__dsub_rn(x, H.lo), H.inv_csx);
    f = fmin(fmax(f, 0.0), (double)(H.nxx - 1));
    return (int)f;
}

__device__ __forceinline__ int64_t cell_of(double a, double b, double c, const Header& H) {
    return ((int64_t)coord(c, H) * H.nx + coord(b, H)) * H.nxx + coord_x(a, H);
}

// ------------------------------------------------------------- per UBI ----
// Query plan of one UBI (uniform across the warp).
struct Plan {
    double ub[9];      // UBI^-1
    double w[3];       // box half-widths
    int64_t lo[3];     // hkl box
    int64_t nh[3];
    bool ok;           // false: plain scan of every regular g
};

__device__ __forceinline__ Plan make_plan(const double u[9], double tmax, const Header& H,
                                          int64_t nreg) {
    Plan P;
    bool ok = true;
#pragma unroll
    for (int e = 0; e < 9; e++) ok = ok && isfinite(u[e]);
    const double c00 = u[4] * u[8] - u[5] * u[7], c01 = u[5] * u[6] - u[3] * u[8],
                 c02 = u[3] * u[7] - u[4] * u[6];
    const double det = u[0] * c00 + u[1] * c01 + u[2] * c02;
    ok = ok && isfinite(det) && det != 0.;
    const double id = 1.0 / det;
    P.ub[0] = c00 * id;
    P.ub[1] = (u[2] * u[7] - u[1] * u[8]) * id;
    P.ub[2] = (u[1] * u[5] - u[2] * u[4]) * id;
    P.ub[3] = c01 * id;
    P.ub[4] = (u[0] * u[8] - u[2] * u[6]) * id;
    P.ub[5] = (u[2] * u[3] - u[0] * u[5]) * id;
    P.ub[6] = c02 * id;
    P.ub[7] = (u[1] * u[6] - u[0] * u[7]) * id;
    P.ub[8] = (u[0] * u[4] - u[1] * u[3]) * id;
    double nu = 0., nb = 0.;
#pragma unroll
    for (int e = 0; e < 9; e++) {
        nu += u[e] * u[e];
        nb += P.ub[e] * P.ub[e];
        ok = ok && isfinite(P.ub[e]);
    }
    ok = ok && sqrt(nu) * sqrt(nb) <= kMaxCond;
    const double G = -H.lo;  // every regular g lies in [-G, G]^3
    double total = 1.;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const double s = fabs(u[3 * r]) + fabs(u[3 * r + 1]) + fabs(u[3 * r + 2]);
        const double hm = s * G + 1.0;
        ok = ok && hm < 1e6;
        const double l = floor(-hm), h = ceil(hm);
        P.lo[r] = ok ? (int64_t)l : 0;
        P.nh[r] = ok ? (int64_t)(h - l) + 1 : 1;
        total *= (h - l) + 1.;
        P.w[r] = (tmax + kHklMargin) *
                 sqrt(P.ub[3 * r] * P.ub[3 * r] + P.ub[3 * r + 1] * P.ub[3 * r + 1] +
                      P.ub[3 * r + 2] * P.ub[3 * r + 2]) * (1. + 1e-9);
        ok = ok && isfinite(P.w[r]);
    }
    ok = ok && total <= (double)nreg;  // more candidate hkl than g: the plain scan is cheaper
    P.ok = ok;
    return P;
}

struct WarpPlan {
    double u[9], ub[9], w[3];
    int lo[3], nh[3];
};

__device__ __forceinline__ unsigned long long pack_hkl(int h, int k, int l) {
    return ((unsigned long long)(unsigned)(h + (1 << 20)) << 42) |
           ((unsigned long long)(unsigned)(k + (1 << 20)) << 21) |
           (unsigned long long)(unsigned)(l + (1 << 20));
}

__device__ __forceinline__ void unpack_hkl(unsigned long long q, double hkl[3]) {
    hkl[0] = (double)((int)((q >> 42) & 0x1fffff) - (1 << 20));
    hkl[1] = (double)((int)((q >> 21) & 0x1fffff) - (1 << 20));
    hkl[2] = (double)((int)(q & 0x1fffff) - (1 << 20));
}

// Largest lane j with excl_j <= f, excl non-decreasing over lanes, excl_0 = 0.
__device__ __forceinline__ int owner(int excl, int f) {
    int j = 0;
#pragma unroll
    for (int st = 16; st > 0; st >>= 1) {
        const int v = __shfl_sync(0xffffffffu, excl, j + st);
        if (v <= f) j += st;
    }
    return j;
}

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int& total) {
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    total = __shfl_sync(0xffffffffu, incl, 31);
    return incl - v;
}

// Plan of UBI i into the warp's shared slot; false: plain scan instead.
__device__ __forceinline__ bool setup_plan(volatile WarpPlan* wp, const double* __restrict__ ubis,
                                           int64_t i, double tmax, const Header& H,
                                           int64_t nreg, int lane) {
    double u[9];
#pragma unroll
    for (int e = 0; e < 9; e++) u[e] = ubis[9 * i + e];
    const Plan P = make_plan(u, tmax, H, nreg);
    const bool ok = P.ok && P.nh[0] < (1 << 20) && P.nh[1] < (1 << 20) && P.nh[2] < (1 << 20);
    if (lane == 0) {
#pragma unroll
        for (int e = 0; e < 9; e++) {
            wp->u[e] = u[e];
            wp->ub[e] = P.ub[e];
        }
#pragma unroll
        for (int r = 0; r < 3; r++) {
            wp->w[r] = P.w[r];
            wp->lo[r] = ok ? (int)P.lo[r] : 0;
            wp->nh[r] = ok ? (int)P.nh[r] : 0;
        }
    }
    __syncwarp();
    return ok;
}

// Euclidean norms of columns 0 and 1 of the plan's UB (the h and k directions).
__device__ __forceinline__ void ub_column_norms(const volatile WarpPlan* wp, double& n0,
                                                double& n1) {
    n0 = sqrt(wp->ub[0] * wp->ub[0] + wp->ub[3] * wp->ub[3] + wp->ub[6] * wp->ub[6]);
    n1 = sqrt(wp->ub[1] * wp->ub[1] + wp->ub[4] * wp->ub[4] + wp->ub[7] * wp->ub[7]);
}

// The l of the (h, k) column whose lattice point UB.(h, k, l) lies within R of
// the origin, clipped to the plan's l range: [l0, l0 + len), len = 0 if none.
// The column is the line a + l b (a = UB.(h, k, 0), b = UB's column 2); its
// l range, the roots of |a + l b|^2 = R^2, is taken in FP64 with every
// rounding bounded, so no lattice point inside the ball is left out:
//   a is rounded by at most 2 eps (|h| n0 + |k| n1), which is added to R;
//   the discriminant ab^2 - bb (aa - R^2) by at most 17 eps bb aa + 9 eps bb R^2
//   (ab^2 <= aa bb), and 4e-15 bb (aa + R^2) (> 20 eps) is added to it, so a
//   column that meets the ball is never dropped at a tangent;
//   each root by at most 9 eps (|ab| + sq) / bb (sum, product, reciprocal,
//   and |root| <= (|ab| + sq) / bb), and the range takes the integers within
//   2e-15 (|ab| + sq) / bb + 1e-6 of the roots.
// So the range holds the lattice points of the ball and few others: widening
// each end by a whole l instead ran a quarter more candidates through the
// binned join's enumeration (1.33 x on 20,000 trial UBIs of 1.1M g: binned
// scoring 3.05 -> 2.96 ms, the same boxes).
__device__ __forceinline__ void column_l_range(const volatile WarpPlan* wp, double n0, double n1,
                                               int h, int k, double R, int& l0, int& len) {
    const double bx = wp->ub[2], by = wp->ub[5], bz = wp->ub[8];
    const double bb = bx * bx + by * by + bz * bz;
    const double ax = wp->ub[0] * h + wp->ub[1] * k, ay = wp->ub[3] * h + wp->ub[4] * k,
                 az = wp->ub[6] * h + wp->ub[7] * k;
    const double ab = ax * bx + ay * by + az * bz;
    const double aa = ax * ax + ay * ay + az * az;
    const double llo = (double)wp->lo[2], lhi = (double)(wp->lo[2] + wp->nh[2] - 1);
    l0 = 0;
    len = 0;
    const double Rc = R + 1e-15 * (fabs((double)h) * n0 + fabs((double)k) * n1);
    const double r2 = Rc * Rc;
    const double disc = ab * ab - bb * (aa - r2) + 4e-15 * bb * (aa + r2);
    if (disc >= 0.) {
        const double sq = sqrt(disc), ib = 1.0 / bb;
        const double m = 2e-15 * (fabs(ab) + sq) * ib + 1e-6;
        const double la = fmax(ceil((-ab - sq) * ib - m), llo);
        const double lb = fmin(floor((-ab + sq) * ib + m), lhi);
        if (la <= lb) {
            l0 = (int)la;
            len = (int)(lb - la) + 1;
        }
    }
}

// Every hkl whose box [UB.hkl - w, UB.hkl + w] can reach a regular g (inside
// the data cube and within rmax of the origin), for the (h, k) columns of work
// item `part` of `parts`.  32 (h, k) columns at a time, each lane solving for
// the range of l whose lattice point lies within rmax + |w| of the origin, the
// 32 ranges flattened across the warp.  emit(pass, h, k, l, c) is called by
// every lane of the warp together (warp-synchronous); pass says whether the
// lane holds a box, c is its centre UB.hkl.
template <class Emit>
__device__ __forceinline__ void enumerate_boxes(const volatile WarpPlan* wp, int part, int parts,
                                                int lane, const Header& H, Emit& emit) {
    const int nh0 = wp->nh[0];
    const int64_t nhk = (int64_t)nh0 * wp->nh[1];
    double n0, n1;
    ub_column_norms(wp, n0, n1);
    for (int64_t hb = (int64_t)part * 32; hb < nhk; hb += 32 * (int64_t)parts) {
        const int64_t hk = hb + lane;
        int len = 0, l0 = 0, h = 0, k = 0;
        if (hk < nhk) {
            h = wp->lo[0] + (int)(hk % nh0);
            k = wp->lo[1] + (int)(hk / nh0);
            const double R = (H.rmax + sqrt(wp->w[0] * wp->w[0] + wp->w[1] * wp->w[1] +
                                            wp->w[2] * wp->w[2])) * (1. + 1e-9) + 1e-12;
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
            bool pass = false;
            double c[3] = {0., 0., 0.};
            if (f < total) {
                const double hkl[3] = {(double)hj, (double)kj, (double)lj};
                bool in = true;
                double d2 = 0.;
                const double G = -H.lo;
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    c[r] = wp->ub[3 * r] * hkl[0] + wp->ub[3 * r + 1] * hkl[1] +
                           wp->ub[3 * r + 2] * hkl[2];
                    const double wr = wp->w[r];
                    in = in && (c[r] - wr <= G) && (c[r] + wr >= -G);
                    const double e = fmax(fabs(c[r]) - wr, 0.);
                    d2 += e * e;
                }
                pass = in && d2 <= H.rmax * H.rmax * (1. + 1e-9);
            }
            emit(pass, hj, kj, lj, c);
        }
    }
}

// host helpers defined in gvec_grid.cu
int num_sms();
unsigned grid_for(int64_t items, int per);
int scan(const int* x, int64_t len, int* y, int* tot, cudaStream_t st);
int score_parts(int64_t m);
bool grid_dims_ok(int32_t nx, int32_t xsub);

}  // namespace grid
}  // namespace id11b
