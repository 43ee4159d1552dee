// Reciprocal-space cell index over the g-vectors, and scoring by hkl lookup.
//
// The reference's score() (ImageD11 src/closest.c:227-248) tests every g
// against a UBI.  A g-vector is counted iff |UBI.g - round(UBI.g)|^2 < tol^2,
// i.e. iff it lies inside the ellipsoid of radius tol (in hkl units) around
// UB.hkl for hkl = round(UBI.g), UB = UBI^-1.  This file bins the g-vectors
// into a uniform grid of cells (square in y and z, x cut finer; x fastest, so
// a row of cells along x is one contiguous range of the cell-sorted g), then
// for each UBI enumerates
// the integer hkl whose ellipsoid can reach the data and tests only the g in
// the cells overlapping a conservative bounding box of that ellipsoid.  Every
// tested pair is evaluated with the reference's exact FP64 arithmetic
// (drlv2_exact) and counted only under its own hkl (ih == hkl), so each g is
// counted at most once and exactly when the reference counts it.
//
// Conservativeness: with d = UBI.g - hkl, g = UB.hkl + UB.d, so
// |g_j - (UB.hkl)_j| <= |d| * ||row j of UB||.  The box half-widths use
// (tol + 1e-6) in place of |d|: 1e-6 in hkl units is far above the FP64
// rounding of h, of UB = inv(UBI) (condition number capped at 1e6) and of
// UB.hkl (|hkl| capped).  Cell coordinates come from one monotone function
// of a coordinate, used by the build and the query alike, so a g inside the
// box is always inside the scanned cells.  UBIs outside the caps (non-finite,
// singular, ill-conditioned, or with more candidate hkl than g-vectors) are
// scored by a plain scan of every regular g; g-vectors outside the regular
// range (non-finite or |g_j| > 1024), or outside the cube and ball of radius
// rmax the index was built for, by a scan over that list.
#include "grid.cuh"

namespace id11b {
namespace grid {

// scoring CTAs: warps (one per work item) and the resident CTAs per SM the
// register budget is compiled for.  Occupancy decides the speed of the
// latency-bound lookups: 20,000 UBIs x 1.1M g on B200 took 13.0 ms at 8 warps
// x 2 CTAs (107 registers), 9.9 ms at 8 x 3, 9.5 ms at 2 x 12, 9.4 ms at
// 1 x 24 (80 registers) and 8.0 ms at 1 x 32 (64 registers, a few spilled).
#ifndef ID11B_GRID_WARPS
#define ID11B_GRID_WARPS 1
#endif
#ifndef ID11B_GRID_MINB
#define ID11B_GRID_MINB 32
#endif
constexpr int kSW = ID11B_GRID_WARPS;
constexpr int kST = 32 * kSW;

// ------------------------------------------------------------------ build --
// max |g_j| and max |g| over regular g, as float bits rounded up
__global__ void __launch_bounds__(kGT)
k_bounds(const double* __restrict__ gv, int64_t n, unsigned int* __restrict__ out) {
    float gm = 0.f, rm = 0.f;
    for (int64_t k = (int64_t)blockIdx.x * kGT + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * kGT) {
        double a = gv[3 * k], b = gv[3 * k + 1], c = gv[3 * k + 2];
        if (!regular(a, b, c)) continue;
        gm = fmaxf(gm, __double2float_ru(fmax(fabs(a), fmax(fabs(b), fabs(c)))));
        rm = fmaxf(rm, __double2float_ru(sqrt(a * a + b * b + c * c) * (1. + 1e-12)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        gm = fmaxf(gm, __shfl_xor_sync(0xffffffffu, gm, o));
        rm = fmaxf(rm, __shfl_xor_sync(0xffffffffu, rm, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, __float_as_uint(gm));
        atomicMax(out + 1, __float_as_uint(rm));
    }
}

__global__ void __launch_bounds__(kGT)
k_count(const double* __restrict__ gv, int64_t n, const Header* __restrict__ Hp,
        int* __restrict__ cnt, int* __restrict__ flag) {
    const Header H = *Hp;
    for (int64_t k = (int64_t)blockIdx.x * kGT + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * kGT) {
        double a = gv[3 * k], b = gv[3 * k + 1], c = gv[3 * k + 2];
        const bool reg = indexed(a, b, c, H);
        flag[k] = reg ? 0 : 1;
        if (reg) atomicAdd(cnt + cell_of(a, b, c, H), 1);
    }
}

// exclusive scan of x[0..len) into y, CTA totals into tot (pass 1)
__global__ void __launch_bounds__(kScanT)
k_scan_local(const int* __restrict__ x, int64_t len, int* __restrict__ y, int* __restrict__ tot) {
    __shared__ int s_w[kScanT / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanPer + 4 * threadIdx.x;
    int v[4], sum = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        v[q] = base + q < len ? x[base + q] : 0;
        sum += v[q];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int w = s_w[lane];
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        s_w[lane] = wi - w;  // exclusive over warps
        if (lane == 31) tot[blockIdx.x] = wi;
    }
    __syncthreads();
    int run = s_w[wid] + incl - sum;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (base + q < len) y[base + q] = run;
        run += v[q];
    }
}

// exclusive scan of the CTA totals in place (one CTA, sequential chunks)
__global__ void __launch_bounds__(kScanT) k_scan_totals(int* __restrict__ tot, int nb) {
    __shared__ int s_w[kScanT / 32];
    __shared__ int s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int b0 = 0; b0 < nb; b0 += kScanT) {
        const int i = b0 + threadIdx.x;
        const int v = i < nb ? tot[i] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) s_w[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            int w = s_w[lane], wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += t;
            }
            s_w[lane] = wi - w;
        }
        __syncthreads();
        const int carry = s_carry;
        if (i < nb) tot[i] = carry + s_w[wid] + incl - v;
        __syncthreads();
        if (threadIdx.x == kScanT - 1) s_carry = carry + s_w[wid] + incl;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kScanT)
k_scan_add(int* __restrict__ y, int64_t len, const int* __restrict__ tot) {
    const int64_t base = (int64_t)blockIdx.x * kScanPer + 4 * threadIdx.x;
    const int add = tot[blockIdx.x];
#pragma unroll
    for (int q = 0; q < 4; q++)
        if (base + q < len) y[base + q] += add;
}

__global__ void __launch_bounds__(kGT)
k_scatter(const double* __restrict__ gv, int64_t n, const Header* __restrict__ Hp,
          const int* __restrict__ start, int* __restrict__ cursor, double* __restrict__ gs,
          int* __restrict__ gidx, const int* __restrict__ spos, int* __restrict__ spec) {
    const Header H = *Hp;
    for (int64_t k = (int64_t)blockIdx.x * kGT + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * kGT) {
        double a = gv[3 * k], b = gv[3 * k + 1], c = gv[3 * k + 2];
        if (!indexed(a, b, c, H)) {
            spec[spos[k]] = (int)k;
            continue;
        }
        const int64_t cid = cell_of(a, b, c, H);
        const int p = start[cid] + atomicAdd(cursor + cid, 1);
        gs[3 * (int64_t)p] = a;
        gs[3 * (int64_t)p + 1] = b;
        gs[3 * (int64_t)p + 2] = c;
        gidx[p] = (int)k;
    }
}

// Each cell's entries ordered by original index (the layout, and so every
// result, does not depend on the order the scatter's atomics ran in) and the
// FP32 (round to nearest) copy of the sorted g for staging, with the g's x cell
// (as int bits) in w.  One thread per position; the thread at a cell's first
// position sorts the cell and writes its copies.  Threads at the cell's other
// positions may read coordinates the sort is moving, but every value there is
// a coordinate of a g of that cell, so they find the same cell and skip it.
__global__ void __launch_bounds__(kGT)
k_sort_cells_f32(const int* __restrict__ start, const Header* __restrict__ Hp, double* gs,
                 int* gidx, float4* __restrict__ g4) {
    const Header H = *Hp;
    const int64_t nreg = start[H.ncells];
    for (int64_t p = (int64_t)blockIdx.x * kGT + threadIdx.x; p < nreg;
         p += (int64_t)gridDim.x * kGT) {
        const int64_t c = cell_of(gs[3 * p], gs[3 * p + 1], gs[3 * p + 2], H);
        const int a = start[c];
        if (a != p) continue;
        const int b = start[c + 1];
        for (int i = a + 1; i < b; i++) {
            const int key = gidx[i];
            const double x = gs[3 * (int64_t)i], y = gs[3 * (int64_t)i + 1],
                         z = gs[3 * (int64_t)i + 2];
            int j = i - 1;
            while (j >= a && gidx[j] > key) {
                gidx[j + 1] = gidx[j];
                gs[3 * (int64_t)j + 3] = gs[3 * (int64_t)j];
                gs[3 * (int64_t)j + 4] = gs[3 * (int64_t)j + 1];
                gs[3 * (int64_t)j + 5] = gs[3 * (int64_t)j + 2];
                j--;
            }
            gidx[j + 1] = key;
            gs[3 * (int64_t)j + 3] = x;
            gs[3 * (int64_t)j + 4] = y;
            gs[3 * (int64_t)j + 5] = z;
        }
        for (int64_t q = a; q < b; q++)
            g4[q] = make_float4(__double2float_rn(gs[3 * q]), __double2float_rn(gs[3 * q + 1]),
                                __double2float_rn(gs[3 * q + 2]),
                                __int_as_float(coord_x(gs[3 * q], H)));
    }
}

// Per-warp queue of hkl that reach the data.  Enumeration: 32 (h, k) columns
// at a time, each lane solving for the range of l whose lattice point lies
// within rmax + |w| of the origin (every hkl whose box can reach a regular g
// is inside it), the 32 ranges flattened across the warp; candidates passing
// the box test are queued (packed hkl) in ballot order, and whenever 32 are
// queued the warp runs the 32 lookups together (lookup_batch).  The UBI's plan
// lives in shared memory, not in registers.
constexpr int kQueue = 64;

// Per-warp scratch for one batch of up to 32 lookups.
struct Batch {
    double c[32][3];
    unsigned long long hkl[32];
    int ix0[32], ix1[32], iy0[32], ny[32], iz0[32];
    // g found inside a box, waiting for the FP64 evaluation (32 at a time)
    double cg[64][3];
    unsigned long long ch[64];
    int cp[64];
    int cn;
};

// Evaluate the first `take` waiting candidates (one per lane) in the
// reference's FP64 arithmetic, hand them to act, and drop them from the list.
template <class Act>
__device__ __forceinline__ void eval_candidates(const volatile WarpPlan* wp, Batch* bt, int take,
                                                int lane, Act& act) {
    if (lane < take) {
        double u[9], ih[3], hkl[3];
#pragma unroll
        for (int e = 0; e < 9; e++) u[e] = wp->u[e];
        const double g[3] = {bt->cg[lane][0], bt->cg[lane][1], bt->cg[lane][2]};
        const double sv = drlv2_exact(u, g[0], g[1], g[2], ih);
        unpack_hkl(bt->ch[lane], hkl);
        act(bt->cp[lane], sv, ih[0] == hkl[0] && ih[1] == hkl[1] && ih[2] == hkl[2], g, ih);
    }
    __syncwarp();
    const int rest = bt->cn - take;  // < 32
    double a = 0., b = 0., c = 0.;
    unsigned long long h = 0;
    int q = 0;
    if (lane < rest) {
        a = bt->cg[take + lane][0];
        b = bt->cg[take + lane][1];
        c = bt->cg[take + lane][2];
        h = bt->ch[take + lane];
        q = bt->cp[take + lane];
    }
    __syncwarp();
    if (lane < rest) {
        bt->cg[lane][0] = a;
        bt->cg[lane][1] = b;
        bt->cg[lane][2] = c;
        bt->ch[lane] = h;
        bt->cp[lane] = q;
    }
    __syncwarp();
    if (lane == 0) bt->cn = rest;
    __syncwarp();
}

// The lookups of `take` queued hkl (slot = lane), warp-cooperatively: the
// cell rows of all of them are flattened across the lanes, then the g of
// each 32 rows, so the lanes stay converged whatever the per-query sizes.
// Every g inside a box is evaluated in the reference's FP64 arithmetic and
// handed to act(pos, drlv2, own, g, ih), own = (ih, the rounded h, == the
// box's hkl).
template <class Act>
__device__ __forceinline__ void lookup_batch(const volatile WarpPlan* wp, Batch* bt,
                                             const unsigned long long* q_w, int take, int lane,
                                             const Header& H, const int* __restrict__ start,
                                             const double* __restrict__ gs, Act& act) {
    int nrows = 0;
    if (lane < take) {
        const unsigned long long q = q_w[lane];
        double hkl[3], c[3];
        unpack_hkl(q, hkl);
#pragma unroll
        for (int r = 0; r < 3; r++) {
            c[r] = wp->ub[3 * r] * hkl[0] + wp->ub[3 * r + 1] * hkl[1] + wp->ub[3 * r + 2] * hkl[2];
            bt->c[lane][r] = c[r];
        }
        bt->hkl[lane] = q;
        const int iy0 = coord(c[1] - wp->w[1], H), iy1 = coord(c[1] + wp->w[1], H);
        const int iz0 = coord(c[2] - wp->w[2], H), iz1 = coord(c[2] + wp->w[2], H);
        bt->ix0[lane] = coord_x(c[0] - wp->w[0], H);
        bt->ix1[lane] = coord_x(c[0] + wp->w[0], H);
        bt->iy0[lane] = iy0;
        bt->ny[lane] = iy1 - iy0 + 1;
        bt->iz0[lane] = iz0;
        nrows = (iy1 - iy0 + 1) * (iz1 - iz0 + 1);
    }
    __syncwarp();
    int rtotal;
    const int rexcl = warp_excl_scan(nrows, lane, rtotal);
    const double w0 = wp->w[0], w1 = wp->w[1], w2 = wp->w[2];
    for (int r0 = 0; r0 < rtotal; r0 += 32) {
        const int rf = r0 + lane;
        const int qj = owner(rexcl, rf);
        const int rr = rf - __shfl_sync(0xffffffffu, rexcl, qj);
        int st = 0, len = 0;
        if (rf < rtotal) {
            const int ny = bt->ny[qj];
            const int iy = bt->iy0[qj] + rr % ny, iz = bt->iz0[qj] + rr / ny;
            const int64_t row = ((int64_t)iz * H.nx + iy) * H.nxx;
            st = __ldg(start + row + bt->ix0[qj]);
            len = __ldg(start + row + bt->ix1[qj] + 1) - st;
        }
        int gtotal;
        const int gexcl = warp_excl_scan(len, lane, gtotal);
        const int off = st - gexcl;
        for (int f0 = 0; f0 < gtotal; f0 += 32) {
            const int f = f0 + lane;
            const int rj = owner(gexcl, f);
            const int pos = f + __shfl_sync(0xffffffffu, off, rj);
            const int qq = __shfl_sync(0xffffffffu, qj, rj);
            bool inb = false;
            double g0 = 0., g1 = 0., g2 = 0.;
            if (f < gtotal) {
                g0 = __ldg(gs + 3 * (int64_t)pos);
                g1 = __ldg(gs + 3 * (int64_t)pos + 1);
                g2 = __ldg(gs + 3 * (int64_t)pos + 2);
                inb = fabs(g0 - bt->c[qq][0]) <= w0 && fabs(g1 - bt->c[qq][1]) <= w1 &&
                      fabs(g2 - bt->c[qq][2]) <= w2;
            }
            const unsigned mk = __ballot_sync(0xffffffffu, inb);
            const int cn = bt->cn;  // < 32 here
            if (inb) {
                const int slot = cn + __popc(mk & ((1u << lane) - 1u));
                bt->cg[slot][0] = g0;
                bt->cg[slot][1] = g1;
                bt->cg[slot][2] = g2;
                bt->ch[slot] = bt->hkl[qq];
                bt->cp[slot] = pos;
            }
            __syncwarp();
            if (lane == 0) bt->cn = cn + __popc(mk);
            __syncwarp();
            if (cn + __popc(mk) >= 32) eval_candidates(wp, bt, 32, lane, act);
        }
    }
    __syncwarp();
}

// Every (UBI, g) pair of work item `part` of `parts` whose drlv2 can be below
// the plan's tolerance goes to act(pos, drlv2, own, g, ih): through the hkl lookup
// when ok, else by a plain scan of the regular g (own = true: each g once).
template <class Act>
__device__ __forceinline__ void walk(volatile WarpPlan* wp, Batch* bt, unsigned long long* q_w,
                                     bool ok, int part, int parts, int lane, const Header& H,
                                     int64_t nreg, const int* __restrict__ start,
                                     const double* __restrict__ gs, Act& act) {
    if (!ok) {
        double u[9];
#pragma unroll
        for (int e = 0; e < 9; e++) u[e] = wp->u[e];
        for (int64_t f = (int64_t)part * 32 + lane; f < nreg; f += 32 * (int64_t)parts) {
            double ih[3];
            const double g[3] = {gs[3 * f], gs[3 * f + 1], gs[3 * f + 2]};
            const double s = drlv2_exact(u, g[0], g[1], g[2], ih);
            act((int)f, s, true, g, ih);
        }
        return;
    }
    int qn = 0;  // queued (uniform)
    if (lane == 0) bt->cn = 0;
    __syncwarp();
    const unsigned lt = (1u << lane) - 1u;
    auto queue = [&](bool pass, int hj, int kj, int lj, const double*) {
        const unsigned mask = __ballot_sync(0xffffffffu, pass);
        if (pass) q_w[qn + __popc(mask & lt)] = pack_hkl(hj, kj, lj);
        qn += __popc(mask);
        __syncwarp();
        if (qn >= 32) {
            lookup_batch(wp, bt, q_w, 32, lane, H, start, gs, act);
            const int rest = qn - 32;
            unsigned long long v = 0;
            if (lane < rest) v = q_w[32 + lane];
            __syncwarp();
            if (lane < rest) q_w[lane] = v;
            __syncwarp();
            qn = rest;
        }
    };
    enumerate_boxes(wp, part, parts, lane, H, queue);
    if (qn > 0) lookup_batch(wp, bt, q_w, qn, lane, H, start, gs, act);
    const int cn = bt->cn;
    if (cn > 0) eval_candidates(wp, bt, cn, lane, act);
}

template <int NT>
__global__ void __launch_bounds__(kST, ID11B_GRID_MINB)
k_score(const double* __restrict__ ubis, int64_t m, int parts, Header* __restrict__ Hp,
        const int* __restrict__ start, const double* __restrict__ gs, Tols tols,
        int* __restrict__ pcnt, double* __restrict__ psum) {
    __shared__ unsigned long long s_q[kSW][kQueue];
    __shared__ WarpPlan s_plan[kSW];
    __shared__ Batch s_batch[kSW];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t wk = ((int64_t)blockIdx.x * kST + threadIdx.x) >> 5;
    if (wk >= m * parts) return;  // uniform per warp
    const int64_t i = wk / parts;
    const int part = (int)(wk % parts);
    const Header H = *Hp;
    const int64_t nreg = start[H.ncells];
    double t2[NT];
    double tmax = 0.;
    int cnt[NT];
    double sum[NT];
#pragma unroll
    for (int j = 0; j < NT; j++) {
        tmax = fmax(tmax, tols.t[j]);
        t2[j] = tols.t[j] * tols.t[j];
        cnt[j] = 0;
        sum[j] = 0.;
    }
    unsigned long long tested = 0;
    const bool ok = setup_plan(s_plan + w, ubis, i, tmax, H, nreg, lane);
    auto act = [&](int, double s, bool own, const double*, const double*) {
        tested++;
        if (own) {
#pragma unroll
            for (int j = 0; j < NT; j++)
                if (s < t2[j]) {
                    cnt[j]++;
                    sum[j] += s;
                }
        }
    };
    walk(s_plan + w, s_batch + w, s_q[w], ok, part, parts, lane, H, nreg, start, gs, act);
    if (!ok && part == 0 && lane == 0) atomicAdd(&Hp->nfallback, 1ull);
#pragma unroll
    for (int j = 0; j < NT; j++) {
        const int cs = warp_sum(cnt[j]);
        const double ss = warp_sum(sum[j]);
        if (lane == 0) {
            pcnt[(i * parts + part) * NT + j] = cs;
            psum[(i * parts + part) * NT + j] = ss;
        }
    }
    const long long tt = warp_sum((long long)tested);
    if (lane == 0 && tt) atomicAdd(&Hp->ntested, (unsigned long long)tt);
}

// The g-vectors outside the regular range, one warp per UBI: lanes stride the
// list, fixed-tree warp sums, one slot per UBI and tolerance.
__global__ void __launch_bounds__(kGT)
k_score_special(const double* __restrict__ ubis, int64_t m, int ntol, Tols tols,
                const double* __restrict__ gv, const int* __restrict__ special,
                const int* __restrict__ nspecial, int* __restrict__ scnt,
                double* __restrict__ ssum) {
    const int64_t i = ((int64_t)blockIdx.x * kGT + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= m) return;  // uniform per warp
    int c[ID11B_MAX_TOLS] = {0, 0, 0, 0};
    double sm[ID11B_MAX_TOLS] = {0., 0., 0., 0.};
    const int ns = *nspecial;
    if (ns) {
        double u[9];
        for (int e = 0; e < 9; e++) u[e] = ubis[9 * i + e];
        for (int q = lane; q < ns; q += 32) {
            const int64_t k = special[q];
            double ih[3];
            const double v = drlv2_exact(u, gv[3 * k], gv[3 * k + 1], gv[3 * k + 2], ih);
            for (int j = 0; j < ntol; j++)
                if (v < tols.t[j] * tols.t[j]) {
                    c[j]++;
                    sm[j] += v;
                }
        }
    }
    for (int j = 0; j < ntol; j++) {
        const int cs = warp_sum(c[j]);
        const double ss = warp_sum(sm[j]);
        if (lane == 0) {
            scnt[i * ntol + j] = cs;
            ssum[i * ntol + j] = ss;
        }
    }
}

// One thread per UBI: CTA-part partials in a fixed order, then the slot of
// the g-vectors outside the regular range.
__global__ void __launch_bounds__(kGT)
k_score_finish(int64_t m, int parts, int ntol, const int* __restrict__ pcnt,
               const double* __restrict__ psum, const int* __restrict__ scnt,
               const double* __restrict__ ssum, int* __restrict__ counts,
               double* __restrict__ sums) {
    const int64_t i = (int64_t)blockIdx.x * kGT + threadIdx.x;
    if (i >= m) return;
    int c[ID11B_MAX_TOLS] = {0, 0, 0, 0};
    double s[ID11B_MAX_TOLS] = {0., 0., 0., 0.};
    for (int p = 0; p < parts; p++)
        for (int j = 0; j < ntol; j++) {
            c[j] += pcnt[(i * parts + p) * ntol + j];
            s[j] += psum[(i * parts + p) * ntol + j];
        }
    for (int j = 0; j < ntol; j++) {
        counts[i * ntol + j] = c[j] + scnt[i * ntol + j];
        if (sums) sums[i * ntol + j] = s[j] + ssum[i * ntol + j];
    }
}

// ------------------------------------------------------------ refinement --
// score_and_refine (ImageD11 src/closest.c:267-345) for many UBIs against all
// g through the index: the pairs with drlv2 < tol^2 are exactly the ones the
// lookup hands over with own = true; each adds ih.g^T, ih.ih^T, drlv2 and 1 to
// the normal equations in the reference's FP64 operations, per lane in shared
// memory ([field][lane]), then warp trees, per-part partials and a fixed-order
// finish per UBI that applies the reference's update.
constexpr int kLsqF = 17;  // R 9 (g_i ih_j at 3i+j), H 6 (00 10 20 11 21 22), sum, n

__device__ __forceinline__ void lsq_add(double* acc, double s, const double* g,
                                        const double* ih) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) acc[(3 * i + j) * 32] = dadd(acc[(3 * i + j) * 32], dmul(ih[j], g[i]));
    acc[9 * 32] = dadd(acc[9 * 32], dmul(ih[0], ih[0]));
    acc[10 * 32] = dadd(acc[10 * 32], dmul(ih[1], ih[0]));
    acc[11 * 32] = dadd(acc[11 * 32], dmul(ih[2], ih[0]));
    acc[12 * 32] = dadd(acc[12 * 32], dmul(ih[1], ih[1]));
    acc[13 * 32] = dadd(acc[13 * 32], dmul(ih[2], ih[1]));
    acc[14 * 32] = dadd(acc[14 * 32], dmul(ih[2], ih[2]));
    acc[15 * 32] = dadd(acc[15 * 32], s);
    acc[16 * 32] += 1.0;
}

__global__ void __launch_bounds__(kST, ID11B_GRID_MINB)
k_refine(const double* __restrict__ ubis, int64_t m, int parts, const Header* __restrict__ Hp,
         const int* __restrict__ start, const double* __restrict__ gs, double tol,
         double* __restrict__ part_out) {
    __shared__ unsigned long long s_q[kSW][kQueue];
    __shared__ WarpPlan s_plan[kSW];
    __shared__ Batch s_batch[kSW];
    __shared__ double s_lsq[kSW][kLsqF * 32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t wk = ((int64_t)blockIdx.x * kST + threadIdx.x) >> 5;
    if (wk >= m * parts) return;  // uniform per warp
    const int64_t i = wk / parts;
    const int part = (int)(wk % parts);
    const Header H = *Hp;
    const int64_t nreg = start[H.ncells];
    const double t2 = tol * tol;
    double* acc = s_lsq[w] + lane;
#pragma unroll
    for (int f = 0; f < kLsqF; f++) acc[f * 32] = 0.;
    const bool ok = setup_plan(s_plan + w, ubis, i, tol, H, nreg, lane);
    auto act = [&](int, double s, bool own, const double* g, const double* ih) {
        if (own && s < t2) lsq_add(acc, s, g, ih);
    };
    walk(s_plan + w, s_batch + w, s_q[w], ok, part, parts, lane, H, nreg, start, gs, act);
    __syncwarp();
#pragma unroll 1
    for (int f = 0; f < kLsqF; f++) {
        const double v = warp_sum(acc[f * 32]);
        if (lane == 0) part_out[(i * parts + part) * kLsqF + f] = v;
    }
}

// The g-vectors outside the regular range, one warp per UBI: normal-equation
// terms of the pairs below tol^2 (lanes stride the list, fixed-tree sums).
__global__ void __launch_bounds__(kGT)
k_refine_special(const double* __restrict__ ubis, int64_t m, double tol,
                 const double* __restrict__ gv, const int* __restrict__ special,
                 const int* __restrict__ nspecial, double* __restrict__ spart) {
    __shared__ double s_lsq[kGT / 32][kLsqF * 32];
    const int64_t i = ((int64_t)blockIdx.x * kGT + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= m) return;  // uniform per warp
    double* acc = s_lsq[threadIdx.x >> 5] + lane;
    for (int f = 0; f < kLsqF; f++) acc[f * 32] = 0.;
    const int ns = *nspecial;
    if (ns) {
        double u[9];
        for (int e = 0; e < 9; e++) u[e] = ubis[9 * i + e];
        for (int q = lane; q < ns; q += 32) {
            const int64_t k = special[q];
            double ih[3];
            const double g[3] = {gv[3 * k], gv[3 * k + 1], gv[3 * k + 2]};
            const double sv = drlv2_exact(u, g[0], g[1], g[2], ih);
            if (sv < tol * tol) lsq_add(acc, sv, g, ih);
        }
    }
    __syncwarp();
    for (int f = 0; f < kLsqF; f++) {
        const double v = warp_sum(acc[f * 32]);
        if (lane == 0) spart[i * kLsqF + f] = v;
    }
}

// One thread per UBI: partials in part order, then the slot of the g outside
// the regular range, then the reference's update; n and mean drlv2 of the UBI
// as it was on entry.
__global__ void __launch_bounds__(kGT)
k_refine_finish(double* __restrict__ ubis, int64_t m, int parts,
                const double* __restrict__ part_in, const double* __restrict__ spart,
                int* __restrict__ npk, double* __restrict__ mean) {
    const int64_t i = (int64_t)blockIdx.x * kGT + threadIdx.x;
    if (i >= m) return;
    double t[kLsqF];
    for (int f = 0; f < kLsqF; f++) t[f] = 0.;
    for (int p = 0; p < parts; p++)
        for (int f = 0; f < kLsqF; f++) t[f] += part_in[(i * parts + p) * kLsqF + f];
    for (int f = 0; f < kLsqF; f++) t[f] += spart[i * kLsqF + f];
    double u[9];
    for (int e = 0; e < 9; e++) u[e] = ubis[9 * i + e];
    double R[9], Hm[9];
    for (int f = 0; f < 9; f++) R[f] = t[f];
    Hm[0] = t[9];  Hm[1] = t[10]; Hm[2] = t[11];
    Hm[3] = t[10]; Hm[4] = t[12]; Hm[5] = t[13];
    Hm[6] = t[11]; Hm[7] = t[13]; Hm[8] = t[14];
    lsq_update_exact(R, Hm, u);
    for (int e = 0; e < 9; e++) ubis[9 * i + e] = u[e];
    const long long n = (long long)t[16];
    if (npk) npk[i] = (int)n;
    if (mean) mean[i] = n > 0 ? t[15] / (double)n : 0.;
}

// ------------------------------------------------------------ assignment --
// Batched score_and_assign (ImageD11 src/closest.c:366-397) over m grains in
// order: for each g the reference's sequence of calls leaves the label of the
// first grain reaching the smallest drlv2 among those below tol^2 and below
// the g's initial drlv2, and that drlv2.  Pass 0 takes the minimum (FP64 bits
// of non-negative values order like the values), pass 1 the lowest grain index
// reaching it; both passes evaluate the same pairs with the same arithmetic.
template <int PASS>
__global__ void __launch_bounds__(kST, ID11B_GRID_MINB)
k_assign(const double* __restrict__ ubis, int64_t m, int parts, const Header* __restrict__ Hp,
         const int* __restrict__ start, const double* __restrict__ gs,
         const int* __restrict__ gidx, double tol, const double* __restrict__ drlv2,
         unsigned long long* __restrict__ best, int* __restrict__ lab, int64_t base) {
    __shared__ unsigned long long s_q[kSW][kQueue];
    __shared__ WarpPlan s_plan[kSW];
    __shared__ Batch s_batch[kSW];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t wk = ((int64_t)blockIdx.x * kST + threadIdx.x) >> 5;
    if (wk >= m * parts) return;  // uniform per warp
    const int64_t i = wk / parts;
    const int part = (int)(wk % parts);
    const Header H = *Hp;
    const int64_t nreg = start[H.ncells];
    const double t2 = tol * tol;
    const bool ok = setup_plan(s_plan + w, ubis, i, tol, H, nreg, lane);
    auto act = [&](int pos, double s, bool own, const double*, const double*) {
        if (!own || !(s < t2)) return;
        const int k = __ldg(gidx + pos);
        if (!(s < __ldg(drlv2 + k))) return;
        const unsigned long long b = (unsigned long long)__double_as_longlong(s);
        if (PASS == 0)
            atomicMin(best + k, b);
        else if (best[k] == b)
            atomicMin(lab + k, (int)(base + i));
    };
    walk(s_plan + w, s_batch + w, s_q[w], ok, part, parts, lane, H, nreg, start, gs, act);
}

constexpr unsigned long long kNoBest = 0x7fffffffffffffffull;

__global__ void __launch_bounds__(kGT)
k_assign_init(int64_t n, unsigned long long* __restrict__ best, int* __restrict__ lab) {
    for (int64_t k = (int64_t)blockIdx.x * kGT + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * kGT) {
        best[k] = kNoBest;  // above the bits of every finite drlv2, and positive as int64
        lab[k] = INT_MAX;
    }
}

// is v one of the grain labels (strictly increasing; null: 0 .. m-1)?
__device__ __forceinline__ bool is_grain_label(int v, const int* __restrict__ gl, int64_t m) {
    if (!gl) return v >= 0 && (int64_t)v < m;
    int64_t lo = 0, hi = m;  // binary search
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        const int x = gl[mid];
        if (x == v) return true;
        if (x < v) lo = mid + 1; else hi = mid;
    }
    return false;
}

// regular g (by sorted position): write the winner, or apply the reference's
// "it does not belong after all" reset when the g held a grain's label
__global__ void __launch_bounds__(kGT)
k_assign_final(const int* __restrict__ start, int64_t ncells, const int* __restrict__ gidx,
               const unsigned long long* __restrict__ best, const int* __restrict__ lab,
               const int* __restrict__ gl, int64_t m, double* __restrict__ drlv2,
               int* __restrict__ labels, int* __restrict__ npk) {
    const int64_t nreg = start[ncells];
    for (int64_t p = (int64_t)blockIdx.x * kGT + threadIdx.x; p < nreg;
         p += (int64_t)gridDim.x * kGT) {
        const int k = gidx[p];
        const int w = lab[k];
        if (w != INT_MAX) {
            labels[k] = gl ? gl[w] : w;
            drlv2[k] = __longlong_as_double((long long)best[k]);
            if (npk) atomicAdd(npk + w, 1);
        } else if (is_grain_label(labels[k], gl, m)) {
            labels[k] = -1;
        }
    }
}

// g outside the regular range: the reference's sequence of calls, literally
__global__ void __launch_bounds__(kGT)
k_assign_special(const double* __restrict__ ubis, int64_t m, const double* __restrict__ gv,
                 const int* __restrict__ spec, const int* __restrict__ nspec, double tol,
                 const int* __restrict__ gl, double* __restrict__ drlv2,
                 int* __restrict__ labels, int* __restrict__ npk) {
    const int ns = *nspec;
    const double t2 = tol * tol;
    for (int q = blockIdx.x * kGT + threadIdx.x; q < ns; q += gridDim.x * kGT) {
        const int64_t k = spec[q];
        const double g0 = gv[3 * k], g1 = gv[3 * k + 1], g2 = gv[3 * k + 2];
        double d = drlv2[k];
        int l = labels[k];
        int64_t win = -1;
        for (int64_t i = 0; i < m; i++) {
            double u[9], ih[3];
            for (int e = 0; e < 9; e++) u[e] = ubis[9 * i + e];
            const double s = drlv2_exact(u, g0, g1, g2, ih);
            const int li = gl ? gl[i] : (int)i;
            if (s < t2 && s < d) {
                l = li;
                d = s;
                win = i;
            } else if (l == li) {
                l = -1;
                win = -1;
            }
        }
        labels[k] = l;
        drlv2[k] = d;
        if (npk && win >= 0) atomicAdd(npk + win, 1);
    }
}

}  // namespace grid
}  // namespace id11b

namespace id11b {
namespace grid {

int num_sms() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 148;
}

unsigned grid_for(int64_t items, int per) {
    int64_t b = (items + per - 1) / per;
    int64_t cap = (int64_t)num_sms() * 8;
    if (b > cap) b = cap;
    return (unsigned)(b > 0 ? b : 1);
}

// exclusive scan of x[0..len) into y (len >= 1), tot: scratch
int scan(const int* x, int64_t len, int* y, int* tot, cudaStream_t st) {
    const int64_t nb = (len + kScanPer - 1) / kScanPer;
    k_scan_local<<<(unsigned)nb, kScanT, 0, st>>>(x, len, y, tot);
    ID11B_CHECK_LAUNCH();
    k_scan_totals<<<1, kScanT, 0, st>>>(tot, (int)nb);
    ID11B_CHECK_LAUNCH();
    k_scan_add<<<(unsigned)nb, kScanT, 0, st>>>(y, len, tot);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

// work items (warps) per UBI: enough warps for ~4 waves of 8 warps x 8 CTAs per SM
int score_parts(int64_t m) {
    if (m <= 0) return 1;
    int64_t want = (int64_t)num_sms() * 64 * 4;
    int64_t p = (want + m - 1) / m;
    if (p > kMaxParts) p = kMaxParts;
    return (int)(p < 1 ? 1 : p);
}

}  // namespace grid
}  // namespace id11b

using namespace id11b::grid;

extern "C" int id11b_dev_gvec_bounds(const double* gv, int64_t n, uint32_t* bounds, void* stream) {
    if (n < 0 || !bounds || (n > 0 && !gv)) return ID11B_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    ID11B_CHECK(cudaMemsetAsync(bounds, 0, 2 * sizeof(uint32_t), st));
    if (n == 0) return ID11B_OK;
    k_bounds<<<grid_for(n, kGT), kGT, 0, st>>>(gv, n, bounds);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_grid_plan(float gmax, int64_t n, double cell, int32_t* nx, double* cs) {
    if (!nx || !cs || n < 0 || !(gmax >= 0.f) || !(cell >= 0.)) return ID11B_ERR_ARG;
    const double G = (double)gmax * (1. + 1e-6) + 1e-300;
    double c = cell;
    if (c == 0.) c = 2. * G / fmax(1., cbrt((double)n));  // ~one g per cell of the cube
    int64_t k = (int64_t)ceil(2. * G / c);
    if (k < 1) k = 1;
    if (k > 400) {  // at most 6.4e7 cells
        k = 400;
    }
    *nx = (int32_t)k;
    *cs = fmax(c, 2. * G / (double)k);
    return ID11B_OK;
}

namespace id11b {
namespace grid {
bool grid_dims_ok(int32_t nx, int32_t xsub) {
    return nx >= 1 && nx <= 400 && xsub >= 1 && xsub <= 16 && (int64_t)nx * nx * nx * xsub <= (1 << 26);
}
}  // namespace grid
}  // namespace id11b

extern "C" int64_t id11b_grid_bytes(int64_t n, int32_t nx, int32_t xsub) {
    if (n < 0 || !grid_dims_ok(nx, xsub)) return -1;
    return (int64_t)layout(n, (int64_t)nx * nx * nx * xsub).bytes;
}

extern "C" int id11b_dev_build_grid(const double* gv, int64_t n, float gmax, float rmax, double cs,
                                    int32_t nx, int32_t xsub, void* gridbuf, int64_t grid_bytes,
                                    void* stream) {
    if (n < 0 || !grid_dims_ok(nx, xsub) || !gridbuf || (n > 0 && !gv) || !(cs > 0.) ||
        !(gmax >= 0.f) || !(rmax >= 0.f))
        return ID11B_ERR_ARG;
    if ((uintptr_t)gridbuf & 255) return ID11B_ERR_ALIGN;
    if (n > INT32_MAX - 1) return ID11B_ERR_SIZE;
    const int64_t ncells = (int64_t)nx * nx * nx * xsub;
    const Layout L = layout(n, ncells);
    if (grid_bytes < (int64_t)L.bytes) return ID11B_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    char* b = (char*)gridbuf;
    Header h;
    memset(&h, 0, sizeof(h));
    h.lo = -((double)gmax * (1. + 1e-6) + 1e-300);
    h.cs = cs;
    h.inv_cs = 1.0 / cs;
    h.inv_csx = (double)xsub / cs;
    h.rmax = (double)rmax;
    h.ncells = ncells;
    h.n = n;
    h.nx = nx;
    h.nxx = nx * xsub;
    static_assert(sizeof(Header) <= 256, "header");
    // a copy from pageable memory returns once the source has been staged,
    // so the stack value may go out of scope
    ID11B_CHECK(cudaMemcpyAsync(b + L.header, &h, sizeof(h), cudaMemcpyHostToDevice, st));
    int* cnt = (int*)(b + L.cnt);
    int* start = (int*)(b + L.start);
    int* flag = (int*)(b + L.flag);
    int* spos = (int*)(b + L.spos);
    int* tot = (int*)(b + L.tot);
    ID11B_CHECK(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(ncells + 1), st));
    ID11B_CHECK(cudaMemsetAsync(flag, 0, sizeof(int) * (size_t)(n + 1), st));
    const Header* H = (const Header*)(b + L.header);
    if (n > 0) {
        k_count<<<grid_for(n, kGT), kGT, 0, st>>>(gv, n, H, cnt, flag);
        ID11B_CHECK_LAUNCH();
    }
    int rc = scan(cnt, ncells + 1, start, tot, st);
    if (rc) return rc;
    rc = scan(flag, n + 1, spos, tot, st);
    if (rc) return rc;
    ID11B_CHECK(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(ncells + 1), st));  // cursors
    if (n > 0) {
        k_scatter<<<grid_for(n, kGT), kGT, 0, st>>>(gv, n, H, start, cnt, (double*)(b + L.g),
                                                    (int*)(b + L.idx), spos, (int*)(b + L.spec));
        ID11B_CHECK_LAUNCH();
        k_sort_cells_f32<<<grid_for(n, kGT), kGT, 0, st>>>(start, H, (double*)(b + L.g),
                                                            (int*)(b + L.idx),
                                                            (float4*)(b + L.g4));
        ID11B_CHECK_LAUNCH();
    }
    return ID11B_OK;
}

// partials: (m * parts + m) x ntol ints, then the same doubles (the last m x
// ntol of each: the g outside the regular range)
extern "C" int64_t id11b_grid_score_workspace_bytes(int64_t m, int ntol) {
    if (m < 0 || ntol < 1 || ntol > ID11B_MAX_TOLS) return -1;
    const int64_t mm = m > 0 ? m : 1;
    const int64_t items = (mm * score_parts(m) + mm) * ntol;
    return (int64_t)(al256(sizeof(int) * (size_t)items) + al256(sizeof(double) * (size_t)items));
}

extern "C" int id11b_dev_score_grid(const double* ubis, int64_t m, const double* gv, int64_t n,
                                    int32_t nx, int32_t xsub, const void* gridbuf,
                                    const double* tols_host, int ntol, int32_t* counts,
                                    double* sums, void* ws, int64_t ws_bytes, void* stream) {
    if (!tols_host || ntol < 1 || ntol > ID11B_MAX_TOLS || m < 0 || n < 0 ||
        !grid_dims_ok(nx, xsub) || !gridbuf || !ws || (m > 0 && (!ubis || !counts)) ||
        (n > 0 && !gv))
        return ID11B_ERR_ARG;
    Tols T;
    T.fix = 0.;  // the lookup's sums are fixed-order FP64
    for (int j = 0; j < ID11B_MAX_TOLS; j++) T.t[j] = j < ntol ? tols_host[j] : 0.;
    for (int j = 0; j < ntol; j++)
        if (!(tols_host[j] >= 0.) || !(tols_host[j] < 1e3)) return ID11B_ERR_ARG;
    if (((uintptr_t)gridbuf & 255) || ((uintptr_t)ws & 255)) return ID11B_ERR_ALIGN;
    if (ws_bytes < id11b_grid_score_workspace_bytes(m, ntol)) return ID11B_ERR_SIZE;
    if (m > INT32_MAX) return ID11B_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    const Layout L = layout(n, (int64_t)nx * nx * nx * xsub);
    char* b = (char*)gridbuf;
    Header* H = (Header*)b;
    ID11B_CHECK(cudaMemsetAsync(&H->nfallback, 0, 3 * sizeof(unsigned long long), st));
    if (m == 0) return ID11B_OK;
    const int parts = score_parts(m);
    const int64_t items = (m * parts + m) * ntol;
    int* pcnt = (int*)ws;
    double* psum = (double*)((char*)ws + al256(sizeof(int) * (size_t)items));
    int* scnt = pcnt + m * parts * ntol;
    double* ssum = psum + m * parts * ntol;
    const int64_t warps = m * parts;
    const unsigned blocks = (unsigned)((warps + kSW - 1) / kSW);
    const int* start = (const int*)(b + L.start);
    const double* gs = (const double*)(b + L.g);
    switch (ntol) {
        case 1: k_score<1><<<blocks, kST, 0, st>>>(ubis, m, parts, H, start, gs, T, pcnt, psum); break;
        case 2: k_score<2><<<blocks, kST, 0, st>>>(ubis, m, parts, H, start, gs, T, pcnt, psum); break;
        case 3: k_score<3><<<blocks, kST, 0, st>>>(ubis, m, parts, H, start, gs, T, pcnt, psum); break;
        default: k_score<4><<<blocks, kST, 0, st>>>(ubis, m, parts, H, start, gs, T, pcnt, psum); break;
    }
    ID11B_CHECK_LAUNCH();
    k_score_special<<<(unsigned)((m * 32 + kGT - 1) / kGT), kGT, 0, st>>>(
        ubis, m, ntol, T, gv, (const int*)(b + L.spec), (const int*)(b + L.spos) + n, scnt,
        ssum);
    ID11B_CHECK_LAUNCH();
    k_score_finish<<<(unsigned)((m + kGT - 1) / kGT), kGT, 0, st>>>(m, parts, ntol, pcnt, psum,
                                                                    scnt, ssum, counts, sums);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_grid_stats(const void* gridbuf, int64_t* nregular, int64_t* nspecial,
                                int64_t* nfallback, int64_t* ntested, int64_t* npairs,
                                void* stream) {
    if (!gridbuf) return ID11B_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    Header h;
    ID11B_CHECK(cudaMemcpyAsync(&h, gridbuf, sizeof(h), cudaMemcpyDeviceToHost, st));
    ID11B_CHECK(cudaStreamSynchronize(st));
    const Layout L = layout(h.n, h.ncells);
    int nr = 0, ns = 0;
    ID11B_CHECK(cudaMemcpyAsync(&nr, (const char*)gridbuf + L.start + sizeof(int) * h.ncells,
                                sizeof(int), cudaMemcpyDeviceToHost, st));
    ID11B_CHECK(cudaMemcpyAsync(&ns, (const char*)gridbuf + L.spos + sizeof(int) * h.n,
                                sizeof(int), cudaMemcpyDeviceToHost, st));
    ID11B_CHECK(cudaStreamSynchronize(st));
    if (nregular) *nregular = nr;
    if (nspecial) *nspecial = ns;
    if (nfallback) *nfallback = (int64_t)h.nfallback;
    if (ntested) *ntested = (int64_t)h.ntested;
    if (npairs) *npairs = (int64_t)h.npairs;
    return ID11B_OK;
}

extern "C" int64_t id11b_assign_workspace_bytes(int64_t n) {
    if (n < 0) return -1;
    const size_t nn = (size_t)(n > 0 ? n : 1);
    return (int64_t)(al256(sizeof(unsigned long long) * nn) + al256(sizeof(int) * nn));
}

extern "C" int id11b_dev_score_and_assign_grid(const double* ubis, int64_t m,
                                               const int32_t* grain_labels, const double* gv,
                                               int64_t n, int32_t nx, int32_t xsub,
                                               const void* gridbuf, double tol, double* drlv2,
                                               int32_t* labels, int32_t* npk, void* ws,
                                               int64_t ws_bytes, void* stream) {
    if (m < 0 || n < 0 || !grid_dims_ok(nx, xsub) || !gridbuf || !ws || (m > 0 && !ubis) ||
        (n > 0 && (!gv || !drlv2 || !labels)) || !(tol >= 0.) || !(tol < 1e3))
        return ID11B_ERR_ARG;
    if (((uintptr_t)gridbuf & 255) || ((uintptr_t)ws & 255)) return ID11B_ERR_ALIGN;
    if (ws_bytes < id11b_assign_workspace_bytes(n)) return ID11B_ERR_SIZE;
    if (m > INT32_MAX - 1) return ID11B_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    if (npk && m > 0) ID11B_CHECK(cudaMemsetAsync(npk, 0, sizeof(int32_t) * (size_t)m, st));
    if (m == 0 || n == 0) return ID11B_OK;
    const int64_t ncells = (int64_t)nx * nx * nx * xsub;
    const Layout L = layout(n, ncells);
    const char* b = (const char*)gridbuf;
    const Header* H = (const Header*)b;
    const int* start = (const int*)(b + L.start);
    const double* gs = (const double*)(b + L.g);
    const int* gidx = (const int*)(b + L.idx);
    unsigned long long* best = (unsigned long long*)ws;
    int* lab = (int*)((char*)ws + al256(sizeof(unsigned long long) * (size_t)n));
    k_assign_init<<<grid_for(n, kGT), kGT, 0, st>>>(n, best, lab);
    ID11B_CHECK_LAUNCH();
    const int parts = score_parts(m);
    const unsigned blocks = (unsigned)((m * parts + kSW - 1) / kSW);
    k_assign<0><<<blocks, kST, 0, st>>>(ubis, m, parts, H, start, gs, gidx, tol, drlv2, best, lab,
                                        0);
    ID11B_CHECK_LAUNCH();
    k_assign<1><<<blocks, kST, 0, st>>>(ubis, m, parts, H, start, gs, gidx, tol, drlv2, best, lab,
                                        0);
    ID11B_CHECK_LAUNCH();
    k_assign_final<<<grid_for(n, kGT), kGT, 0, st>>>(start, ncells, gidx, best, lab, grain_labels,
                                                     m, drlv2, labels, npk);
    ID11B_CHECK_LAUNCH();
    k_assign_special<<<grid_for(n, kGT), kGT, 0, st>>>(ubis, m, gv, (const int*)(b + L.spec),
                                                       (const int*)(b + L.spos) + n, tol,
                                                       grain_labels, drlv2, labels, npk);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

// partials: m * parts + m slots of 17 doubles (the last m: the g outside the
// regular range)
extern "C" int64_t id11b_grid_refine_workspace_bytes(int64_t m) {
    if (m < 0) return -1;
    const size_t mm = (size_t)(m > 0 ? m : 1);
    return (int64_t)al256(sizeof(double) * kLsqF * (mm * score_parts(m) + mm));
}

extern "C" int id11b_dev_refine_grid(double* ubis, int64_t m, const double* gv, int64_t n,
                                     int32_t nx, int32_t xsub, const void* gridbuf, double tol,
                                     int iters, int32_t* npk, double* mean, void* ws,
                                     int64_t ws_bytes, void* stream) {
    if (m < 0 || n < 0 || iters < 0 || !grid_dims_ok(nx, xsub) || !gridbuf || !ws ||
        (m > 0 && !ubis) || (n > 0 && !gv) || !(tol >= 0.) || !(tol < 1e3))
        return ID11B_ERR_ARG;
    if (((uintptr_t)gridbuf & 255) || ((uintptr_t)ws & 255)) return ID11B_ERR_ALIGN;
    if (ws_bytes < id11b_grid_refine_workspace_bytes(m)) return ID11B_ERR_SIZE;
    if (m > INT32_MAX) return ID11B_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    if (m == 0) return ID11B_OK;
    const Layout L = layout(n, (int64_t)nx * nx * nx * xsub);
    const char* b = (const char*)gridbuf;
    const Header* H = (const Header*)b;
    const int parts = score_parts(m);
    const unsigned blocks = (unsigned)((m * parts + kSW - 1) / kSW);
    double* part = (double*)ws;
    for (int it = 0; it < iters; it++) {
        k_refine<<<blocks, kST, 0, st>>>(ubis, m, parts, H, (const int*)(b + L.start),
                                         (const double*)(b + L.g), tol, part);
        ID11B_CHECK_LAUNCH();
        double* spart = part + m * parts * kLsqF;
        k_refine_special<<<(unsigned)((m * 32 + kGT - 1) / kGT), kGT, 0, st>>>(
            ubis, m, tol, gv, (const int*)(b + L.spec), (const int*)(b + L.spos) + n, spart);
        ID11B_CHECK_LAUNCH();
        k_refine_finish<<<(unsigned)((m + kGT - 1) / kGT), kGT, 0, st>>>(ubis, m, parts, part,
                                                                         spart, npk, mean);
        ID11B_CHECK_LAUNCH();
    }
    return ID11B_OK;
}

// The assignment in pieces, for grains sharded over ranks: every rank runs
// pass -1 (reset) and pass 0 over its share of the grains, the best arrays are
// reduced with MIN over ranks (int64 view), pass 1 over the share, the lab
// arrays reduced with MIN (int32), and every rank then applies
// id11b_dev_assign_grid_final with all m grains (for the g outside the
// regular range, which follow the reference's sequence of calls).
extern "C" int id11b_dev_assign_grid_pass(const double* ubis, int64_t m, int64_t index_base,
                                          int64_t n, int32_t nx, int32_t xsub,
                                          const void* gridbuf, double tol, const double* drlv2,
                                          int pass, uint64_t* best, int32_t* lab, void* stream) {
    if (m < 0 || n < 0 || index_base < 0 || index_base + m > INT32_MAX - 1 ||
        !grid_dims_ok(nx, xsub) || !gridbuf || !best || !lab || (m > 0 && !ubis) ||
        (n > 0 && !drlv2) || !(tol >= 0.) || !(tol < 1e3) || pass < -1 || pass > 1)
        return ID11B_ERR_ARG;
    if ((uintptr_t)gridbuf & 255) return ID11B_ERR_ALIGN;
    cudaStream_t st = (cudaStream_t)stream;
    if (n == 0) return ID11B_OK;
    if (pass == -1) {
        k_assign_init<<<grid_for(n, kGT), kGT, 0, st>>>(n, (unsigned long long*)best, lab);
        ID11B_CHECK_LAUNCH();
        return ID11B_OK;
    }
    if (m == 0) return ID11B_OK;
    const Layout L = layout(n, (int64_t)nx * nx * nx * xsub);
    const char* b = (const char*)gridbuf;
    const int parts = score_parts(m);
    const unsigned blocks = (unsigned)((m * parts + kSW - 1) / kSW);
    if (pass == 0)
        k_assign<0><<<blocks, kST, 0, st>>>(ubis, m, parts, (const Header*)b,
                                            (const int*)(b + L.start), (const double*)(b + L.g),
                                            (const int*)(b + L.idx), tol, drlv2,
                                            (unsigned long long*)best, lab, index_base);
    else
        k_assign<1><<<blocks, kST, 0, st>>>(ubis, m, parts, (const Header*)b,
                                            (const int*)(b + L.start), (const double*)(b + L.g),
                                            (const int*)(b + L.idx), tol, drlv2,
                                            (unsigned long long*)best, lab, index_base);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_assign_grid_final(const double* ubis, int64_t m,
                                           const int32_t* grain_labels, const double* gv,
                                           int64_t n, int32_t nx, int32_t xsub,
                                           const void* gridbuf, double tol, const uint64_t* best,
                                           const int32_t* lab, double* drlv2, int32_t* labels,
                                           int32_t* npk, void* stream) {
    if (m < 0 || n < 0 || !grid_dims_ok(nx, xsub) || !gridbuf || !best || !lab ||
        (m > 0 && !ubis) || (n > 0 && (!gv || !drlv2 || !labels)) || !(tol >= 0.) ||
        !(tol < 1e3) || m > INT32_MAX - 1)
        return ID11B_ERR_ARG;
    if ((uintptr_t)gridbuf & 255) return ID11B_ERR_ALIGN;
    cudaStream_t st = (cudaStream_t)stream;
    if (npk && m > 0) ID11B_CHECK(cudaMemsetAsync(npk, 0, sizeof(int32_t) * (size_t)m, st));
    if (m == 0 || n == 0) return ID11B_OK;
    const int64_t ncells = (int64_t)nx * nx * nx * xsub;
    const Layout L = layout(n, ncells);
    const char* b = (const char*)gridbuf;
    k_assign_final<<<grid_for(n, kGT), kGT, 0, st>>>(
        (const int*)(b + L.start), ncells, (const int*)(b + L.idx),
        (const unsigned long long*)best, lab, grain_labels, m, drlv2, labels, npk);
    ID11B_CHECK_LAUNCH();
    k_assign_special<<<grid_for(n, kGT), kGT, 0, st>>>(ubis, m, gv, (const int*)(b + L.spec),
                                                       (const int*)(b + L.spos) + n, tol,
                                                       grain_labels, drlv2, labels, npk);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}
