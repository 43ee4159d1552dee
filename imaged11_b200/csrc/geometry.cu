// Detector geometry kernels: compute_gv, compute_geometry, compute_xlylzl (FP64).
//
// Streaming, HBM-bound.  One CTA of 256 threads owns a tile of 256 peaks at a
// time (grid-stride over tiles, grid = a multiple of the SM count).  The AoS
// (n,3) inputs and outputs are staged through shared memory so that every
// global access is a fully coalesced 8-byte-per-lane sweep of the tile's
// 6 KB, instead of three 24-byte-strided accesses per lane.
#include <math.h>

#include <cmath>

#include "common.cuh"
#include "tma.cuh"

namespace id11b {

struct GvParams {
    double m[9];      // chi.wedge matrix built on the host like the reference
    double t[3];      // grain translation
    double omegasign;
    double ds;        // 1 / wavelength
};

constexpr int kGeoThreads = 256;
constexpr double kRad = 3.14159265358979323846 / 180.0;
constexpr double kDeg = 180.0 / 3.14159265358979323846;

// Per-peak body of ImageD11 src/cdiffraction.c:143-167 in the reference's
// operation order (no FMA).  sin/cos come from CUDA's sincos (<= 2 ulp), the
// only difference from the reference's libm.
struct PeakGeo {
    double so, co, d0, d1, d2, inv, k0, k1, k2, g0, g1, g2;
};

//
// Two specialisations give results identical to the general expression
// (apart from the sign of a zero) and are chosen on the host:
//  HAS_T = false: t == (0,0,0), so u = (+-0, +-0, 0), o = +-0 and d = xyz;
//                 taken only for a finite angle (otherwise NaN must propagate
//                 through o exactly as in the reference);
//  ROT   = false: the chi.wedge matrix is exactly the identity (wedge = chi =
//                 0) and t is finite, so M.u = u, and M^T.k = k whenever k is
//                 finite (checked per peak; 0*inf would give NaN otherwise).
template <bool HAS_T = true, bool ROT = true>
__device__ __forceinline__ void peak_geometry(const GvParams& P, double x0, double x1,
                                              double x2, double om, PeakGeo& r) {
    double ang = dmul(dmul(kRad, om), P.omegasign);
    sincos(ang, &r.so, &r.co);
    const double so = r.so, co = r.co;
    if (HAS_T || !isfinite(ang)) {
        double u0 = dsub(dmul(co, P.t[0]), dmul(so, P.t[1]));
        double u1 = dadd(dmul(so, P.t[0]), dmul(co, P.t[1]));
        double u2 = P.t[2];
        double o0 = u0, o1 = u1, o2 = u2;
        if (ROT) {
            o0 = ddot3(P.m[0], P.m[1], P.m[2], u0, u1, u2);
            o1 = ddot3(P.m[3], P.m[4], P.m[5], u0, u1, u2);
            o2 = ddot3(P.m[6], P.m[7], P.m[8], u0, u1, u2);
        }
        r.d0 = dsub(x0, o0);
        r.d1 = dsub(x1, o1);
        r.d2 = dsub(x2, o2);
    } else {
        r.d0 = x0;
        r.d1 = x1;
        r.d2 = x2;
    }
    r.inv = ddiv(1., __dsqrt_rn(ddot3(r.d0, r.d1, r.d2, r.d0, r.d1, r.d2)));
    r.k0 = dmul(P.ds, dsub(dmul(r.d0, r.inv), 1.));
    r.k1 = dmul(dmul(P.ds, r.d1), r.inv);
    r.k2 = dmul(dmul(P.ds, r.d2), r.inv);
    double v0, v1, v2;
    if (!ROT && isfinite(r.k0) && isfinite(r.k1) && isfinite(r.k2)) {
        v0 = r.k0;
        v1 = r.k1;
        v2 = r.k2;
    } else {
        v0 = ddot3(P.m[0], P.m[3], P.m[6], r.k0, r.k1, r.k2);
        v1 = ddot3(P.m[1], P.m[4], P.m[7], r.k0, r.k1, r.k2);
        v2 = ddot3(P.m[2], P.m[5], P.m[8], r.k0, r.k1, r.k2);
    }
    r.g0 = dadd(dmul(co, v0), dmul(so, v1));
    r.g1 = dadd(dmul(-so, v0), dmul(co, v1));
    r.g2 = v2;
}

// tth, eta, ds, g of one peak (ImageD11 src/cdiffraction.c:74-91)
__device__ __forceinline__ void geometry_out(const PeakGeo& r, double* o) {
    o[0] = dmul(kDeg, atan2(__dsqrt_rn(dadd(dmul(r.d1, r.d1), dmul(r.d2, r.d2))), r.d0));
    o[1] = dmul(kDeg, atan2(-r.d1, r.d2));
    o[2] = __dsqrt_rn(ddot3(r.k0, r.k1, r.k2, r.k0, r.k1, r.k2));
    o[3] = r.g0;
    o[4] = r.g1;
    o[5] = r.g2;
}

// MODE 0: gv (n,3); MODE 1: geometry out (n,6)
template <int MODE>
__global__ void __launch_bounds__(kGeoThreads)
k_geometry(const double* __restrict__ xyz, const double* __restrict__ omega, GvParams P,
           double* __restrict__ out, float4* __restrict__ g4, int64_t n) {
    constexpr int OUTW = MODE == 0 ? 3 : 6;
    __shared__ double s_in[3 * kGeoThreads];
    __shared__ double s_out[OUTW * kGeoThreads];
    const int tid = threadIdx.x;
    for (int64_t base = (int64_t)blockIdx.x * kGeoThreads; base < n;
         base += (int64_t)gridDim.x * kGeoThreads) {
        const int cnt = (int)min((int64_t)kGeoThreads, n - base);
        const double* src = xyz + 3 * base;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            int e = tid + j * kGeoThreads;
            if (e < 3 * cnt) s_in[e] = __ldcs(src + e);
        }
        double om = tid < cnt ? __ldcs(omega + base + tid) : 0.;
        __syncthreads();
        if (tid < cnt) {
            PeakGeo r;
            peak_geometry(P, s_in[3 * tid], s_in[3 * tid + 1], s_in[3 * tid + 2], om, r);
            if (MODE == 0) {
                s_out[3 * tid] = r.g0;
                s_out[3 * tid + 1] = r.g1;
                s_out[3 * tid + 2] = r.g2;
                if (g4)
                    g4[base + tid] = make_float4((float)r.g0, (float)r.g1, (float)r.g2, 0.f);
            } else {
                geometry_out(r, s_out + 6 * tid);
            }
        }
        __syncthreads();
        double* dst = out + OUTW * base;
#pragma unroll
        for (int j = 0; j < OUTW; j++) {
            int e = tid + j * kGeoThreads;
            if (e < OUTW * cnt) __stcs(dst + e, s_out[e]);
        }
        __syncthreads();
    }
}

// Pipelined variant for 16-byte-aligned inputs: a persistent CTA walks its
// tiles (blockIdx.x, +gridDim.x, ...) with a 4-stage ring of 1-D TMA bulk
// copies (xyz 6 KB + omega 2 KB per tile) completed on mbarriers, so the loads
// of the next three tiles are in flight while the current one is computed and
// stored.  The final partial tile, whose byte counts need not be multiples of
// 16, is read with ordinary loads.  Bounded waits: on a timeout the CTA stops
// and counts the event in g_geo_timeouts.
__device__ unsigned int g_geo_timeouts = 0;

template <int MODE, bool HAS_T = true, bool ROT = true>
__global__ void __launch_bounds__(kGeoThreads, 4)
k_geometry_tma(const double* __restrict__ xyz, const double* __restrict__ omega, GvParams P,
               double* __restrict__ out, float4* __restrict__ g4, int64_t n) {
    constexpr int OUTW = MODE == 0 ? 3 : 6;
    constexpr int S = 4;
    __shared__ __align__(128) double s_x[S][3 * kGeoThreads];
    __shared__ __align__(128) double s_w[S][kGeoThreads];
    __shared__ __align__(16) double s_out[OUTW * kGeoThreads];
    __shared__ __align__(8) uint64_t s_bar[S];
    const int tid = threadIdx.x;
    const int64_t ntiles = (n + kGeoThreads - 1) / kGeoThreads;
    const int64_t nfull = n / kGeoThreads;
    auto issue = [&](int stage, int64_t t) {
        mbar_arrive_expect_tx(&s_bar[stage], (3 + 1) * kGeoThreads * sizeof(double));
        tma_load_1d(s_x[stage], xyz + 3 * t * kGeoThreads, 3 * kGeoThreads * sizeof(double),
                    &s_bar[stage]);
        tma_load_1d(s_w[stage], omega + t * kGeoThreads, kGeoThreads * sizeof(double),
                    &s_bar[stage]);
    };
    if (tid == 0) {
        for (int s = 0; s < S; s++) mbar_init(&s_bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int s = 0; s < S; s++) {
            int64_t t = blockIdx.x + (int64_t)s * gridDim.x;
            if (t < nfull) issue(s, t);
        }
    for (int64_t i = 0;; i++) {
        const int64_t t = blockIdx.x + i * gridDim.x;
        if (t >= ntiles) break;
        const int stage = (int)(i % S);
        const int64_t base = t * kGeoThreads;
        const int cnt = (int)min((int64_t)kGeoThreads, n - base);
        double x0 = 0., x1 = 0., x2 = 0., om = 0.;
        if (t < nfull) {
            if (!__syncthreads_and(mbar_wait_bounded(&s_bar[stage], (uint32_t)((i / S) & 1)))) {
                if (tid == 0) {
                    atomicAdd(&g_geo_timeouts, 1u);
                    for (int64_t j = i; j < i + S; j++)  // copies still in flight
                        if (blockIdx.x + j * gridDim.x < nfull)
                            mbar_wait_bounded(&s_bar[j % S], (uint32_t)((j / S) & 1), 1u << 16);
                }
                return;
            }
            x0 = s_x[stage][3 * tid];
            x1 = s_x[stage][3 * tid + 1];
            x2 = s_x[stage][3 * tid + 2];
            om = s_w[stage][tid];
        } else if (tid < cnt) {  // final partial tile
            x0 = xyz[3 * (base + tid)];
            x1 = xyz[3 * (base + tid) + 1];
            x2 = xyz[3 * (base + tid) + 2];
            om = omega[base + tid];
        }
        if (tid < cnt) {
            PeakGeo r;
            peak_geometry<HAS_T, ROT>(P, x0, x1, x2, om, r);
            if (MODE == 0) {
                s_out[3 * tid] = r.g0;
                s_out[3 * tid + 1] = r.g1;
                s_out[3 * tid + 2] = r.g2;
                if (g4) g4[base + tid] = make_float4((float)r.g0, (float)r.g1, (float)r.g2, 0.f);
            } else {
                geometry_out(r, s_out + 6 * tid);
            }
        }
        __syncthreads();  // stage consumed by every lane; s_out complete
        if (tid == 0) {
            const int64_t tn = blockIdx.x + (i + S) * gridDim.x;
            if (tn < nfull) {
                fence_proxy_async_smem();
                issue(stage, tn);
            }
        }
        double* dst = out + OUTW * base;
#pragma unroll
        for (int j = 0; j < OUTW; j++) {
            int e = tid + j * kGeoThreads;
            if (e < OUTW * cnt) dst[e] = s_out[e];
        }
        __syncthreads();  // s_out free for the next tile
    }
}

// ImageD11 src/cdiffraction.c:190-224: xlylzl_j = r[3j+1]*v1 + r[3j+2]*v2 + dist_j
struct XyzParams {
    double p[4];
    double r[9];
    double dist[3];
};

__global__ void __launch_bounds__(kGeoThreads)
k_xlylzl(const double* __restrict__ s, const double* __restrict__ f, XyzParams P,
         double* __restrict__ out, int64_t n) {
    __shared__ double s_out[3 * kGeoThreads];
    const int tid = threadIdx.x;
    for (int64_t base = (int64_t)blockIdx.x * kGeoThreads; base < n;
         base += (int64_t)gridDim.x * kGeoThreads) {
        const int cnt = (int)min((int64_t)kGeoThreads, n - base);
        if (tid < cnt) {
            double v1 = dmul(dsub(__ldcs(f + base + tid), P.p[1]), P.p[3]);
            double v2 = dmul(dsub(__ldcs(s + base + tid), P.p[0]), P.p[2]);
#pragma unroll
            for (int j = 0; j < 3; j++)
                s_out[3 * tid + j] =
                    dadd(dadd(dmul(P.r[3 * j + 1], v1), dmul(P.r[3 * j + 2], v2)), P.dist[j]);
        }
        __syncthreads();
        double* dst = out + 3 * base;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            int e = tid + j * kGeoThreads;
            if (e < 3 * cnt) __stcs(dst + e, s_out[e]);
        }
        __syncthreads();
    }
}

// Detector position -> lab position -> geometry in one pass (the two calls of
// columnfile.updateGeometry's fast path, ImageD11/columnfile.py:497-504:
// Ctransform.sf2xyz = compute_xlylzl, then xyz2geometry = compute_geometry).
// The lab positions never leave registers unless asked for, and each value is
// produced by the same operations as the two separate kernels, so the results
// are identical to calling them in turn.  sc, fc, omega are read once with
// the next tile's loads issued before the current tile is computed.
template <bool XYZ, bool G4>
__global__ void __launch_bounds__(kGeoThreads, 4)
k_update_geometry(const double* __restrict__ sc, const double* __restrict__ fc,
                  const double* __restrict__ omega, XyzParams X, GvParams P,
                  double* __restrict__ xyz, double* __restrict__ out, float4* __restrict__ g4,
                  int64_t n) {
    __shared__ double s_xyz[XYZ ? 3 * kGeoThreads : 1];
    __shared__ double s_out[6 * kGeoThreads];
    const int tid = threadIdx.x;
    const int64_t ntiles = (n + kGeoThreads - 1) / kGeoThreads;
    double sn = 0., fn = 0., on = 0.;
    auto load = [&](int64_t t) {
        const int64_t k = t * kGeoThreads + tid;
        if (t < ntiles && k < n) {
            sn = __ldcs(sc + k);
            fn = __ldcs(fc + k);
            on = __ldcs(omega + k);
        }
    };
    load(blockIdx.x);
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const double s = sn, f = fn, om = on;
        load(t + gridDim.x);
        const int64_t base = t * kGeoThreads;
        const int cnt = (int)min((int64_t)kGeoThreads, n - base);
        if (tid < cnt) {
            const double v1 = dmul(dsub(f, X.p[1]), X.p[3]);
            const double v2 = dmul(dsub(s, X.p[0]), X.p[2]);
            double x[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                x[j] = dadd(dadd(dmul(X.r[3 * j + 1], v1), dmul(X.r[3 * j + 2], v2)), X.dist[j]);
                if (XYZ) s_xyz[3 * tid + j] = x[j];
            }
            PeakGeo r;
            peak_geometry(P, x[0], x[1], x[2], om, r);
            geometry_out(r, s_out + 6 * tid);
            if (G4) g4[base + tid] = make_float4((float)r.g0, (float)r.g1, (float)r.g2, 0.f);
        }
        __syncthreads();
        if (XYZ) {
            double* dx = xyz + 3 * base;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const int e = tid + j * kGeoThreads;
                if (e < 3 * cnt) __stcs(dx + e, s_xyz[e]);
            }
        }
        double* dst = out + 6 * base;
#pragma unroll
        for (int j = 0; j < 6; j++) {
            const int e = tid + j * kGeoThreads;
            if (e < 6 * cnt) __stcs(dst + e, s_out[e]);
        }
        __syncthreads();
    }
}

// Chi.wedge matrix exactly as ImageD11 src/cdiffraction.c:117-142 (host libm,
// the reference's own sin/cos; the macro RAD expands to (x*pi)/180 here).
static void wedgechi_host(double wedge, double chi, double m[9]) {
    const double pi = 3.14159265358979323846;
    double sw = sin(wedge * pi / 180.0), cw = cos(wedge * pi / 180.0);
    double sc = sin(chi * pi / 180.0), cc = cos(chi * pi / 180.0);
    double w[9] = {cw, 0.0, -sw, 0., 1.0, 0., sw, 0.0, cw};
    double c[9] = {1., 0.0, 0., 0., cc, -sc, 0., sc, cc};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            volatile double a = c[j] * w[3 * i];
            volatile double b = c[3 + j] * w[3 * i + 1];
            volatile double d = c[6 + j] * w[3 * i + 2];
            volatile double ab = a + b;
            m[3 * i + j] = ab + d;
        }
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

static int geo_grid_tma(int64_t n) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int64_t tiles = (n + kGeoThreads - 1) / kGeoThreads;
    int64_t g = (int64_t)sms * 4;  // 4 persistent CTAs per SM (shared memory <= 44 KB each)
    return (int)(tiles < g ? (tiles > 0 ? tiles : 1) : g);
}

static int geo_grid(int64_t n) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int64_t tiles = (n + kGeoThreads - 1) / kGeoThreads;
    int64_t g = (int64_t)sms * 8;  // 8 CTAs of 256 threads resident per SM
    return (int)(tiles < g ? (tiles > 0 ? tiles : 1) : g);
}

}  // namespace id11b

using namespace id11b;

static GvParams make_gv_params(double omegasign, double wvln, double wedge, double chi,
                               const double* t) {
    GvParams P;
    wedgechi_host(wedge, chi, P.m);
    for (int i = 0; i < 3; i++) P.t[i] = t[i];
    P.omegasign = omegasign;
    volatile double one = 1.;
    P.ds = one / wvln;
    return P;
}

extern "C" int id11b_dev_compute_gv(const double* xlylzl, const double* omega,
                                    double omegasign, double wvln, double wedge, double chi,
                                    const double* t_host, double* gv, float* g4, int64_t n,
                                    void* stream) {
    if (n < 0 || !t_host) return ID11B_ERR_ARG;
    if (n == 0) return ID11B_OK;
    if (!xlylzl || !omega || !gv) return ID11B_ERR_ARG;
    if (g4 && ((uintptr_t)g4 & 15)) return ID11B_ERR_ALIGN;
    GvParams P = make_gv_params(omegasign, wvln, wedge, chi, t_host);
    const bool has_t = !(t_host[0] == 0. && t_host[1] == 0. && t_host[2] == 0.);
    bool rot = !(std::isfinite(t_host[0]) && std::isfinite(t_host[1]) && std::isfinite(t_host[2]));
    for (int i = 0; i < 9; i++) rot = rot || P.m[i] != (i % 4 == 0 ? 1. : 0.);
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = geo_grid_tma(n);
    if (aligned16(xlylzl) && aligned16(omega)) {
        if (has_t && rot)
            k_geometry_tma<0, true, true><<<grid, kGeoThreads, 0, st>>>(xlylzl, omega, P, gv,
                                                                        (float4*)g4, n);
        else if (has_t)
            k_geometry_tma<0, true, false><<<grid, kGeoThreads, 0, st>>>(xlylzl, omega, P, gv,
                                                                         (float4*)g4, n);
        else if (rot)
            k_geometry_tma<0, false, true><<<grid, kGeoThreads, 0, st>>>(xlylzl, omega, P, gv,
                                                                         (float4*)g4, n);
        else
            k_geometry_tma<0, false, false><<<grid, kGeoThreads, 0, st>>>(xlylzl, omega, P, gv,
                                                                          (float4*)g4, n);
    } else
        k_geometry<0><<<geo_grid(n), kGeoThreads, 0, (cudaStream_t)stream>>>(
            xlylzl, omega, P, gv, (float4*)g4, n);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_compute_geometry(const double* xlylzl, const double* omega,
                                          double omegasign, double wvln, double wedge,
                                          double chi, const double* t_host, double* out,
                                          int64_t n, void* stream) {
    if (n < 0 || !t_host) return ID11B_ERR_ARG;
    if (n == 0) return ID11B_OK;
    if (!xlylzl || !omega || !out) return ID11B_ERR_ARG;
    GvParams P = make_gv_params(omegasign, wvln, wedge, chi, t_host);
    if (aligned16(xlylzl) && aligned16(omega))
        k_geometry_tma<1><<<geo_grid_tma(n), kGeoThreads, 0, (cudaStream_t)stream>>>(
            xlylzl, omega, P, out, nullptr, n);
    else
        k_geometry<1><<<geo_grid(n), kGeoThreads, 0, (cudaStream_t)stream>>>(xlylzl, omega, P,
                                                                             out, nullptr, n);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_compute_xlylzl(const double* s, const double* f,
                                        const double* p_host, const double* r_host,
                                        const double* dist_host, double* xlylzl, int64_t n,
                                        void* stream) {
    if (n < 0 || !p_host || !r_host || !dist_host) return ID11B_ERR_ARG;
    if (n == 0) return ID11B_OK;
    if (!s || !f || !xlylzl) return ID11B_ERR_ARG;
    XyzParams P;
    for (int i = 0; i < 4; i++) P.p[i] = p_host[i];
    for (int i = 0; i < 9; i++) P.r[i] = r_host[i];
    for (int i = 0; i < 3; i++) P.dist[i] = dist_host[i];
    k_xlylzl<<<geo_grid(n), kGeoThreads, 0, (cudaStream_t)stream>>>(s, f, P, xlylzl, n);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_update_geometry(const double* sc, const double* fc, const double* omega,
                                         const double* p_host, const double* r_host,
                                         const double* dist_host, double omegasign, double wvln,
                                         double wedge, double chi, const double* t_host,
                                         double* xlylzl, double* out, float* g4, int64_t n,
                                         void* stream) {
    if (n < 0 || !p_host || !r_host || !dist_host || !t_host) return ID11B_ERR_ARG;
    if (n == 0) return ID11B_OK;
    if (!sc || !fc || !omega || !out) return ID11B_ERR_ARG;
    if (g4 && ((uintptr_t)g4 & 15)) return ID11B_ERR_ALIGN;
    XyzParams X;
    for (int i = 0; i < 4; i++) X.p[i] = p_host[i];
    for (int i = 0; i < 9; i++) X.r[i] = r_host[i];
    for (int i = 0; i < 3; i++) X.dist[i] = dist_host[i];
    GvParams P = make_gv_params(omegasign, wvln, wedge, chi, t_host);
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = geo_grid_tma(n);
    if (xlylzl && g4)
        k_update_geometry<true, true><<<grid, kGeoThreads, 0, st>>>(sc, fc, omega, X, P, xlylzl,
                                                                    out, (float4*)g4, n);
    else if (xlylzl)
        k_update_geometry<true, false><<<grid, kGeoThreads, 0, st>>>(sc, fc, omega, X, P, xlylzl,
                                                                     out, nullptr, n);
    else if (g4)
        k_update_geometry<false, true><<<grid, kGeoThreads, 0, st>>>(sc, fc, omega, X, P, nullptr,
                                                                     out, (float4*)g4, n);
    else
        k_update_geometry<false, false><<<grid, kGeoThreads, 0, st>>>(sc, fc, omega, X, P,
                                                                      nullptr, out, nullptr, n);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}
