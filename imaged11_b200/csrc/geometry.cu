// Detector geometry kernels: compute_gv, compute_geometry, compute_xlylzl (FP64).
//
// Streaming, HBM-bound.  One CTA of 256 threads owns a tile of 256 peaks at a
// time (grid-stride over tiles, grid = a multiple of the SM count).  The AoS
// (n,3) inputs and outputs are staged through shared memory so that every
// global access is a fully coalesced 8-byte-per-lane sweep of the tile's
// 6 KB, instead of three 24-byte-strided accesses per lane.
#include <math.h>

#include "common.cuh"

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

__device__ __forceinline__ void peak_geometry(const GvParams& P, double x0, double x1,
                                              double x2, double om, PeakGeo& r) {
    double ang = dmul(dmul(kRad, om), P.omegasign);
    sincos(ang, &r.so, &r.co);
    const double so = r.so, co = r.co;
    double u0 = dsub(dmul(co, P.t[0]), dmul(so, P.t[1]));
    double u1 = dadd(dmul(so, P.t[0]), dmul(co, P.t[1]));
    double u2 = P.t[2];
    double o0 = ddot3(P.m[0], P.m[1], P.m[2], u0, u1, u2);
    double o1 = ddot3(P.m[3], P.m[4], P.m[5], u0, u1, u2);
    double o2 = ddot3(P.m[6], P.m[7], P.m[8], u0, u1, u2);
    r.d0 = dsub(x0, o0);
    r.d1 = dsub(x1, o1);
    r.d2 = dsub(x2, o2);
    r.inv = ddiv(1., __dsqrt_rn(ddot3(r.d0, r.d1, r.d2, r.d0, r.d1, r.d2)));
    r.k0 = dmul(P.ds, dsub(dmul(r.d0, r.inv), 1.));
    r.k1 = dmul(dmul(P.ds, r.d1), r.inv);
    r.k2 = dmul(dmul(P.ds, r.d2), r.inv);
    double v0 = ddot3(P.m[0], P.m[3], P.m[6], r.k0, r.k1, r.k2);
    double v1 = ddot3(P.m[1], P.m[4], P.m[7], r.k0, r.k1, r.k2);
    double v2 = ddot3(P.m[2], P.m[5], P.m[8], r.k0, r.k1, r.k2);
    r.g0 = dadd(dmul(co, v0), dmul(so, v1));
    r.g1 = dadd(dmul(-so, v0), dmul(co, v1));
    r.g2 = v2;
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
                // ImageD11 src/cdiffraction.c:74-91
                double* o = s_out + 6 * tid;
                o[0] = dmul(kDeg, atan2(__dsqrt_rn(dadd(dmul(r.d1, r.d1), dmul(r.d2, r.d2))),
                                        r.d0));
                o[1] = dmul(kDeg, atan2(-r.d1, r.d2));
                o[2] = __dsqrt_rn(ddot3(r.k0, r.k1, r.k2, r.k0, r.k1, r.k2));
                o[3] = r.g0;
                o[4] = r.g1;
                o[5] = r.g2;
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
