// Per-grain translation refinement: the objective of
// ImageD11/refinegrains.py refinepositions (:639-660) / gof (:517-560),
// minimised by damped Gauss-Newton for every grain at once instead of a
// Nelder-Mead simplex per grain.
//
// For grain G with fixed UBI and peaks k (lab positions x_k, omega_k), the
// reference's gof is sum over peaks with drlv2 < tol^2 of
//   drlv2_k(t) = |UBI.g_k(t) - round(UBI.g_k(t))|^2,
// g_k(t) from compute_gv (ImageD11 src/cdiffraction.c:143-167) with the grain
// translation t.  With the rounded hkl held for one step, r_k = UBI.g_k(t) - hkl
// is smooth in t and its 3x3 Jacobian is
//   dr/dt = UBI . B . M^T . (ds/|d|)(I - n n^T) . (-M . A),
// A = dR_omega/dt (the omega rotation of t), B the omega rotation of g,
// d = x - M.A.t, n = d/|d|.  Each iteration sums J^T J, J^T r and the cost over
// the grain's peaks (fixed-order CTA reduction) and takes a Levenberg-Marquardt
// step; a step that raises the cost is undone and the damping raised.  One CTA
// per grain, every iteration in one launch.
#include <math.h>

#include "common.cuh"

namespace id11b {
namespace trans {

// threads per grain (500 grains of ~650 peaks, 30 iterations on B200: 64 and 128
// threads 0.44 ms, 256 threads 0.53 ms, the call's host work included)
#ifndef ID11B_TRANS_THREADS
#define ID11B_TRANS_THREADS 64
#endif
constexpr int kTT = ID11B_TRANS_THREADS;
constexpr double kRad = 3.14159265358979323846 / 180.0;

struct Geo {
    double m[9];  // chi.wedge
    double omegasign, ds;
    double tol2;
};

// sums of one peak: J^T J (6, upper), J^T r (3), cost, n
struct Acc {
    double a[11];
};

__device__ __forceinline__ void peak_terms(const Geo& P, const double u[9], const double t[3],
                                           double x0, double x1, double x2, double om,
                                           Acc& acc) {
    double so, co;
    sincos(kRad * om * P.omegasign, &so, &co);
    const double* M = P.m;
    // o = M.A.t, A = [[co,-so,0],[so,co,0],[0,0,1]]
    const double at0 = co * t[0] - so * t[1], at1 = so * t[0] + co * t[1], at2 = t[2];
    const double d0 = x0 - (M[0] * at0 + M[1] * at1 + M[2] * at2);
    const double d1 = x1 - (M[3] * at0 + M[4] * at1 + M[5] * at2);
    const double d2 = x2 - (M[6] * at0 + M[7] * at1 + M[8] * at2);
    const double inv = 1.0 / sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    const double n0 = d0 * inv, n1 = d1 * inv, n2 = d2 * inv;
    const double k0 = P.ds * (n0 - 1.0), k1 = P.ds * n1, k2 = P.ds * n2;
    const double v0 = M[0] * k0 + M[3] * k1 + M[6] * k2;
    const double v1 = M[1] * k0 + M[4] * k1 + M[7] * k2;
    const double v2 = M[2] * k0 + M[5] * k1 + M[8] * k2;
    const double g0 = co * v0 + so * v1, g1 = -so * v0 + co * v1, g2 = v2;
    double r[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const double h = u[3 * i] * g0 + u[3 * i + 1] * g1 + u[3 * i + 2] * g2;
        r[i] = h - rint(h);
    }
    const double s = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    if (!(s < P.tol2)) return;
    // columns j of dd/dt = -M.A e_j
    const double A[3][3] = {{co, -so, 0.}, {so, co, 0.}, {0., 0., 1.}};
    double J[3][3];  // J[i][j] = dr_i / dt_j
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const double a0 = A[0][j], a1 = A[1][j], a2 = A[2][j];
        const double e0 = -(M[0] * a0 + M[1] * a1 + M[2] * a2);
        const double e1 = -(M[3] * a0 + M[4] * a1 + M[5] * a2);
        const double e2 = -(M[6] * a0 + M[7] * a1 + M[8] * a2);
        // dk = ds * inv * (e - n (n.e))
        const double ne = n0 * e0 + n1 * e1 + n2 * e2;
        const double q0 = P.ds * inv * (e0 - n0 * ne), q1 = P.ds * inv * (e1 - n1 * ne),
                     q2 = P.ds * inv * (e2 - n2 * ne);
        const double w0 = M[0] * q0 + M[3] * q1 + M[6] * q2;
        const double w1 = M[1] * q0 + M[4] * q1 + M[7] * q2;
        const double w2 = M[2] * q0 + M[5] * q1 + M[8] * q2;
        const double dg0 = co * w0 + so * w1, dg1 = -so * w0 + co * w1, dg2 = w2;
#pragma unroll
        for (int i = 0; i < 3; i++) J[i][j] = u[3 * i] * dg0 + u[3 * i + 1] * dg1 + u[3 * i + 2] * dg2;
    }
    int q = 0;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = a; b < 3; b++) {
            acc.a[q++] += J[0][a] * J[0][b] + J[1][a] * J[1][b] + J[2][a] * J[2][b];
        }
#pragma unroll
    for (int a = 0; a < 3; a++) acc.a[6 + a] += J[0][a] * r[0] + J[1][a] * r[1] + J[2][a] * r[2];
    acc.a[9] += s;
    acc.a[10] += 1.0;
}

// (H + lambda diag H) x = -b for a symmetric 3x3 H (upper: h00 h01 h02 h11 h12 h22)
__device__ __forceinline__ bool solve3(const double h[6], const double b[3], double lam,
                                       double x[3]) {
    const double a00 = h[0] * (1. + lam), a01 = h[1], a02 = h[2];
    const double a11 = h[3] * (1. + lam), a12 = h[4], a22 = h[5] * (1. + lam);
    const double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22,
                 c02 = a01 * a12 - a02 * a11;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    if (!(fabs(det) > 0.) || !isfinite(det)) return false;
    const double c11 = a00 * a22 - a02 * a02, c12 = a01 * a02 - a00 * a12,
                 c22 = a00 * a11 - a01 * a01;
    const double id = -1.0 / det;
    x[0] = id * (c00 * b[0] + c01 * b[1] + c02 * b[2]);
    x[1] = id * (c01 * b[0] + c11 * b[1] + c12 * b[2]);
    x[2] = id * (c02 * b[0] + c12 * b[1] + c22 * b[2]);
    return isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]);
}

__global__ void __launch_bounds__(kTT)
k_refine_translations(const double* __restrict__ xyz, const double* __restrict__ omega,
                      const int64_t* __restrict__ offsets, int32_t ngrains,
                      const double* __restrict__ ubis, double* __restrict__ tr, Geo P, int iters,
                      double* __restrict__ cost_out, int32_t* __restrict__ npk_out) {
    __shared__ double s_red[kTT / 32][11];
    __shared__ double s_t[3];
    const int gi = blockIdx.x;
    if (gi >= ngrains) return;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int64_t p0 = offsets[gi], p1 = offsets[gi + 1];
    double u[9];
#pragma unroll
    for (int e = 0; e < 9; e++) u[e] = ubis[9 * gi + e];
    double tacc[3] = {tr[3 * gi], tr[3 * gi + 1], tr[3 * gi + 2]};
    double hacc[6] = {0, 0, 0, 0, 0, 0}, bacc[3] = {0, 0, 0}, cacc = 0., nacc = 0.;
    double lam = 1e-3;
    if (tid == 0) {
        s_t[0] = tacc[0];
        s_t[1] = tacc[1];
        s_t[2] = tacc[2];
    }
    __syncthreads();
    for (int it = 0; it <= iters; it++) {
        const double t[3] = {s_t[0], s_t[1], s_t[2]};
        Acc acc;
#pragma unroll
        for (int q = 0; q < 11; q++) acc.a[q] = 0.;
        for (int64_t k = p0 + tid; k < p1; k += kTT)
            peak_terms(P, u, t, xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2], omega[k], acc);
#pragma unroll
        for (int q = 0; q < 11; q++) {
            const double v = warp_sum(acc.a[q]);
            if (lane == 0) s_red[wid][q] = v;
        }
        __syncthreads();
        if (tid == 0) {
            double a[11];
            for (int q = 0; q < 11; q++) {
                a[q] = 0.;
                for (int w = 0; w < kTT / 32; w++) a[q] += s_red[w][q];  // fixed order
            }
            if (it == 0 || a[9] < cacc) {  // accept t (or the start point)
                for (int q = 0; q < 6; q++) hacc[q] = a[q];
                for (int q = 0; q < 3; q++) {
                    bacc[q] = a[6 + q];
                    tacc[q] = t[q];
                }
                cacc = a[9];
                nacc = a[10];
                if (it) lam = fmax(lam * 0.3, 1e-9);
            } else {
                lam = fmin(lam * 10., 1e9);
            }
            double x[3] = {0., 0., 0.};
            if (it < iters && nacc >= 3. && solve3(hacc, bacc, lam, x)) {
                s_t[0] = tacc[0] + x[0];
                s_t[1] = tacc[1] + x[1];
                s_t[2] = tacc[2] + x[2];
            } else {
                s_t[0] = tacc[0];
                s_t[1] = tacc[1];
                s_t[2] = tacc[2];
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        tr[3 * gi] = tacc[0];
        tr[3 * gi + 1] = tacc[1];
        tr[3 * gi + 2] = tacc[2];
        if (cost_out) cost_out[gi] = cacc;
        if (npk_out) npk_out[gi] = (int32_t)nacc;
    }
}

}  // namespace trans
}  // namespace id11b

using namespace id11b::trans;

// chi.wedge as the reference builds it (src/cdiffraction.c:117-142)
static void wedgechi(double wedge, double chi, double m[9]) {
    const double pi = 3.14159265358979323846;
    double sw = sin(wedge * pi / 180.0), cw = cos(wedge * pi / 180.0);
    double sc = sin(chi * pi / 180.0), cc = cos(chi * pi / 180.0);
    double w[9] = {cw, 0.0, -sw, 0., 1.0, 0., sw, 0.0, cw};
    double c[9] = {1., 0.0, 0., 0., cc, -sc, 0., sc, cc};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            m[3 * i + j] = c[j] * w[3 * i] + c[3 + j] * w[3 * i + 1] + c[6 + j] * w[3 * i + 2];
}

extern "C" int id11b_dev_refine_translations(const double* xyz, const double* omega,
                                             const int64_t* offsets, int32_t ngrains,
                                             const double* ubis, double* translations,
                                             double omegasign, double wvln, double wedge,
                                             double chi, double tol, int iters, double* cost,
                                             int32_t* npk, void* stream) {
    if (ngrains < 0 || iters < 0 || iters > 1000 || !(tol > 0.) || !(wvln > 0.))
        return ID11B_ERR_ARG;
    if (ngrains == 0) return ID11B_OK;
    if (!xyz || !omega || !offsets || !ubis || !translations) return ID11B_ERR_ARG;
    Geo P;
    wedgechi(wedge, chi, P.m);
    P.omegasign = omegasign;
    P.ds = 1.0 / wvln;
    P.tol2 = tol * tol;
    k_refine_translations<<<(unsigned)ngrains, kTT, 0, (cudaStream_t)stream>>>(
        xyz, omega, offsets, ngrains, ubis, translations, P, iters, cost, npk);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}
