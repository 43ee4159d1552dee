// Per-grain translation refinement: the objective of
// ImageD11/refinegrains.py refinepositions (:636-660) / gof (:517-560),
// minimised by damped Gauss-Newton for every grain at once instead of a
// Nelder-Mead simplex per grain.
//
// For grain G with peaks k (lab positions x_k, omega_k) and the UBI it was
// read with, U0, the reference's gof at translation t is built by
// refinegrains.refine (:459-498): g_k(t) from compute_gv (ImageD11
// src/cdiffraction.c:112-168), one score_and_refine from U0 at tol (the
// least-squares UBI U1 of the peaks with drlv2 < tol^2, hkl = round(U0.g)),
// then a second score_and_refine at U1 whose mean drlv2 is the objective:
//   cost(t) = sum over peaks with drlv2 < tol^2 of |U1.g_k - round(U1.g_k)|^2.
// Each iteration makes the same two passes over the grain's peaks: the first
// sums R = sum g h^T and H = sum h h^T and solves U1 = (R H^-1)^-1; the
// second takes the cost at U1 and, with U1 and the rounded hkl held for the
// step, the Jacobian of r_k = U1.g_k(t) - hkl,
//   dr/dt = U1 . B . M^T . (ds/|d|)(I - n n^T) . (-M . A),
// A = dR_omega/dt (the omega rotation of t), B the omega rotation of g,
// d = x - M.A.t, n = d/|d| (forward mode, three tangents per peak; the
// adjoint's reverse pass gives J^T r but not the J^T J a Gauss-Newton step
// needs).  Holding U1 is exact for the gradient: at the least-squares U1 the
// derivative of the cost through U1 vanishes.  The sums J^T J, J^T r and the
// cost are reduced in a fixed order and a Levenberg-Marquardt step is taken;
// a step that raises the cost is undone and the damping raised.  One CTA per
// grain, every iteration in one launch.
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

// g of one peak at translation t, with what its tangents need
struct PeakG {
    double so, co, n0, n1, n2, inv, g[3];
};

__device__ __forceinline__ void peak_g(const Geo& P, const double t[3], double x0, double x1,
                                       double x2, double om, PeakG& q) {
    sincos(kRad * om * P.omegasign, &q.so, &q.co);
    const double* M = P.m;
    const double so = q.so, co = q.co;
    // o = M.A.t, A = [[co,-so,0],[so,co,0],[0,0,1]]
    const double at0 = co * t[0] - so * t[1], at1 = so * t[0] + co * t[1], at2 = t[2];
    const double d0 = x0 - (M[0] * at0 + M[1] * at1 + M[2] * at2);
    const double d1 = x1 - (M[3] * at0 + M[4] * at1 + M[5] * at2);
    const double d2 = x2 - (M[6] * at0 + M[7] * at1 + M[8] * at2);
    q.inv = 1.0 / sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    q.n0 = d0 * q.inv;
    q.n1 = d1 * q.inv;
    q.n2 = d2 * q.inv;
    const double k0 = P.ds * (q.n0 - 1.0), k1 = P.ds * q.n1, k2 = P.ds * q.n2;
    const double v0 = M[0] * k0 + M[3] * k1 + M[6] * k2;
    const double v1 = M[1] * k0 + M[4] * k1 + M[7] * k2;
    const double v2 = M[2] * k0 + M[5] * k1 + M[8] * k2;
    q.g[0] = co * v0 + so * v1;
    q.g[1] = -so * v0 + co * v1;
    q.g[2] = v2;
}

// first pass: R (9, R[i][j] = sum h_j g_i) and H (6, upper) of the peaks
// with drlv2(u0) < tol^2, as score_and_refine sums them
__device__ __forceinline__ void refit_terms(const Geo& P, const double u[9], const double t[3],
                                            double x0, double x1, double x2, double om,
                                            double* a) {
    PeakG q;
    peak_g(P, t, x0, x1, x2, om, q);
    double ih[3], r[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const double h = u[3 * i] * q.g[0] + u[3 * i + 1] * q.g[1] + u[3 * i + 2] * q.g[2];
        ih[i] = rint(h);
        r[i] = h - ih[i];
    }
    const double s = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    if (!(s < P.tol2)) return;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) a[3 * i + j] += ih[j] * q.g[i];
    a[9] += ih[0] * ih[0];
    a[10] += ih[0] * ih[1];
    a[11] += ih[0] * ih[2];
    a[12] += ih[1] * ih[1];
    a[13] += ih[1] * ih[2];
    a[14] += ih[2] * ih[2];
}

// second pass: cost and Gauss-Newton sums at u
__device__ __forceinline__ void peak_terms(const Geo& P, const double u[9], const double t[3],
                                           double x0, double x1, double x2, double om,
                                           Acc& acc) {
    PeakG q;
    peak_g(P, t, x0, x1, x2, om, q);
    const double* M = P.m;
    const double so = q.so, co = q.co, n0 = q.n0, n1 = q.n1, n2 = q.n2, inv = q.inv;
    double r[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const double h = u[3 * i] * q.g[0] + u[3 * i + 1] * q.g[1] + u[3 * i + 2] * q.g[2];
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
    int k = 0;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = a; b < 3; b++) {
            acc.a[k++] += J[0][a] * J[0][b] + J[1][a] * J[1][b] + J[2][a] * J[2][b];
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

// U1 = (R H^-1)^-1 from the first pass's sums; false (U1 left as u0) when
// H or R H^-1 is singular, as score_and_refine leaves its UBI
__device__ bool refit_ubi(const double* a, const double u0[9], double u1[9]) {
    double H[9] = {a[9], a[10], a[11], a[10], a[12], a[13], a[11], a[13], a[14]};
#pragma unroll
    for (int e = 0; e < 9; e++) u1[e] = u0[e];
    if (inverse3x3_exact(H) != 0) return false;
    double UB[9];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            UB[3 * i + j] = a[3 * i] * H[j] + a[3 * i + 1] * H[3 + j] + a[3 * i + 2] * H[6 + j];
    if (inverse3x3_exact(UB) != 0) return false;
#pragma unroll
    for (int e = 0; e < 9; e++) u1[e] = UB[e];
    return true;
}

__global__ void __launch_bounds__(kTT)
k_refine_translations(const double* __restrict__ xyz, const double* __restrict__ omega,
                      const int64_t* __restrict__ offsets, int32_t ngrains,
                      const double* __restrict__ ubis, double* __restrict__ tr, Geo P, int iters,
                      double* __restrict__ cost_out, int32_t* __restrict__ npk_out,
                      double* __restrict__ ubi_out) {
    __shared__ double s_red[kTT / 32][15];
    __shared__ double s_t[3];
    __shared__ double s_u[9];
    const int gi = blockIdx.x;
    if (gi >= ngrains) return;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int64_t p0 = offsets[gi], p1 = offsets[gi + 1];
    double u0[9];
#pragma unroll
    for (int e = 0; e < 9; e++) u0[e] = ubis[9 * gi + e];
    double tacc[3] = {tr[3 * gi], tr[3 * gi + 1], tr[3 * gi + 2]};
    double hacc[6] = {0, 0, 0, 0, 0, 0}, bacc[3] = {0, 0, 0}, cacc = 0., nacc = 0.;
    double uacc[9];
#pragma unroll
    for (int e = 0; e < 9; e++) uacc[e] = u0[e];
    double lam = 1e-3;
    if (tid == 0) {
        s_t[0] = tacc[0];
        s_t[1] = tacc[1];
        s_t[2] = tacc[2];
    }
    __syncthreads();
    for (int it = 0; it <= iters; it++) {
        const double t[3] = {s_t[0], s_t[1], s_t[2]};
        // pass 1: least-squares UBI from u0 at t
        double a[15];
#pragma unroll
        for (int q = 0; q < 15; q++) a[q] = 0.;
        for (int64_t k = p0 + tid; k < p1; k += kTT)
            refit_terms(P, u0, t, xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2], omega[k], a);
#pragma unroll
        for (int q = 0; q < 15; q++) {
            const double v = warp_sum(a[q]);
            if (lane == 0) s_red[wid][q] = v;
        }
        __syncthreads();
        if (tid == 0) {
            double r[15];
            for (int q = 0; q < 15; q++) {
                r[q] = 0.;
                for (int w = 0; w < kTT / 32; w++) r[q] += s_red[w][q];  // fixed order
            }
            double u1[9];
            refit_ubi(r, u0, u1);
            for (int e = 0; e < 9; e++) s_u[e] = u1[e];
        }
        __syncthreads();
        double u1[9];
#pragma unroll
        for (int e = 0; e < 9; e++) u1[e] = s_u[e];
        // pass 2: cost and Gauss-Newton sums at u1
        Acc acc;
#pragma unroll
        for (int q = 0; q < 11; q++) acc.a[q] = 0.;
        for (int64_t k = p0 + tid; k < p1; k += kTT)
            peak_terms(P, u1, t, xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2], omega[k], acc);
#pragma unroll
        for (int q = 0; q < 11; q++) {
            const double v = warp_sum(acc.a[q]);
            if (lane == 0) s_red[wid][q] = v;
        }
        __syncthreads();
        if (tid == 0) {
            double r[11];
            for (int q = 0; q < 11; q++) {
                r[q] = 0.;
                for (int w = 0; w < kTT / 32; w++) r[q] += s_red[w][q];  // fixed order
            }
            if (it == 0 || r[9] < cacc) {  // accept t (or the start point)
                for (int q = 0; q < 6; q++) hacc[q] = r[q];
                for (int q = 0; q < 3; q++) {
                    bacc[q] = r[6 + q];
                    tacc[q] = t[q];
                }
                for (int e = 0; e < 9; e++) uacc[e] = u1[e];
                cacc = r[9];
                nacc = r[10];
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
        if (ubi_out)
            for (int e = 0; e < 9; e++) ubi_out[9 * gi + e] = uacc[e];
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
                                             int32_t* npk, double* ubis_refit, void* stream) {
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
        xyz, omega, offsets, ngrains, ubis, translations, P, iters, cost, npk, ubis_refit);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}
