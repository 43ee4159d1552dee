// Residuals of assigned peaks, their hand-written adjoint, and the geometry
// map, all on the device (FP64).
//
// Geometry parameters (12, device memory, in this order): distance,
// y_center, z_center, tilt_x, tilt_y, tilt_z (radians), wavelength, wedge,
// chi (degrees), t_x, t_y, t_z.  Fixed detector constants (7, host): y_size,
// z_size, omegasign, o11, o12, o21, o22.  Every launch rebuilds
//   r = R3(tilt_x).R2(tilt_y).R1(tilt_z).flip   (ImageD11/transform.py:51-82, :688-692)
//   M = W(wedge).C(chi)                          (src/cdiffraction.c:117-142)
// from the device copy of the parameters, so a step of an optimiser never
// copies the geometry to the host.
//
// Forward model for peak k of grain G (peaks stored grain by grain, CSR):
//   detector -> lab (ImageD11 src/cdiffraction.c:190-224)
//     v1 = (f - y_center) * y_size,  v2 = (s - z_center) * z_size
//     xyz = r[:,1] v1 + r[:,2] v2 + (distance, 0, 0)
//   lab -> g (ImageD11 src/cdiffraction.c:112-168)
//     u = Omega(w)^T t,  o = M u,  d = xyz - o,  dh = d / |d|
//     k = (dh - x) / wavelength,  v = M^T k,  g = Omega(w) v
//   residual  res = UBI_G . g - h_k          (h_k: the peak's assigned hkl)
//
// Backward, given a_res = dL/d res for every peak (reverse mode, per peak):
//   dL/dUBI_G += a_res g^T             a_g = UBI_G^T a_res
//   a_v = Omega^T a_g                  a_k = M a_v,   dL/dM += k a_v^T
//   dL/dwavelength += -(a_k . k) / wavelength
//   a_dh = a_k / wavelength            a_d = (a_dh - dh (dh . a_dh)) / |d|
//   a_xyz = a_d                        a_o = -a_d,    dL/dM += a_o u^T
//   a_u = M^T a_o                      dL/dt += Omega a_u
//   dL/dr[:,1] += a_xyz v1,  dL/dr[:,2] += a_xyz v2,  sum a_xyz (-> distance, centres)
// and, once per launch, dL/dM and dL/dr are contracted with dM/d(wedge, chi)
// and dr/d(tilts), the centre and distance terms with r and the pixel sizes
// (k_finish).
//
// One CTA per grain accumulates its peaks' terms in registers and reduces
// them in a fixed tree into a per-grain row; one CTA then sums the rows in
// grain order.  Every result is deterministic.
//
// Variable projection (MODE 3): each grain's UBI is first solved in closed
// form for the current g (UBI = (sum h g^T)(sum g g^T)^-1, the least-squares
// fit), then the loss and geometry gradient are taken at that UBI.  At the
// least-squares UBI dL/dUBI = 0, so the gradient of the projected loss with
// respect to the geometry equals the partial derivative computed here.
#include <algorithm>

#include "common.cuh"

namespace id11b {

constexpr int kAT = 64;         // threads per CTA
constexpr int kNP = 12;         // geometry parameters
constexpr int kGlob = 22;       // dM(9) dlam(1) dt(3) sum_axyz(3) dR1(3) dR2(3)
constexpr int kPart = kGlob + 1;  // + sum of squared residuals

struct AdjDet {
    double y_size, z_size, omegasign, o11, o12, o21, o22;
};

struct AdjGeom {
    double r[9];        // detector rotation . flip (row-major)
    double M[9];        // chi.wedge
    double t[3];        // grain-origin translation
    double wavelength, distance, y_center, z_center, y_size, z_size, omegasign;
};

struct PeakState {
    double so, co, u[3], v1, v2, dh[3], rn, k[3], g[3];  // rn = 1 / |d|
};

__device__ __forceinline__ void mat3mul(const double* a, const double* b, double* c) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            c[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}

// The rotation factors of r and M and their derivatives:
// R[0..2] = R3(tilt_x), R2(tilt_y), R1(tilt_z); dR the same differentiated;
// F the detector flip; W, C and dW, dC per radian.
struct RotFactors {
    double R[3][9], dR[3][9], F[9], W[9], C[9], dW[9], dC[9];
};

__device__ void rot_factors(const double* p, const AdjDet& D, RotFactors& f) {
    double sx, cx, sy, cy, sz, cz, sw, cw, sc, cc;
    sincos(p[3], &sx, &cx);
    sincos(p[4], &sy, &cy);
    sincos(p[5], &sz, &cz);
    const double rad = 3.14159265358979323846 / 180.0;
    sincos(p[7] * rad, &sw, &cw);
    sincos(p[8] * rad, &sc, &cc);
    const double R3[9] = {1, 0, 0, 0, cx, -sx, 0, sx, cx};
    const double R2[9] = {cy, 0, sy, 0, 1, 0, -sy, 0, cy};
    const double R1[9] = {cz, -sz, 0, sz, cz, 0, 0, 0, 1};
    const double dR3[9] = {0, 0, 0, 0, -sx, -cx, 0, cx, -sx};
    const double dR2[9] = {-sy, 0, cy, 0, 0, 0, -cy, 0, -sy};
    const double dR1[9] = {-sz, -cz, 0, cz, -sz, 0, 0, 0, 0};
    const double F[9] = {1, 0, 0, 0, D.o22, D.o21, 0, D.o12, D.o11};
    const double W[9] = {cw, 0, -sw, 0, 1, 0, sw, 0, cw};
    const double C[9] = {1, 0, 0, 0, cc, -sc, 0, sc, cc};
    const double dW[9] = {-sw, 0, -cw, 0, 0, 0, cw, 0, -sw};
    const double dC[9] = {0, 0, 0, 0, -sc, -cc, 0, cc, -sc};
#pragma unroll
    for (int e = 0; e < 9; e++) {
        f.R[0][e] = R3[e];
        f.R[1][e] = R2[e];
        f.R[2][e] = R1[e];
        f.dR[0][e] = dR3[e];
        f.dR[1][e] = dR2[e];
        f.dR[2][e] = dR1[e];
        f.F[e] = F[e];
        f.W[e] = W[e];
        f.C[e] = C[e];
        f.dW[e] = dW[e];
        f.dC[e] = dC[e];
    }
}

// a.b.c.F with one of a, b, c replaced by its derivative (which = 0, 1, 2)
// or none (which = -1).
__device__ void rot_product(const RotFactors& f, int which, double out[9]) {
    double ab[9], abc[9];
    mat3mul(which == 0 ? f.dR[0] : f.R[0], which == 1 ? f.dR[1] : f.R[1], ab);
    mat3mul(ab, which == 2 ? f.dR[2] : f.R[2], abc);
    mat3mul(abc, f.F, out);
}

__device__ void make_geom(const double* p, const AdjDet& D, AdjGeom& P) {
    RotFactors f;
    rot_factors(p, D, f);
    rot_product(f, -1, P.r);
    mat3mul(f.W, f.C, P.M);
    P.t[0] = p[9];
    P.t[1] = p[10];
    P.t[2] = p[11];
    P.wavelength = p[6];
    P.distance = p[0];
    P.y_center = p[1];
    P.z_center = p[2];
    P.y_size = D.y_size;
    P.z_size = D.z_size;
    P.omegasign = D.omegasign;
}

// sin and cos of the peak's omega * omegasign: from the table made by
// id11b_dev_omega_sincos when one is given (omega is fixed for a peak, so
// an optimiser's evaluations need not repeat them), else computed here
__device__ __forceinline__ void peak_sincos(const AdjGeom& P, const double* __restrict__ omega,
                                            const double* __restrict__ osc, int64_t kk,
                                            double& so, double& co) {
    if (osc) {
        const double2 v = __ldg(reinterpret_cast<const double2*>(osc) + kk);
        so = v.x;
        co = v.y;
    } else {
        sincos(3.14159265358979323846 / 180.0 * omega[kk] * P.omegasign, &so, &co);
    }
}

__device__ __forceinline__ void forward_peak(const AdjGeom& P, double s, double f, double so,
                                             double co, PeakState& q) {
    q.so = so;
    q.co = co;
    q.v1 = (f - P.y_center) * P.y_size;
    q.v2 = (s - P.z_center) * P.z_size;
    double xyz[3];
#pragma unroll
    for (int j = 0; j < 3; j++) xyz[j] = P.r[3 * j + 1] * q.v1 + P.r[3 * j + 2] * q.v2;
    xyz[0] += P.distance;
    q.u[0] = q.co * P.t[0] - q.so * P.t[1];
    q.u[1] = q.so * P.t[0] + q.co * P.t[1];
    q.u[2] = P.t[2];
    double d[3];
#pragma unroll
    for (int i = 0; i < 3; i++)
        d[i] = xyz[i] - (P.M[3 * i] * q.u[0] + P.M[3 * i + 1] * q.u[1] + P.M[3 * i + 2] * q.u[2]);
    q.rn = 1.0 / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
#pragma unroll
    for (int i = 0; i < 3; i++) q.dh[i] = d[i] * q.rn;
    // divided, not multiplied by a rounded 1/wavelength: the rounding then
    // stays independent from peak to peak as wavelength varies
    q.k[0] = (q.dh[0] - 1.0) / P.wavelength;
    q.k[1] = q.dh[1] / P.wavelength;
    q.k[2] = q.dh[2] / P.wavelength;
    double v[3];
#pragma unroll
    for (int i = 0; i < 3; i++) v[i] = P.M[i] * q.k[0] + P.M[3 + i] * q.k[1] + P.M[6 + i] * q.k[2];
    q.g[0] = q.co * v[0] + q.so * v[1];
    q.g[1] = -q.so * v[0] + q.co * v[1];
    q.g[2] = v[2];
}

// Reverse-mode terms of one peak given a_res; gl = the 22 global sums.
__device__ __forceinline__ void adjoint_peak(const AdjGeom& P, const PeakState& q,
                                             const double U[9], const double ar[3],
                                             double* dU, double* gl) {
    if (dU) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) dU[3 * i + j] += ar[i] * q.g[j];
    }
    double ag[3], av[3], ak[3];
#pragma unroll
    for (int j = 0; j < 3; j++) ag[j] = U[j] * ar[0] + U[3 + j] * ar[1] + U[6 + j] * ar[2];
    av[0] = q.co * ag[0] - q.so * ag[1];
    av[1] = q.so * ag[0] + q.co * ag[1];
    av[2] = ag[2];
#pragma unroll
    for (int i = 0; i < 3; i++)
        ak[i] = P.M[3 * i] * av[0] + P.M[3 * i + 1] * av[1] + P.M[3 * i + 2] * av[2];
    // dL/dM from v = M^T k: dM[j][i] += k_j av_i
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int i = 0; i < 3; i++) gl[3 * j + i] += q.k[j] * av[i];
    const double akk = ak[0] * q.k[0] + ak[1] * q.k[1] + ak[2] * q.k[2];
    gl[9] += -akk / P.wavelength;
    double adh[3];
#pragma unroll
    for (int i = 0; i < 3; i++) adh[i] = ak[i] / P.wavelength;
    const double dd = q.dh[0] * adh[0] + q.dh[1] * adh[1] + q.dh[2] * adh[2];
    double ad[3];
#pragma unroll
    for (int i = 0; i < 3; i++) ad[i] = (adh[i] - q.dh[i] * dd) * q.rn;
    // o = M u: dM[i][j] += a_o_i u_j with a_o = -a_d
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) gl[3 * i + j] -= ad[i] * q.u[j];
    double au[3];
#pragma unroll
    for (int j = 0; j < 3; j++) au[j] = -(P.M[j] * ad[0] + P.M[3 + j] * ad[1] + P.M[6 + j] * ad[2]);
    gl[10] += q.co * au[0] + q.so * au[1];
    gl[11] += -q.so * au[0] + q.co * au[1];
    gl[12] += au[2];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        gl[13 + i] += ad[i];
        gl[16 + i] += ad[i] * q.v1;
        gl[19 + i] += ad[i] * q.v2;
    }
}

// Fixed-order CTA reduction of acc[NA]: warp butterflies, then the warps'
// partials summed in warp order.  Result in red[0][e] for every thread.
template <int NA>
__device__ __forceinline__ void cta_reduce(double* acc, double (*red)[NA]) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
#pragma unroll
    for (int e = 0; e < NA; e++) acc[e] = warp_sum(acc[e]);
    if (lane == 0)
#pragma unroll
        for (int e = 0; e < NA; e++) red[w][e] = acc[e];
    __syncthreads();
    for (int e = tid; e < NA; e += kAT) {
        double t = red[0][e];
        for (int q = 1; q < kAT / 32; q++) t += red[q][e];
        red[0][e] = t;
    }
    __syncthreads();
}

// MODE 0: residuals (+ g, + per-grain sum of squares); ubis == nullptr
//         gives g only.
// MODE 1: adjoint of given dL/dres.
// MODE 2: loss 0.5 sum res^2 and its gradient (a_res = res) in one pass.
// MODE 3: variable projection: least-squares UBI per grain, then MODE 2 at it.
// MODE 4: least-squares UBI per grain only.
template <int MODE>
__global__ void __launch_bounds__(kAT)
k_residual(const double* __restrict__ params, AdjDet D, const double* __restrict__ sc,
           const double* __restrict__ fc, const double* __restrict__ omega,
           const double* __restrict__ osc,
           const double* __restrict__ hkl, const int64_t* __restrict__ off,
           const double* __restrict__ ubis, int ngrains, double* __restrict__ res,
           double* __restrict__ gout, double* __restrict__ ssq,
           const double* __restrict__ ares, double* __restrict__ dubi,
           double* __restrict__ partial, double* __restrict__ ubis_out) {
    constexpr bool kAdj = MODE == 1 || MODE == 2 || MODE == 3;
    constexpr int NA = MODE == 0 ? 1 : (MODE == 4 ? 15 : 9 + kPart);
    constexpr int NR = NA > 15 ? NA : 15;
    __shared__ AdjGeom sP;
    __shared__ double s_red[kAT / 32][NR];
    __shared__ double s_U[9];
    const int tid = threadIdx.x;
    if (tid == 0) make_geom(params, D, sP);
    __syncthreads();
    const AdjGeom& P = sP;
    for (int G = blockIdx.x; G < ngrains; G += gridDim.x) {
        const int64_t k0 = off[G], k1 = off[G + 1];
        double U[9];
        if (MODE == 3 || MODE == 4) {
            // pass 1: A = sum h g^T (9), B = sum g g^T (6, upper triangle)
            double a[15];
#pragma unroll
            for (int e = 0; e < 15; e++) a[e] = 0.;
            for (int64_t kk = k0 + tid; kk < k1; kk += kAT) {
                PeakState q;
                double so, co;
                peak_sincos(P, omega, osc, kk, so, co);
                forward_peak(P, sc[kk], fc[kk], so, co, q);
                const double h[3] = {hkl[3 * kk], hkl[3 * kk + 1], hkl[3 * kk + 2]};
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int j = 0; j < 3; j++) a[3 * i + j] += h[i] * q.g[j];
                a[9] += q.g[0] * q.g[0];
                a[10] += q.g[0] * q.g[1];
                a[11] += q.g[0] * q.g[2];
                a[12] += q.g[1] * q.g[1];
                a[13] += q.g[1] * q.g[2];
                a[14] += q.g[2] * q.g[2];
            }
            cta_reduce<15>(a, reinterpret_cast<double(*)[15]>(&s_red[0][0]));
            if (tid == 0) {
                const double* r = s_red[0];
                double B[9] = {r[9], r[10], r[11], r[10], r[12], r[13], r[11], r[13], r[14]};
                // B is positive semi-definite; fewer than three independent
                // g leave it singular up to rounding, so the test is
                // relative: det <= 1e-10 trace^3 counts as singular
                const double tr = B[0] + B[4] + B[8];
                const double det = B[0] * (B[4] * B[8] - B[5] * B[7]) -
                                   B[1] * (B[3] * B[8] - B[5] * B[6]) +
                                   B[2] * (B[3] * B[7] - B[4] * B[6]);
                double X[9];
                if (det > 1e-10 * tr * tr * tr && inverse3x3_exact(B) == 0) {
                    mat3mul(r, B, X);   // UBI = A B^-1
                } else {
#pragma unroll
                    for (int e = 0; e < 9; e++) X[e] = 0.;   // singular: UBI 0
                }
#pragma unroll
                for (int e = 0; e < 9; e++) s_U[e] = X[e];
            }
            __syncthreads();
#pragma unroll
            for (int e = 0; e < 9; e++) U[e] = s_U[e];
            if (ubis_out && tid < 9) ubis_out[9 * (int64_t)G + tid] = s_U[tid];
            if (MODE == 4) {
                __syncthreads();
                continue;
            }
        } else if (ubis) {
#pragma unroll
            for (int e = 0; e < 9; e++) U[e] = ubis[9 * (int64_t)G + e];
        } else {
#pragma unroll
            for (int e = 0; e < 9; e++) U[e] = 0.;
        }
        double acc[NA];
#pragma unroll
        for (int e = 0; e < NA; e++) acc[e] = 0.;
        for (int64_t kk = k0 + tid; kk < k1; kk += kAT) {
            PeakState q;
            double so, co;
            peak_sincos(P, omega, osc, kk, so, co);
            forward_peak(P, sc[kk], fc[kk], so, co, q);
            if (MODE == 0) {
                if (gout) {
#pragma unroll
                    for (int i = 0; i < 3; i++) gout[3 * kk + i] = q.g[i];
                }
                if (ubis) {
                    double ss = 0.;
#pragma unroll
                    for (int i = 0; i < 3; i++) {
                        const double ri = U[3 * i] * q.g[0] + U[3 * i + 1] * q.g[1] +
                                          U[3 * i + 2] * q.g[2] - hkl[3 * kk + i];
                        if (res) res[3 * kk + i] = ri;
                        ss += ri * ri;
                    }
                    acc[0] += ss;
                }
            } else if (kAdj) {
                double ar[3];
                if (MODE == 1) {
#pragma unroll
                    for (int i = 0; i < 3; i++) ar[i] = ares[3 * kk + i];
                } else {
#pragma unroll
                    for (int i = 0; i < 3; i++)
                        ar[i] = U[3 * i] * q.g[0] + U[3 * i + 1] * q.g[1] + U[3 * i + 2] * q.g[2] -
                                hkl[3 * kk + i];
                    acc[9 + kGlob] += ar[0] * ar[0] + ar[1] * ar[1] + ar[2] * ar[2];
                }
                adjoint_peak(P, q, U, ar, MODE == 3 ? nullptr : acc, acc + 9);
            }
        }
        cta_reduce<NA>(acc, reinterpret_cast<double(*)[NA]>(&s_red[0][0]));
        for (int e = tid; e < NA; e += kAT) {
            const double t = s_red[0][e];
            if (MODE == 0) {
                if (ssq) ssq[G] = t;
            } else if (e < 9) {
                if (dubi) dubi[9 * (int64_t)G + e] = t;
            } else {
                partial[(int64_t)G * kPart + (e - 9)] = t;
            }
        }
        __syncthreads();
    }
}

// Sums the per-grain rows (rows x kPart) in grain order (one warp per
// column: lane l sums rows l, l+32, ..., then a fixed butterfly) and maps the
// sums onto the 12 geometry parameters; loss = 0.5 * sum of squares.
__global__ void __launch_bounds__(32 * kPart)
k_finish(const double* __restrict__ partial, int rows, const double* __restrict__ params,
         AdjDet D, double* __restrict__ grad, double* __restrict__ loss) {
    __shared__ double col[kPart];
    const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
    double t = 0.;
    for (int r = lane; r < rows; r += 32) t += partial[(int64_t)r * kPart + c];
    t = warp_sum(t);
    if (lane == 0) col[c] = t;
    __syncthreads();
    if (threadIdx.x != 0) return;
    if (loss) *loss = 0.5 * col[kGlob];
    if (!grad) return;
    RotFactors f;
    rot_factors(params, D, f);
    double r[9];
    rot_product(f, -1, r);
    const double* dM = col;          // dL/dM (row-major)
    const double* A = col + 13;      // sum of dL/dxyz
    const double* dR1 = col + 16;    // dL/dr[:,1]
    const double* dR2 = col + 19;    // dL/dr[:,2]
    grad[0] = A[0];
    grad[1] = -D.y_size * (r[1] * A[0] + r[4] * A[1] + r[7] * A[2]);
    grad[2] = -D.z_size * (r[2] * A[0] + r[5] * A[1] + r[8] * A[2]);
    for (int k = 0; k < 3; k++) {    // tilt_x, tilt_y, tilt_z
        double dr[9];
        rot_product(f, k, dr);
        double s = 0.;
        for (int i = 0; i < 3; i++) s += dr[3 * i + 1] * dR1[i] + dr[3 * i + 2] * dR2[i];
        grad[3 + k] = s;
    }
    grad[6] = col[9];
    const double rad = 3.14159265358979323846 / 180.0;
    double dMw[9], dMc[9];
    mat3mul(f.dW, f.C, dMw);
    mat3mul(f.W, f.dC, dMc);
    double sw = 0., sc = 0.;
    for (int e = 0; e < 9; e++) {
        sw += dM[e] * dMw[e];
        sc += dM[e] * dMc[e];
    }
    grad[7] = sw * rad;
    grad[8] = sc * rad;
    grad[9] = col[10];
    grad[10] = col[11];
    grad[11] = col[12];
}

// Bragg angle of each assigned reflection computed from its grain's UB and
// its derivative, as ImageD11 src/deriv.c:38-53 (g_to_k) computes them:
//   g = UB h,  t = wavelength |g| / 2,  theta = asin(t) (degrees),
//   dtheta/dUB_ij = (180/pi) wavelength / (2 |g| sqrt(1 - t^2)) g_i h_j.
// BACKWARD: grad_ub_G = sum over the grain's peaks of a_theta dtheta/dUB,
// reduced in a fixed order.
template <bool BACKWARD>
__global__ void __launch_bounds__(kAT)
k_bragg(const double* __restrict__ ubs, const double* __restrict__ hkl,
        const int64_t* __restrict__ off, int ngrains, double wavelength,
        double* __restrict__ theta, double* __restrict__ jac,
        const double* __restrict__ atheta, double* __restrict__ gub) {
    __shared__ double s_red[kAT / 32][9];
    const double deg = 180.0 / 3.14159265358979323846;
    for (int G = blockIdx.x; G < ngrains; G += gridDim.x) {
        double B[9];
#pragma unroll
        for (int e = 0; e < 9; e++) B[e] = ubs[9 * (int64_t)G + e];
        double acc[9];
#pragma unroll
        for (int e = 0; e < 9; e++) acc[e] = 0.;
        for (int64_t kk = off[G] + threadIdx.x; kk < off[G + 1]; kk += kAT) {
            const double h[3] = {hkl[3 * kk], hkl[3 * kk + 1], hkl[3 * kk + 2]};
            double g[3];
#pragma unroll
            for (int i = 0; i < 3; i++) g[i] = B[3 * i] * h[0] + B[3 * i + 1] * h[1] + B[3 * i + 2] * h[2];
            const double modg = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
            const double t = wavelength * modg / 2.0;
            const double c = deg * wavelength / (2.0 * modg * sqrt(1.0 - t * t));
            if (BACKWARD) {
                const double a = atheta[kk] * c;
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int j = 0; j < 3; j++) acc[3 * i + j] += a * g[i] * h[j];
            } else {
                theta[kk] = deg * asin(t);
                if (jac)
#pragma unroll
                    for (int i = 0; i < 3; i++)
#pragma unroll
                        for (int j = 0; j < 3; j++) jac[9 * kk + 3 * i + j] = c * g[i] * h[j];
            }
        }
        if (BACKWARD) {
            cta_reduce<9>(acc, s_red);
            if (threadIdx.x < 9) gub[9 * (int64_t)G + threadIdx.x] = s_red[0][threadIdx.x];
            __syncthreads();
        }
    }
}

// sin and cos of omega * omegasign (degrees) per peak, interleaved
__global__ void k_omega_sincos(const double* __restrict__ omega, int64_t n, double omegasign,
                               double* __restrict__ out) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        double so, co;
        sincos(3.14159265358979323846 / 180.0 * omega[k] * omegasign, &so, &co);
        out[2 * k] = so;
        out[2 * k + 1] = co;
    }
}

static int adj_grid(int ngrains) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
    const int cap = sms * 16;
    return ngrains < cap ? ngrains : cap;
}

static int adj_det(const double* d, AdjDet& D) {
    if (!d) return ID11B_ERR_ARG;
    D.y_size = d[0];
    D.z_size = d[1];
    D.omegasign = d[2];
    D.o11 = d[3];
    D.o12 = d[4];
    D.o21 = d[5];
    D.o22 = d[6];
    return ID11B_OK;
}

}  // namespace id11b

using namespace id11b;

extern "C" int64_t id11b_adjoint_workspace_bytes(int32_t ngrains) {
    return (int64_t)sizeof(double) * kPart * (ngrains > 0 ? ngrains : 1);
}

// omega_sincos (optional, 16-byte aligned): the table id11b_dev_omega_sincos
// makes for these peaks; NULL computes sin and cos of omega in the kernels
static bool osc_misaligned(const double* osc) { return osc && ((uintptr_t)osc & 15); }

extern "C" int id11b_dev_residuals(const double* params, const double* detector,
                                   const double* sc, const double* fc, const double* omega,
                                   const double* omega_sincos, const double* hkl,
                                   const int64_t* offsets, const double* ubis, int32_t ngrains,
                                   double* res, double* gvec, double* ssq, void* stream) {
    AdjDet D;
    if (!params || adj_det(detector, D) || ngrains < 0) return ID11B_ERR_ARG;
    if (osc_misaligned(omega_sincos)) return ID11B_ERR_ALIGN;
    if (ngrains == 0) return ID11B_OK;
    if (!offsets || !sc || !fc || !omega) return ID11B_ERR_ARG;
    if (ubis && (!hkl || !res)) return ID11B_ERR_ARG;
    if (!ubis && !gvec) return ID11B_ERR_ARG;
    k_residual<0><<<adj_grid(ngrains), kAT, 0, (cudaStream_t)stream>>>(
        params, D, sc, fc, omega, omega_sincos, hkl, offsets, ubis, ngrains, res, gvec,
        ubis ? ssq : nullptr, nullptr, nullptr, nullptr, nullptr);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_residuals_adjoint(const double* params, const double* detector,
                                           const double* sc, const double* fc,
                                           const double* omega, const double* omega_sincos,
                                           const double* hkl, const int64_t* offsets,
                                           const double* ubis, int32_t ngrains,
                                           const double* grad_res, double* grad_ubis,
                                           double* grad_params, void* workspace,
                                           int64_t ws_bytes, void* stream) {
    AdjDet D;
    if (!params || adj_det(detector, D) || ngrains < 0 || !grad_params) return ID11B_ERR_ARG;
    if (osc_misaligned(omega_sincos)) return ID11B_ERR_ALIGN;
    cudaStream_t st = (cudaStream_t)stream;
    if (ngrains == 0) {
        ID11B_CHECK(cudaMemsetAsync(grad_params, 0, sizeof(double) * kNP, st));
        return ID11B_OK;
    }
    if (!offsets || !sc || !fc || !omega || !hkl || !ubis || !grad_res || !workspace)
        return ID11B_ERR_ARG;
    if (ws_bytes < id11b_adjoint_workspace_bytes(ngrains)) return ID11B_ERR_SIZE;
    double* partial = (double*)workspace;
    k_residual<1><<<adj_grid(ngrains), kAT, 0, st>>>(params, D, sc, fc, omega, omega_sincos, hkl,
                                                     offsets, ubis, ngrains, nullptr, nullptr,
                                                     nullptr, grad_res, grad_ubis, partial,
                                                     nullptr);
    ID11B_CHECK_LAUNCH();
    k_finish<<<1, 32 * kPart, 0, st>>>(partial, ngrains, params, D, grad_params, nullptr);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_residual_loss(const double* params, const double* detector,
                                       const double* sc, const double* fc, const double* omega,
                                       const double* omega_sincos, const double* hkl,
                                       const int64_t* offsets, const double* ubis,
                                       int32_t ngrains, double* loss, double* grad_ubis,
                                       double* grad_params, double* ubis_out, void* workspace,
                                       int64_t ws_bytes, void* stream) {
    AdjDet D;
    if (!params || adj_det(detector, D) || ngrains < 0 || !loss) return ID11B_ERR_ARG;
    if (!ubis && grad_ubis) return ID11B_ERR_ARG;
    if (osc_misaligned(omega_sincos)) return ID11B_ERR_ALIGN;
    cudaStream_t st = (cudaStream_t)stream;
    if (ngrains == 0) {
        ID11B_CHECK(cudaMemsetAsync(loss, 0, sizeof(double), st));
        if (grad_params) ID11B_CHECK(cudaMemsetAsync(grad_params, 0, sizeof(double) * kNP, st));
        return ID11B_OK;
    }
    if (!offsets || !sc || !fc || !omega || !hkl || !workspace) return ID11B_ERR_ARG;
    if (ws_bytes < id11b_adjoint_workspace_bytes(ngrains)) return ID11B_ERR_SIZE;
    double* partial = (double*)workspace;
    const int grid = adj_grid(ngrains);
    if (ubis)
        k_residual<2><<<grid, kAT, 0, st>>>(params, D, sc, fc, omega, omega_sincos, hkl, offsets,
                                            ubis, ngrains, nullptr, nullptr, nullptr, nullptr,
                                            grad_ubis, partial, nullptr);
    else
        k_residual<3><<<grid, kAT, 0, st>>>(params, D, sc, fc, omega, omega_sincos, hkl, offsets,
                                            nullptr, ngrains, nullptr, nullptr, nullptr, nullptr,
                                            nullptr, partial, ubis_out);
    ID11B_CHECK_LAUNCH();
    k_finish<<<1, 32 * kPart, 0, st>>>(partial, ngrains, params, D, grad_params, loss);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_best_ubis(const double* params, const double* detector,
                                   const double* sc, const double* fc, const double* omega,
                                   const double* omega_sincos, const double* hkl,
                                   const int64_t* offsets, int32_t ngrains, double* ubis_out,
                                   void* stream) {
    AdjDet D;
    if (!params || adj_det(detector, D) || ngrains < 0) return ID11B_ERR_ARG;
    if (osc_misaligned(omega_sincos)) return ID11B_ERR_ALIGN;
    if (ngrains == 0) return ID11B_OK;
    if (!offsets || !sc || !fc || !omega || !hkl || !ubis_out) return ID11B_ERR_ARG;
    k_residual<4><<<adj_grid(ngrains), kAT, 0, (cudaStream_t)stream>>>(
        params, D, sc, fc, omega, omega_sincos, hkl, offsets, nullptr, ngrains, nullptr,
        nullptr, nullptr, nullptr, nullptr, nullptr, ubis_out);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_bragg_theta(const double* ubs, const double* hkl,
                                     const int64_t* offsets, int32_t ngrains, double wavelength,
                                     double* theta, double* dtheta_dub, void* stream) {
    if (ngrains < 0) return ID11B_ERR_ARG;
    if (ngrains == 0) return ID11B_OK;
    if (!ubs || !hkl || !offsets || !theta) return ID11B_ERR_ARG;
    k_bragg<false><<<adj_grid(ngrains), kAT, 0, (cudaStream_t)stream>>>(
        ubs, hkl, offsets, ngrains, wavelength, theta, dtheta_dub, nullptr, nullptr);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_bragg_theta_adjoint(const double* ubs, const double* hkl,
                                             const int64_t* offsets, int32_t ngrains,
                                             double wavelength, const double* grad_theta,
                                             double* grad_ubs, void* stream) {
    if (ngrains < 0) return ID11B_ERR_ARG;
    if (ngrains == 0) return ID11B_OK;
    if (!ubs || !hkl || !offsets || !grad_theta || !grad_ubs) return ID11B_ERR_ARG;
    k_bragg<true><<<adj_grid(ngrains), kAT, 0, (cudaStream_t)stream>>>(
        ubs, hkl, offsets, ngrains, wavelength, nullptr, nullptr, grad_theta, grad_ubs);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_omega_sincos(const double* omega, int64_t n, double omegasign,
                                      double* sincos_out, void* stream) {
    if (n < 0) return ID11B_ERR_ARG;
    if (n == 0) return ID11B_OK;
    if (!omega || !sincos_out) return ID11B_ERR_ARG;
    if ((uintptr_t)sincos_out & 15) return ID11B_ERR_ALIGN;
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 32);
    k_omega_sincos<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(omega, n, omegasign,
                                                                      sincos_out);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}
