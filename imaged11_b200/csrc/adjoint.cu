// Residuals of assigned peaks and their hand-written adjoint (FP64).
//
// Forward model for peak k of grain G (peaks stored grain by grain, CSR):
//   detector -> lab (ImageD11 src/cdiffraction.c:190-224)
//     v1 = (f - y_center) * y_size,  v2 = (s - z_center) * z_size
//     xyz = r[:,1] v1 + r[:,2] v2 + (distance, 0, 0),     r = tilts . flip
//   lab -> g (ImageD11 src/cdiffraction.c:112-168)
//     u = Omega(w)^T t,  o = M u,  d = xyz - o,  dh = d / |d|
//     k = (dh - x) / wavelength,  v = M^T k,  g = Omega(w) v,   M = chi.wedge
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
//
// One CTA per grain accumulates its peaks' terms in registers and reduces
// them in a fixed tree, so dL/dUBI and the 22 global sums are deterministic;
// the global sums go to a per-grain partial array that one CTA then reduces in
// grain order.  The caller (imaged11_b200/adjoint.py) maps dL/dM, dL/dr and the
// centre/distance sums onto wedge, chi, tilts, centres and distance.
#include "common.cuh"

namespace id11b {

constexpr int kAT = 64;         // threads per CTA
constexpr int kGlob = 22;       // dM(9) dlam(1) dt(3) sum_axyz(3) dR1(3) dR2(3)

struct AdjGeom {
    double r[9];        // detector rotation . flip (row-major)
    double M[9];        // chi.wedge
    double t[3];        // grain-origin translation
    double wavelength, distance, y_center, z_center, y_size, z_size, omegasign;
};

struct PeakState {
    double so, co, u[3], v1, v2, dh[3], n, k[3], g[3];
};

__device__ __forceinline__ void forward_peak(const AdjGeom& P, double s, double f, double om,
                                             PeakState& q) {
    const double rad = 3.14159265358979323846 / 180.0;
    q.v1 = (f - P.y_center) * P.y_size;
    q.v2 = (s - P.z_center) * P.z_size;
    double xyz[3];
#pragma unroll
    for (int j = 0; j < 3; j++) xyz[j] = P.r[3 * j + 1] * q.v1 + P.r[3 * j + 2] * q.v2;
    xyz[0] += P.distance;
    sincos(rad * om * P.omegasign, &q.so, &q.co);
    q.u[0] = q.co * P.t[0] - q.so * P.t[1];
    q.u[1] = q.so * P.t[0] + q.co * P.t[1];
    q.u[2] = P.t[2];
    double d[3];
#pragma unroll
    for (int i = 0; i < 3; i++)
        d[i] = xyz[i] - (P.M[3 * i] * q.u[0] + P.M[3 * i + 1] * q.u[1] + P.M[3 * i + 2] * q.u[2]);
    q.n = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
#pragma unroll
    for (int i = 0; i < 3; i++) q.dh[i] = d[i] / q.n;
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

// MODE 0: residuals (+ per-grain sum of squares); MODE 1: adjoint.
template <int MODE>
__global__ void __launch_bounds__(kAT)
k_residual(AdjGeom P, const double* __restrict__ sc, const double* __restrict__ fc,
           const double* __restrict__ omega, const double* __restrict__ hkl,
           const int64_t* __restrict__ off, const double* __restrict__ ubis, int ngrains,
           double* __restrict__ res, double* __restrict__ gout, double* __restrict__ ssq,
           const double* __restrict__ ares, double* __restrict__ dubi,
           double* __restrict__ partial) {
    constexpr int NA = MODE == 0 ? 1 : 9 + kGlob;
    __shared__ double s_red[kAT / 32][NA];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int G = blockIdx.x; G < ngrains; G += gridDim.x) {
        double U[9];
#pragma unroll
        for (int e = 0; e < 9; e++) U[e] = ubis[9 * (int64_t)G + e];
        double acc[NA];
#pragma unroll
        for (int e = 0; e < NA; e++) acc[e] = 0.;
        for (int64_t kk = off[G] + tid; kk < off[G + 1]; kk += kAT) {
            PeakState q;
            forward_peak(P, sc[kk], fc[kk], omega[kk], q);
            if (MODE == 0) {
                double ss = 0.;
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    const double ri = U[3 * i] * q.g[0] + U[3 * i + 1] * q.g[1] +
                                      U[3 * i + 2] * q.g[2] - hkl[3 * kk + i];
                    res[3 * kk + i] = ri;
                    if (gout) gout[3 * kk + i] = q.g[i];
                    ss += ri * ri;
                }
                acc[0] += ss;
            } else {
                const double ar[3] = {ares[3 * kk], ares[3 * kk + 1], ares[3 * kk + 2]};
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int j = 0; j < 3; j++) acc[3 * i + j] += ar[i] * q.g[j];  // dL/dUBI
                double ag[3], av[3], ak[3];
#pragma unroll
                for (int j = 0; j < 3; j++) ag[j] = U[j] * ar[0] + U[3 + j] * ar[1] + U[6 + j] * ar[2];
                av[0] = q.co * ag[0] - q.so * ag[1];
                av[1] = q.so * ag[0] + q.co * ag[1];
                av[2] = ag[2];
#pragma unroll
                for (int i = 0; i < 3; i++)
                    ak[i] = P.M[3 * i] * av[0] + P.M[3 * i + 1] * av[1] + P.M[3 * i + 2] * av[2];
                double* gl = acc + 9;
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
                for (int i = 0; i < 3; i++) ad[i] = (adh[i] - q.dh[i] * dd) / q.n;
                // o = M u: dM[i][j] += a_o_i u_j with a_o = -a_d
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int j = 0; j < 3; j++) gl[3 * i + j] -= ad[i] * q.u[j];
                double au[3];
#pragma unroll
                for (int j = 0; j < 3; j++)
                    au[j] = -(P.M[j] * ad[0] + P.M[3 + j] * ad[1] + P.M[6 + j] * ad[2]);
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
        }
#pragma unroll
        for (int e = 0; e < NA; e++) acc[e] = warp_sum(acc[e]);
        if (lane == 0)
#pragma unroll
            for (int e = 0; e < NA; e++) s_red[w][e] = acc[e];
        __syncthreads();
        for (int e = tid; e < NA; e += kAT) {
            double t = 0.;
            for (int q = 0; q < kAT / 32; q++) t += s_red[q][e];
            if (MODE == 0) {
                ssq[G] = t;
            } else if (e < 9) {
                dubi[9 * (int64_t)G + e] = t;
            } else {
                partial[(int64_t)G * kGlob + (e - 9)] = t;
            }
        }
        __syncthreads();
    }
}

// Column sums of x (rows x cols) -> out (cols); one CTA, one warp per column:
// lane l sums rows l, l+32, ... in order, then a fixed butterfly, so the
// result does not depend on timing.
__global__ void k_sum_rows(const double* __restrict__ x, int rows, int cols,
                           double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    for (int c = threadIdx.x >> 5; c < cols; c += blockDim.x >> 5) {
        double t = 0.;
        for (int r = lane; r < rows; r += 32) t += x[(int64_t)r * cols + c];
        t = warp_sum(t);
        if (lane == 0) out[c] = t;
    }
}

}  // namespace id11b

using namespace id11b;

static int adj_geom(const double* g, AdjGeom& P) {
    if (!g) return ID11B_ERR_ARG;
    for (int i = 0; i < 9; i++) P.r[i] = g[i];
    for (int i = 0; i < 9; i++) P.M[i] = g[9 + i];
    for (int i = 0; i < 3; i++) P.t[i] = g[18 + i];
    P.wavelength = g[21];
    P.distance = g[22];
    P.y_center = g[23];
    P.z_center = g[24];
    P.y_size = g[25];
    P.z_size = g[26];
    P.omegasign = g[27];
    return ID11B_OK;
}

extern "C" int64_t id11b_adjoint_workspace_bytes(int32_t ngrains) {
    return (int64_t)sizeof(double) * kGlob * (ngrains > 0 ? ngrains : 1);
}

extern "C" int id11b_dev_residuals(const double* geom_host, const double* sc, const double* fc,
                                   const double* omega, const double* hkl,
                                   const int64_t* offsets, const double* ubis, int32_t ngrains,
                                   double* res, double* gvec, double* ssq, void* stream) {
    AdjGeom P;
    if (adj_geom(geom_host, P) || ngrains < 0) return ID11B_ERR_ARG;
    if (ngrains == 0) return ID11B_OK;
    if (!offsets || !ubis || !res || !ssq) return ID11B_ERR_ARG;
    k_residual<0><<<ngrains, kAT, 0, (cudaStream_t)stream>>>(
        P, sc, fc, omega, hkl, offsets, ubis, ngrains, res, gvec, ssq, nullptr, nullptr, nullptr);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

extern "C" int id11b_dev_residuals_adjoint(const double* geom_host, const double* sc,
                                           const double* fc, const double* omega,
                                           const double* hkl, const int64_t* offsets,
                                           const double* ubis, int32_t ngrains,
                                           const double* grad_res, double* grad_ubis,
                                           double* grad_global, void* workspace,
                                           int64_t ws_bytes, void* stream) {
    AdjGeom P;
    if (adj_geom(geom_host, P) || ngrains < 0 || !grad_global) return ID11B_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (ngrains == 0) {
        ID11B_CHECK(cudaMemsetAsync(grad_global, 0, sizeof(double) * kGlob, st));
        return ID11B_OK;
    }
    if (!offsets || !ubis || !grad_res || !grad_ubis || !workspace) return ID11B_ERR_ARG;
    if (ws_bytes < id11b_adjoint_workspace_bytes(ngrains)) return ID11B_ERR_SIZE;
    double* partial = (double*)workspace;
    k_residual<1><<<ngrains, kAT, 0, st>>>(P, sc, fc, omega, hkl, offsets, ubis, ngrains,
                                           nullptr, nullptr, nullptr, grad_res, grad_ubis,
                                           partial);
    ID11B_CHECK_LAUNCH();
    k_sum_rows<<<1, 32 * kGlob, 0, st>>>(partial, ngrains, kGlob, grad_global);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}
