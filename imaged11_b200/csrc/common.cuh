// Shared device helpers for the imaged11_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/imaged11_b200.h"

namespace id11b {

// ---------------------------------------------------------------------------
// Exact FP64.  The reference C is compiled without FMA contraction and sums
// left to right (ImageD11 src/closest.c:236-243).  These wrappers are never
// fused by nvcc, so kernels written with them reproduce the reference's
// rounding operation by operation.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Round to nearest, ties to even, through the magic constant 1.5*2^52, the
// same two additions as ImageD11 src/closest.c:84-85.
constexpr double kMagic = 6755399441055744.0;
__device__ __forceinline__ double dround(double x) { return dsub(dadd(x, kMagic), kMagic); }

// (a0*b0 + a1*b1) + a2*b2 without contraction.
__device__ __forceinline__ double ddot3(double a0, double a1, double a2, double b0,
                                        double b1, double b2) {
    return dadd(dadd(dmul(a0, b0), dmul(a1, b1)), dmul(a2, b2));
}

// The reference's per-peak test: h = UBI.g, t = h - round(h),
// sumsq = (t0^2 + t1^2) + t2^2.  Returns sumsq; ih receives round(h).
__device__ __forceinline__ double drlv2_exact(const double u[9], double g0, double g1,
                                              double g2, double ih[3]) {
    double h0 = ddot3(u[0], u[1], u[2], g0, g1, g2);
    double h1 = ddot3(u[3], u[4], u[5], g0, g1, g2);
    double h2 = ddot3(u[6], u[7], u[8], g0, g1, g2);
    ih[0] = dround(h0);
    ih[1] = dround(h1);
    ih[2] = dround(h2);
    double t0 = dsub(h0, ih[0]), t1 = dsub(h1, ih[1]), t2 = dsub(h2, ih[2]);
    return dadd(dadd(dmul(t0, t0), dmul(t1, t1)), dmul(t2, t2));
}

// Cofactor inverse with the reference's exact expression order
// (ImageD11 src/closest.c:38-76).  Returns -1 and leaves m alone if det == 0.
__device__ __forceinline__ int inverse3x3_exact(double m[9]) {
    double a00 = m[0], a01 = m[1], a02 = m[2], a10 = m[3], a11 = m[4], a12 = m[5],
           a20 = m[6], a21 = m[7], a22 = m[8];
    double det = dadd(dsub(dmul(a00, dsub(dmul(a22, a11), dmul(a21, a12))),
                           dmul(a10, dsub(dmul(a22, a01), dmul(a21, a02)))),
                      dmul(a20, dsub(dmul(a12, a01), dmul(a11, a02))));
    if (!(det != 0.)) return -1;
    double r[9];
    r[0] = ddiv(dsub(dmul(a22, a11), dmul(a21, a12)), det);
    r[1] = ddiv(-dsub(dmul(a22, a01), dmul(a21, a02)), det);
    r[2] = ddiv(dsub(dmul(a12, a01), dmul(a11, a02)), det);
    r[3] = ddiv(-dsub(dmul(a22, a10), dmul(a20, a12)), det);
    r[4] = ddiv(dsub(dmul(a22, a00), dmul(a20, a02)), det);
    r[5] = ddiv(-dsub(dmul(a12, a00), dmul(a10, a02)), det);
    r[6] = ddiv(dsub(dmul(a21, a10), dmul(a20, a11)), det);
    r[7] = ddiv(-dsub(dmul(a21, a00), dmul(a20, a01)), det);
    r[8] = ddiv(dsub(dmul(a11, a00), dmul(a10, a01)), det);
#pragma unroll
    for (int i = 0; i < 9; i++) m[i] = r[i];
    return 0;
}

// UB = R.inv(H), UBI = inv(UB); ubi is replaced only when both inverses exist
// (ImageD11 src/closest.c:326-340).  UB(i,j) sums l = 0,1,2 starting from 0.
__device__ __forceinline__ void lsq_update_exact(double R[9], double H[9], double ubi[9]) {
    double UB[9];
    int k = inverse3x3_exact(H);
    if (k != 0) return;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double s = 0.;
            s = dadd(s, dmul(R[3 * i + 0], H[0 + j]));
            s = dadd(s, dmul(R[3 * i + 1], H[3 + j]));
            s = dadd(s, dmul(R[3 * i + 2], H[6 + j]));
            UB[3 * i + j] = s;
        }
    if (inverse3x3_exact(UB) == 0) {
#pragma unroll
        for (int i = 0; i < 9; i++) ubi[i] = UB[i];
    }
}

// Order-free sums of non-negative terms (drlv2): each term rounded to a
// multiple of 1/scale and added as a 64-bit integer into the 8 bytes of its
// double output slot (zeroed first), so that the total is the same whatever
// order the atomics land in; id11b_fixsum_finish turns the slots back into
// doubles.  fixsum_scale picks the largest power of two for which n terms
// below tmax^2 cannot pass 2^62 (2^48 for 1.1M g at tol 0.1: a term is then
// off by at most 2^-49).
__device__ __forceinline__ void fixsum_add(double* slot, double x, double scale) {
    atomicAdd(reinterpret_cast<unsigned long long*>(slot), __double2ull_rn(x * scale));
}
inline double fixsum_scale(int64_t n, double tmax) {
    const double t2 = tmax * tmax > 1e-300 ? tmax * tmax : 1e-300;
    int e = 0;
    frexp(4.611686018427387904e18 / ((double)(n > 0 ? n : 1) * t2), &e);  // 2^62 / worst
    e -= 1;                                                                 // floor(log2)
    e = e < 20 ? 20 : (e > 60 ? 60 : e);
    return ldexp(1.0, e);
}

// Warp sums (fixed butterfly order, so results are reproducible run to run).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ long long warp_sum(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace id11b

// Status from a launch: 0, or ID11B_ERR_CUDA with the CUDA code recorded.
int id11b_record_cuda(cudaError_t e);
// The n slots that fixsum_add accumulated with this scale, converted to
// doubles in place.
int id11b_fixsum_finish(double* sums, int64_t n, double scale, cudaStream_t st);
#define ID11B_CHECK_LAUNCH()                                             \
    do {                                                                 \
        cudaError_t _e = cudaGetLastError();                             \
        if (_e != cudaSuccess) return id11b_record_cuda(_e);             \
    } while (0)
#define ID11B_CHECK(call)                                                \
    do {                                                                 \
        cudaError_t _e = (call);                                         \
        if (_e != cudaSuccess) return id11b_record_cuda(_e);             \
    } while (0)
