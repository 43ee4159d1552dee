/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the grain-scoring path.
 *
 * This file restates, in plain C99, the arithmetic of ImageD11's native
 * grain-scoring functions so that the CUDA kernels of imaged11_b200 can be
 * checked against it.  Nothing in the product links or calls this code: only
 * tests/, the smoke check and the CPU-baseline leg of bench.py load it.
 *
 * Every function follows the operation order of the reference so that, with
 * FMA contraction disabled (-ffp-contract=off, see the Makefile), results are
 * bit-identical to the reference's compiled C on the same host:
 *   - products and sums are evaluated left to right, e.g. (a*b + c*d) + e*f;
 *   - rounding to the nearest integer uses the magic-constant add/subtract
 *     (x + 6755399441055744.0) - 6755399441055744.0 (round half to even);
 *   - acceptance is the strict test sumsq < tol*tol.
 * Parity of this restatement with the reference is pinned by the golden
 * vectors in tests/golden (made by tests/golden/make_golden.py from the
 * reference's own compiled C and its numpy transform module).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846
#define ORC_MAGIC 6755399441055744.0

/* ImageD11 src/closest.c:84-85 (conv_double_to_int_fast). */
static inline double orc_round(double x) { return (x + ORC_MAGIC) - ORC_MAGIC; }

/* ImageD11 src/closest.c:100-119 (verify_rounding): compare the magic-constant
 * rounding with floor(x + 0.5) on a grid that avoids exact halves. */
int orc_verify_rounding(int n) {
    int bad = 0;
    for (int pass = 0; pass < 2; pass++) {
        for (int i = -100; i < 200; i++) {
            double v = (pass == 0 ? n : -n) + i * 50.0;
            int fast = (int)orc_round(v);
            int slow = (int)floor(v + 0.5);
            bad += (fast != slow);
        }
    }
    return bad;
}

/* ImageD11 src/closest.c:38-76 (inverse3x3): cofactor inverse divided by the
 * determinant, in place; returns -1 (and leaves m alone) when det == 0. */
int orc_inverse3x3(double m[9]) {
    double a00 = m[0], a01 = m[1], a02 = m[2];
    double a10 = m[3], a11 = m[4], a12 = m[5];
    double a20 = m[6], a21 = m[7], a22 = m[8];
    double det = a00 * (a22 * a11 - a21 * a12) - a10 * (a22 * a01 - a21 * a02) +
                 a20 * (a12 * a01 - a11 * a02);
    if (!(det != 0.))
        return -1;
    double r[9];
    r[0] = (a22 * a11 - a21 * a12) / det;
    r[1] = -(a22 * a01 - a21 * a02) / det;
    r[2] = (a12 * a01 - a11 * a02) / det;
    r[3] = -(a22 * a10 - a20 * a12) / det;
    r[4] = (a22 * a00 - a20 * a02) / det;
    r[5] = -(a12 * a00 - a10 * a02) / det;
    r[6] = (a21 * a10 - a20 * a11) / det;
    r[7] = -(a21 * a00 - a20 * a01) / det;
    r[8] = (a11 * a00 - a10 * a01) / det;
    memcpy(m, r, sizeof(r));
    return 0;
}

/* Chi.wedge matrix as built at ImageD11 src/cdiffraction.c:117-142.  The
 * reference's RAD macro expands textually, so sin(wedge*RAD) evaluates
 * (wedge*pi)/180. */
static void orc_wedgechi(double wedge, double chi, double mat[9]) {
    double sw = sin(wedge * ORC_PI / 180.0), cw = cos(wedge * ORC_PI / 180.0);
    double sc = sin(chi * ORC_PI / 180.0), cc = cos(chi * ORC_PI / 180.0);
    double w[9] = {cw, 0.0, -sw, 0., 1.0, 0., sw, 0.0, cw};
    double c[9] = {1., 0.0, 0., 0., cc, -sc, 0., sc, cc};
    /* element (i,j) = sum_k c[3k+j] * w[3i+k], summed k = 0,1,2 */
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            mat[3 * i + j] = c[j] * w[3 * i] + c[3 + j] * w[3 * i + 1] +
                             c[6 + j] * w[3 * i + 2];
}

void orc_wedgechi_matrix(double wedge, double chi, double mat[9]) {
    orc_wedgechi(wedge, chi, mat);
}

/* ImageD11 src/cdiffraction.c:112-168 (compute_gv). */
void orc_compute_gv(const double *xlylzl, const double *omega, double omegasign,
                    double wvln, double wedge, double chi, const double *t,
                    double *gv, int64_t n) {
    double m[9];
    orc_wedgechi(wedge, chi, m);
    const double rad = ORC_PI / 180.0;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        double ang = rad * omega[i] * omegasign;
        double so = sin(ang), co = cos(ang);
        double u0 = co * t[0] - so * t[1];
        double u1 = so * t[0] + co * t[1];
        double u2 = t[2];
        double o0 = m[0] * u0 + m[1] * u1 + m[2] * u2;
        double o1 = m[3] * u0 + m[4] * u1 + m[5] * u2;
        double o2 = m[6] * u0 + m[7] * u1 + m[8] * u2;
        double d0 = xlylzl[3 * i] - o0;
        double d1 = xlylzl[3 * i + 1] - o1;
        double d2 = xlylzl[3 * i + 2] - o2;
        double inv = 1. / sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        double ds = 1. / wvln;
        double k0 = ds * (d0 * inv - 1.);
        double k1 = ds * d1 * inv;
        double k2 = ds * d2 * inv;
        double v0 = m[0] * k0 + m[3] * k1 + m[6] * k2;
        double v1 = m[1] * k0 + m[4] * k1 + m[7] * k2;
        double v2 = m[2] * k0 + m[5] * k1 + m[8] * k2;
        gv[3 * i] = co * v0 + so * v1;
        gv[3 * i + 1] = -so * v0 + co * v1;
        gv[3 * i + 2] = v2;
    }
}

/* ImageD11 src/cdiffraction.c:31-94 (compute_geometry): tth, eta, ds, g. */
void orc_compute_geometry(const double *xlylzl, const double *omega,
                          double omegasign, double wvln, double wedge,
                          double chi, const double *t, double *out, int64_t n) {
    double m[9];
    orc_wedgechi(wedge, chi, m);
    const double rad = ORC_PI / 180.0;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        double ang = rad * omega[i] * omegasign;
        double so = sin(ang), co = cos(ang);
        double u0 = co * t[0] - so * t[1];
        double u1 = so * t[0] + co * t[1];
        double u2 = t[2];
        double o0 = m[0] * u0 + m[1] * u1 + m[2] * u2;
        double o1 = m[3] * u0 + m[4] * u1 + m[5] * u2;
        double o2 = m[6] * u0 + m[7] * u1 + m[8] * u2;
        double d0 = xlylzl[3 * i] - o0;
        double d1 = xlylzl[3 * i + 1] - o1;
        double d2 = xlylzl[3 * i + 2] - o2;
        double inv = 1. / sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        double *o = out + 6 * i;
        o[0] = 180.0 / ORC_PI * atan2(sqrt(d1 * d1 + d2 * d2), d0);
        double ds = 1. / wvln;
        double k0 = ds * (d0 * inv - 1.);
        double k1 = ds * d1 * inv;
        double k2 = ds * d2 * inv;
        o[1] = 180.0 / ORC_PI * atan2(-d1, d2);
        o[2] = sqrt(k0 * k0 + k1 * k1 + k2 * k2);
        double v0 = m[0] * k0 + m[3] * k1 + m[6] * k2;
        double v1 = m[1] * k0 + m[4] * k1 + m[7] * k2;
        double v2 = m[2] * k0 + m[5] * k1 + m[8] * k2;
        o[3] = co * v0 + so * v1;
        o[4] = -so * v0 + co * v1;
        o[5] = v2;
    }
}

/* ImageD11 src/cdiffraction.c:190-224 (compute_xlylzl).
 * p = [s_cen, f_cen, s_size, f_size]; r is 3x3 row-major; dist is 3. */
void orc_compute_xlylzl(const double *s, const double *f, const double *p,
                        const double *r, const double *dist, double *xlylzl,
                        int64_t n) {
    for (int64_t i = 0; i < n; i++) {
        double v1 = (f[i] - p[1]) * p[3];
        double v2 = (s[i] - p[0]) * p[2];
        for (int j = 0; j < 3; j++)
            xlylzl[3 * i + j] = r[3 * j + 1] * v1 + r[3 * j + 2] * v2 + dist[j];
    }
}

/* h = UBI.g for one g (row sums left to right), ImageD11 src/closest.c:236-241 */
static inline void orc_hkl(const double *u, const double *g, double h[3]) {
    h[0] = u[0] * g[0] + u[1] * g[1] + u[2] * g[2];
    h[1] = u[3] * g[0] + u[4] * g[1] + u[5] * g[2];
    h[2] = u[6] * g[0] + u[7] * g[1] + u[8] * g[2];
}

/* ImageD11 src/closest.c:227-248 (score). */
int orc_score(const double *ubi, const double *gv, double tol, int64_t ng) {
    double tolsq = tol * tol;
    int n = 0;
    for (int64_t k = 0; k < ng; k++) {
        double h[3];
        orc_hkl(ubi, gv + 3 * k, h);
        double t0 = h[0] - orc_round(h[0]);
        double t1 = h[1] - orc_round(h[1]);
        double t2 = h[2] - orc_round(h[2]);
        double sumsq = t0 * t0 + t1 * t1 + t2 * t2;
        if (sumsq < tolsq)
            n++;
    }
    return n;
}

/* Least-squares update shared by score_and_refine and refine_assigned:
 * UB = R.inv(H); UBI = inv(UB); ubi untouched unless both inverses exist.
 * ImageD11 src/closest.c:326-340 and :460-473. */
static void orc_lsq_update(double R[9], double H[9], double *ubi) {
    double UB[9] = {0};
    int k = orc_inverse3x3(H);
    if (k == 0) {
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                for (int l = 0; l < 3; l++)
                    UB[3 * i + j] += R[3 * i + l] * H[3 * l + j];
    }
    if (k == 0 && orc_inverse3x3(UB) == 0)
        memcpy(ubi, UB, sizeof(UB));
}

/* ImageD11 src/closest.c:267-345 (score_and_refine).  Writes the count and
 * the mean drlv2 of the accepted peaks (both before the update). */
void orc_score_and_refine(double *ubi, const double *gv, double tol,
                          int *n_out, double *mean_drlv2, int64_t ng) {
    double R[9] = {0}, H[9] = {0};
    double tolsq = tol * tol, sumdrlv2 = 0.;
    int n = 0;
    for (int64_t k = 0; k < ng; k++) {
        const double *g = gv + 3 * k;
        double h[3];
        orc_hkl(ubi, g, h);
        double t0 = h[0] - orc_round(h[0]);
        double t1 = h[1] - orc_round(h[1]);
        double t2 = h[2] - orc_round(h[2]);
        double sumsq = t0 * t0 + t1 * t1 + t2 * t2;
        if (sumsq < tolsq) {
            n++;
            sumdrlv2 += sumsq;
            double ih[3] = {orc_round(h[0]), orc_round(h[1]), orc_round(h[2])};
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    R[3 * i + j] = R[3 * i + j] + ih[j] * g[i];
                    H[3 * i + j] = H[3 * i + j] + ih[j] * ih[i];
                }
        }
    }
    orc_lsq_update(R, H, ubi);
    if (n > 0)
        sumdrlv2 /= n;
    *n_out = n;
    *mean_drlv2 = sumdrlv2;
}

/* ImageD11 src/closest.c:416-474 (refine_assigned). */
void orc_refine_assigned(double *ubi, const double *gv, const int32_t *labels,
                         int label, int *npk, double *mean_drlv2, int64_t ng) {
    double R[9] = {0}, H[9] = {0}, sumsqtot = 0;
    int n = 0;
    for (int64_t k = 0; k < ng; k++) {
        if (label != labels[k])
            continue;
        n++;
        const double *g = gv + 3 * k;
        double h[3], ih[3], t[3];
        orc_hkl(ubi, g, h);
        for (int j = 0; j < 3; j++) {
            ih[j] = orc_round(h[j]);
            t[j] = h[j] - ih[j];
        }
        sumsqtot += t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                R[3 * i + j] = R[3 * i + j] + ih[j] * g[i];
                H[3 * i + j] = H[3 * i + j] + ih[j] * ih[i];
            }
    }
    *npk = n;
    *mean_drlv2 = n > 0 ? sumsqtot / n : 0.;
    orc_lsq_update(R, H, ubi);
}

/* ImageD11 src/closest.c:366-397 (score_and_assign). */
int orc_score_and_assign(const double *ubi, const double *gv, double tol,
                         double *drlv2, int32_t *labels, int label, int64_t ng) {
    double tolsq = tol * tol;
    int n = 0;
#pragma omp parallel for reduction(+ : n) schedule(static, 4096)
    for (int64_t k = 0; k < ng; k++) {
        double h[3];
        orc_hkl(ubi, gv + 3 * k, h);
        double t0 = h[0] - orc_round(h[0]);
        double t1 = h[1] - orc_round(h[1]);
        double t2 = h[2] - orc_round(h[2]);
        double sumsq = t0 * t0 + t1 * t1 + t2 * t2;
        if ((sumsq < tolsq) && (sumsq < drlv2[k])) {
            labels[k] = label;
            drlv2[k] = sumsq;
            n++;
        } else if (labels[k] == label) {
            labels[k] = -1;
        }
    }
    return n;
}

/* ---- batched helpers (loops of the single-call functions above) ---- */

/* counts[m*T + j] = score(ubis[m], gv, tols[j]); OpenMP over UBIs. */
void orc_score_many(const double *ubis, int64_t m, const double *gv, int64_t ng,
                    const double *tols, int ntol, int32_t *counts) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < m; i++)
        for (int j = 0; j < ntol; j++)
            counts[i * ntol + j] = orc_score(ubis + 9 * i, gv, tols[j], ng);
}

/* Per grain g: `iters` score_and_refine calls over its own CSR segment
 * gv[offsets[g] : offsets[g+1]]; ubis updated in place; n and mean drlv2 of
 * the last iteration written out.  OpenMP over grains. */
void orc_refine_csr(double *ubis, const double *gv, const int64_t *offsets,
                    int64_t ngrains, double tol, int iters, int32_t *npk,
                    double *drlv2) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t g = 0; g < ngrains; g++) {
        int n = 0;
        double d = 0.;
        for (int it = 0; it < iters; it++)
            orc_score_and_refine(ubis + 9 * g, gv + 3 * offsets[g], tol, &n, &d,
                                 offsets[g + 1] - offsets[g]);
        npk[g] = n;
        drlv2[g] = d;
    }
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
