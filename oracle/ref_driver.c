/*
 * TEST INFRASTRUCTURE ONLY -- batch drivers around the reference's own C.
 *
 * Linked with the unmodified ImageD11 sources src/closest.c,
 * src/cdiffraction.c and src/cimaged11utils.c (compiled where they lie by
 * oracle/Makefile, output in oracle/_ref/).  The reference has no batched
 * entry point, and its Python `score` wrapper holds the GIL, so the CPU
 * baseline calls the reference functions from OpenMP loops here: one
 * reference call per (UBI, tolerance) or per (grain, iteration), exactly the
 * calls the reference's own Python callers make in a loop
 * (ImageD11/indexing.py:800, ImageD11/refinegrains.py:467).
 */
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double vec[3];
/* reference prototypes, ImageD11 src/closest.c:227, :267 */
int score(vec ubi[3], vec gv[], double tol, int ng);
void score_and_refine(vec ubi[3], vec gv[], double tol, int *n_arg,
                      double *sumdrlv2_arg, int ng);
/* ImageD11 src/closest.c:366 */
int score_and_assign(vec *ubi, vec *gv, double tol, double *drlv2, int *labels, int label,
                     int ng);

void ref_score_many(const double *ubis, int64_t m, const double *gv, int64_t ng,
                    const double *tols, int ntol, int32_t *counts) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < m; i++)
        for (int j = 0; j < ntol; j++)
            counts[i * ntol + j] =
                score((vec *)(ubis + 9 * i), (vec *)gv, tols[j], (int)ng);
}

void ref_refine_csr(double *ubis, const double *gv, const int64_t *offsets,
                    int64_t ngrains, double tol, int iters, int32_t *npk,
                    double *drlv2) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t g = 0; g < ngrains; g++) {
        int n = 0;
        double d = 0.;
        for (int it = 0; it < iters; it++)
            score_and_refine((vec *)(ubis + 9 * g), (vec *)(gv + 3 * offsets[g]),
                             tol, &n, &d, (int)(offsets[g + 1] - offsets[g]));
        npk[g] = n;
        drlv2[g] = d;
    }
}

/* score_and_assign for grains 0 .. m-1 in order, as fight_over_peaks calls it
   (ImageD11/indexing.py); the reference parallelises each call over the g. */
void ref_assign_seq(const double *ubis, int64_t m, const double *gv, int64_t ng, double tol,
                    double *drlv2, int32_t *labels) {
    for (int64_t i = 0; i < m; i++)
        score_and_assign((vec *)(ubis + 9 * i), (vec *)gv, tol, drlv2, (int *)labels, (int)i,
                         (int)ng);
}

int ref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
