/*
 * imaged11_b200 -- C ABI of the B200 (sm_100a) grain-scoring path.
 *
 * Two layers:
 *
 *  1. Reference-signature entry points (id11b_<name>): the exact C signatures
 *     that ImageD11's f2py module binds (src/_cImageD11.pyf), with HOST
 *     pointers.  Each call copies its inputs to the GPU, runs the kernels and
 *     copies the results back before returning, so a binding that today points
 *     at ImageD11's src/closest.c / src/cdiffraction.c can point here instead.
 *     Calls run on the calling thread's per-thread default stream and stage
 *     through device and pinned host buffers kept per host thread and device
 *     (up to 64 MB, grown on demand and held until the thread exits; larger
 *     calls draw from the CUDA stream-ordered pool), so concurrent calls from
 *     different host threads are safe (the reference marks score_and_refine
 *     and refine_assigned "threadsafe").
 *
 *  2. Device entry points (id11b_dev_<name>): DEVICE pointers for every array,
 *     scalars by value, small fixed-size parameter vectors (t[3], p[4], r[9],
 *     dist[3]) as HOST pointers read during the call, and a cudaStream_t passed
 *     as void*.  They only enqueue work; nothing is synchronised.  Kernels that
 *     need scratch memory take a caller-provided workspace whose size is given
 *     by the matching *_workspace_bytes() query.
 *
 * Every entry point returns an int status (ID11B_OK == 0) except where the
 * reference's own signature returns a value; those report failure as noted.
 * Scalar FP64 arithmetic that decides an assignment (rounding to hkl, the
 * strict drlv2 < tol^2 test) is bit-exact with the reference C.
 */
#ifndef IMAGED11_B200_H
#define IMAGED11_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define ID11B_OK 0
#define ID11B_ERR_ARG 1     /* bad argument (negative size, null pointer, ntol > 4) */
#define ID11B_ERR_CUDA 2    /* a CUDA call failed: see id11b_last_cuda_error()   */
#define ID11B_ERR_ALIGN 3   /* pointer not aligned as the kernel requires        */
#define ID11B_ERR_SIZE 4    /* size beyond a documented maximum                  */
#define ID11B_ERR_TIMEOUT 5 /* a bounded device wait gave up                     */
#define ID11B_ERR_NODEV 6   /* no CUDA device                                    */

#define ID11B_MAX_TOLS 4

/* ABI version (major*100 + minor). */
int id11b_version(void);
/* Human-readable text for a status code. */
const char *id11b_status_string(int status);
/* The cudaError_t behind the calling thread's last ID11B_ERR_CUDA. */
int id11b_last_cuda_error(void);

/* =====================================================================
 * Layer 1: reference signatures, host pointers.
 * ===================================================================== */

/* Replaces compute_gv, ImageD11 src/cdiffraction.c:112-168
 * (f2py: src/_cImageD11.pyf:551-564).  xlylzl (n,3), omega (n), t (3),
 * gv (n,3) written.  Returns nothing, like the reference; failures are
 * reported through id11b_last_status(). */
void id11b_compute_gv(double xlylzl[][3], double omega[], double omegasign,
                      double wvln, double wedge, double chi, double t[3],
                      double gv[][3], int n);

/* Replaces compute_geometry, ImageD11 src/cdiffraction.c:31-94
 * (f2py: src/_cImageD11.pyf:534-549).  out (n,6) = tth, eta, ds, gx, gy, gz. */
void id11b_compute_geometry(double xlylzl[][3], double omega[], double omegasign,
                            double wvln, double wedge, double chi, double t[3],
                            double out[][6], int n);

/* Replaces compute_xlylzl, ImageD11 src/cdiffraction.c:190-224
 * (f2py: src/_cImageD11.pyf:566-583).  p = [s_cen, f_cen, s_size, f_size],
 * r (9) = detector rotation . flip, row-major; dist (3). */
void id11b_compute_xlylzl(double s[], double f[], double p[4], double r[9],
                          double dist[3], double xlylzl[][3], int n);

/* Replaces score, ImageD11 src/closest.c:227-248 (f2py: src/_cImageD11.pyf:106-120).
 * Returns the count, or -1 on failure (see id11b_last_status()). */
int id11b_score(double ubi[3][3], double gv[][3], double tol, int ng);

/* Replaces score_and_refine, ImageD11 src/closest.c:267-345
 * (f2py: src/_cImageD11.pyf:123-136).  ubi is refined in place; *n_arg and
 * *sumdrlv2_arg receive the count and mean drlv2 before the update. */
void id11b_score_and_refine(double ubi[3][3], double gv[][3], double tol,
                            int *n_arg, double *sumdrlv2_arg, int ng);

/* Replaces refine_assigned, ImageD11 src/closest.c:416-474
 * (f2py: src/_cImageD11.pyf:156-170).  Uses peaks with labels[k] == label. */
void id11b_refine_assigned(double ubi[3][3], double gv[][3], int labels[], int label,
                           int *npk, double *sumdrlv2, int ng);

/* Replaces score_and_assign, ImageD11 src/closest.c:366-397
 * (f2py: src/_cImageD11.pyf:138-154).  drlv2 and labels updated in place.
 * Returns the count, or -1 on failure. */
int id11b_score_and_assign(double ubi[3][3], double gv[][3], double tol,
                           double drlv2[], int labels[], int label, int ng);

/* Replaces verify_rounding, ImageD11 src/closest.c:100-119
 * (f2py: src/_cImageD11.pyf:69-74): runs the check
 * with the GPU's rounding.  Returns the number of mismatches (0 = good), or
 * -1 on failure. */
int id11b_verify_rounding(int n);

/* Status of the calling thread's last layer-1 call. */
int id11b_last_status(void);

/* =====================================================================
 * Layer 2: device pointers + stream.
 * ===================================================================== */

/* compute_gv on device arrays.  If g4 is non-null it also receives an FP32
 * copy of every g as (gx, gy, gz, 0) float4 for the batched scorers (16-byte
 * aligned). */
int id11b_dev_compute_gv(const double *xlylzl, const double *omega, double omegasign,
                         double wvln, double wedge, double chi, const double *t_host,
                         double *gv, float *g4, int64_t n, void *stream);

int id11b_dev_compute_geometry(const double *xlylzl, const double *omega,
                               double omegasign, double wvln, double wedge, double chi,
                               const double *t_host, double *out, int64_t n,
                               void *stream);

int id11b_dev_compute_xlylzl(const double *s, const double *f, const double *p_host,
                             const double *r_host, const double *dist_host,
                             double *xlylzl, int64_t n, void *stream);

/* score: *count (device int32) = number of g with drlv2 < tol^2. */
int id11b_dev_score(const double *ubi, const double *gv, double tol, int64_t ng,
                    int32_t *count, void *stream);

/* Workspace for dev_score_and_refine / dev_refine_assigned. */
int64_t id11b_lsq_workspace_bytes(int64_t ng);

/* score_and_refine on device: ubi (9, device) refined in place; *n (int32)
 * and *mean_drlv2 (double) written on the device. */
int id11b_dev_score_and_refine(double *ubi, const double *gv, double tol, int64_t ng,
                               int32_t *n, double *mean_drlv2, void *workspace,
                               int64_t workspace_bytes, void *stream);

int id11b_dev_refine_assigned(double *ubi, const double *gv, const int32_t *labels,
                              int label, int64_t ng, int32_t *npk, double *mean_drlv2,
                              void *workspace, int64_t workspace_bytes, void *stream);

/* No counterpart in the reference.  score_and_refine on device pointers that
 * allocates nothing, for callers that cannot allocate device memory (a process
 * that has reserved the GPU's memory up front and forbids later allocations, or
 * a host running inside another framework's capped memory pool).  Same
 * arguments and results as id11b_dev_score_and_refine minus the workspace: the
 * scratch is a library-owned device array of id11b_noalloc_scratch_bytes()
 * bytes (136 KiB) that every GPU loading the library holds until the process
 * exits.  CUDA loads the module holding that array lazily, so the first call in
 * each context takes device memory: make one warm-up call per device (one
 * g-vector is enough) before reserving memory or capping the pool, and before
 * any stream capture.  The array's device address is cached per CUDA context
 * (a context recreated after cudaDeviceReset is looked up afresh).  ng beyond
 * 2^31-1 returns ID11B_ERR_SIZE.  All calls on a device share the array: calls
 * that overlap on the GPU race, so serialise them (one stream, or explicit
 * ordering). */
int64_t id11b_noalloc_scratch_bytes(void);
int id11b_dev_score_and_refine_noalloc(double *ubi, const double *gv, double tol, int64_t ng,
                                       int32_t *n, double *mean_drlv2, void *stream);

/* score_and_assign on device; *count (int32, device) receives the count. */
int id11b_dev_score_and_assign(const double *ubi, const double *gv, double tol,
                               double *drlv2, int32_t *labels, int label, int64_t ng,
                               int32_t *count, void *stream);

/* verify_rounding on the device; *bad (int32, device) = mismatches. */
int id11b_dev_verify_rounding(int n, int32_t *bad, void *stream);

/* =====================================================================
 * Batched extensions (no single reference function: each replaces a Python
 * loop of reference calls, as noted).  Device pointers + stream.
 * ===================================================================== */

/* Plain FP64 batched score: counts[m*ntol + j] = score(ubis[m], gv, tols[j]),
 * the loop of ImageD11/indexing.py:800 / :1095.  Reference arithmetic on the
 * GPU, one thread per g; the baseline the FP32 kernels are measured against. */
int id11b_dev_score_many_fp64(const double *ubis, int64_t m, const double *gv, int64_t ng,
                              const double *tols_host, int ntol, int32_t *counts,
                              void *stream);

/* compute_xlylzl followed by compute_geometry in one pass (the fast path of
 * ImageD11/columnfile.py updateGeometry, :497-504: Ctransform.sf2xyz then
 * xyz2geometry, ImageD11/transform.py:695-706, :754-774): slow/fast detector
 * positions sc, fc and omega (n doubles each) -> out (n,6) = tth, eta, ds,
 * gx, gy, gz, identical to the two reference calls in turn.  p, r, dist as
 * for compute_xlylzl; omegasign, wvln, wedge, chi, t as for compute_geometry.
 * xlylzl (n,3, optional) receives the lab positions; g4 (n float4, optional,
 * 16-byte aligned) the FP32 g copy of id11b_dev_prepare_gvecs.  No reference
 * counterpart as one function. */
int id11b_dev_update_geometry(const double *sc, const double *fc, const double *omega,
                              const double *p_host, const double *r_host,
                              const double *dist_host, double omegasign, double wvln,
                              double wedge, double chi, const double *t_host, double *xlylzl,
                              double *out, float *g4, int64_t n, void *stream);

/* Prepare g-vectors for the FP32 batched kernels: g4 (n float4, 16-byte
 * aligned) receives FP32 copies; gws (id11b_gvec_workspace_bytes(n), 256-byte
 * aligned) receives max|g| and the list of g evaluated in FP64 only
 * (non-finite, or a component beyond 1024). */
int64_t id11b_gvec_workspace_bytes(int64_t n);
int id11b_dev_prepare_gvecs(const double *gv, int64_t n, float *g4, void *gws,
                            int64_t gws_bytes, void *stream);

/* Workspace for id11b_dev_score_batch (refine = 0) / id11b_dev_refine_batch
 * (refine = 1) with m UBIs and n g-vectors. */
int64_t id11b_batch_workspace_bytes(int64_t m, int64_t n, int refine);

/* Batched score, FP32 screening with exact FP64 recheck of every pair within
 * a proven error band of tol^2: counts identical to the reference's score()
 * (ImageD11 src/closest.c:227-248) for every (UBI, tol).  counts (m, ntol)
 * int32; sums (m, ntol) double, optional: sum of drlv2 of the counted pairs
 * (FP32 values, relative error below 1e-5), accumulated in fixed point so
 * that they repeat bit for bit.  ntol <= ID11B_MAX_TOLS; a tolerance >= 0.45
 * sends every pair through exact FP64. */
int id11b_dev_score_batch(const double *ubis, int64_t m, const double *gv, const float *g4,
                          int64_t n, const void *gws, const double *tols_host, int ntol,
                          int32_t *counts, double *sums, void *ws, int64_t ws_bytes,
                          void *stream);

/* id11b_dev_score_batch with an explicit tile shape (no reference counterpart:
 * the reference scores one UBI per call).  A CTA holds 256 * ubis_per_thread
 * UBIs in registers (2 or 4; 0 = the build default, 4) and streams 1/gsplit of
 * the g-vectors through shared memory in 1,024-vector tiles (gsplit 0 = the
 * built-in heuristic, about four waves of CTAs; larger values are clamped to
 * one tile per CTA).  Counts do not depend on the tile shape.
 * id11b_score_tile_default reports the shape the heuristic picks. */
int id11b_score_tile_default(int64_t m, int64_t n, int *ubis_per_thread, int *gsplit);
int id11b_dev_score_batch_tiled(const double *ubis, int64_t m, const double *gv,
                                const float *g4, int64_t n, const void *gws,
                                const double *tols_host, int ntol, int32_t *counts,
                                double *sums, int ubis_per_thread, int gsplit, void *ws,
                                int64_t ws_bytes, void *stream);

/* Reciprocal-space cell index (no reference counterpart; it replaces the
 * reference's test of every g against every UBI in score(), ImageD11
 * src/closest.c:227-248, with a lookup of the g near each UB.hkl).
 * Regular g-vectors (finite, every |g_j| <= 1024) inside [-gmax, gmax]^3 and
 * within rmax of the origin are binned into nx^3 cubic cells of side cs over
 * that cube, sorted by cell (x fastest; within a cell by index); the others
 * are kept in an index list and scored by a plain scan (so bounds smaller
 * than the data's cost speed, never counts).
 *   1. id11b_dev_gvec_bounds: bounds[0] = max |g_j|, bounds[1] = max |g| over
 *      regular g, as float bits rounded up (device, 2 x uint32);
 *   2. id11b_grid_plan (host): nx and cs for n g-vectors; cell = 0 picks about
 *      one g per cell of the cube, else the requested side (nx <= 400);
 *   3. id11b_dev_build_grid into gridbuf (id11b_grid_bytes(n, nx, xsub),
 *      256-byte aligned): y and z cut into nx cells of side cs, x into
 *      nx * xsub cells of side cs / xsub (xsub 1..16, nx^3 * xsub <= 2^26).
 * id11b_dev_score_grid then gives the counts (and optional sums of drlv2) of
 * id11b_dev_score_batch, identical to the reference's score() for every
 * (UBI, tol): every candidate pair is evaluated in the reference's FP64
 * arithmetic.  A UBI whose lookup would cost more than a plain scan
 * (non-finite, singular, condition number above 1e6, more candidate hkl
 * than g) is scored by a plain scan.  id11b_grid_stats reports the regular and
 * listed g, and for the last score call the UBIs scanned plainly, the pairs
 * evaluated in FP64 and (binned calls) the (box, g) pairs screened in FP32. */
int id11b_dev_gvec_bounds(const double *gv, int64_t n, uint32_t *bounds, void *stream);
int id11b_grid_plan(float gmax, int64_t n, double cell, int32_t *nx, double *cs);
int64_t id11b_grid_bytes(int64_t n, int32_t nx, int32_t xsub);
int id11b_dev_build_grid(const double *gv, int64_t n, float gmax, float rmax, double cs,
                         int32_t nx, int32_t xsub, void *gridbuf, int64_t grid_bytes,
                         void *stream);
int64_t id11b_grid_score_workspace_bytes(int64_t m, int ntol);
int id11b_dev_score_grid(const double *ubis, int64_t m, const double *gv, int64_t n, int32_t nx,
                         int32_t xsub, const void *gridbuf, const double *tols_host, int ntol,
                         int32_t *counts, double *sums, void *ws, int64_t ws_bytes,
                         void *stream);
int id11b_grid_stats(const void *gridbuf, int64_t *nregular, int64_t *nspecial,
                     int64_t *nfallback, int64_t *ntested, int64_t *npairs, void *stream);

/* The same counts (and optional FP64 sums of the counted drlv2) as
 * id11b_dev_score_grid -- identical to the reference's score() for every
 * (UBI, tol), ImageD11 src/closest.c:227-248 -- by a spatial join instead of
 * per-box lookups: every (UBI, hkl) box that can reach the data is enumerated
 * once, the boxes are sorted by the grid cell holding their centre, and each
 * run of 32 boxes along a row of cells is tested against the g-vectors of
 * its region (the cells it spans widened by the largest box half width),
 * staged in shared memory, with the FP32 screening arithmetic; pairs inside
 * the proven error band are re-evaluated with the reference's FP64
 * arithmetic.  Tolerances must lie in [0, 0.4) (else ID11B_ERR_ARG: use
 * id11b_dev_score_grid; also for grids beyond 65,536 rows of cells or 8,191
 * x cells per row, ID11B_ERR_SIZE).  The workspace (256-byte aligned) holds
 * per-UBI and per-row tables plus 16 bytes per box:
 * id11b_grid_bins_workspace_bytes(m, nx, xsub, boxes) for a box capacity;
 * with fewer bytes than the call needs, the UBIs are processed in ranges that
 * fit (ID11B_ERR_SIZE when one UBI's boxes alone do not fit).  The call reads
 * the box total back to the host (one stream synchronisation).  Sums, when
 * asked for, are of FP64 drlv2 values, accumulated in fixed point (steps of
 * 2^-(62 - ceil(log2(n tmax^2))), 2^-49 for 1.1M g at tol 0.1) so that they
 * repeat bit for bit; counts are exact. */
int64_t id11b_grid_bins_workspace_bytes(int64_t m, int32_t nx, int32_t xsub, int64_t boxes);
/* Measurement hook: the calling thread's next id11b_dev_score_grid_bins call
 * records start_event before its first join launch and stop_event after its
 * last (both cudaEvent_t, created by the caller; NULL, NULL clears). */
int id11b_grid_bins_time_join(void *start_event, void *stop_event);
int id11b_dev_score_grid_bins(const double *ubis, int64_t m, const double *gv, int64_t n,
                              int32_t nx, int32_t xsub, const void *gridbuf,
                              const double *tols_host, int ntol, int32_t *counts, double *sums,
                              void *ws, int64_t ws_bytes, void *stream);

/* id11b_dev_score_and_assign_grid in pieces, for grains sharded over ranks
 * (one process per GPU): each rank runs pass -1 (reset of best (n uint64) and
 * lab (n int32)) and pass 0 over its share ubis[base : base+m]; best is
 * reduced with MIN over the ranks as int64; pass 1 over the share; lab reduced
 * with MIN as int32; then every rank calls id11b_dev_assign_grid_final with
 * all grains (the g outside the regular range follow the reference's
 * sequence of calls) and ends with the same drlv2 and labels. */
int id11b_dev_assign_grid_pass(const double *ubis, int64_t m, int64_t index_base, int64_t n,
                               int32_t nx, int32_t xsub, const void *gridbuf, double tol,
                               const double *drlv2, int pass, uint64_t *best, int32_t *lab,
                               void *stream);
/* Passes 0 and 1 of id11b_dev_assign_grid_pass for all m grains at once
 * (index_base 0) through the binned join of id11b_dev_score_grid_bins (ws of
 * id11b_grid_bins_workspace_bytes; tol < 0.4; the grid within the join's row
 * and x-cell limits): best and lab as pass -1 leaves them, then
 * id11b_dev_assign_grid_final.  Every pair the FP32 screen cannot exclude
 * from tol^2 is evaluated in the reference's FP64 arithmetic, so best and lab
 * end as the lookup passes leave them. */
int id11b_dev_assign_grid_bins(const double *ubis, int64_t m, const double *gv, int64_t n,
                               int32_t nx, int32_t xsub, const void *gridbuf, double tol,
                               const double *drlv2, uint64_t *best, int32_t *lab, void *ws,
                               int64_t ws_bytes, void *stream);
int id11b_dev_assign_grid_final(const double *ubis, int64_t m, const int32_t *grain_labels,
                                const double *gv, int64_t n, int32_t nx, int32_t xsub,
                                const void *gridbuf, double tol, const uint64_t *best,
                                const int32_t *lab, double *drlv2, int32_t *labels,
                                int32_t *npk, void *stream);

/* `iters` rounds of score_and_refine (ImageD11 src/closest.c:267-345) for each
 * of m UBIs against all n g-vectors through the cell index: the result of
 * id11b_dev_refine_batch (every pair below tol^2 accumulated in the
 * reference's FP64 arithmetic; sums in a fixed order), found by lookup.
 * ws: id11b_grid_refine_workspace_bytes(m), 256-byte aligned. */
int64_t id11b_grid_refine_workspace_bytes(int64_t m);
int id11b_dev_refine_grid(double *ubis, int64_t m, const double *gv, int64_t n, int32_t nx,
                          int32_t xsub, const void *gridbuf, double tol, int iters,
                          int32_t *npk, double *mean_drlv2, void *ws, int64_t ws_bytes,
                          void *stream);

/* Batched score_and_assign through the cell index: the result of calling the
 * reference's score_and_assign (ImageD11 src/closest.c:366-397) for grain
 * i = 0 .. m-1 in order, score_and_assign(ubis[i], gv, tol, drlv2, labels,
 * grain_labels[i]), as ImageD11/indexing.py fight_over_peaks (:876-905) does:
 * drlv2 (n) and labels (n) are updated in place to the same values, bit for
 * bit.  grain_labels: strictly increasing int32 (m), or NULL for 0 .. m-1
 * (the caller checks the order).  npk (m, optional): peaks holding each
 * grain's label at the end (the histogram fight_over_peaks takes); the
 * per-call return values of the sequential calls are not reproduced.  ws:
 * id11b_assign_workspace_bytes(n), 256-byte aligned. */
int64_t id11b_assign_workspace_bytes(int64_t n);
int id11b_dev_score_and_assign_grid(const double *ubis, int64_t m, const int32_t *grain_labels,
                                    const double *gv, int64_t n, int32_t nx, int32_t xsub,
                                    const void *gridbuf, double tol, double *drlv2,
                                    int32_t *labels, int32_t *npk, void *ws, int64_t ws_bytes,
                                    void *stream);

/* `iters` rounds of score_and_refine (ImageD11 src/closest.c:267-345) for each
 * of m UBIs against all n g-vectors, ubis (m,3,3) updated in place; npk and
 * mean_drlv2 (optional) receive the last round's count and mean drlv2.
 * Candidates are screened in FP32; every accepted pair is evaluated and
 * accumulated in the reference's FP64 arithmetic (per-CTA partials summed in
 * a fixed order). */
int id11b_dev_refine_batch(double *ubis, int64_t m, const double *gv, const float *g4,
                           int64_t n, const void *gws, double tol, int iters, int32_t *npk,
                           double *mean_drlv2, void *ws, int64_t ws_bytes, void *stream);

/* Per-grain refinement over CSR peak lists: grain g refines ubis[g] (9 doubles,
 * in place) against gv[offsets[g] : offsets[g+1]] with `iters` rounds of
 * score_and_refine (ImageD11 src/closest.c:267-345), as the per-grain loop of
 * ImageD11/refinegrains.py:459-498 calls it.  order (optional, ngrains int32)
 * is the processing order (largest grains first balances best).
 * persistent != 0: one launch runs every round of every grain, CTAs pulling
 * grains from a work counter in `workspace` (id11b_refine_csr_workspace_bytes());
 * persistent == 0: one CTA per grain, the plain baseline (call once per round).
 * npk / mean_drlv2 (optional, ngrains) receive the last round's count and mean
 * drlv2.  threads: CTA size 32, 64, 128, 256 or 512 (0 = 128); small CTAs keep
 * more grains in flight (64 is fastest for 2,000 grains of 20..1,500 peaks).  Exact FP64 per pair; the persistent launch (counter reset + kernel)
 * can be captured in a CUDA graph and replayed. */
int64_t id11b_refine_csr_workspace_bytes(void);
int id11b_dev_refine_csr(double *ubis, const double *gv, const int64_t *offsets,
                         const int32_t *order, int32_t ngrains, double tol, int iters,
                         int persistent, int threads, int32_t *npk, double *mean_drlv2,
                         void *workspace, int64_t ws_bytes, void *stream);

/* Per-grain refinement as id11b_dev_refine_csr (persistent, 64-thread CTAs)
 * with FP32 screening -- the proven error band of id11b_dev_score_batch, FP64
 * inside it -- and compensated FP32 normal-equation sums (error-free products
 * and TwoSum; H as exact integers), FP64 3x3 solves.  The same accepted pairs
 * and peak counts; UBIs agree with the FP64 sums to ~1e-14 relative, mean
 * drlv2 to the band (~1e-6 relative).  gmax: a bound on every |g_j| (<= 1024,
 * finite g only); tol < 0.4.  No counterpart in the reference: its
 * score_and_refine sums in FP64 (ImageD11 src/closest.c:267-345). */
int id11b_dev_refine_csr_f32c(double *ubis, const double *gv, const int64_t *offsets,
                              const int32_t *order, int32_t ngrains, double tol, int iters,
                              double gmax, int32_t *npk, double *mean_drlv2, void *workspace,
                              int64_t ws_bytes, void *stream);

/* Per-grain translation refinement: minimises, for every grain G at once, the
 * objective of ImageD11/refinegrains.py refinepositions / gof (:517-560,
 * :636-660) -- by damped Gauss-Newton (analytic 3x3 Jacobian per peak) where
 * the reference runs a Nelder-Mead simplex per grain.  At translation t_G the
 * objective is what gof's refine (:459-498) computes: g from compute_gv
 * (src/cdiffraction.c:112-168) at t_G, U1 = the score_and_refine update of
 * UBI_G (least squares over the peaks with drlv2 < tol^2, hkl rounded at
 * UBI_G), and cost = sum over the peaks with drlv2(U1) < tol^2 of
 * |U1.g - round(U1.g)|^2, npk their count (refinegrains' gof is
 * 1e6 * cost / npk).  Grain G owns xyz/omega rows offsets[G] ..
 * offsets[G+1]-1 (lab positions from compute_xlylzl, omega in degrees);
 * ubis (ngrains,9) are the UBIs read (left unchanged); translations
 * (ngrains,3) in/out; cost, npk and ubis_refit (ngrains,9, the U1 at the
 * final translations) are optional outputs.  iters = 0 evaluates the
 * objective at the given translations only. */
int id11b_dev_refine_translations(const double *xyz, const double *omega,
                                  const int64_t *offsets, int32_t ngrains, const double *ubis,
                                  double *translations, double omegasign, double wvln,
                                  double wedge, double chi, double tol, int iters, double *cost,
                                  int32_t *npk, double *ubis_refit, void *stream);

/* Residuals of assigned peaks and their adjoint (no single reference
 * function: the forward model chains compute_xlylzl and compute_gv,
 * ImageD11 src/cdiffraction.c:190-224 and :112-168, with UBI.g - h, the
 * quantity refinegrains.gof minimises by Nelder-Mead, ImageD11/refinegrains.py
 * :517-560).  Peaks are stored grain by grain: grain G owns peaks
 * offsets[G] .. offsets[G+1]-1, with detector positions sc (slow), fc (fast),
 * omega (degrees) and assigned integer hkl (n,3 doubles).
 *
 * params: 12 doubles in DEVICE memory -- distance, y_center, z_center,
 * tilt_x, tilt_y, tilt_z (radians), wavelength, wedge, chi (degrees), t_x,
 * t_y, t_z (ImageD11 parameter names); every launch builds the detector
 * matrix R3(tilt_x).R2(tilt_y).R1(tilt_z).flip (ImageD11/transform.py:51-82)
 * and chi.wedge from them on the device, so no call reads the geometry on
 * the host.  detector: 7 HOST doubles, the fixed constants y_size, z_size,
 * omegasign, o11, o12, o21, o22 (read during the call).
 *
 * id11b_dev_residuals writes res (n,3) = UBI_G.g - hkl, optionally gvec (n,3),
 * and ssq (ngrains, optional) = per-grain sum of squared residuals; with
 * ubis NULL it writes gvec only (hkl and res unused).
 * id11b_dev_residuals_adjoint takes grad_res = dL/dres (n,3) and writes
 * grad_ubis (ngrains,9, optional) = dL/dUBI and grad_params (12, device) =
 * dL/dparams.
 * id11b_dev_residual_loss writes loss (1, device) = 0.5 sum |res|^2 and its
 * gradients in one pass over the peaks: at the given ubis (grad_ubis
 * optional), or, with ubis NULL, at each grain's least-squares UBI for the
 * current g-vectors (variable projection; the UBIs go to ubis_out when it is
 * not NULL, grad_ubis must be NULL -- it is zero there).
 * id11b_dev_best_ubis writes each grain's least-squares UBI
 * (sum h g^T)(sum g g^T)^-1 for the g-vectors at params; a grain whose
 * normal matrix B = sum g g^T is singular (det B <= 1e-10 trace(B)^3, as
 * for fewer than three independent g) gets UBI 0.
 * omega_sincos (optional, NULL computes them): the table of
 * id11b_dev_omega_sincos for the same peaks.  FP64; reductions in a fixed
 * order (deterministic).  Workspace: id11b_adjoint_workspace_bytes(ngrains). */
int64_t id11b_adjoint_workspace_bytes(int32_t ngrains);
int id11b_dev_residuals(const double *params, const double *detector, const double *sc,
                        const double *fc, const double *omega, const double *omega_sincos,
                        const double *hkl, const int64_t *offsets, const double *ubis,
                        int32_t ngrains, double *res, double *gvec, double *ssq, void *stream);
int id11b_dev_residuals_adjoint(const double *params, const double *detector,
                                const double *sc, const double *fc, const double *omega,
                                const double *omega_sincos, const double *hkl,
                                const int64_t *offsets, const double *ubis, int32_t ngrains,
                                const double *grad_res, double *grad_ubis, double *grad_params,
                                void *workspace, int64_t ws_bytes, void *stream);
int id11b_dev_residual_loss(const double *params, const double *detector, const double *sc,
                            const double *fc, const double *omega, const double *omega_sincos,
                            const double *hkl, const int64_t *offsets, const double *ubis,
                            int32_t ngrains, double *loss, double *grad_ubis,
                            double *grad_params, double *ubis_out, void *workspace,
                            int64_t ws_bytes, void *stream);
int id11b_dev_best_ubis(const double *params, const double *detector, const double *sc,
                        const double *fc, const double *omega, const double *omega_sincos,
                        const double *hkl, const int64_t *offsets, int32_t ngrains,
                        double *ubis_out, void *stream);
/* sin and cos of omega * omegasign (omega in degrees) for n peaks,
 * interleaved (2n doubles, 16-byte aligned): the omega_sincos table the
 * residual entry points take, so that repeated evaluations over the same
 * peaks do not recompute them. */
int id11b_dev_omega_sincos(const double *omega, int64_t n, double omegasign,
                           double *sincos_out, void *stream);

/* Bragg angle of each assigned reflection computed from its grain's UB
 * matrix (ubs: ngrains x 9, row-major; hkl, offsets as above), in degrees,
 * and its derivative with respect to UB, the quantities ImageD11
 * src/deriv.c:38-53 (g_to_k) computes: g = UB h, t = wavelength |g| / 2,
 * theta = asin(t), dtheta/dUB_ij = (180/pi) wavelength g_i h_j /
 * (2 |g| sqrt(1 - t^2)).  dtheta_dub (n,9) is optional.  The adjoint takes
 * grad_theta (n) and writes grad_ubs (ngrains,9) = sum over each grain's
 * peaks of grad_theta dtheta/dUB (fixed order).  FP64. */
int id11b_dev_bragg_theta(const double *ubs, const double *hkl, const int64_t *offsets,
                          int32_t ngrains, double wavelength, double *theta,
                          double *dtheta_dub, void *stream);
int id11b_dev_bragg_theta_adjoint(const double *ubs, const double *hkl,
                                  const int64_t *offsets, int32_t ngrains, double wavelength,
                                  const double *grad_theta, double *grad_ubs, void *stream);

/* Synchronising read of the last batch call's statistics from its workspace:
 * FP64 re-evaluations, UBIs routed wholly to FP64, and the device error flag
 * (returned as the status). */
int id11b_batch_stats(const void *ws, int64_t m, int64_t n, int refine, int64_t *nrecheck,
                      int32_t *nfallback, int32_t *error, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* IMAGED11_B200_H */
