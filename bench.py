"""Benchmark: batched candidate-grain scoring on B200.

Workload (default): 1.1M g-vectors simulated from 2,000 FCC Al grains
(a = 4.05 A, |g| <= 1.5 A^-1, wavelength 0.2846 A, 150 mm, 2048^2 x 75 um
detector, sigma 0.5 px / 0.05 deg centroid noise, 10% uniform noise peaks)
scored against 20,000 trial UBIs (10% true orientations perturbed by 0.5 deg,
90% uniformly random orientations of the same cell) at tol = 0.02, 0.05, 0.1,
counts identical to the reference's score().

Metric: assigned peak x grain pairs per second = M * N * T / step time.
One step = the reciprocal-space cell index rebuilt from the g-vectors + exact
batched scoring through it (binned join: FP32 screening of every (UBI, hkl)
box against the g near it, proven FP64 recheck band), inputs resident in HBM.
Beside it in the same run: the plain FP64 kernel (every pair, reference
arithmetic) on the same 20,000 UBIs, the brute-force FP32 screening kernel,
the per-box lookup scorer, the reference's own C on the host cores, and the
other configurations (uneven refinement, adjoint, translations, the
full-scale scan, the small drop-in sequence), each checked against the
reference.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): every rank scores its own 20,000 trial UBIs against the
same g-vectors (weak scaling, no collective on the data path); the step time
is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

TOLS = [0.02, 0.05, 0.1]
# DRAM bytes (read + write) of one binned-join launch on this workload, from an ncu
# capture of the same command (profiles/): the traffic is the box records
K_JOIN_DRAM_BYTES = 404.0e6
K_JOIN_TRAFFIC_NOTE = ("dram__bytes_read.sum + dram__bytes_write.sum of one k_join<3> launch "
                       "(399.5 + 4.5 MB; 20,000 UBIs, cell factor 0.9, x cut 8x -- the "
                       "autotuner's pick in the runs recorded; 401.0 MB at 0.8 x 4x; ncu "
                       "--set full capture in "
                       "profiles/k_join_binned_20000ubi_1.1Mg.md): mostly the box records, "
                       "read once; the staged g come from L2")
N_GRAINS = 2000
GMAX = 1.5
N_UBI = 20000
SEED = 1234
FLOP_PER_EVAL = 30   # per (UBI, g): 9 FMA (18), 3 rint, 3 sub, 5 for t.t, 1 compare
L2_FLUSH_BYTES = 256 << 20


def measured_hbm_peak():
    """Measured HBM copy bandwidth of this GPU model (GB/s), else the fallback."""
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def compute_gv_measure(torch, ps, dev, n_peaks=10_000_000, steps=5, flush=None):
    """compute_gv (FP64 drop-in kernel) over n_peaks lab positions, inputs
    resident; returns (GB/s of algorithmic traffic, ms per launch)."""
    from imaged11_b200 import cImageD11 as cim
    reps = (n_peaks + len(ps.xyz) - 1) // len(ps.xyz)
    x = torch.tensor(ps.xyz, device=dev).repeat(reps, 1)[:n_peaks].contiguous()
    om = torch.tensor(ps.omega, device=dev).repeat(reps)[:n_peaks].contiguous()
    g = torch.empty_like(x)
    geo = ps.geo

    def run():
        cim.compute_gv(x, om, geo["omegasign"], geo["wavelength"], geo["wedge"], geo["chi"],
                       [0.0, 0.0, 0.0], g)
    for _ in range(3):
        run()
    times = cuda_time_ms(torch, run, steps, flush)
    ms = float(np.mean(times))
    return 56.0 * n_peaks / (ms * 1e-3) / 1e9, ms


def grid_measure(torch, dev, ps, ubis, steps=5, flush=None, check_counts=None, cell=None,
                 xsub=None):
    """Scoring through the reciprocal-space cell index on the same workload:
    index build time, ms per score_grid call (inputs resident, L2 flushed
    between calls) and pairs decided per second."""
    from imaged11_b200 import batch
    gv_d = torch.tensor(ps.gv, device=dev)
    ubis_d = torch.tensor(ubis, device=dev)
    m, n, T = len(ubis), len(ps.gv), len(TOLS)
    batch.GvecGrid(gv_d, cell=cell, xsub=xsub)            # load the kernels
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    grid = batch.GvecGrid(gv_d, cell=cell, xsub=xsub)
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - t0) * 1e3
    ws = batch.BinsWorkspace(m, grid, batch.bins_box_estimate(ubis_d, grid, max(TOLS)))
    counts = torch.empty((m, T), dtype=torch.int32, device=dev)

    def run():
        batch.score_grid(ubis_d, grid, TOLS, workspace=ws, out=counts, method="bins")
    for _ in range(3):
        run()
    same = None
    if check_counts is not None:
        same = bool(torch.equal(counts, check_counts))
    times = cuda_time_ms(torch, run, steps, flush)
    ms = float(np.mean(times))
    st = grid.stats()

    # batched score_and_assign (the fight_over_peaks loop, tol 0.05) against
    # the drop-in kernel called once per grain, on the first 256 UBIs
    d = torch.empty(n, dtype=torch.float64, device=dev)
    lab = torch.empty(n, dtype=torch.int32, device=dev)
    one = torch.empty(1, dtype=torch.int32, device=dev)

    def assign(k):
        d.fill_(2.0)
        lab.fill_(-1)
        batch.score_and_assign_grid(ubis_d[:k], grid, 0.05, d, lab)

    def assign_seq(k):
        d.fill_(2.0)
        lab.fill_(-1)
        for i in range(k):
            batch.lib.id11b_dev_score_and_assign(ubis_d[i].data_ptr(), gv_d.data_ptr(), 0.05,
                                                 d.data_ptr(), lab.data_ptr(), i, n,
                                                 one.data_ptr(), None)
    k = min(256, m)
    assign_seq(k)
    ref_lab, ref_d = lab.clone(), d.clone()
    assign(k)
    same_assign = bool(torch.equal(lab, ref_lab) and torch.equal(d, ref_d))
    t_seq = float(np.mean(cuda_time_ms(torch, lambda: assign_seq(k), 2, flush)))
    t_asg = float(np.mean(cuda_time_ms(torch, lambda: assign(m), steps, flush)))
    # one round of dense score_and_refine for every trial UBI (tol 0.05): through
    # the index, and through the FP32-screened refine_batch
    gs = batch.GvecSet(gv_d)
    rws = batch.BatchWorkspace(m, n, refine=True)
    t_rg = float(np.mean(cuda_time_ms(torch, lambda: batch.refine_grid(ubis_d.clone(), grid, 0.05),
                                      steps, flush)))
    t_rb = float(np.mean(cuda_time_ms(
        torch, lambda: batch.refine_batch(ubis_d.clone(), gs, 0.05, workspace=rws), steps,
        flush)))
    # errors of one indexed round against the reference arithmetic, 32 UBIs
    from oracle import oracle as orcm
    orc = orcm.Reference() if orcm.have_reference() else orcm.Oracle()
    ug, ng_, mg = batch.refine_grid(ubis_d[:32].clone(), grid, 0.05)
    ug, ng_, mg = ug.cpu().numpy().reshape(-1, 9), ng_.cpu().numpy(), mg.cpu().numpy()
    e_u = e_m = 0.0
    same_n = True
    for q in range(32):
        rn, rmean, ru = orc.score_and_refine(ubis[q], ps.gv, 0.05)
        same_n &= int(rn) == int(ng_[q])
        sc = max(np.abs(ru).max(), 1e-300)
        e_u = max(e_u, float(np.abs(ug[q] - np.asarray(ru).reshape(9)).max() / sc))
        if rmean:
            e_m = max(e_m, abs(mg[q] - rmean) / rmean)
    return {"ms": ms, "value": m * n * T / (ms * 1e-3), "unit": "pairs/s",
            "refine": {"ubis": m, "tol": 0.05, "grid_ms": t_rg, "batch_fp32_ms": t_rb,
                       "value": m * n / (t_rg * 1e-3), "batch_value": m * n / (t_rb * 1e-3),
                       "vs_reference_32_ubis": {"npk_identical": bool(same_n),
                                                "ubi_max_rel_err": e_u,
                                                "mean_drlv2_max_rel_err": float(e_m)}},
            "assign": {"ubis": m, "tol": 0.05, "ms": t_asg, "value": m * n / (t_asg * 1e-3),
                       "sequential_plain_fp64_value": k * n / (t_seq * 1e-3),
                       "sequential_ubis": k, "identical_to_sequential": same_assign},
            "build_ms_wall": build_ms, "cells": grid.nx ** 3 * grid.xsub, "cell_A^-1": grid.cs,
            "xsub": grid.xsub,
            "pairs_tested_fp64": st["pairs_tested"],
            "tested_fraction": st["pairs_tested"] / float(m * n),
            "plain_scan_ubis": st["fallback_ubis"], "counts_equal_score_batch": same}


def update_geometry_measure(torch, dev, n_peaks=10_000_000, steps=5, flush=None):
    """Detector positions -> lab positions -> tth, eta, ds, g for n_peaks: the
    fused pass against compute_xlylzl + compute_geometry launched in turn
    (inputs resident, L2 flushed between steps)."""
    from imaged11_b200 import transform
    rng = np.random.default_rng(SEED + 11)
    pars = {"y_center": 1024.3, "z_center": 1021.7, "y_size": 75.0, "z_size": 75.0,
            "distance": 152300.0, "wavelength": 0.2846, "omegasign": 1.0, "tilt_x": 0.004,
            "tilt_y": -0.002, "tilt_z": 0.006, "o11": 1, "o12": 0, "o21": 0, "o22": -1,
            "wedge": 0.01, "chi": 0.02}
    ct = transform.Ctransform(pars)
    sc = torch.tensor(rng.uniform(0, 2048, n_peaks), device=dev)
    fc = torch.tensor(rng.uniform(0, 2048, n_peaks), device=dev)
    om = torch.tensor(rng.uniform(0, 360, n_peaks), device=dev)
    xyz = torch.empty((n_peaks, 3), dtype=torch.float64, device=dev)
    out = torch.empty((n_peaks, 6), dtype=torch.float64, device=dev)
    t = (5.0, -3.0, 2.0)

    def fused():
        ct.sf2geometry(sc, fc, om, *t)

    def separate():
        ct.sf2xyz(sc, fc, out=xyz)
        ct.xyz2geometry(xyz, om, *t, out=out)
    for _ in range(3):
        fused()
        separate()
    mf = float(np.mean(cuda_time_ms(torch, fused, steps, flush)))
    ms = float(np.mean(cuda_time_ms(torch, separate, steps, flush)))
    return {"case": "update_geometry", "peaks": n_peaks, "fused_ms": mf, "separate_ms": ms,
            "fused_gbs": 96.0 * n_peaks / (mf * 1e-3) / 1e9,
            "separate_gbs": 120.0 * n_peaks / (ms * 1e-3) / 1e9,
            "bytes_per_peak": {"fused": 96, "separate": 120}}


def refine_workload(seed=SEED + 7, ngrains=2000):
    """Uneven per-grain refinement: hcp Ti grains (a=2.95, c=4.68 A), per-grain
    peak counts log-uniform in 20..2000, each grain's shortest reflections up to
    that count (a per-grain |g| cutoff) as g-vectors with 5e-4 1/A noise, no
    detector; each UBI 0.2 deg and 0.2% strain off its true value.  (The stated
    total of about 1.2M peaks does not follow from these numbers: counts
    log-uniform over 20..2,000 have mean 430, so 2,000 grains hold about 0.86M.)"""
    from imaged11_b200 import synth
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(20), np.log(2000), ngrains)).astype(int)
    gv, off, ubis = synth.grain_gvectors(counts, "Ti_hcp", rng)
    u0 = synth.perturb_ubis(ubis, 0.2, 0.002, rng)
    return gv, off, u0


def refine_csr_measure(torch, dev, iters=5, tol=0.05, steps=5, flush=None, cpu=True):
    """Batched per-grain refinement: persistent kernel replayed from a CUDA
    graph vs the plain FP64 path (one launch per round), pairs = peaks x rounds."""
    from imaged11_b200 import batch
    gv, off, u0 = refine_workload()
    gs = batch.GrainSet(gv, off, u0)
    u0_dev = gs.ubis.clone()
    graph = gs.capture(tol, iters)

    def reset():
        if flush is not None:
            flush()
        gs.ubis.copy_(u0_dev)

    times_g, times_p = [], []
    for _ in range(3):
        reset()
        graph.replay()
        reset()
        gs.refine(tol, iters, persistent=False)
    st = torch.cuda.current_stream()
    for _ in range(steps):
        for fn, acc in ((graph.replay, times_g),
                        (lambda: gs.refine(tol, iters, persistent=False), times_p)):
            reset()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            e1.synchronize()
            acc.append(e0.elapsed_time(e1))
    pairs = gs.peaks * iters
    out = {"grains": gs.ngrains, "peaks": gs.peaks, "rounds": iters, "tol": tol,
           "peaks_per_grain_min_max": [int(np.diff(off).min()), int(np.diff(off).max())],
           "graph_ms": float(np.mean(times_g)), "plain_fp64_ms": float(np.mean(times_p)),
           "value": pairs / (np.mean(times_g) * 1e-3), "unit": "pairs/s",
           "plain_fp64_value": pairs / (np.mean(times_p) * 1e-3)}
    out["ratio_vs_plain_fp64"] = out["value"] / out["plain_fp64_value"]
    # compensated FP32 sums (FP32 screening, FP64 solves) against the FP64 sums
    fp64_u = gs.ubis.clone()
    reset()
    graph.replay()
    torch.cuda.synchronize()
    fp64_u.copy_(gs.ubis)
    fp64_n = gs.npk.clone()
    t32 = []
    for _ in range(steps + 1):
        reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        gs.refine(tol, iters, precision="f32c")
        e1.record(st)
        e1.synchronize()
        t32.append(e0.elapsed_time(e1))
    u32 = gs.ubis.view(-1, 9)
    scale64 = fp64_u.view(-1, 9).abs().max(1, keepdim=True).values.clamp_min(1e-300)
    out["compensated_fp32"] = {
        "ms": float(np.mean(t32[1:])), "value": pairs / (np.mean(t32[1:]) * 1e-3),
        "npk_equal_fp64_sums": bool(torch.equal(gs.npk, fp64_n)),
        "ubi_max_rel_diff_vs_fp64_sums": float(((u32 - fp64_u.view(-1, 9)).abs() /
                                                scale64).max().item()),
        "note": "FP32 screening with the proven band + compensated FP32 normal equations, "
                "FP64 3x3 solves, one launch (not graph-captured)"}
    if cpu:
        from oracle import oracle as orc
        lib = orc.Reference() if orc.have_reference() else orc.Oracle()
        t0 = time.perf_counter()
        ref_u, ref_n, ref_m = lib.refine_csr(u0, gv, off, tol, iters)
        dt = time.perf_counter() - t0
        # the graph's result against the reference's: the max error of every UBI
        # element (relative to the grain's largest element) and of mean drlv2
        reset()
        graph.replay()
        torch.cuda.synchronize()
        gu = gs.ubis.cpu().numpy().reshape(-1, 9)
        ru = np.asarray(ref_u).reshape(-1, 9)
        scale = np.abs(ru).max(1, keepdims=True)
        scale[scale == 0] = 1.0
        gm, rm = gs.mean.cpu().numpy(), np.asarray(ref_m)
        nz = rm != 0
        out["vs_reference"] = {
            "npk_identical": bool(np.array_equal(gs.npk.cpu().numpy(), np.asarray(ref_n))),
            "ubi_max_rel_err": float((np.abs(gu - ru) / scale).max()),
            "mean_drlv2_max_rel_err": float((np.abs(gm[nz] - rm[nz]) / rm[nz]).max())
            if nz.any() else 0.0}
        out["cpu_baseline"] = {"value": pairs / dt, "unit": "pairs/s",
                               "cores": lib.max_threads(),
                               "kind": "reference" if isinstance(lib, orc.Reference) else "port",
                               "sample": "whole workload, %d peaks x %d rounds (%.1f ms)" % (len(gv), iters, dt * 1e3)}
    return out


# the cfg4 scan's starting geometry: the truth offset by these amounts (um,
# px, rad, deg)
CFG4_START_OFFSETS = dict(distance=300., y_center=0.4, z_center=-0.3, tilt_y=4e-4,
                          tilt_z=-3e-4, wedge=0.005)
CFG3_TRUTH = dict(distance=152300., y_center=1024 + 3.7, z_center=1024 - 2.1, tilt_x=0.004,
                  tilt_y=-0.002, tilt_z=0.006, wedge=0.01, chi=0.02, t_x=5., t_y=-3., t_z=2.)


def translations_measure(torch, dev, steps=5, cpu=True):
    """Per-grain translation refinement (the refinepositions objective): 500
    FCC Al grains, |g| <= 1.75, each at its own position (uniform +-60 um),
    0.5 px / 0.05 deg noise, UBIs fixed at truth, start at t = 0, 30
    iterations, all grains in one launch; the reference's method (a
    Nelder-Mead simplex on the oracle's compute_gv + score_and_refine, as
    refinegrains.gof) on a few grains on the host for comparison."""
    from imaged11_b200 import batch, synth
    from imaged11_b200 import cImageD11 as cim
    truth = synth.default_geometry(**CFG3_TRUTH)
    ps = synth.simulate(500, "Al", gmax=1.75, seed=SEED + 17, geo=truth, noise_frac=0.0,
                        translations_um=60.0)
    idx, off = ps.grain_offsets()
    p, r, dist = synth.xlylzl_params(truth)
    s_d = torch.tensor(ps.s[idx], device=dev)
    f_d = torch.tensor(ps.f[idx], device=dev)
    om = torch.tensor(ps.omega[idx], device=dev)
    xyz = torch.empty((len(idx), 3), dtype=torch.float64, device=dev)
    cim.compute_xlylzl(s_d, f_d, p, r.ravel(), dist, xyz)
    ng = len(off) - 1
    z = np.zeros((ng, 3))

    def run():
        return batch.refine_translations(xyz, om, off, ps.ubis, z, truth["omegasign"],
                                         truth["wavelength"], truth["wedge"], truth["chi"],
                                         iters=30)
    for _ in range(3):
        run()
    ms = float(np.mean(cuda_time_ms(torch, run, steps)))
    t, cost, npk = run()
    err = np.abs(t.cpu().numpy() - ps.translations)
    out = {"grains": ng, "peaks": int(off[-1]), "iterations": 30, "ms": ms,
           "grains_per_s": ng / (ms * 1e-3),
           "error_um_median_max": [float(np.median(err)), float(err.max())]}
    if cpu:
        from scipy.optimize import minimize
        from oracle import oracle as orcm
        orc = orcm.Reference() if orcm.have_reference() else orcm.Oracle()
        xyz_h = xyz.cpu().numpy()
        om_h = ps.omega[idx]
        t0 = time.perf_counter()
        nev = 0
        k = 8
        for g in range(k):
            a, b = off[g], off[g + 1]

            def gof(tt, a=a, b=b, g=g):
                gv = orc.compute_gv(xyz_h[a:b], om_h[a:b], truth["omegasign"],
                                    truth["wavelength"], truth["wedge"], truth["chi"], tt)
                n, mean, _ = orc.score_and_refine(ps.ubis[g], gv, 1.0)
                return n * mean
            res = minimize(gof, np.zeros(3), method="Nelder-Mead",
                           options={"xatol": 1e-3, "fatol": 1e-12, "maxiter": 2000})
            nev += res.nfev
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": k / dt, "unit": "grains/s", "cores": orc.max_threads(),
                               "kind": "reference" if isinstance(orc, orcm.Reference) else "port",
                               "sample": "Nelder-Mead on %d grains, %d objective evaluations"
                                         % (k, nev)}
        out["ratio_vs_cpu_nelder_mead"] = out["grains_per_s"] / (k / dt)
    return out


def adjoint_measure(torch, dev, steps=5, refine=True):
    """Joint grain + geometry refinement workload: 500 FCC Al grains (~325k
    peaks, |g| <= 1.75) simulated with tilts, wedge, chi, translation and
    offset centres, 0.5 px / 0.05 deg noise; gradient of the residuals with
    respect to 12 geometry parameters and 500 x 9 UBI elements."""
    from imaged11_b200 import adjoint, synth
    truth = synth.default_geometry(**CFG3_TRUTH)
    ps = synth.simulate(500, "Al", gmax=1.75, seed=SEED + 11, geo=truth, noise_frac=0.0,
                        translation=(5., -3., 2.))
    idx, off = ps.grain_offsets()
    peaks = adjoint.PeakTable(ps.s[idx], ps.f[idx], ps.omega[idx], ps.hkl[idx], off, truth)
    nominal = dict(truth, distance=150000., y_center=1024., z_center=1024., tilt_x=0.,
                   tilt_y=0., tilt_z=0., wedge=0., chi=0., t_x=0., t_y=0., t_z=0.)
    p0 = adjoint.params_tensor(nominal)
    u0 = adjoint.best_ubis(p0, peaks)

    def grad_eval():
        p = p0.clone().requires_grad_(True)
        u = u0.clone().requires_grad_(True)
        adjoint.loss(p, u, peaks).backward()
        return p.grad, u.grad

    def projected_eval():
        p = p0.clone().requires_grad_(True)
        adjoint.projected_loss(p, peaks).backward()
        return p.grad

    for _ in range(3):
        grad_eval()
        projected_eval()
    times = cuda_time_ms(torch, grad_eval, steps)
    tproj = cuda_time_ms(torch, projected_eval, steps)
    out = {"grains": peaks.ngrains, "peaks": peaks.n, "params": 12 + 9 * peaks.ngrains,
           "gradient_ms": float(np.mean(times)),
           "gradient_peaks_per_s": peaks.n / (np.mean(times) * 1e-3),
           "projected_gradient_ms": float(np.mean(tproj)),
           "note": "gradient_ms: loss and its gradient in the 12 geometry parameters and "
                   "the 500 x 9 UBI elements through torch.autograd (one fused residual + "
                   "adjoint kernel, one reduction, geometry kept on the device); "
                   "projected_gradient_ms: the same with every grain's UBI solved in "
                   "closed form inside the kernel (one L-BFGS evaluation of refine_geometry)"}
    if refine:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        p, _, hist = adjoint.refine_geometry(peaks, p0, max_iter=100)
        torch.cuda.synchronize()
        got = dict(zip(adjoint.PARAMS, p.cpu().numpy()))
        out["refine"] = {"seconds": time.perf_counter() - t0, "evaluations": len(hist),
                         "loss_start": hist[0], "loss_end": hist[-1],
                         "error_vs_truth": {k: float(got[k] - truth[k])
                                            for k in adjoint.PARAMS if k != "wavelength"}}
    return out


def pipeline_measure(torch, dev, n_ubi=100_000, tol=0.05, rounds=5, cpu=True):
    """Full-scale scan: 20,000 grains (70% hcp Ti, 30% bcc beta-Ti, |g| <= 1.27,
    15% noise peaks, cfg3 geometry), end to end on the device:
    compute_xlylzl + compute_gv -> cell index + scoring of n_ubi trial UBIs
    (binned join) -> batched score_and_assign of every peak to the 20,000
    grains (their UBIs 0.2 deg / 0.2% off truth) -> peaks grouped by label ->
    `rounds` rounds of per-grain refinement -> hkl of the assigned peaks from
    the refined UBIs -> a geometry step (3 L-BFGS iterations on the 12
    geometry parameters, every grain's UBI re-solved in closed form inside the
    adjoint kernel at each evaluation).
    Each stage's output is checked against the reference's own C on a sample
    (cpu=True): compute_gv on 1M peaks, score() of 256 trials over all peaks,
    the sequential score_and_assign of all 20,000 grains on 100k peaks, and 5
    score_and_refine rounds of 64 grains on the same grouped peaks.  The FP32
    screening kernel on the same trials is timed beside it."""
    from imaged11_b200 import adjoint, batch, synth
    from imaged11_b200 import cImageD11 as cim
    from imaged11_b200._lib import lib, check
    truth = synth.default_geometry(**CFG3_TRUTH)
    # the pipeline runs from the experiment's starting estimate of the
    # geometry, a little off the truth the peaks were simulated with; the
    # geometry step moves it towards the truth
    est = dict(truth, **{k: truth[k] + d for k, d in CFG4_START_OFFSETS.items()})
    ng = 20000
    rng = np.random.default_rng(SEED + 13)
    cells = ["Ti_hcp" if x < 0.7 else "Ti_beta" for x in rng.random(ng)]
    ps = synth.simulate(ng, gmax=1.27, seed=SEED + 13, geo=truth, noise_frac=0.15,
                        translation=(5., -3., 2.), cells=cells)
    n = len(ps)
    trials = np.concatenate([
        synth.trial_ubis(ps.ubis[np.array(cells) == c], int(n_ubi * frac), 0.1, 0.5, rng, cell=c)
        for c, frac in (("Ti_hcp", 0.7), ("Ti_beta", 0.3))])
    p, r, dist = synth.xlylzl_params(est)
    s_d = torch.tensor(ps.s, device=dev)
    f_d = torch.tensor(ps.f, device=dev)
    om_d = torch.tensor(ps.omega, device=dev)
    xyz = torch.empty((n, 3), dtype=torch.float64, device=dev)
    gv = torch.empty((n, 3), dtype=torch.float64, device=dev)
    g4 = torch.empty((n, 4), dtype=torch.float32, device=dev)
    ub_d = torch.tensor(trials, device=dev)
    u_ref = synth.perturb_ubis(ps.ubis, 0.2, 0.002, rng)
    u_ref_d = torch.tensor(u_ref, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    t_arr = np.array([est["t_x"], est["t_y"], est["t_z"]])
    cbuf = torch.empty((len(trials), 1), dtype=torch.int32, device=dev)
    d2 = torch.empty(n, dtype=torch.float64, device=dev)
    lab = torch.empty(n, dtype=torch.int32, device=dev)
    out = {}
    state = {}

    def run(ev, shape=None):
        ev[0].record()
        cim.compute_xlylzl(s_d, f_d, p, r.ravel(), dist, xyz)
        check(lib.id11b_dev_compute_gv(xyz.data_ptr(), om_d.data_ptr(), est["omegasign"],
                                       est["wavelength"], est["wedge"], est["chi"],
                                       t_arr.ctypes.data, gv.data_ptr(), g4.data_ptr(), n,
                                       stream), "compute_gv")
        ev[1].record()
        grid = batch.GvecGrid(gv) if shape is None else \
            batch.GvecGrid(gv, cell=state["cs"], xsub=state["xsub"])
        if "ws" not in state or (state["ws"].nx, state["ws"].xsub) != (grid.nx, grid.xsub):
            state["boxes"] = batch.bins_box_estimate(ub_d, grid, tol)
            state["ws"] = batch.BinsWorkspace(len(trials), grid, state["boxes"])
        batch.score_grid(ub_d, grid, [tol], workspace=state["ws"], out=cbuf)
        ev[2].record()
        d2.fill_(2.0)
        lab.fill_(-1)
        if state.get("assign_bins"):
            # the binned join on the scoring's index
            batch.score_and_assign_grid(u_ref_d, grid, tol, d2, lab, method="bins",
                                        workspace=state["aws"])
        else:
            # the lookup, on an index of the lookup's best shape when that
            # differs from the scoring's (its build is timed here)
            agrid = grid if shape is None or state.get("walk_shape") in (None, tuple(shape)) \
                else batch.GvecGrid(gv, cell=state["base_cs"] * state["walk_shape"][0],
                                    xsub=state["walk_shape"][1])
            batch.score_and_assign_grid(u_ref_d, agrid, tol, d2, lab)
        ev[3].record()
        lab_s, order = torch.sort(lab, stable=True)
        first = int((lab_s < 0).sum().item())
        order, gl = order[first:], lab_s[first:].long()
        off = torch.zeros(ng + 1, dtype=torch.int64, device=dev)
        off[1:] = torch.cumsum(torch.bincount(gl, minlength=ng), 0)
        grains = batch.GrainSet(gv.index_select(0, order), off, u_ref_d.clone())
        grains.refine(tol, rounds)
        ev[4].record()
        ub_pk = grains.ubis.view(-1, 3, 3).index_select(0, gl)
        hkl = torch.round(torch.einsum("nij,nj->ni", ub_pk, grains.gv))
        peaks = adjoint.PeakTable(s_d.index_select(0, order), f_d.index_select(0, order),
                                  om_d.index_select(0, order), hkl, off, est)
        p0 = adjoint.params_tensor(est)
        p1, _, hist = adjoint.refine_geometry(peaks, p0, max_iter=3)
        ev[5].record()
        ev[5].synchronize()
        moved = dict(zip(adjoint.PARAMS, p1.cpu().numpy()))
        keys = ("distance", "y_center", "z_center", "tilt_y", "tilt_z", "wedge")
        out.update(assigned=int(n - first), refined_peaks=grains.peaks,
                   npk_median=int(grains.npk.median().item()),
                   geometry_step={"loss_before": hist[0], "loss_after": hist[-1],
                                  "evaluations": len(hist),
                                  "loss_reduced": bool(hist[-1] < hist[0]),
                                  "error_vs_truth_before": {k: est[k] - truth[k] for k in keys},
                                  "error_vs_truth_after": {k: float(moved[k] - truth[k])
                                                           for k in keys}})
        state.update(grid=grid, order=order, off=off, grains=grains)

    run([torch.cuda.Event(enable_timing=True) for _ in range(6)])   # warm-up (module loads)
    # index shape for this peak set from the autotuner, on all the trials (a
    # tenth of them favours larger cells: per-row staging weighs more against
    # fewer boxes) -- untimed setup; the counts do not depend on it
    from imaged11_b200 import tune
    base = batch.GvecGrid(gv, xsub=1)
    shape, ptable = tune.tune_grid(ub_d, gv, [tol],
                                   cell_factors=None, xsubs=(4, 8, 16),
                                   reps=1)
    walk = [(t_, ms) for t_, ms in ptable if t_[2] == "walk"]
    state.update(cs=base.cs * shape[0], xsub=shape[1], base_cs=base.cs,
                 walk_shape=tuple(min(walk, key=lambda x: x[1])[0][:2]) if walk else None)
    del base
    # the binned join's workspace for the tuned shape, sized before the timed
    # run (untimed setup, as the workspace a caller keeps between scans)
    g_t = batch.GvecGrid(gv, cell=state["cs"], xsub=state["xsub"])
    state["boxes"] = batch.bins_box_estimate(ub_d, g_t, tol)
    state["ws"] = batch.BinsWorkspace(len(trials), g_t, state["boxes"])
    # the assignment's method, each timed twice on the grains (untimed setup):
    # the binned join on this index, or the lookup on an index of its own shape
    amodes = {}
    if tol < batch.BINS_TOL_LIMIT and batch.bins_fit(g_t):
        state["aws"] = batch.BinsWorkspace(ng, g_t, batch.bins_box_estimate(u_ref_d, g_t, tol))
        amodes["bins"] = lambda: batch.score_and_assign_grid(u_ref_d, g_t, tol, d2, lab,
                                                             method="bins",
                                                             workspace=state["aws"])
    if state["walk_shape"] is not None:
        g_w = batch.GvecGrid(gv, cell=state["base_cs"] * state["walk_shape"][0],
                             xsub=state["walk_shape"][1])
        amodes["walk"] = lambda: batch.score_and_assign_grid(u_ref_d, g_w, tol, d2, lab)
    amode_ms = {}
    for k_, fn in amodes.items():
        for _ in range(2):
            d2.fill_(2.0)
            lab.fill_(-1)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record()
            fn()
            a1.record()
            a1.synchronize()
        amode_ms[k_] = a0.elapsed_time(a1)
    state["assign_bins"] = bool(amode_ms) and min(amode_ms, key=amode_ms.get) == "bins"
    amodes.clear()
    del g_t
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    run(ev, shape)
    names = ["compute_xlylzl+compute_gv", "cell_index+score_grid", "score_and_assign",
             "group+refine_csr", "adjoint_geometry_step"]
    stages = {nm: ev[i].elapsed_time(ev[i + 1]) for i, nm in enumerate(names)}
    # the FP32 screening kernel on the same trial UBIs, for comparison
    gs = batch.GvecSet(gv)
    ws = batch.BatchWorkspace(len(trials), n, refine=False)
    c32 = batch.score_batch(ub_d, gs, [tol], workspace=ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    c32 = batch.score_batch(ub_d, gs, [tol], workspace=ws)
    e1.record()
    e1.synchronize()
    pairs = (len(trials) * n + ng * n + rounds * out["refined_peaks"] +
             out["geometry_step"]["evaluations"] * out["refined_peaks"])
    device_ms = sum(stages.values())
    res = {"grains": ng, "peaks": n, "trial_ubis": int(len(trials)), "tol": tol,
           "stage_ms": stages, "pairs": pairs, "device_ms": device_ms,
           "value": pairs / (device_ms * 1e-3), "unit": "pairs/s",
           "assigned_peaks": out["assigned"], "peaks_per_grain_median": out["npk_median"],
           "geometry_step": out["geometry_step"],
           "index_shape": {"cell_factor": shape[0], "xsub": shape[1],
                           "method": tune.grid_method(n),
                           "assignment": {
                               "method": "bins" if state["assign_bins"] else "walk",
                               "ms_untimed_trial": amode_ms,
                               "walk_index": None if state["walk_shape"] is None else
                               {"cell_factor": state["walk_shape"][0],
                                "xsub": state["walk_shape"][1]}},
                           "tuning_ms": {"%g,%d,%s" % t_: round(ms, 2)
                                                         for t_, ms in ptable}},
           "score_batch_fp32_ms": e0.elapsed_time(e1),
           "score_grid_counts_equal_fp32": bool(torch.equal(c32, cbuf)),
           "trial_counts_median_max": [int(cbuf[:, 0].median().item()),
                                       int(cbuf[:, 0].max().item())],
           "note": "wall between events: host glue (grouping, GrainSet, PeakTable) included"}
    if cpu:
        from oracle import oracle as orcm
        ref = orcm.Reference() if orcm.have_reference() else orcm.Oracle()
        chk = {"kind": "reference" if isinstance(ref, orcm.Reference) else "port"}
        gv_h = gv.cpu().numpy()
        # compute_gv on 1M peaks (the reference C from the same lab positions)
        xyz_h = xyz[:1_000_000].cpu().numpy()
        rgv = ref.compute_gv(xyz_h, ps.omega[:1_000_000], est["omegasign"],
                             est["wavelength"], est["wedge"], est["chi"], t_arr)
        chk["compute_gv_1M_max_abs_err"] = float(np.abs(rgv - gv_h[:1_000_000]).max())
        # score() of 256 trials over every peak
        rc = ref.score_many(trials[:256], gv_h, [tol])
        chk["trial_counts_identical_256"] = bool(np.array_equal(rc, cbuf[:256].cpu().numpy()))
        # the reference's sequential score_and_assign of all grains on 100k peaks
        # (each peak's outcome depends on that peak alone)
        sel = np.sort(np.random.default_rng(SEED + 14).choice(n, 100_000, replace=False))
        rd = np.full(len(sel), 2.0)
        rl = np.full(len(sel), -1, np.int32)
        ref.assign_seq(u_ref, np.ascontiguousarray(gv_h[sel]), tol, rd, rl)
        chk["assign_labels_identical_100k"] = bool(np.array_equal(rl, lab.cpu().numpy()[sel]))
        chk["assign_drlv2_identical_100k"] = bool(np.array_equal(rd, d2.cpu().numpy()[sel]))
        # 5 score_and_refine rounds of 64 grains on the same grouped peaks
        order = state["order"].cpu().numpy()
        off = state["off"].cpu().numpy()
        k = 64
        gsub = np.ascontiguousarray(gv_h[order[:off[k]]])
        ru, rn, _ = ref.refine_csr(u_ref[:k], gsub, off[:k + 1], tol, rounds)
        gu = state["grains"].ubis.view(-1, 3, 3)[:k].cpu().numpy()
        gn = state["grains"].npk[:k].cpu().numpy()
        scale = np.abs(ru).max(axis=(1, 2))
        chk["refine_64_npk_identical"] = bool(np.array_equal(gn, rn))
        chk["refine_64_ubi_max_rel_err"] = float((np.abs(gu - ru).max(axis=(1, 2)) / scale).max())
        chk["all_identical"] = bool(chk["trial_counts_identical_256"] and
                                    chk["assign_labels_identical_100k"] and
                                    chk["assign_drlv2_identical_100k"] and
                                    chk["refine_64_npk_identical"] and
                                    chk["refine_64_ubi_max_rel_err"] <= 1e-9)
        res["vs_reference"] = chk
    return res


def workload(rank=0, n_ubi=N_UBI):
    from imaged11_b200 import synth
    ps = synth.simulate(N_GRAINS, "Al", gmax=GMAX, seed=SEED, noise_frac=0.10)
    rng = np.random.default_rng(SEED + 1 + rank)
    ubis = synth.trial_ubis(ps.ubis, n_ubi, 0.10, 0.5, rng)
    return ps, ubis


def config_dict(n, m):
    return {
        "workload": "batched candidate scoring: %d g-vectors (2000 FCC Al grains, |g|<=%.1f, "
                    "10%% noise peaks) x %d trial UBIs x tols %s" % (n, GMAX, m, TOLS),
        "n_gvectors": n, "n_ubis_per_gpu": m, "tols": TOLS, "seed": SEED,
        "pairs_per_step": "M*N*T", "l2": "flushed between timed steps (256 MB write)",
    }


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 20 ms by a reader
    thread that stamps each sample on arrival; the sampler is live before the
    timed region starts, and summary() keeps the samples taken inside it (or,
    for a region shorter than one interval, the ones on either side)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 20

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.samples = []   # (arrival time, line)
        self.t0 = self.t1 = None

    def _read(self):
        for line in self.proc.stdout:
            if line.strip():
                self.samples.append((time.monotonic(), line))

    def __enter__(self):
        import threading
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
            t_end = time.monotonic() + 10.0
            while not self.samples and time.monotonic() < t_end and self.proc.poll() is None:
                time.sleep(0.005)
        except OSError:
            self.proc = None
        self.t0 = time.monotonic()
        return self

    def __exit__(self, *a):
        self.t1 = time.monotonic()
        if self.proc is not None:
            time.sleep(2.5 * self.PERIOD_MS / 1e3)   # the sample that covers the end
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.reader.join(timeout=5)

    def summary(self):
        inside = [l for t, l in self.samples
                  if self.t0 is not None and self.t0 <= t <= self.t1 + self.PERIOD_MS / 1e3]
        where = "inside the timed region"
        if not inside and self.samples:
            before = [l for t, l in self.samples if t < self.t0][-1:]
            after = [l for t, l in self.samples if t > self.t1][:1]
            inside = before + after
            where = "the samples on either side of a timed region shorter than %d ms" % \
                self.PERIOD_MS
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in inside:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "sampled": where,
                "window_ms": None if self.t0 is None else (self.t1 - self.t0) * 1e3}


def cuda_time_ms(torch, fn, steps, flush=None):
    """Per-step CUDA-event times (ms) on the current stream, L2 flushed between."""
    times = []
    st = torch.cuda.current_stream()
    for _ in range(steps):
        if flush is not None:
            flush()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times


def cpu_reference_rate(ps, ubis, seconds=10.0, kind="reference"):
    """The reference's own C score() over UBIs (OpenMP, all host threads) on a
    bounded sample of the workload: (pairs/s record, the sample's counts
    (m, T) for the first m UBIs)."""
    from oracle import oracle as orc
    lib = orc.Reference() if (kind == "reference" and orc.have_reference()) else orc.Oracle()
    kind = "reference" if isinstance(lib, orc.Reference) else "port"
    gv = np.ascontiguousarray(ps.gv)
    cores = lib.max_threads()
    # calibrate on a few UBIs, then size the sample to about `seconds`
    k = max(cores, 8)
    t0 = time.perf_counter()
    lib.score_many(ubis[:k], gv, TOLS)
    dt = time.perf_counter() - t0
    m = int(min(len(ubis), max(k, k * seconds / max(dt, 1e-3))))
    t0 = time.perf_counter()
    counts = lib.score_many(ubis[:m], gv, TOLS)
    dt = time.perf_counter() - t0
    pairs = m * len(gv) * len(TOLS)
    return ({"value": pairs / dt, "unit": "pairs/s", "cores": cores, "kind": kind,
             "sample": "%d UBIs x %d g x %d tols (%.1f s)" % (m, len(gv), len(TOLS), dt)},
            counts)


def count_launches(torch, fn):
    """Kernels launched by one call of fn, from the CUDA profiler's activity
    record (memsets and copies excluded); None when profiling is unavailable."""
    try:
        from torch.profiler import ProfilerActivity, profile
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
        names = [e.name for e in prof.events()
                 if str(getattr(e, "device_type", "")).endswith("CUDA")]
        kernels = [nm for nm in names if not any(w in nm.lower() for w in
                                                 ("memset", "memcpy", "memcpyasync"))]
        return len(kernels), sorted(set(k.split("(")[0][:60] for k in kernels))
    except Exception as e:  # noqa: BLE001  (the profiler is optional here)
        return None, [repr(e)[:200]]


def cfg0_measure(cpu=True, reps=3):
    """Plain FP64 method, small: 50 FCC Al grains (|g| <= 1.0, 10% noise
    peaks), compute_gv over every peak in FP64, then 3 score_and_refine
    iterations at tol 0.05 for each of the 50 true UBIs perturbed by 0.1 deg and
    0.1% strain -- through the drop-in module (imaged11_b200.cImageD11) with
    host numpy buffers, one call at a time as an unchanged refinegrains caller
    makes them, timed on the host clock; beside it the same call sequence on
    the reference's compiled C."""
    from imaged11_b200 import cImageD11 as cim, synth
    ps = synth.simulate(50, "Al", gmax=1.0, seed=SEED + 21, noise_frac=0.10)
    rng = np.random.default_rng(SEED + 22)
    u0 = synth.perturb_ubis(ps.ubis, 0.1, 0.001, rng)
    geo = ps.geo
    xyz = np.ascontiguousarray(ps.xyz)
    om = np.ascontiguousarray(ps.omega)
    args = (geo["omegasign"], geo["wavelength"], geo["wedge"], geo["chi"])

    def run_dropin():
        gv = np.empty_like(xyz)
        cim.compute_gv(xyz, om, *args, [0.0, 0.0, 0.0], gv)
        out = []
        for u in u0:
            uu = np.array(u, order="C")
            for _ in range(3):
                n, d = cim.score_and_refine(uu, gv, 0.05)
            out.append((uu, n, d))
        return gv, out

    run_dropin()
    t0 = time.perf_counter()
    for _ in range(reps):
        gv, res = run_dropin()
    ms = (time.perf_counter() - t0) / reps * 1e3
    out = {"grains": 50, "peaks": int(len(xyz)), "iterations": 3, "tol": 0.05,
           "calls_per_run": 1 + 3 * 50, "dropin_ms": ms,
           "note": "host numpy buffers through the drop-in module, host clock"}
    if cpu:
        from oracle import oracle as orcm
        ref = orcm.Reference() if orcm.have_reference() else orcm.Oracle()
        t0 = time.perf_counter()
        for _ in range(reps):
            rgv = ref.compute_gv(xyz, om, *args, np.zeros(3))
            rres = []
            for u in u0:
                uu = np.array(u, order="C")
                for _ in range(3):
                    n, d, uu = ref.score_and_refine(uu, rgv, 0.05)
                rres.append((uu, n, d))
        rms = (time.perf_counter() - t0) / reps * 1e3
        scale = np.abs(np.asarray([r[0] for r in rres])).max(axis=(1, 2))
        out["reference_ms"] = rms
        out["reference_kind"] = "reference" if isinstance(ref, orcm.Reference) else "port"
        out["vs_reference"] = {
            "gv_max_abs_err": float(np.abs(gv - rgv).max()),
            "npk_identical": bool(all(a[1] == b[1] for a, b in zip(res, rres))),
            "ubi_max_rel_err": float(max(np.abs(a[0] - b[0]).max() / s
                                         for a, b, s in zip(res, rres, scale))),
            "mean_drlv2_max_rel_err": float(max(abs(a[2] - b[2]) / max(abs(b[2]), 1e-300)
                                                for a, b in zip(res, rres)))}
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    ps, ubis = workload()
    from oracle import oracle as orc
    lib = orc.Reference() if orc.have_reference() else orc.Oracle()
    kind = "reference" if isinstance(lib, orc.Reference) else "port"
    gv = np.ascontiguousarray(ps.gv)
    cores = lib.max_threads()
    m = max(cores * 4, 64)         # each step: a bounded sample of the workload
    for _ in range(args.warmup):
        lib.score_many(ubis[:m], gv, TOLS)
    times = []
    for i in range(args.steps):
        u = ubis[(i * m) % (len(ubis) - m):][:m]
        t0 = time.perf_counter()
        lib.score_many(u, gv, TOLS)
        times.append(time.perf_counter() - t0)
    pairs = m * len(gv) * len(TOLS)
    value = pairs * len(times) / sum(times)
    line = {
        "impl": "reference", "metric": "assigned peak x grain pairs/s", "value": value,
        "unit": "pairs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(len(gv), N_UBI),
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": kind,
                         "sample": "%d UBIs x %d g x %d tols per step" % (m, len(gv), len(TOLS))},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from imaged11_b200 import batch

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ps, ubis = workload(rank, args.ubis)
    if args.case == "adjoint":  # residual gradient (+ joint refinement)
        print(json.dumps(adjoint_measure(torch, dev, steps=args.steps)))
        return 0
    if args.case == "pipeline":  # full-scale scan, end to end on the device
        print(json.dumps(pipeline_measure(torch, dev)))
        return 0
    if args.case == "refine":   # per-grain CSR refinement alone
        print(json.dumps(refine_csr_measure(torch, dev, steps=args.steps, cpu=False)))
        return 0
    if args.case == "grid":     # cell-index scoring alone (profiling case)
        for cell in (args.cell or [None]):
            for xsub in (args.xsub or [None]):
                print(json.dumps(grid_measure(torch, dev, ps, ubis, steps=args.steps, cell=cell,
                                              xsub=xsub)))
        return 0
    if args.case == "cfg0":     # the small drop-in sequence with host buffers
        print(json.dumps(cfg0_measure()))
        return 0
    if args.case == "translations":  # per-grain translation refinement
        print(json.dumps(translations_measure(torch, dev, steps=args.steps)))
        return 0
    if args.case == "geometry":  # fused detector -> geometry pass (profiling case)
        print(json.dumps(update_geometry_measure(torch, dev, args.peaks, args.steps)))
        return 0
    if args.case == "gv":       # compute_gv alone (profiling case)
        gbs, ms = compute_gv_measure(torch, ps, dev, args.peaks, args.steps)
        print(json.dumps({"case": "compute_gv", "peaks": args.peaks, "GB/s": gbs, "ms": ms}))
        return 0
    n, m, T = len(ps.gv), len(ubis), len(TOLS)
    pairs = m * n * T
    gv_d = torch.tensor(ps.gv, device=dev)
    ubis_d = torch.tensor(ubis, device=dev)
    flush_buf = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def flush():
        flush_buf.fill_(1)

    from imaged11_b200 import tune
    # --- headline: exact batched scoring through the reciprocal-space cell
    # index, binned join (index shape from the autotuner: untimed setup)
    shape, grid_table = tune.tune_grid(ubis_d, gv_d, TOLS,
                                       cell_factors=(0.8, 0.85, 0.9, 1.0, 1.25),
                                       xsubs=(4, 8), reps=2, method="bins")
    base = batch.GvecGrid(gv_d, xsub=1)
    grid = batch.GvecGrid(gv_d, cell=base.cs * shape[0], xsub=shape[1])
    del base
    ws = batch.BinsWorkspace(m, grid, batch.bins_box_estimate(ubis_d, grid, max(TOLS)))
    counts = torch.empty((m, T), dtype=torch.int32, device=dev)

    def step():
        grid.refresh()      # the index rebuilt from the g-vectors every step
        batch.score_grid(ubis_d, grid, TOLS, workspace=ws, out=counts, method="bins")

    step()
    if args.kernel_only:        # profiling case: warm-up + timed steps, nothing else
        for _ in range(args.warmup):
            step()
        kt = cuda_time_ms(torch, step, args.steps, flush)
        torch.cuda.synchronize()
        print(json.dumps({"case": "score_grid_bins", "ubis": m, "gvectors": n,
                          "ms_per_step": sum(kt) / len(kt),
                          "pairs_per_s": pairs / (sum(kt) / len(kt) * 1e-3)}))
        return 0

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        times = cuda_time_ms(torch, step, args.steps, flush)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t = torch.tensor([sum(times)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = pairs * world / (ms_per_step * 1e-3)
    gstats = grid.stats()

    # the join kernel alone: CUDA events around its launches, recorded on the
    # launching stream by the library, over the same steps
    join_ms = []
    st_ = torch.cuda.current_stream()
    for _ in range(args.steps):
        flush()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st_)
        e1.record(st_)  # creates both events
        batch.lib.id11b_grid_bins_time_join(e0.cuda_event, e1.cuda_event)
        step()
        e1.synchronize()
        join_ms.append(e0.elapsed_time(e1))
    join_ms = float(np.mean(join_ms))
    launches, launch_names = count_launches(torch, step)

    # plain FP64 kernel (reference arithmetic): every tolerance in one pass and
    # one launch per tolerance, on the same 20,000 UBIs; counts compared
    gs = batch.GvecSet(gv_d)
    c64 = batch.score_many_fp64(ubis_d, gs, TOLS)
    p64_fused = cuda_time_ms(torch, lambda: batch.score_many_fp64(ubis_d, gs, TOLS, out=c64),
                             2, flush)
    p64_per_tol = cuda_time_ms(torch, lambda: [batch.score_many_fp64(ubis_d, gs, [t_])
                                               for t_ in TOLS], 1, flush)
    rate64f = pairs / (np.mean(p64_fused) * 1e-3)
    rate64 = pairs / (np.mean(p64_per_tol) * 1e-3)
    same64 = bool(torch.equal(c64, counts))

    # FP32 screening kernel (every pair tested, proven FP64 recheck band)
    sws = batch.BatchWorkspace(m, n, refine=False)
    gs.prepare()
    tile, tune_table = tune.tune_score(ubis_d, gs, TOLS, reps=2)
    c32 = torch.empty((m, T), dtype=torch.int32, device=dev)
    batch.score_batch(ubis_d, gs, TOLS, workspace=sws, out=c32)
    k_times = cuda_time_ms(torch, lambda: batch.score_batch(ubis_d, gs, TOLS, workspace=sws,
                                                           out=c32), max(2, args.steps), flush)
    k_ms = float(np.mean(k_times))
    nrecheck, nfallback = sws.stats()
    same32 = bool(torch.equal(c32, counts))

    # the lookup scorer on the same index (per-box lookups, FP64 candidates)
    cw = batch.score_grid(ubis_d, grid, TOLS, method="walk")
    w_times = cuda_time_ms(torch, lambda: batch.score_grid(ubis_d, grid, TOLS, method="walk",
                                                          out=cw), max(2, args.steps), flush)
    same_walk = bool(torch.equal(cw, counts))

    # compute_gv (HBM-bound FP64 streaming kernel), 10M peaks
    gv_gbs, gv_ms = compute_gv_measure(torch, ps, dev, 10_000_000, max(3, args.steps), flush)
    hbm_peak, hbm_kind = measured_hbm_peak()
    gv_cpu = None
    if world == 1:  # the reference's OpenMP compute_gv on the host cores, 2M peaks
        from oracle import oracle as orcm
        ref = orcm.Reference() if orcm.have_reference() else orcm.Oracle()
        reps = -(-2_000_000 // len(ps.xyz))
        xh = np.ascontiguousarray(np.tile(ps.xyz, (reps, 1))[:2_000_000])
        oh = np.ascontiguousarray(np.tile(ps.omega, reps)[:2_000_000])
        geo = ps.geo
        ref.compute_gv(xh[:1000], oh[:1000], geo["omegasign"], geo["wavelength"], 0., 0.,
                       np.zeros(3))
        t0 = time.perf_counter()
        ref.compute_gv(xh, oh, geo["omegasign"], geo["wavelength"], 0., 0., np.zeros(3))
        dt = time.perf_counter() - t0
        gv_cpu = {"value": 56.0 * len(oh) / dt / 1e9, "unit": "GB/s",
                  "cores": ref.max_threads(),
                  "kind": "reference" if isinstance(ref, orcm.Reference) else "port",
                  "sample": "2,000,000 peaks (%.3f s)" % dt}

    # uneven per-grain refinement (persistent kernel in a CUDA graph)
    refine = refine_csr_measure(torch, dev, steps=max(3, args.steps), flush=flush,
                                cpu=(world == 1))
    adj = adjoint_measure(torch, dev, steps=max(3, args.steps))
    trans = translations_measure(torch, dev, steps=max(3, args.steps), cpu=(world == 1))
    # the full-scale scan (cfg4) and the small drop-in sequence (cfg0)
    pipe = pipeline_measure(torch, dev, cpu=(world == 1))
    cfg0 = cfg0_measure(cpu=(world == 1))

    # end to end through the public API: pinned host inputs -> counts on host
    gv_h = torch.tensor(ps.gv).pin_memory()
    ub_h = torch.tensor(ubis).pin_memory()
    ews = batch.BinsWorkspace(m, grid, ws.boxes)

    def e2e_step():
        g = batch.GvecGrid(gv_h.to(dev, non_blocking=True), cell=grid.cs, xsub=grid.xsub)
        c = batch.score_grid(ub_h.to(dev, non_blocking=True), g, TOLS, workspace=ews,
                             method="bins")
        return c.cpu()

    for _ in range(2):
        e2e_step()
    serial_ms = float(np.mean(cuda_time_ms(torch, e2e_step, max(2, args.steps), flush)))
    # the timed step's calls (index rebuilt in place by refresh, then scored)
    # with each step's inputs uploaded on a copy stream while the previous step
    # computes (two indexes, each over its own g buffer): one timed region over
    # all steps -- every upload, L2 flush, index rebuild, scoring and counts read
    # back inside it -- divided by the steps
    main = torch.cuda.current_stream()
    copy_st = torch.cuda.Stream()
    gbuf = [gv_h.to(dev) for _ in range(2)]
    ubuf = [torch.empty(ub_h.shape, dtype=ub_h.dtype, device=dev) for _ in range(2)]
    egrid = [batch.GvecGrid(gbuf[j], cell=grid.cs, xsub=grid.xsub) for j in range(2)]
    assert all(eg.gv.data_ptr() == gbuf[j].data_ptr() for j, eg in enumerate(egrid))

    cbuf_h = [torch.empty((m, T), dtype=torch.int32).pin_memory() for _ in range(2)]

    def e2e_pipelined(k):
        up = [torch.cuda.Event() for _ in range(2)]
        done = [torch.cuda.Event() for _ in range(2)]
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)

        def upload(j):
            # buffers j % 2 were last read by step j - 2: wait for its end
            with torch.cuda.stream(copy_st):
                if j >= 2:
                    copy_st.wait_event(done[j % 2])
                gbuf[j % 2].copy_(gv_h, non_blocking=True)
                ubuf[j % 2].copy_(ub_h, non_blocking=True)
                up[j % 2].record(copy_st)

        e0.record(main)
        copy_st.wait_event(e0)
        upload(0)
        for i in range(k):
            if i + 1 < k:
                upload(i + 1)
            flush()
            main.wait_event(up[i % 2])
            egrid[i % 2].refresh()
            c = batch.score_grid(ubuf[i % 2], egrid[i % 2], TOLS, workspace=ews,
                                 method="bins")
            cbuf_h[i % 2].copy_(c, non_blocking=True)   # the step's counts to the host
            done[i % 2].record(main)
            if i > 0:
                done[(i - 1) % 2].synchronize()         # the previous step's counts arrived
        done[(k - 1) % 2].synchronize()
        e1.record(main)
        e1.synchronize()
        return e0.elapsed_time(e1) / k

    e2e_pipelined(2)
    e2e_steps = max(3, args.steps)
    e2e_ms = e2e_pipelined(e2e_steps)
    e2e_counts_equal = bool(torch.equal(cbuf_h[(e2e_steps - 1) % 2], counts.cpu()))
    e2e_t = torch.tensor([e2e_ms, serial_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = pairs * world / (float(e2e_t[0].item()) * 1e-3)
    e2e_serial = pairs * world / (float(e2e_t[1].item()) * 1e-3)

    if rank != 0:
        return 0

    clocks = clk.summary()
    sm_mhz = clocks["sm_mhz"] or 1965.0
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    fp32_peak = nsm * 128 * 2 * sm_mhz * 1e6 / 1e12
    screened = gstats["pairs_screened"]
    achieved = screened * FLOP_PER_EVAL / (join_ms * 1e-3) / 1e12
    achieved32 = (m * n * FLOP_PER_EVAL) / (k_ms * 1e-3) / 1e12
    cpu, ref_counts = cpu_reference_rate(ps, ubis) if world == 1 else (None, None)
    parity = {"cfg1": {
        "vs": "the reference's own score() (oracle/_ref, the unmodified src/closest.c)",
        "ubis_checked": int(len(ref_counts)) if ref_counts is not None else 0,
        "counts_identical": bool(np.array_equal(
            counts[:len(ref_counts)].cpu().numpy(), ref_counts))
        if ref_counts is not None else None,
        "counts_equal_plain_fp64_all_ubis": same64,
        "counts_equal_fp32_screening_all_ubis": same32,
        "counts_equal_lookup_scorer_all_ubis": same_walk}}
    if "vs_reference" in pipe:
        parity["cfg4"] = pipe["vs_reference"]
    if "vs_reference" in cfg0:
        parity["cfg0"] = cfg0["vs_reference"]
    line = {
        "metric": "assigned peak x grain pairs/s", "value": value, "unit": "pairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64recheck", "data": "synthetic",
        "config": dict(config_dict(n, m),
                       method="exact batched scoring through the reciprocal-space cell index "
                              "(binned join: FP32 screening of (UBI, hkl) boxes against the "
                              "g of their cell rows, proven FP64 recheck band); the index is "
                              "rebuilt from the g-vectors in every step",
                       index_shape={"cell_factor": shape[0], "xsub": shape[1],
                                    "cell_A^-1": grid.cs, "nx": grid.nx}),
        "tuning_ms": {"%g,%d,%s" % t_: round(ms, 3) for t_, ms in grid_table},
        "e2e": {"value": e2e_value, "unit": "pairs/s",
                "h2d_bytes_per_step": int(ps.gv.nbytes + ubis.nbytes),
                "d2h_bytes_per_step": int(m * T * 4),
                "ms_per_step": float(e2e_t[0].item()),
                "how": "the timed step's calls (GvecGrid.refresh + score_grid) on inputs "
                       "copied from pinned host memory into the index's g buffer, counts "
                       "read back to the host (pinned) every step; step i+1's copies run "
                       "on a second stream during step i (two indexes), and the host "
                       "queues step i+1 before waiting for step i's counts; one timed "
                       "region over the steps (L2 flushed before each step inside it)",
                "counts_equal_device_step": e2e_counts_equal,
                "serial_value": e2e_serial,
                "serial_how": "a new GvecGrid (bounds read back) + score_grid each step, "
                              "its copies before its compute (CUDA events around each step)"},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "traffic": K_JOIN_DRAM_BYTES,
                     "traffic_note": K_JOIN_TRAFFIC_NOTE,
                     "kernel": "k_join<3> (binned join)",
                     "join_ms": join_ms, "pairs_screened": screened,
                     "peak_note": "CUDA-core FP32 = SMs x 128 x 2 x median SM clock under load; "
                                  "%d FLOP per screened (box, g) pair" % FLOP_PER_EVAL},
        "gpu_launches": None if launches is None else launches * args.steps,
        "gpu_launches_note": "kernels one step launches (CUDA profiler activity record) x steps",
        "gpu_kernels": launch_names,
        "plain_fp64": {"value_all_tols": rate64f, "value_per_tol_launch": rate64,
                       "unit": "pairs/s", "ubis": m, "ms_all_tols": float(np.mean(p64_fused)),
                       "ratio_vs_plain_fp64_all_tols": value / rate64f,
                       "ratio_vs_plain_fp64_per_tol_launch": value / rate64,
                       "counts_equal": same64},
        "fp32_screening": {"value": pairs / (k_ms * 1e-3), "ms": k_ms,
                           "tile": {"ubis_per_thread": tile[0], "gsplit": tile[1]},
                           "roofline": {"bound": "fp32", "achieved": achieved32,
                                        "peak": fp32_peak, "frac": achieved32 / fp32_peak,
                                        "kernel": "k_batch<%d,3,score>" % tile[0]},
                           "recheck": {"fp64_pairs": nrecheck, "fraction": nrecheck / (m * n),
                                       "fallback_ubis": nfallback},
                           "counts_equal": same32},
        "cell_index_lookup": {"value": pairs / (float(np.mean(w_times)) * 1e-3),
                              "ms": float(np.mean(w_times)), "counts_equal": same_walk},
        "cell_index": {"fp64_rechecks": gstats["pairs_tested"],
                       "pairs_screened_fp32": screened,
                       "screened_fraction_of_all_pairs": screened / float(m * n),
                       "plain_scan_ubis": gstats["fallback_ubis"],
                       "boxes_capacity": ws.boxes},
        "parity": parity,
        "refine_csr": refine,
        "adjoint": adj,
        "translations": trans,
        "pipeline": pipe,
        "cfg0": cfg0,
        "compute_gv": {"peaks": 10_000_000, "ms": gv_ms, "achieved_gbs": gv_gbs,
                       "cpu_baseline": gv_cpu,
                       "peak_gbs": hbm_peak, "peak_kind": hbm_kind,
                       "frac": gv_gbs / hbm_peak, "bytes_per_peak": 56},
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ubis", type=int, default=N_UBI, help="trial UBIs per GPU")
    ap.add_argument("--kernel-only", action="store_true",
                    help="only warm-up + timed steps of the scoring step (profiling case)")
    ap.add_argument("--case", default="score",
                    choices=["score", "gv", "geometry", "grid", "translations", "refine", "adjoint",
                             "pipeline", "cfg0"],
                    help="gv: compute_gv alone on --peaks lab positions; refine: per-grain "
                         "CSR refinement alone (profiling cases)")
    ap.add_argument("--peaks", type=int, default=10_000_000)
    ap.add_argument("--cell", type=float, nargs="*", help="grid case: cell sides (1/A) to time")
    ap.add_argument("--xsub", type=int, nargs="*", help="grid case: x subdivisions to time")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
