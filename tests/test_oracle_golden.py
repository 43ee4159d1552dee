"""Pin the CPU oracle (C restatement) to the reference's own outputs.

The golden vectors were produced by the reference's compiled C and its numpy
transform module (tests/golden/make_golden.py).  Every oracle result must be
bit-identical to the reference C; the reference numpy path is a second,
independent check at the reference test's own tolerance.
"""
import numpy as np


def test_verify_rounding(oracle):
    for n in (0, 1, 20, 12345, -7):
        assert oracle.verify_rounding(n) == 0


def test_compute_gv_bitexact(oracle, golden):
    d = golden["compute_gv"]
    for i in range(int(d["gv_ncases"])):
        osg, wl, w, c, tx, ty, tz = d["gv%d_params" % i]
        gv = oracle.compute_gv(d["gv_xlylzl"], d["gv_omega"], osg, wl, w, c, [tx, ty, tz])
        assert np.array_equal(gv, d["gv%d_out" % i]), i
        # reference numpy path, test/test_cImageD11.py:47 uses np.allclose
        assert np.allclose(gv, d["gv%d_numpy" % i])
        geo = oracle.compute_geometry(d["gv_xlylzl"], d["gv_omega"], osg, wl, w, c, [tx, ty, tz])
        assert np.array_equal(geo, d["gv%d_geometry" % i]), i
    osg, wl, w, c, tx, ty, tz = d["rand_params"]
    gv = oracle.compute_gv(d["rand_xlylzl"], d["rand_omega"], osg, wl, w, c, [tx, ty, tz])
    assert np.array_equal(gv, d["rand_gv"])
    geo = oracle.compute_geometry(d["rand_xlylzl"], d["rand_omega"], osg, wl, w, c, [tx, ty, tz])
    assert np.array_equal(geo, d["rand_geometry"])


def test_compute_xlylzl_bitexact(oracle, golden):
    d = golden["compute_xlylzl"]
    for r, out, npy in zip(d["xl_r"], d["xl_out"], d["xl_numpy"]):
        x = oracle.compute_xlylzl(d["xl_s"], d["xl_f"], d["xl_p"], r, d["xl_dist"])
        assert np.array_equal(x, out)
        assert np.abs(x - npy).max() < 1e-6      # test/test_cImageD11.py:188


def test_score_family_bitexact(oracle, golden):
    d = golden["scoring"]
    gv, ubis, tols = d["sc_gv"], d["sc_ubis"], d["sc_tols"]
    counts = oracle.score_many(ubis, gv, tols)
    assert np.array_equal(counts, d["sc_counts"])
    for i, u in enumerate(ubis):
        for j, t in enumerate(tols):
            n, m, u2 = oracle.score_and_refine(u, gv, t)
            assert n == d["sar_n"][i, j]
            assert m == d["sar_drlv2"][i, j]
            assert np.array_equal(u2, d["sar_ubi"][i, j])
    for i, u in enumerate(ubis[:20]):
        uu = u.copy()
        for _ in range(3):
            _, _, uu = oracle.score_and_refine(uu, gv, 0.05)
        assert np.array_equal(uu, d["sar3_ubi"][i])


def test_refine_assigned_bitexact(oracle, golden):
    d = golden["scoring"]
    for gi in range(8):
        n, m, u = oracle.refine_assigned(d["sc_ubis"][gi], d["sc_gv"], d["ra_labels"], gi)
        assert n == d["ra_n"][gi] and m == d["ra_drlv2"][gi]
        assert np.array_equal(u, d["ra_ubi"][gi])


def test_score_and_assign_bitexact(oracle, golden):
    d = golden["scoring"]
    gv = d["sc_gv"]
    drl = np.full(len(gv), 2.0)
    lab = np.full(len(gv), -1, np.int32)
    for i, u in enumerate(d["sc_ubis"][:24]):
        k, drl, lab = oracle.score_and_assign(u, gv, 0.05, drl, lab, i)
        assert k == d["sa_n"][i]
    assert np.array_equal(drl, d["sa_drlv2"])
    assert np.array_equal(lab, d["sa_labels"])


def test_adversarial_and_singular(oracle, golden):
    d = golden["scoring"]
    u0, g = d["adv_ubi"], d["adv_gv"]
    for j, t in enumerate(d["sc_tols"]):
        assert oracle.score(u0, g, t) == d["adv_counts"][j]
        n, m, u = oracle.score_and_refine(u0, g[:-6], t)
        assert n == d["adv_sar_n"][j] and m == d["adv_sar_drlv2"][j]
        assert np.array_equal(u, d["adv_sar_ubi"][j])
    for i, row in enumerate(d["sing_results"]):
        n, m, u = oracle.score_and_refine(u0, d["sing%d_gv" % i], 0.05)
        assert n == row[0] and m == row[1] and np.array_equal(u.ravel(), row[2:])


def test_batch_helpers_match_single_calls(oracle, golden):
    d = golden["scoring"]
    gv = d["sc_gv"]
    ubis = d["sc_ubis"][:6]
    off = np.array([0, 300, 300, 900, 1500, 2000, 2600], np.int64)
    u, npk, drl = oracle.refine_csr(ubis, gv, off, 0.05, 2)
    for g in range(6):
        uu = ubis[g].copy()
        for _ in range(2):
            n, m, uu = oracle.score_and_refine(uu, gv[off[g]:off[g + 1]], 0.05)
        assert np.array_equal(u[g], uu) and npk[g] == n and drl[g] == m
