"""Generate tests/golden/refinegrains.npz from the REFERENCE's own
refinegrains.refinepositions.

Run where an ImageD11 checkout exists, naming its root (argument or the
IMAGED11_REF environment variable), after ``make -C oracle REF=<root>``:

    python tests/golden/make_refinegrains.py /path/to/ImageD11

ImageD11.refinegrains is imported from the checkout with the stand-ins of
make_indexer.py (xfab, h5py, fabio; ImageD11.cImageD11 served by the
reference's own C in oracle/_ref/libimaged11_ref.so).  A refinegrains object
is set up as loadparameters / readubis / loadfiltered / generate_grains would
(in memory: the parameters, the UBIs read, and a columnfile of one simulated
scan of fcc Al grains at different positions), and refinepositions()
(ImageD11/refinegrains.py:636-660) runs its Nelder-Mead simplex per grain.

The fixture holds the scan geometry, each grain's peaks as assignlabels left
them (peaks_xyz, omega), the UBIs read, the starting translations, the
translations refinepositions wrote and the reference's gof at them (gof with
that grain alone and tolerance 1.0, as refinepositions evaluates it).  Only
the .npz file is read by the tests.
"""
import contextlib
import io
import logging
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from imaged11_b200 import synth  # noqa: E402
import make_indexer  # noqa: E402

GEOKEYS = ("distance", "y_center", "z_center", "y_size", "z_size", "tilt_x", "tilt_y",
           "tilt_z", "o11", "o12", "o21", "o22", "omegasign", "wavelength", "wedge", "chi",
           "t_x", "t_y", "t_z")


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IMAGED11_REF")
    if not ref_root:
        sys.exit("usage: make_refinegrains.py /path/to/ImageD11 (or set IMAGED11_REF)")
    so = os.path.join(REPO, "oracle", "_ref", "libimaged11_ref.so")
    if not os.path.exists(so):
        sys.exit("build the reference's C first: make -C oracle REF=" + ref_root)
    logging.disable(logging.CRITICAL)
    make_indexer.import_reference_indexing(ref_root, so)
    import importlib
    rgm = importlib.import_module("ImageD11.refinegrains")
    colm = importlib.import_module("ImageD11.columnfile")

    geo = synth.default_geometry(distance=152300., y_center=1024 + 3.7, z_center=1024 - 2.1,
                                 tilt_x=0.001, tilt_y=-0.002, tilt_z=0.003, wedge=0.02,
                                 chi=-0.03, t_x=0., t_y=0., t_z=0.)
    ng = 10
    ps = synth.simulate(ng, "Al", gmax=1.0, seed=61, geo=geo, noise_frac=0.05,
                        translations_um=120.0, sigma_px=0.3, sigma_om=0.03)
    rng = np.random.default_rng(62)
    ubis = synth.perturb_ubis(ps.ubis, 0.03, 0.0003, rng)
    with contextlib.redirect_stdout(io.StringIO()):
        rg = rgm.refinegrains(tolerance=0.1, OmFloat=False)
    for k in GEOKEYS:
        rg.parameterobj.parameters[k] = float(geo[k])
    for i in range(ng):               # as readubis
        rg.grainnames.append(i)
        rg.ubisread[i] = ubis[i].copy()
        rg.translationsread[i] = None
    col = colm.colfile_from_dict({"sc": ps.s, "fc": ps.f, "omega": ps.omega})
    name = "scan0"                    # as loadfiltered
    rg.scannames.append(name)
    col.addcolumn(np.ones(col.nrows, float), "drlv2")
    col.addcolumn(np.ones(col.nrows, float) - 2, "labels")
    rg.scantitles[name] = col.titles
    rg.scandata[name] = col
    with contextlib.redirect_stdout(io.StringIO()):
        rg.generate_grains()
    keys = sorted(rg.grains.keys())
    t0 = np.array([np.array(rg.grains[k].translation, dtype=np.float64) for k in keys])
    with contextlib.redirect_stdout(io.StringIO()):
        rg.refinepositions(maxiters=100)
    t_ref = np.array([np.array(rg.grains[k].translation, dtype=np.float64) for k in keys])
    # the reference's gof at the translations it wrote, as refinepositions
    # evaluates it (one grain, tolerance 1.0)
    gof = []
    rg.tolerance = 1.0
    rg.parameterobj.varylist = ["t_x", "t_y", "t_z"]
    with contextlib.redirect_stdout(io.StringIO()):
        for k, t in zip(keys, t_ref):
            rg.grains_to_refine = [k]
            gof.append(rg.gof(list(t)))
    xyz = [np.asarray(rg.grains[k].peaks_xyz, dtype=np.float64) for k in keys]
    om = [np.asarray(rg.grains[k].om, dtype=np.float64) for k in keys]
    off = np.zeros(ng + 1, np.int64)
    off[1:] = np.cumsum([len(o) for o in om])
    out = dict(geo=np.array([geo[k] for k in GEOKEYS]), keys=np.array([k[0] for k in keys]),
               xyz=np.concatenate(xyz), omega=np.concatenate(om), offsets=off,
               ubis=np.array([rg.ubisread[k[0]] for k in keys]), t0=t0, t_ref=t_ref,
               gof_ref=np.array(gof), t_true=ps.translations)
    path = os.path.join(HERE, "refinegrains.npz")
    np.savez_compressed(path, **out)
    print("%d grains, %d assigned peaks; reference gof %s" % (ng, off[-1], np.round(gof, 3)))
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
