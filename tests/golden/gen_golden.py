"""Generate the golden vectors under tests/golden/ (run in the build container).

The reference ships no tests or fixtures for this path, so the pins are:

* ``bkproj_ref_tiny.npz`` -- the reference's own CPU backprojector, KatsevichBkProj.cpp
  compiled unchanged from the CTRecon sources (oracle/_ref, built by oracle/Makefile), run
  on a small helical geometry whose FProj comes from the FP64 filter oracle. Stores the
  ellipsoids, the geometry and the reference's output image for the FProj stored in
  ``filter_tiny.npz``
  (an image pre-filled with a sentinel, so the untouched voxels are visible).
* ``geometry_kat.npz`` -- the detector sizing of FunctionKat_v6.m:49-57 for the reference's
  own default scan, and the constants the reference recorded from it
  (KatsevichFiltering_GPU.cu:997, KatsevichBkProj_GPU.cu:465-479).
* ``filter_tiny.npz`` -- the FP64 filter oracle's output for the same small scan, to pin the
  restatement against regressions (MATLAB/Octave, needed to run KatsevichFiltering.m, are
  not available).

Usage: python tests/golden/gen_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from ctrecon_b200.geometry import small_config  # noqa: E402

SENTINEL = 7.25


def golden_scan():
    return small_config(name="golden", YL=32, ZL=8, views_per_turn=90, turns=3, NX=20, NY=20,
                        NZ=12, voxel=None, n_ellipsoids=5, seed=11)


def main():
    s = golden_scan()
    fp = O.filter_params(ProjScale=float(s.views_per_turn), DecWidth=s.DecWidth,
                         DecHeigh=s.DecHeigh, ScanR=s.ScanR, StdDis=s.StdDis, HelicP=s.HelicP,
                         FilterCoeFF=s.filter_coeff, DeltaAngle=s.delta, FilteringMode=0,
                         YL=s.YL, ZL=s.ZL, ProjNumber=s.P)
    g = O.bp_geom(s.locus(), s.detector(), s.object(), honour_extras=False)
    ell = s.ellipsoids()
    proj = O.project_ellipsoids(g, ell)
    fproj = O.katsevich_filter(fp, proj)
    if not O.ref_available():
        raise SystemExit("oracle/_ref is not built: run `make -C oracle` with the CTRecon sources")
    img = np.full(s.vol_shape, SENTINEL)
    O.ref_bkproj(s.geom_struct(), fproj, img)
    np.savez_compressed(os.path.join(HERE, "bkproj_ref_tiny.npz"), ell=ell,
                        locus=np.array(s.locus()), detector=np.array(s.detector()),
                        object=np.array(s.object()), image=img, sentinel=SENTINEL)
    np.savez_compressed(os.path.join(HERE, "filter_tiny.npz"), proj=proj, fproj=fproj,
                        params=np.array(s.filter_args()))
    # FunctionKat_v6.m:18-27 defaults and the constants recorded in the reference
    w, h, d = O.geometry_sizing(75.0, 150.0, 12.5, 25.0, 300, 40)
    np.savez(os.path.join(HERE, "geometry_kat.npz"),
             inputs=np.array([75.0, 150.0, 12.5, 25.0, 300, 40]),
             computed=np.array([w, h, d]),
             recorded=np.array([106.7778696422639, 18.005134774901215, 2.461918834681550]))
    print("wrote golden vectors to", HERE)


if __name__ == "__main__":
    main()
