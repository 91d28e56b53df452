"""Test configuration: the `gpu` marker, import paths and shared fixtures.

CPU tests (`-m "not gpu"`) check the FP64 oracle against the reference's own
KatsevichBkProj.cpp and the golden vectors, the host-side tables and the C ABI surface.
GPU tests (`-m gpu`) compare the CUDA path, called through the C ABI, with the oracle.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) GPU")


def rel_rmse(x, ref, mask=None):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if mask is not None:
        x, ref = x[mask], ref[mask]
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))


def max_abs(x, ref, mask=None):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if mask is not None:
        x, ref = x[mask], ref[mask]
    return float(np.max(np.abs(x - ref))) if x.size else 0.0


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    return oracle


@pytest.fixture(scope="session")
def tiny_scan():
    from ctrecon_b200.geometry import small_config
    return small_config()


def oracle_filter_params(O, s):
    return O.filter_params(ProjScale=float(s.views_per_turn), DecWidth=s.DecWidth,
                           DecHeigh=s.DecHeigh, ScanR=s.ScanR, StdDis=s.StdDis, HelicP=s.HelicP,
                           FilterCoeFF=s.filter_coeff, DeltaAngle=s.delta,
                           FilteringMode=s.filtering_mode, YL=s.YL, ZL=s.ZL, ProjNumber=s.P)


def oracle_geom(O, s, honour_extras=True):
    return O.bp_geom(s.locus(), s.detector(), s.object(), honour_extras=honour_extras)


def central_block(O, s, n=48):
    """A central n^3 block of scan s at the scan's voxel pitch, posed the way the reference's
    KatsevichBkProj accepts it (ObjR = n/2 voxels, so that its default pitch 2*ObjR/N is the
    scan's), and restricted to the views [lo, hi) that the block's PI intervals need, with a
    3-view margin so that loop bounds and endpoint weights are those of the full scan
    (KatsevichBkProj.cpp:177-234). Returns (locus, detector, object, lo, hi)."""
    dx = s.voxel_size[0]
    obj = [dx * n / 2.0, float(n), float(n), float(n), dx, dx, dx]
    g = O.bp_geom(s.locus(), s.detector(), obj, honour_extras=True)
    pit = O.pi_table(g)
    v = pit["valid"]
    lo = max(0, int(np.floor(pit["B"][v].min())) - 3)
    hi = min(s.P, int(np.ceil(pit["T"][v].max())) + 4)
    locus = s.locus()
    locus[4] = float(lo + 1)          # ProjBeginIndex (one-based)
    locus[5] = float(hi)              # ProjEndIndex
    return locus, s.detector(), obj, lo, hi
