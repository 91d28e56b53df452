"""ctypes wrapper of the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may import
this module; the product never does. It wraps ``liborc.so`` (the C restatement in
``katsevich_oracle.c``) and ``_ref/libkatsevich_bkproj_ref.so`` (the reference's own
``KatsevichBkProj.cpp``, compiled unchanged by ``oracle/Makefile``).

Array conventions (numpy C order == the reference's MATLAB column-major arrays):
  proj / fproj : shape (P, ZL, YL)   -- MATLAB Proj(YL, ZL, P)
  image        : shape (NX, NY, NZ)  -- linear index (x*NY + y)*NZ + z
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")
REF_BKPROJ_PATH = os.path.join(HERE, "_ref", "libkatsevich_bkproj_ref.so")
REF_PROJSLICE_PATH = os.path.join(HERE, "_ref", "libcreateprojslice_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_up = ctypes.POINTER(ctypes.c_ubyte)


class FilterParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "ProjScale", "DecWidth", "DecHeigh", "ScanR", "StdDis", "HelicP", "FilterCoeFF",
        "DeltaAngle")] + [(n, ctypes.c_int) for n in ("FilteringMode", "YL", "ZL", "ProjNumber")]


class BPGeom(ctypes.Structure):
    _fields_ = [("locus", ctypes.c_double * 7), ("detector", ctypes.c_double * 6),
                ("object", ctypes.c_double * 7), ("n_detector", ctypes.c_int),
                ("n_object", ctypes.c_int), ("honour_extras", ctypes.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} missing: run `make -C oracle`")
        L = ctypes.CDLL(LIB_PATH)
        L.orc_geometry_sizing.argtypes = [ctypes.c_double] * 4 + [ctypes.c_int] * 2 + [_dp] * 3
        L.orc_num_kappa.argtypes = [ctypes.c_int, _ip]
        L.orc_filter_tables.argtypes = [ctypes.POINTER(FilterParams), _dp, _dp, _dp, _ip, _dp,
                                        _dp, _ip, _ip, _dp, _dp]
        L.orc_hilbert_taps.argtypes = [ctypes.c_int, _dp]
        L.orc_filter.argtypes = [ctypes.POINTER(FilterParams), _dp, _dp, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int]
        L.orc_filter_direct.argtypes = [ctypes.POINTER(FilterParams), _dp, _dp, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int]
        L.orc_filter_view_stages.argtypes = [ctypes.POINTER(FilterParams), _dp, ctypes.c_int,
                                             _dp, _dp, _dp]
        L.orc_pisegment.argtypes = [ctypes.c_double] * 3 + [_dp, _dp]
        L.orc_pisegment.restype = None
        L.orc_bkproj.argtypes = [ctypes.POINTER(BPGeom), _dp, _dp] + [ctypes.c_int] * 5 + [
            ctypes.POINTER(ctypes.c_longlong), _up]
        L.orc_pi_table.argtypes = [ctypes.POINTER(BPGeom), _dp, _dp, _ip, _ip, _up, ctypes.c_int]
        L.orc_project_ellipsoids.argtypes = [ctypes.POINTER(BPGeom), _dp, ctypes.c_int, _dp,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


class OracleError(RuntimeError):
    pass


def _check(rc, what):
    if rc != 0:
        raise OracleError(f"{what} failed with code {rc}")


# ---------------------------------------------------------------------------------------
def geometry_sizing(ScanR, StdDis, HelicP, ObjR, YL, ZL):
    """FunctionKat_v6.m:49-57 -> (DecWidth, DecHeigh, delta)."""
    w, h, d = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    lib().orc_geometry_sizing(ScanR, StdDis, HelicP, ObjR, YL, ZL, ctypes.byref(w),
                              ctypes.byref(h), ctypes.byref(d))
    return w.value, h.value, d.value


def num_kappa(ZL):
    qq = ctypes.c_int()
    al = lib().orc_num_kappa(ZL, ctypes.byref(qq))
    return al, qq.value


def filter_params(**kw) -> FilterParams:
    fp = FilterParams()
    for k, v in kw.items():
        setattr(fp, k, v)
    return fp


def filter_tables(fp: FilterParams) -> dict:
    AL, QQ = num_kappa(fp.ZL)
    YL, ZL = fp.YL, fp.ZL
    out = dict(AZCor=np.zeros((AL, YL)), coef=np.zeros((AL, YL)), Rato=np.zeros(AL),
               lw=np.zeros((AL, YL), np.int32), w_lw=np.zeros((AL, YL)),
               w_up=np.zeros((AL, YL)), bAL=np.zeros((ZL, YL), np.int32),
               eAL=np.zeros((ZL, YL), np.int32), bC=np.zeros((ZL, YL)), eC=np.zeros((ZL, YL)))
    rc = lib().orc_filter_tables(
        ctypes.byref(fp), _ptr(out["AZCor"]), _ptr(out["coef"]), _ptr(out["Rato"]),
        _ptr(out["lw"], _ip), _ptr(out["w_lw"]), _ptr(out["w_up"]), _ptr(out["bAL"], _ip),
        _ptr(out["eAL"], _ip), _ptr(out["bC"]), _ptr(out["eC"]))
    _check(rc, "orc_filter_tables")
    out["AL"], out["QQ"] = AL, QQ
    return out


def hilbert_taps(YL) -> np.ndarray:
    h = np.zeros(2 * YL - 1)
    _check(lib().orc_hilbert_taps(YL, _ptr(h)), "orc_hilbert_taps")
    return h


def katsevich_filter_direct(fp: FilterParams, proj: np.ndarray, p_begin=0, p_end=0,
                            nthreads=0):
    """KatsevichFiltering_T.m (DerMode 0: direct half-view derivative) -> FProj."""
    proj = np.ascontiguousarray(proj, dtype=np.float64)
    assert proj.shape == (fp.ProjNumber, fp.ZL, fp.YL)
    out = np.zeros_like(proj)
    _check(lib().orc_filter_direct(ctypes.byref(fp), _ptr(proj), _ptr(out), p_begin, p_end,
                                   nthreads), "orc_filter_direct")
    return out


def derivative_direct(fp: FilterParams, proj: np.ndarray, p: int):
    """KatsevichFiltering_T.m:50-101 for view p -> GF (ZL, YL)."""
    proj = np.ascontiguousarray(proj, dtype=np.float64)
    gf = np.zeros((fp.ZL, fp.YL))
    L = lib()
    L.orc_derivative_direct.argtypes = [ctypes.POINTER(FilterParams), _dp, ctypes.c_int, _dp]
    _check(L.orc_derivative_direct(ctypes.byref(fp), _ptr(proj), p, _ptr(gf)),
           "orc_derivative_direct")
    return gf


def katsevich_filter(fp: FilterParams, proj: np.ndarray, p_begin=0, p_end=0, nthreads=0):
    """KatsevichFiltering.m (CPU branch) on views [p_begin, p_end) -> FProj (same shape)."""
    proj = np.ascontiguousarray(proj, dtype=np.float64)
    assert proj.shape == (fp.ProjNumber, fp.ZL, fp.YL)
    out = np.zeros_like(proj)
    _check(lib().orc_filter(ctypes.byref(fp), _ptr(proj), _ptr(out), p_begin, p_end, nthreads),
           "orc_filter")
    return out


def filter_view_stages(fp: FilterParams, proj: np.ndarray, p: int):
    AL, _ = num_kappa(fp.ZL)
    proj = np.ascontiguousarray(proj, dtype=np.float64)
    gf = np.zeros((fp.ZL, fp.YL))
    xin = np.zeros((AL, fp.YL))
    xout = np.zeros((AL, fp.YL))
    _check(lib().orc_filter_view_stages(ctypes.byref(fp), _ptr(proj), p, _ptr(gf), _ptr(xin),
                                        _ptr(xout)), "orc_filter_view_stages")
    return gf, xin, xout


def find_tau(ratio=2.0 / 3.0, tol=1e-4):
    """FindTau.m:6-22."""
    L = lib()
    L.orc_find_tau.restype = ctypes.c_double
    L.orc_find_tau.argtypes = [ctypes.c_double, ctypes.c_double]
    return L.orc_find_tau(ratio, tol)


def pisegment(x, y, z):
    b, t = ctypes.c_double(), ctypes.c_double()
    lib().orc_pisegment(x, y, z, ctypes.byref(b), ctypes.byref(t))
    return b.value, t.value


def bp_geom(locus, detector, obj, honour_extras=True) -> BPGeom:
    g = BPGeom()
    for i, v in enumerate(locus):
        g.locus[i] = v
    for i, v in enumerate(detector):
        g.detector[i] = v
    for i, v in enumerate(obj):
        g.object[i] = v
    g.n_detector = len(detector)
    g.n_object = len(obj)
    g.honour_extras = 1 if honour_extras else 0
    return g


def _vol_shape(g: BPGeom):
    return int(g.object[1]), int(g.object[2]), int(g.object[3])


def bkproj(g: BPGeom, fproj: np.ndarray, image: np.ndarray | None = None, x_range=(0, 0),
           z_range=(0, 0), nthreads=0, want_touched=False):
    """KatsevichBkProj.cpp restated. Returns (image, n_updates[, touched])."""
    fproj = np.ascontiguousarray(fproj, dtype=np.float64)
    if image is None:
        image = np.zeros(_vol_shape(g))
    assert image.dtype == np.float64 and image.flags.c_contiguous
    n = ctypes.c_longlong()
    touched = np.zeros(_vol_shape(g), np.uint8) if want_touched else None
    rc = lib().orc_bkproj(ctypes.byref(g), _ptr(fproj), _ptr(image), x_range[0], x_range[1],
                          z_range[0], z_range[1], nthreads, ctypes.byref(n),
                          _ptr(touched, _up) if touched is not None else None)
    _check(rc, "orc_bkproj")
    if want_touched:
        return image, n.value, touched
    return image, n.value


def pi_table(g: BPGeom, nthreads=0):
    shp = _vol_shape(g)
    B, T = np.zeros(shp), np.zeros(shp)
    lb, le = np.zeros(shp, np.int32), np.zeros(shp, np.int32)
    valid = np.zeros(shp, np.uint8)
    _check(lib().orc_pi_table(ctypes.byref(g), _ptr(B), _ptr(T), _ptr(lb, _ip), _ptr(le, _ip),
                              _ptr(valid, _up), nthreads), "orc_pi_table")
    return dict(B=B, T=T, loop_begin=lb, loop_end=le, valid=valid.astype(bool))


def project_ellipsoids(g: BPGeom, ell: np.ndarray, p_begin=0, p_end=0, nthreads=0):
    P = int(g.locus[5]) - int(g.locus[4]) + 1
    YL, ZL = int(g.detector[1]), int(g.detector[3])
    ell = np.ascontiguousarray(ell, dtype=np.float64).reshape(-1, 10)
    proj = np.zeros((P, ZL, YL))
    _check(lib().orc_project_ellipsoids(ctypes.byref(g), _ptr(ell), ell.shape[0], _ptr(proj),
                                        p_begin, p_end, nthreads), "orc_project_ellipsoids")
    return proj


# ---------------------------------------------------------------------------------------
def ref_available() -> bool:
    return os.path.exists(REF_BKPROJ_PATH)


def ref_bkproj(geom: dict, fproj: np.ndarray, image: np.ndarray):
    """Run the reference's own KatsevichBkProj.cpp mexFunction (in place on `image`)."""
    import sys
    root = os.path.dirname(HERE)
    if root not in sys.path:
        sys.path.insert(0, root)
    from ctrecon_b200.mexharness import MexModule
    m = MexModule(REF_BKPROJ_PATH)
    m.set_print(False)
    m.call([geom, fproj, image], nlhs=0)
    return image


# The head phantom of CreateProjSlice.cpp:13-24, rows (a, b, c, x0, y0, z0, phi in degrees,
# density) in units of the object radius: the reference's own projector, kept here as the test
# input that pins the analytic projectors against it.
HEAD_PHANTOM = np.array([
    [0.6900, 0.920, 0.900, 0, 0, 0, 0, 2.0],
    [0.6624, 0.874, 0.880, 0, 0, 0, 0, -0.98],
    [0.4100, 0.160, 0.210, -0.22, 0, -0.25, 108, -0.02],
    [0.3100, 0.110, 0.220, 0.22, 0, -0.25, 72, -0.02],
    [0.2100, 0.250, 0.500, 0, 0.35, -0.25, 0, 0.02],
    [0.0460, 0.046, 0.046, 0, 0.1, -0.25, 0, 0.02],
    [0.0460, 0.023, 0.020, -0.08, -0.65, -0.25, 0, 0.01],
    [0.0460, 0.023, 0.020, 0.06, -0.65, -0.25, 90, 0.01],
    [0.0560, 0.040, 0.100, 0.06, -0.105, 0.625, 90, 0.02],
    [0.0560, 0.056, 0.100, 0, 0.100, 0.625, 0, -0.02]])


def head_phantom_ellipsoids(pi=3.14159265358979):
    """HEAD_PHANTOM as rows (cx cy cz a b c phi theta psi rho) of the analytic projectors: a
    rotation about z by phi (CreateProjSlice.cpp:79-81,106-111), no tilt."""
    H = HEAD_PHANTOM
    z = np.zeros(len(H))
    return np.column_stack([H[:, 3], H[:, 4], H[:, 5], H[:, 0], H[:, 1], H[:, 2],
                            H[:, 6] * pi / 180, z, z, H[:, 7]])


def ref_projslice_available() -> bool:
    return os.path.exists(REF_PROJSLICE_PATH)


def ref_create_proj_slice(theta, pou, heli, YL, ZL, DW, DH):
    """Run the reference's own CreateProjSlice.cpp mexFunction (FunctionKat_v6.m:73): one view
    of the head phantom at source angle theta, source radius pou, pitch heli, a YL x ZL flat
    detector through the axis of width DW and height DH. Returns numpy (ZL, YL)."""
    import sys
    root = os.path.dirname(HERE)
    if root not in sys.path:
        sys.path.insert(0, root)
    from ctrecon_b200.mexharness import MexModule
    m = MexModule(REF_PROJSLICE_PATH)
    m.set_print(False)
    return m.call([float(theta), float(pou), float(heli), float(YL), float(ZL), float(DW),
                   float(DH)], nlhs=1)[0]


def rebin_to_panel(proj, c, w, D):
    """rebinToPanel.m:1-36 on numpy (prj_num, det_hei, det_num); returns (out, detWidth)."""
    proj = np.ascontiguousarray(proj, dtype=np.float64)
    P, H, N = proj.shape
    out = np.empty_like(proj)
    L = lib()
    L.orc_rebin_to_panel.restype = ctypes.c_double
    L.orc_rebin_to_panel.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp]
    width = L.orc_rebin_to_panel(_ptr(proj), N, H, P, c, w, D, _ptr(out))
    return out, width
