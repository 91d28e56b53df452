"""Python face of the C ABI, mirroring the reference's MEX interface.

Host functions take numpy arrays in the reference's MATLAB layouts (C-order shape
``(P, ZL, YL)`` for projections, ``(NX, NY, NZ)`` for the image) and behave like the MEX
functions they replace:

* :func:`KatsevichFiltering_GPU` -- 14 arguments, filtered result written in place into
  the 14th (``KatsevichFiltering_GPU.cu:939-978``);
* :func:`KatsevichBkProj` / :func:`KatsevichBkProj_GPU` -- ``(geom, FProj, RecMatrix)``,
  image updated in place (``KatsevichBkProj.cpp:314-352``).

Device functions take CUDA tensors (torch is only the device-memory and stream plumbing)
and run on the tensors' device, ordered on the current torch stream.
"""
from __future__ import annotations

import ctypes
import os
from typing import Mapping, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import BPGeom, FilterParams, check, lib


# ---- argument packing -----------------------------------------------------------------------
def filter_params(ProjScale, DecWidth, DecHeigh, ScanR, StdDis, HelicP, FilterCoeFF, DeltaAngle,
                  FilteringMode, YL, ZL, ProjNumber) -> FilterParams:
    """Pack inputs 2..13 of KatsevichFiltering_GPU (ints truncated like the reference)."""
    p = FilterParams()
    p.proj_scale = float(int(ProjScale))
    p.dec_width = float(DecWidth)
    p.dec_height = float(DecHeigh)
    p.scan_r = float(ScanR)
    p.std_dis = float(StdDis)
    p.helic_p = float(HelicP)
    p.filter_coeff = float(FilterCoeFF)
    p.delta_angle = float(DeltaAngle)
    p.filtering_mode = int(FilteringMode)
    p.yl = int(YL)
    p.zl = int(ZL)
    p.proj_number = int(ProjNumber)
    return p


def bp_geom(geom) -> BPGeom:
    """Pack a geom struct (mapping with Locus, Detector, Object in that order, as built at
    FunctionKat_v6.m:110-112) or a (locus, detector, object) triple."""
    if isinstance(geom, BPGeom):
        return geom
    if isinstance(geom, Mapping):
        vals = list(geom.values())
    else:
        vals = list(geom)
    locus, det, obj = (np.asarray(v, dtype=np.float64).ravel() for v in vals[:3])
    if locus.size < 7 or det.size < 4 or obj.size < 4:
        raise ValueError("geom needs Locus[7], Detector[>=4], Object[>=4]")
    g = BPGeom()
    for i in range(7):
        g.locus[i] = locus[i]
    for i in range(min(6, det.size)):
        g.detector[i] = det[i]
    for i in range(min(7, obj.size)):
        g.object[i] = obj[i]
    g.n_detector = min(6, det.size)
    g.n_object = min(7, obj.size)
    return g


def scan_filter_params(scan) -> FilterParams:
    return filter_params(*scan.filter_args())


def num_kappa(zl: int) -> int:
    return lib().ctrecon_num_kappa(int(zl))


def geometry_sizing(ScanR, StdDis, HelicP, ObjR, YL, ZL):
    w, h, d = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    lib().ctrecon_geometry_sizing(ScanR, StdDis, HelicP, ObjR, int(YL), int(ZL),
                                  ctypes.byref(w), ctypes.byref(h), ctypes.byref(d))
    return w.value, h.value, d.value


def filter_tables(p: FilterParams) -> dict:
    """The filter's FP64 host tables (see ctrecon_filter_tables); no GPU needed."""
    AL, YL, ZL = num_kappa(p.zl), p.yl, p.zl
    ip = ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    t = dict(r0=np.zeros((AL, YL), np.int32), r1=np.zeros((AL, YL), np.int32),
             wa=np.zeros((AL, YL)), wb=np.zeros((AL, YL)), b=np.zeros((ZL, YL), np.int32),
             e=np.zeros((ZL, YL), np.int32), gb=np.zeros((ZL, YL)), ge=np.zeros((ZL, YL)))
    st = lib().ctrecon_filter_tables(
        ctypes.byref(p), t["r0"].ctypes.data_as(ip), t["r1"].ctypes.data_as(ip),
        t["wa"].ctypes.data_as(dp), t["wb"].ctypes.data_as(dp), t["b"].ctypes.data_as(ip),
        t["e"].ctypes.data_as(ip), t["gb"].ctypes.data_as(dp), t["ge"].ctypes.data_as(dp))
    check(st, None)
    return t


def _f64(a: np.ndarray, name: str, n: int) -> np.ndarray:
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError(f"{name} must be a C-contiguous float64 numpy array")
    if a.size < n:
        raise ValueError(f"{name} has {a.size} elements, needs {n}")
    return a


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _stream_handle(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _tptr(t, dtype_name: str, name: str) -> int:
    if t is None:
        return None
    if not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if dtype_name and str(t.dtype) != f"torch.{dtype_name}":
        raise TypeError(f"{name} must be torch.{dtype_name}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t.data_ptr()


# ---- context ---------------------------------------------------------------------------------
class Context:
    """One ctrecon context on one device (not thread-safe; one per host thread)."""

    def __init__(self, device: int = 0, hilbert: int = _lib.HILBERT_FP32,
                 pi_solver: int = _lib.PI_BISECT):
        h = ctypes.c_void_p()
        check(lib().ctrecon_ctx_create(int(device), ctypes.byref(h)), None)
        self._h = h
        self.device = device
        self.set_option(_lib.OPT_HILBERT, hilbert)
        self.set_option(_lib.OPT_PI_SOLVER, pi_solver)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().ctrecon_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_option(self, opt: int, value: int):
        check(lib().ctrecon_set_option(self._h, int(opt), int(value)), self._h)

    def get_option(self, opt: int) -> int:
        v = ctypes.c_int()
        check(lib().ctrecon_get_option(self._h, int(opt), ctypes.byref(v)), self._h)
        return v.value

    def kernel_times(self) -> dict:
        """{kind: (ms, launches)} of the launches timed since the last call (with
        OPT_KERNEL_TIMING on); waits for them."""
        from . import _lib
        n = len(_lib.KERNEL_KINDS)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_ulonglong * n)()
        check(lib().ctrecon_kernel_times(self._h, ms, cnt, n), self._h)
        return {k: (ms[i], int(cnt[i])) for i, k in enumerate(_lib.KERNEL_KINDS)}

    # -- host FP64 (MEX-equivalent) --------------------------------------------------------
    def filter_host(self, p: FilterParams, proj: np.ndarray, fproj: Optional[np.ndarray] = None):
        n = p.yl * p.zl * p.proj_number
        _f64(proj, "Proj", n)
        if fproj is None:
            fproj = np.empty_like(proj)
        _f64(fproj, "FProj", n)
        check(lib().ctrecon_filter_host_f64(self._h, ctypes.byref(p), _dptr(proj), _dptr(fproj)),
              self._h)
        return fproj

    def bkproj_host(self, geom, fproj: np.ndarray, image: np.ndarray) -> np.ndarray:
        g = bp_geom(geom)
        check(lib().ctrecon_bkproj_host_f64(self._h, ctypes.byref(g), _dptr(fproj), _dptr(image)),
              self._h)
        return image

    def recon_host(self, p: FilterParams, geom, proj: np.ndarray, image: np.ndarray):
        g = bp_geom(geom)
        check(lib().ctrecon_recon_host_f64(self._h, ctypes.byref(p), ctypes.byref(g), _dptr(proj),
                                           _dptr(image)), self._h)
        return image

    # -- device FP32 (torch tensors) -----------------------------------------------------------
    def filter_dev(self, p: FilterParams, d_proj, d_fproj, stream=None):
        check(lib().ctrecon_filter_dev_f32(self._h, _stream_handle(stream), ctypes.byref(p),
                                           _tptr(d_proj, "float32", "d_proj"),
                                           _tptr(d_fproj, "float32", "d_fproj")), self._h)

    def filter_mode1_dev(self, p: FilterParams, d_proj, d_fproj, stream=None):
        """FilteringMode 1 (FunctionKat_v6.m:86-90): mean of the filters with FilterCoeFF and
        1 - FilterCoeFF."""
        check(lib().ctrecon_filter_mode1_dev_f32(self._h, _stream_handle(stream), ctypes.byref(p),
                                                 _tptr(d_proj, "float32", "d_proj"),
                                                 _tptr(d_fproj, "float32", "d_fproj")), self._h)

    @staticmethod
    def pi_table_bytes(geom) -> int:
        g = bp_geom(geom)
        n = ctypes.c_size_t()
        check(lib().ctrecon_pi_table_bytes(ctypes.byref(g), ctypes.byref(n)), None)
        return n.value

    def pi_dev(self, geom, d_pitab, d_updates=None, stream=None):
        g = bp_geom(geom)
        check(lib().ctrecon_pi_dev(self._h, _stream_handle(stream), ctypes.byref(g),
                                   _tptr(d_pitab, "", "d_pitab"),
                                   _tptr(d_updates, "int64", "d_updates")), self._h)

    def bkproj_dev(self, geom, d_fproj, d_image, d_pitab=None, stream=None):
        g = bp_geom(geom)
        check(lib().ctrecon_bkproj_dev_f32(self._h, _stream_handle(stream), ctypes.byref(g),
                                           _tptr(d_fproj, "float32", "d_fproj"),
                                           _tptr(d_pitab, "", "d_pitab"),
                                           _tptr(d_image, "float32", "d_image")), self._h)

    # -- arc detector to flat panel (rebinToPanel.m) ------------------------------------------
    def rebin_to_panel_dev(self, d_proj, det_center_idx: float, det_cell_width: float,
                           sour_to_det: float, d_out, stream=None) -> float:
        """d_proj, d_out: device tensors (prj_num, det_hei, det_num), float32 or float64 (the
        latter reproduces the reference's arithmetic exactly). Returns the panel width."""
        P, H, N = d_proj.shape
        dt = str(d_proj.dtype).replace("torch.", "")
        fn = {"float32": lib().ctrecon_rebin_to_panel_dev_f32,
              "float64": lib().ctrecon_rebin_to_panel_dev_f64}[dt]
        width = ctypes.c_double()
        check(fn(self._h, _stream_handle(stream), _tptr(d_proj, dt, "d_proj"), N, H, P,
                 float(det_center_idx), float(det_cell_width), float(sour_to_det),
                 _tptr(d_out, dt, "d_out"), ctypes.byref(width)), self._h)
        return width.value

    # -- autotuner -----------------------------------------------------------------------------
    def tune_bkproj(self, geom, d_fproj, d_image, d_pitab=None, stream=None) -> dict:
        """Times the backprojector forms on this data, records the fastest for the geometry
        (used under OPT_BP_VARIANT = BP_AUTO) and returns {variant: ms} plus the best."""
        g = bp_geom(geom)
        r = _lib.TuneResult()
        check(lib().ctrecon_tune_bkproj(self._h, _stream_handle(stream), ctypes.byref(g),
                                        _tptr(d_fproj, "float32", "d_fproj"),
                                        _tptr(d_pitab, "", "d_pitab"),
                                        _tptr(d_image, "float32", "d_image"), ctypes.byref(r)),
              self._h)
        return _tune_dict(r)

    def tune_save(self, path: str):
        check(lib().ctrecon_tune_save(self._h, os.fsencode(path)), self._h)

    def tune_load(self, path: str):
        check(lib().ctrecon_tune_load(self._h, os.fsencode(path)), self._h)

    def phantom_dev(self, geom, ell: np.ndarray, d_proj, photons: float = 0.0, seed: int = 0,
                    stream=None):
        g = bp_geom(geom)
        ell = np.ascontiguousarray(ell, dtype=np.float64).reshape(-1, 10)
        check(lib().ctrecon_phantom_project_dev(
            self._h, _stream_handle(stream), ctypes.byref(g), _dptr(ell), ell.shape[0],
            float(photons), int(seed) & ((1 << 64) - 1), _tptr(d_proj, "float32", "d_proj")),
            self._h)


class Batch:
    """Many scans reconstructed together (ctrecon_batch_*): per-scan filters and PI solves, one
    persistent backprojection launch over all scans, optionally replayed as a CUDA graph."""

    def __init__(self, ctx: Context, scans):
        self.ctx = ctx
        self.n = len(scans)
        fps = (FilterParams * self.n)(*[scan_filter_params(s) for s in scans])
        gs = (BPGeom * self.n)(*[bp_geom(s.geom_struct()) for s in scans])
        h = ctypes.c_void_p()
        check(lib().ctrecon_batch_create(ctx.handle, self.n, fps, gs, ctypes.byref(h)), ctx.handle)
        self._h = h

    def close(self):
        if self._h:
            lib().ctrecon_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_variant(self, variant: int):
        check(lib().ctrecon_batch_set_variant(self._h, int(variant)), self.ctx.handle)

    def run(self, d_projs, d_fprojs, d_images, stream=None, use_graph=True):
        arr = lambda ts, name, dt: (ctypes.c_void_p * self.n)(*[_tptr(t, dt, name) for t in ts])
        check(lib().ctrecon_batch_run_dev(self._h, _stream_handle(stream),
                                          arr(d_projs, "d_proj", "float32"),
                                          arr(d_fprojs, "d_fproj", "float32"),
                                          arr(d_images, "d_image", "float32"),
                                          1 if use_graph else 0), self.ctx.handle)

    def updates(self):
        out = (ctypes.c_ulonglong * self.n)()
        check(lib().ctrecon_batch_updates(self._h, out), self.ctx.handle)
        return [int(v) for v in out]

    def tune(self, d_projs, d_fprojs, d_images, stream=None) -> dict:
        """One run of the batch, then the persistent backprojection timed for every candidate
        form; the fastest becomes the batch's form."""
        arr = lambda ts, name, dt: (ctypes.c_void_p * self.n)(*[_tptr(t, dt, name) for t in ts])
        r = _lib.TuneResult()
        check(lib().ctrecon_batch_tune(self._h, _stream_handle(stream),
                                       arr(d_projs, "d_proj", "float32"),
                                       arr(d_fprojs, "d_fproj", "float32"),
                                       arr(d_images, "d_image", "float32"), ctypes.byref(r)),
              self.ctx.handle)
        d = _tune_dict(r)
        d["per_scan"] = self.variants()
        return d

    def set_variants(self, variants):
        """One backprojector form per scan (scans sharing a form share a launch)."""
        arr = (ctypes.c_int * self.n)(*[int(v) for v in variants])
        check(lib().ctrecon_batch_set_variants(self._h, arr, self.n), self.ctx.handle)

    def variants(self):
        """The backprojector form of each scan."""
        out = (ctypes.c_int * self.n)()
        check(lib().ctrecon_batch_get_variants(self._h, out, self.n), self.ctx.handle)
        return [int(v) for v in out]


def _tune_dict(r) -> dict:
    return {"best_variant": r.best_variant, "best_ms": r.best_ms,
            "ms": {int(r.variants[i]): float(r.ms[i]) for i in range(r.n)}}


_default: Optional[Context] = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(0)
    return _default


# ---- the reference's MEX functions -------------------------------------------------------------
def KatsevichFiltering_GPU(Proj, ProjScale, DecWidth, DecHeigh, ScanR, StdDis, HelicP,
                           FilterCoeFF, DeltaAngle, FilteringMode, YL, ZL, ProjNumber, FProj):
    """KatsevichFiltering_GPU.cu:939-978: filter Proj, result written in place into FProj."""
    p = filter_params(ProjScale, DecWidth, DecHeigh, ScanR, StdDis, HelicP, FilterCoeFF,
                      DeltaAngle, FilteringMode, YL, ZL, ProjNumber)
    default_context().filter_host(p, Proj, FProj)


def KatsevichBkProj(geom, FProj, RecMatrix):
    """KatsevichBkProj.cpp:314-352: backproject FProj into RecMatrix in place."""
    _f64(FProj, "FProj", 1)
    _f64(RecMatrix, "RecMatrix", 1)
    default_context().bkproj_host(geom, FProj, RecMatrix)


KatsevichBkProj_GPU = KatsevichBkProj
