"""ctypes bindings of ``libctrecon.so`` (the C ABI declared in ``include/ctrecon.h``).

The library is built in-tree (``ctrecon_b200/lib/``) by ``ctrecon_b200/csrc/Makefile``;
there is no fallback: if it is missing, loading raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libctrecon.so")
MEX_DIR = os.path.join(LIB_DIR, "mex")

# status codes (ctrecon_status)
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_GEOMETRY = 2
ERR_CUDA = 3
ERR_OUT_OF_MEMORY = 4
ERR_NO_DEVICE = 5
ERR_TIMEOUT = 6
ERR_UNSUPPORTED = 7
ERR_INTERNAL = 8

HILBERT_FP32, HILBERT_BF16X3, HILBERT_TF32 = 0, 1, 2
PI_BISECT, PI_NEWTON, PI_LEARNED = 0, 1, 2
OPT_HILBERT, OPT_PI_SOLVER, OPT_FILTER_CHUNK, OPT_BP_VARIANT, OPT_VERBOSE = 1, 2, 3, 4, 5
OPT_DERIVATIVE = 6
OPT_BP_WINDOW = 7
OPT_PINET_MODE = 8
OPT_KERNEL_TIMING = 9
OPT_TC_FORM = 10
TC_PARITY_SPLIT, TC_SINGLE_PASS = 0, 1
OPT_K1_FORM = 11
OPT_HOST_THREADS = 12
K1_STAGED, K1_PER_VIEW = 0, 1
KERNEL_KINDS = ("deriv_rebin", "hilbert_simt", "hilbert_tc", "pi_solve", "cell_records",
                "backproject")
PINET_VOXEL_FP32, PINET_VOXEL_BF16, PINET_GRID = 0, 1, 2
DERIV_DIRECT, DERIV_CHAIN = 0, 1


class FilterParams(ctypes.Structure):
    _fields_ = [("proj_scale", ctypes.c_double), ("dec_width", ctypes.c_double),
                ("dec_height", ctypes.c_double), ("scan_r", ctypes.c_double),
                ("std_dis", ctypes.c_double), ("helic_p", ctypes.c_double),
                ("filter_coeff", ctypes.c_double), ("delta_angle", ctypes.c_double),
                ("filtering_mode", ctypes.c_int), ("yl", ctypes.c_int), ("zl", ctypes.c_int),
                ("proj_number", ctypes.c_int)]


class ProjFileHeader(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "source_to_center", "source_to_detector", "det_reso_u", "det_reso_v", "det_pixel_u",
        "det_pixel_v", "det_center_u", "det_center_v", "is_arc", "start_angle_deg", "start_z",
        "pitch", "total_views", "views_per_turn")] + [("storage_order", ctypes.c_double * 3)]


class ImgFileHeader(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double * 3) for n in ("reso", "pixel", "ctr_idx", "center",
                                                    "storage_order")]


BP_AUTO = -1
TUNE_MAX = 16


class TuneResult(ctypes.Structure):
    _fields_ = [("best_variant", ctypes.c_int), ("best_ms", ctypes.c_float), ("n", ctypes.c_int),
                ("variants", ctypes.c_int * TUNE_MAX), ("ms", ctypes.c_float * TUNE_MAX)]


class BPGeom(ctypes.Structure):
    _fields_ = [("locus", ctypes.c_double * 7), ("detector", ctypes.c_double * 6),
                ("object", ctypes.c_double * 7), ("n_detector", ctypes.c_int),
                ("n_object", ctypes.c_int)]


_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_st = ctypes.c_int

# (name, restype, argtypes) of every exported entry point of include/ctrecon.h
SIGNATURES = [
    ("ctrecon_ctx_create", _st, [ctypes.c_int, ctypes.POINTER(_vp)]),
    ("ctrecon_ctx_destroy", None, [_vp]),
    ("ctrecon_last_error", ctypes.c_char_p, [_vp]),
    ("ctrecon_status_string", ctypes.c_char_p, [_st]),
    ("ctrecon_abi_version", ctypes.c_int, []),
    ("ctrecon_set_option", _st, [_vp, ctypes.c_int, ctypes.c_int]),
    ("ctrecon_get_option", _st, [_vp, ctypes.c_int, _ip]),
    ("ctrecon_filter_host_f64", _st, [_vp, ctypes.POINTER(FilterParams), _dp, _dp]),
    ("ctrecon_bkproj_host_f64", _st, [_vp, ctypes.POINTER(BPGeom), _dp, _dp]),
    ("ctrecon_recon_host_f64", _st, [_vp, ctypes.POINTER(FilterParams), ctypes.POINTER(BPGeom),
                                     _dp, _dp]),
    ("ctrecon_filter_dev_f32", _st, [_vp, _vp, ctypes.POINTER(FilterParams), _vp, _vp]),
    ("ctrecon_pi_table_bytes", _st, [ctypes.POINTER(BPGeom), ctypes.POINTER(ctypes.c_size_t)]),
    ("ctrecon_pi_dev", _st, [_vp, _vp, ctypes.POINTER(BPGeom), _vp, _vp]),
    ("ctrecon_bkproj_dev_f32", _st, [_vp, _vp, ctypes.POINTER(BPGeom), _vp, _vp, _vp]),
    ("ctrecon_filter_mode1_dev_f32", _st, [_vp, _vp, ctypes.POINTER(FilterParams), _vp, _vp]),
    ("ctrecon_filter_noalloc_dev_f32", _st, [_vp, ctypes.POINTER(FilterParams), _vp, _vp]),
    ("ctrecon_selftest_bounded_wait", _st, [_vp, _vp, ctypes.c_int]),
    ("ctrecon_sync", _st, [_vp, _vp]),
    ("ctrecon_pi_dev_stats", _st, [_vp, _vp, ctypes.POINTER(BPGeom), _vp, _vp, _vp]),
    ("ctrecon_kernel_times", _st, [_vp, _dp, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int]),
    ("ctrecon_batch_create", _st, [_vp, ctypes.c_int, ctypes.POINTER(FilterParams),
                                   ctypes.POINTER(BPGeom), ctypes.POINTER(_vp)]),
    ("ctrecon_batch_destroy", None, [_vp]),
    ("ctrecon_batch_set_variant", _st, [_vp, ctypes.c_int]),
    ("ctrecon_batch_get_variants", _st, [_vp, _ip, ctypes.c_int]),
    ("ctrecon_batch_set_variants", _st, [_vp, _ip, ctypes.c_int]),
    ("ctrecon_batch_run_dev", _st, [_vp, _vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                    ctypes.POINTER(_vp), ctypes.c_int]),
    ("ctrecon_batch_updates", _st, [_vp, ctypes.POINTER(ctypes.c_ulonglong)]),
    ("ctrecon_tune_bkproj", _st, [_vp, _vp, ctypes.POINTER(BPGeom), _vp, _vp, _vp,
                                  ctypes.POINTER(TuneResult)]),
    ("ctrecon_batch_tune", _st, [_vp, _vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                 ctypes.POINTER(_vp), ctypes.POINTER(TuneResult)]),
    ("ctrecon_tune_save", _st, [_vp, ctypes.c_char_p]),
    ("ctrecon_tune_load", _st, [_vp, ctypes.c_char_p]),
    ("ctrecon_pinet_num_params", ctypes.c_int, []),
    ("ctrecon_pinet_train", _st, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_uint64,
                                  ctypes.POINTER(ctypes.c_float)]),
    ("ctrecon_pinet_get_params", _st, [_vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
    ("ctrecon_pinet_set_params", _st, [_vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int,
                                       ctypes.c_double]),
    ("ctrecon_pinet_loss_grad", _st, [_vp, _vp, _vp, _vp, ctypes.c_int, _vp, _vp]),
    ("ctrecon_pinet_predict", _st, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    ("ctrecon_num_kappa", ctypes.c_int, [ctypes.c_int]),
    ("ctrecon_find_tau", _st, [ctypes.c_double, ctypes.c_double, _dp]),
    ("ctrecon_filter_tables", _st, [ctypes.POINTER(FilterParams), _ip, _ip, _dp, _dp, _ip, _ip,
                                    _dp, _dp]),
    ("ctrecon_geometry_sizing", None, [ctypes.c_double] * 4 + [ctypes.c_int] * 2 + [_dp] * 3),
    ("ctrecon_phantom_project_dev", _st, [_vp, _vp, ctypes.POINTER(BPGeom), _dp, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_uint64, _vp]),
    ("ctrecon_rebin_to_panel_dev_f32", _st, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, _vp, _dp]),
    ("ctrecon_rebin_to_panel_dev_f64", _st, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, _vp, _dp]),
    ("ctrecon_projfile_read", _st, [ctypes.c_char_p, ctypes.POINTER(ProjFileHeader), _dp,
                                    ctypes.c_size_t]),
    ("ctrecon_projfile_write", _st, [ctypes.c_char_p, ctypes.POINTER(ProjFileHeader), _dp]),
    ("ctrecon_imgfile_read", _st, [ctypes.c_char_p, ctypes.POINTER(ImgFileHeader), _dp,
                                   ctypes.c_size_t]),
    ("ctrecon_imgfile_write", _st, [ctypes.c_char_p, ctypes.POINTER(ImgFileHeader), _dp]),
]

_lib = None


def lib():
    """Load libctrecon.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with "
                              f"`make -C ctrecon_b200/csrc` or __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class CtreconError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status
        self.message = message


def check(status: int, ctx=None) -> None:
    if status != OK:
        msg = lib().ctrecon_last_error(ctx)
        raise CtreconError(status, (msg or b"").decode(errors="replace") or
                           lib().ctrecon_status_string(status).decode())
