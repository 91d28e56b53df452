"""ctrecon_b200 -- CTRecon's Katsevich helical cone-beam reconstruction on one NVIDIA B200.

The compute path is hand-written sm_100a CUDA behind the C ABI of ``include/ctrecon.h``
(``ctrecon_b200/lib/libctrecon.so``); this package binds it with ctypes and mirrors the
reference's MEX entry points. Importing the package does not load the library; the first
call that needs it does, and raises if it was not built.
"""
from ._lib import (HILBERT_BF16X3, HILBERT_FP32, HILBERT_TF32, PI_BISECT, PI_LEARNED, PI_NEWTON,
                   CtreconError)
from .api import (Batch, Context, KatsevichBkProj, KatsevichBkProj_GPU, KatsevichFiltering_GPU, bp_geom,
                  default_context, filter_params, filter_tables, geometry_sizing, num_kappa,
                  scan_filter_params)

__all__ = [
    "Context", "CtreconError", "KatsevichBkProj", "KatsevichBkProj_GPU", "KatsevichFiltering_GPU",
    "bp_geom", "default_context", "filter_params", "filter_tables", "geometry_sizing",
    "num_kappa", "scan_filter_params", "HILBERT_FP32", "HILBERT_BF16X3", "HILBERT_TF32",
    "PI_BISECT", "PI_NEWTON", "PI_LEARNED",
]
