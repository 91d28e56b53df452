"""Standalone MEX harness: call a MEX module's ``mexFunction`` without MATLAB.

A MEX module here is a shared library built against the project's ``mex.h`` shim
(``ctrecon_b200/mex``); each module carries its own copy of the shim, so arrays are
created, wrapped and passed through the module's own ``mx*`` functions and errors raised
with ``mexErrMsgTxt`` come back as :class:`MexError` (MATLAB would raise a MATLAB error).

Arrays follow MATLAB's column-major layout: a numpy array in C order with shape
``(P, ZL, YL)`` is the MATLAB array ``YL x ZL x P`` -- the layout of ``Proj`` and
``FProj`` in ``KatsevichFiltering.m:33`` -- and is passed without copying, so MEX
functions that write into an input (``KatsevichFiltering_GPU.cu:976``,
``KatsevichBkProj.cpp:265``) update the numpy buffer in place, as in MATLAB.
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Mapping, Sequence

import numpy as np

MX_DOUBLE_CLASS = 6
MX_SINGLE_CLASS = 7


class MexError(RuntimeError):
    """A MEX function raised mexErrMsgTxt."""


class MexModule:
    """One MEX shared library (exports ``mexFunction`` and the shim's ``mx*`` API)."""

    def __init__(self, path: str):
        self.path = path
        self.lib = ctypes.CDLL(path)
        L = self.lib
        vp, sz = ctypes.c_void_p, ctypes.c_size_t
        L.mexshim_wrap_numeric.restype = vp
        L.mexshim_wrap_numeric.argtypes = [sz, ctypes.POINTER(sz), ctypes.c_int, vp]
        L.mxCreateStructMatrix.restype = vp
        L.mxCreateStructMatrix.argtypes = [sz, sz, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
        L.mxSetFieldByNumber.restype = None
        L.mxSetFieldByNumber.argtypes = [vp, sz, ctypes.c_int, vp]
        L.mxDestroyArray.restype = None
        L.mxDestroyArray.argtypes = [vp]
        L.mexshim_call.restype = ctypes.c_int
        L.mexshim_call.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.c_int,
                                   ctypes.POINTER(vp), ctypes.c_char_p, sz]
        L.mexshim_set_print.restype = None
        L.mexshim_set_print.argtypes = [ctypes.c_int]
        L.mxGetPr.restype = vp
        L.mxGetPr.argtypes = [vp]
        L.mxGetClassID.restype = ctypes.c_int
        L.mxGetClassID.argtypes = [vp]
        L.mxGetNumberOfDimensions.restype = sz
        L.mxGetNumberOfDimensions.argtypes = [vp]
        L.mxGetDimensions.restype = ctypes.POINTER(sz)
        L.mxGetDimensions.argtypes = [vp]
        self._entry = ctypes.cast(L.mexFunction, vp)

    def set_print(self, enabled: bool) -> None:
        self.lib.mexshim_set_print(1 if enabled else 0)

    # -- argument construction -------------------------------------------------------
    def _wrap(self, arr: np.ndarray, keep: list, dims: Sequence[int] | None = None):
        if arr.dtype == np.float64:
            cls = MX_DOUBLE_CLASS
        elif arr.dtype == np.float32:
            cls = MX_SINGLE_CLASS
        else:
            raise TypeError(f"unsupported dtype {arr.dtype}")
        if not arr.flags.c_contiguous:
            raise ValueError("arrays must be C-contiguous (MATLAB column-major reversed)")
        if dims is None:
            dims = tuple(reversed(arr.shape)) if arr.ndim else (1, 1)
        dims = list(dims) + [1] * max(0, 2 - len(dims))
        d = (ctypes.c_size_t * len(dims))(*dims)
        keep.append(arr)
        h = self.lib.mexshim_wrap_numeric(len(dims), d, cls, arr.ctypes.data)
        return h

    def _arg(self, value, keep: list):
        if isinstance(value, Mapping):
            names = list(value.keys())
            cnames = (ctypes.c_char_p * len(names))(*[n.encode() for n in names])
            s = self.lib.mxCreateStructMatrix(1, 1, len(names), cnames)
            for i, n in enumerate(names):
                v = np.ascontiguousarray(np.atleast_1d(np.asarray(value[n], dtype=np.float64)))
                # MATLAB row vector 1 x n, as written by struct('Locus', [...])
                h = self._wrap(v, keep, dims=(1, v.size))
                self.lib.mxSetFieldByNumber(s, 0, i, h)
            return s, True
        if isinstance(value, np.ndarray):
            return self._wrap(value, keep), False
        if isinstance(value, (int, float, np.floating, np.integer)):
            v = np.array([float(value)], dtype=np.float64)
            return self._wrap(v, keep, dims=(1, 1)), False
        raise TypeError(f"unsupported MEX argument type {type(value)}")

    def _take(self, h) -> np.ndarray:
        """Copy a left-hand side the MEX function created into numpy (C order, the MATLAB
        dimensions reversed) and free it."""
        try:
            nd = int(self.lib.mxGetNumberOfDimensions(h))
            dims = self.lib.mxGetDimensions(h)
            shape = tuple(int(dims[i]) for i in range(nd))[::-1]
            cls = int(self.lib.mxGetClassID(h))
            if cls not in (MX_DOUBLE_CLASS, MX_SINGLE_CLASS):
                raise MexError(f"unsupported output class {cls}")
            ct = ctypes.c_double if cls == MX_DOUBLE_CLASS else ctypes.c_float
            n = int(np.prod(shape)) if shape else 1
            ptr = self.lib.mxGetPr(h)
            buf = (ct * n).from_address(ptr) if n else (ct * 0)()
            return np.ctypeslib.as_array(buf).reshape(shape).copy()
        finally:
            self.lib.mxDestroyArray(h)

    def call(self, args: Iterable, nlhs: int = 0) -> list:
        """Invoke mexFunction(nlhs, plhs, nrhs, prhs) with the given right-hand sides; returns
        the nlhs outputs it created, as numpy arrays."""
        keep: list = []
        handles, owned = [], []
        try:
            for a in args:
                h, is_struct = self._arg(a, keep)
                handles.append(h)
                owned.append(h)
            n = len(handles)
            prhs = (ctypes.c_void_p * max(n, 1))(*handles)
            plhs = (ctypes.c_void_p * max(nlhs, 1))()
            err = ctypes.create_string_buffer(1024)
            rc = self.lib.mexshim_call(self._entry, nlhs, plhs, n, prhs, err, len(err))
            if rc != 0:
                raise MexError(err.value.decode(errors="replace"))
            return [self._take(plhs[i]) for i in range(nlhs) if plhs[i]]
        finally:
            for h in owned:
                self.lib.mxDestroyArray(h)
