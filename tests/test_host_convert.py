"""The host threads' FP64 <-> FP32 conversions of the host calls (csrc/host_convert.h), CPU only.

The host calls convert their FP64 inputs to FP32 on the host, and widen the filter's FP32
results for pageable arrays back to FP64, with SSE2 loads and streaming stores around a scalar
head and tail. Their results must be the C casts' bit for bit (round to nearest even, exact
widening) for every start alignment and length, including subnormals, infinities, ties and
values past the FP32 range: the GPU tests check them only on phantom projections. The header is
compiled here into a small shared library with the product's own compiler flags.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "ctrecon_b200", "csrc")

SRC = r"""
#include "host_convert.h"
extern "C" void narrow(const double* s, float* d, size_t n) { ctr::convert_stream(s, d, n); }
extern "C" void widen(const float* s, double* d, size_t n) { ctr::widen_stream(s, d, n); }
"""


@pytest.fixture(scope="module")
def conv(tmp_path_factory):
    d = tmp_path_factory.mktemp("host_convert")
    src, lib = d / "hc.cpp", d / "libhc.so"
    src.write_text(SRC)
    subprocess.check_call(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-I" + HEADER_DIR,
                           str(src), "-o", str(lib)])
    L = ctypes.CDLL(str(lib))
    for f, a, b in ((L.narrow, ctypes.c_double, ctypes.c_float),
                    (L.widen, ctypes.c_float, ctypes.c_double)):
        f.argtypes = [ctypes.POINTER(a), ctypes.POINTER(b), ctypes.c_size_t]
        f.restype = None
    return L


def _values(rng, n):
    x = rng.standard_normal(n) * 10.0 ** rng.integers(-45, 39, n)
    special = np.array([0.0, -0.0, np.inf, -np.inf, 1e-40, -1e-45, 1.4e-45, 7e-46,
                        3.4028235677973366e38, 3.5e38, -1e300, 1e-300,
                        1.0 + 2.0 ** -24, 1.0 + 3 * 2.0 ** -24, 0.1, 1 / 3])
    x[: len(special)] = special[: n]
    return rng.permutation(x)


@pytest.mark.parametrize("offset", [0, 1, 2, 3])
def test_narrow_equals_cast(conv, offset):
    rng = np.random.default_rng(5 + offset)
    for n in list(range(0, 13)) + [37, 64, 1001]:
        src = np.zeros(n + 8)
        src[offset:offset + n] = _values(rng, n) if n else []
        out = np.full(n + 8, 7.0, dtype=np.float32)
        s = src[offset:]
        d = out[offset:]
        with np.errstate(over="ignore"):
            conv.narrow(s.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                        d.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n)
            want = s[:n].astype(np.float32)
        assert np.array_equal(d[:n].view(np.uint32), want.view(np.uint32)), (n, offset)
        assert np.all(out[:offset] == 7.0) and np.all(d[n:] == 7.0)  # nothing outside


@pytest.mark.parametrize("offset", [0, 1, 2, 3])
def test_widen_is_exact(conv, offset):
    rng = np.random.default_rng(11 + offset)
    for n in list(range(0, 13)) + [37, 64, 1001]:
        with np.errstate(over="ignore"):
            vals = _values(rng, n).astype(np.float32)
        src = np.zeros(n + 8, dtype=np.float32)
        src[offset:offset + n] = vals
        out = np.full(n + 8, 7.0)
        s = src[offset:]
        d = out[offset:]
        conv.widen(s.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                   d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n)
        assert np.array_equal(d[:n].view(np.uint64), s[:n].astype(np.float64).view(np.uint64))
        assert np.all(out[:offset] == 7.0) and np.all(d[n:] == 7.0)


def test_narrow_nan_stays_nan(conv):
    src = np.array([np.nan, -np.nan, 1.0, np.nan, 2.0, 3.0, np.nan])
    out = np.zeros(len(src), dtype=np.float32)
    conv.narrow(src.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(src))
    assert np.array_equal(np.isnan(out), np.isnan(src))
    assert np.array_equal(out[~np.isnan(out)], src[~np.isnan(src)].astype(np.float32))
