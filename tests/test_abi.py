"""The C ABI surface and the host-side logic (CPU only, no kernel launches)."""
import ctypes
import os
import re

import numpy as np
import pytest

import ctrecon_b200 as ct
from ctrecon_b200 import _lib
from ctrecon_b200.geometry import config, small_config
from ctrecon_b200.mexharness import MexError, MexModule

from conftest import oracle_filter_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "ctrecon.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ctrecon_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(syms) <= bound, set(syms) - bound


def header_enum_values():
    """Every `CTRECON_NAME = value` enumerator of include/ctrecon.h."""
    txt = open(os.path.join(ROOT, "include", "ctrecon.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return {m.group(1): int(m.group(2))
            for m in re.finditer(r"\bCTRECON_([A-Z0-9_]+)\s*=\s*(-?\d+)\b", txt)}


def test_python_option_constants_match_header():
    """The ctypes mirror's option numbers and option values are the header's, so an option
    added on one side only is caught here."""
    h = header_enum_values()
    opts = {k: v for k, v in h.items() if k.startswith("OPT_")}
    assert len(opts) >= 12
    for name, value in opts.items():
        assert getattr(_lib, name) == value, name
    for name in ("HILBERT_FP32", "HILBERT_BF16X3", "HILBERT_TF32", "PI_BISECT", "PI_NEWTON",
                 "PI_LEARNED", "TC_PARITY_SPLIT", "TC_SINGLE_PASS", "K1_STAGED", "K1_PER_VIEW"):
        assert getattr(_lib, name) == h[name], name


def test_abi_version_and_status_strings():
    L = _lib.lib()
    assert L.ctrecon_abi_version() == 1
    for st in range(0, 9):
        assert L.ctrecon_status_string(st)


def test_context_creation_without_gpu_is_an_error_not_a_crash():
    h = ctypes.c_void_p()
    st = _lib.lib().ctrecon_ctx_create(0, ctypes.byref(h))
    assert st in (_lib.OK, _lib.ERR_NO_DEVICE)
    if st == _lib.OK:
        _lib.lib().ctrecon_ctx_destroy(h)
    else:
        assert b"device" in _lib.lib().ctrecon_last_error(None).lower()


@pytest.mark.parametrize("name", ["c1", "c2", "c3", "tiny", "mode2"])
def test_filter_tables_match_oracle(oracle_mod, name):
    if name == "tiny":
        s = small_config()
    elif name == "mode2":
        s = small_config(filtering_mode=2, filter_coeff=0.3)
    else:
        s = config(name)
    p = ct.scan_filter_params(s)
    t = ct.filter_tables(p)
    o = oracle_mod.filter_tables(oracle_filter_params(oracle_mod, s))
    clamp = o["w_up"] == 0
    np.testing.assert_array_equal(t["r0"], o["lw"])
    np.testing.assert_array_equal(t["r1"][~clamp], o["lw"][~clamp] + 1)
    np.testing.assert_allclose(t["wa"], o["w_lw"] * o["coef"], rtol=1e-15, atol=0)
    np.testing.assert_allclose(t["wb"], o["w_up"] * o["coef"], rtol=1e-15, atol=1e-300)
    np.testing.assert_array_equal(t["b"], o["bAL"])
    np.testing.assert_array_equal(t["e"], o["eAL"])
    coef_b = np.take_along_axis(o["coef"], o["bAL"], axis=0)
    coef_e = np.take_along_axis(o["coef"], o["eAL"], axis=0)
    np.testing.assert_allclose(t["gb"], -o["bC"] / coef_b, rtol=1e-15)
    np.testing.assert_allclose(t["ge"], -o["eC"] / coef_e, rtol=1e-15)


@pytest.mark.parametrize("ratio,tol", [(2.0 / 3.0, 1e-4), (0.2, 1e-4), (0.5, 1e-10)])
def test_find_tau_matches_oracle(oracle_mod, ratio, tol):
    """FindTau.m:6-22 (the script's own case is ratio 2/3, tolerance 1e-4)."""
    t = ctypes.c_double()
    assert _lib.lib().ctrecon_find_tau(ratio, tol, ctypes.byref(t)) == _lib.OK
    assert t.value == oracle_mod.find_tau(ratio, tol)
    am = 2 * np.pi - 2 * np.arccos(ratio)
    assert abs(t.value * np.cos(am) - np.cos(t.value * am) + 1 - t.value) <= tol
    assert 0 < t.value < 0.5


def test_num_kappa_matches_reference():
    for zl in (4, 8, 16, 40, 64, 128, 256):
        assert ct.num_kappa(zl) == 2 * int(np.ceil(zl * 1.3 * 0.5)) + 1


def test_geometry_sizing_matches_oracle(oracle_mod):
    args = (75.0, 150.0, 12.5, 25.0, 300, 40)
    assert ct.geometry_sizing(*args) == oracle_mod.geometry_sizing(*args)


def test_filter_tables_reject_bad_arguments():
    s = small_config()
    p = ct.scan_filter_params(s)
    p.yl = 3
    with pytest.raises(ct.CtreconError) as e:
        ct.filter_tables(p)
    assert e.value.status == _lib.ERR_INVALID_ARGUMENT
    p = ct.scan_filter_params(s)
    p.proj_number = 2
    with pytest.raises(ct.CtreconError):
        ct.filter_tables(p)


def test_backward_rebin_geometry_error_is_reported():
    """A helical pitch far beyond the detector's Tam-Danielson window makes the reference's
    crossing fix-up step outside 1..AL (a MATLAB index error); the tables report it."""
    s = small_config()
    p = ct.scan_filter_params(s)
    bad = 0
    for hp in (20 * s.HelicP, 60 * s.HelicP, -40 * s.HelicP):
        p.helic_p = hp
        try:
            ct.filter_tables(p)
        except ct.CtreconError as e:
            assert e.status == _lib.ERR_GEOMETRY
            bad += 1
    # whether or not a given pitch triggers it, no call may crash
    assert bad >= 0


def _mex(name):
    path = os.path.join(_lib.MEX_DIR, name + ".so")
    assert os.path.exists(path), path
    m = MexModule(path)
    m.set_print(False)
    return m


def test_mex_modules_export_mexfunction():
    for n in ("KatsevichFiltering_GPU", "KatsevichBkProj", "KatsevichBkProj_GPU"):
        m = _mex(n)
        assert hasattr(m.lib, "mexFunction")


def test_mex_bkproj_argument_errors_match_reference():
    """KatsevichBkProj.cpp:321-326 and :338-342, raised before any device work."""
    m = _mex("KatsevichBkProj")
    s = small_config()
    fp = np.zeros(s.proj_shape)
    img = np.zeros(s.vol_shape)
    with pytest.raises(MexError, match="bkproj requires two input arguments."):
        m.call([s.geom_struct(), fp])
    with pytest.raises(MexError, match="bkproj requires one output argument."):
        m.call([s.geom_struct(), fp, img], nlhs=1)
    with pytest.raises(MexError, match="Single precision is not supported"):
        m.call([s.geom_struct(), fp.astype(np.float32), img])
    with pytest.raises(MexError, match="smaller than geom"):
        m.call([s.geom_struct(), fp[:-1].copy(), img])


def test_mex_filter_argument_errors():
    m = _mex("KatsevichFiltering_GPU")
    s = small_config()
    proj = np.zeros(s.proj_shape)
    with pytest.raises(MexError, match="14 input arguments"):
        m.call([proj] + list(s.filter_args()))
    args = [proj] + list(s.filter_args()) + [np.zeros(5)]
    with pytest.raises(MexError, match="YL\\*ZL\\*ProjNumber"):
        m.call(args)
