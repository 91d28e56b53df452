"""DerMode 0 of the reference's driver: KatsevichFiltering_T.m, the Katsevich filter with the
direct half-view derivative (FunctionKat_v6.m:95-102).

CPU: the C oracle's derivative (oracle/katsevich_oracle.c::view_derivative_direct) against a
literal Python transcription of KatsevichFiltering_T.m:50-101. GPU (marked): the library's
filter with CTRECON_DERIV_DIRECT against the oracle's whole DerMode 0 filter.
"""
import math

import numpy as np
import pytest

from conftest import oracle_filter_params, oracle_geom, rel_rmse

PI = 3.14159265358979  # KatsevichFiltering_T.m:31


def _transcription(proj, fp, p):
    """KatsevichFiltering_T.m:33-101 statement by statement for output view p (0-based) on
    numpy (P, ZL, YL); MATLAB's Proj(Y, Z, view) is proj[view - 1, Z - 1, Y - 1]."""
    P, ZL, YL = proj.shape
    DeltaL = 2 * PI / fp.ProjScale
    DeltaU = fp.DecWidth / YL
    DeltaV = fp.DecHeigh / ZL
    HalfZ = (ZL + 1) / 2
    HalfY = (YL + 1) / 2
    y = (np.arange(1, YL + 1) - HalfY) * DeltaU
    z = (np.arange(1, ZL + 1) - HalfZ) * DeltaV
    DeltaL2 = DeltaL / 2
    StdDis = fp.StdDis

    def check(d, lo, hi):  # CheckData.m
        return lo if d < lo else (hi if d > hi else d)

    def resampled(view, Dzc, Uy):
        GF = np.zeros((ZL, YL))
        for Yindex in range(1, YL + 1):
            for Zindex in range(1, ZL + 1):
                ycor = Uy[Yindex - 1] / DeltaU + HalfY
                zcor = (Dzc[Yindex - 1] * z[Zindex - 1]) / DeltaV + HalfZ
                YD = math.floor(ycor)
                ZD = math.floor(zcor)
                YU = YD + 1
                ZU = ZD + 1
                alfa = ycor - YD
                beta = zcor - ZD
                YD, YU = check(YD, 1, YL), check(YU, 1, YL)
                ZD, ZU = check(ZD, 1, ZL), check(ZU, 1, ZL)
                Pr = lambda yy, zz: proj[view, zz - 1, yy - 1]
                GF[Zindex - 1, Yindex - 1] = (Pr(YD, ZD) * (1 - alfa) * (1 - beta) +
                                              Pr(YD, ZU) * (1 - alfa) * beta +
                                              Pr(YU, ZD) * alfa * (1 - beta) +
                                              Pr(YU, ZU) * alfa * beta)
        return GF

    Dzc1 = StdDis / (StdDis * math.cos(DeltaL2) - y * math.sin(DeltaL2))
    Uy1 = (y * math.cos(DeltaL2) + StdDis * math.sin(DeltaL2)) * Dzc1
    Dzc2 = StdDis / (StdDis * math.cos(DeltaL2) + y * math.sin(DeltaL2))
    Uy2 = (y * math.cos(DeltaL2) - StdDis * math.sin(DeltaL2)) * Dzc2
    q = P - 2 if p == P - 1 else p  # GF(:,:,ProjNumber) = GF(:,:,ProjNumber-1)
    return (resampled(q + 1, Dzc1, Uy1) - resampled(q, Dzc2, Uy2)) / DeltaL


@pytest.fixture(scope="module")
def tiny(oracle_mod):
    from ctrecon_b200.geometry import small_config
    s = small_config()
    O = oracle_mod
    proj = O.project_ellipsoids(oracle_geom(O, s), s.ellipsoids())
    return s, proj


@pytest.mark.parametrize("p", [0, 37, 539])
def test_oracle_direct_derivative_matches_transcription(oracle_mod, tiny, p):
    s, proj = tiny
    fp = oracle_filter_params(oracle_mod, s)
    got = oracle_mod.derivative_direct(fp, proj, p)
    want = _transcription(proj, fp, p)
    assert np.allclose(got, want, rtol=1e-13, atol=1e-9 * np.abs(want).max())


@pytest.mark.gpu
@pytest.mark.parametrize("mode,bound", [("fp32", 1e-5), ("bf16x3", 5e-5)])
def test_gpu_direct_filter_matches_oracle(oracle_mod, tiny, mode, bound):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    s, proj = tiny
    ref = oracle_mod.katsevich_filter_direct(oracle_filter_params(oracle_mod, s), proj)
    hil = ct.HILBERT_FP32 if mode == "fp32" else ct.HILBERT_BF16X3
    with ct.Context(0, hilbert=hil) as cx:
        cx.set_option(_lib.OPT_DERIVATIVE, _lib.DERIV_DIRECT)
        d = torch.from_numpy(proj.astype(np.float32)).cuda()
        out = torch.empty_like(d)
        cx.filter_dev(ct.scan_filter_params(s), d, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        host = cx.filter_host(ct.scan_filter_params(s), proj)
    err = rel_rmse(got, ref)
    print(f"DerMode 0 filter {mode}: rel RMSE {err:.2e}")
    assert err < bound
    assert rel_rmse(host, ref) < bound
