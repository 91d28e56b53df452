"""A second, independent restatement of the reference's CPU filter, KatsevichFiltering.m:39-287,
statement by statement in NumPy, checked against the C oracle's filter (oracle/katsevich_oracle.c).

The C oracle replaces the reference's FFT convolution by the exact direct Toeplitz sum, keeps the
host tables in its own records and folds the pre- and post-weights into them. This file does none
of that: it keeps MATLAB's arrays (Proj(YL, ZL, P) as `Proj[Y-1, Z-1, p-1]`), its one-based loops
(written as `for Yindex in range(1, YL + 1)` and indexed `[Yindex - 1]`), its order of operations,
the kernel of CreateHSP.m:11-23 laid out in a length-nn2 buffer as at :160-167, and
`real(ifft(fft(row, nn2) .* FFT_F))` for every kappa row (numpy's FFT in place of MATLAB's). The
forward-rebin clamp (:134-145) and the backward-rebin search and crossing fix-up (:192-287) are
the MATLAB control flow, including the values BeginAL / EndAL keep from the previous Zindex.
MATLAB and Octave are not installed, so this transliteration stands in for running the .m file.
CPU only.
"""
import math

import numpy as np
import pytest

from conftest import oracle_filter_params, oracle_geom

PI = 3.14159265358979  # KatsevichFiltering.m:32, CreateHSP.m:15


def nextpow2(n):
    """MATLAB nextpow2 for a positive integer: the smallest p with 2^p >= n."""
    p = 0
    while 2 ** p < n:
        p += 1
    return p


def CreateHSP(XS, index=1):
    """CreateHSP.m:11-44 with the rectangle window (WindowType = 1, KatsevichFiltering.m:22)."""
    Length = XS
    HS = np.ones(Length)
    Center = Length / 2 + 1
    HS[1 - 1] = 0
    for i in range(2, int(Center - 1) + 1):
        HS[i - 1] = 2 * math.sin(PI * (i - Center) / 2) ** 2 / (PI * (i - Center))
    HS[int(Center) - 1] = 0
    for i in range(int(Center) + 1, Length + 1):
        HS[i - 1] = 2 * math.sin(PI * (i - Center) / 2) ** 2 / (PI * (i - Center))
    Window = np.ones(Length)
    return HS * Window


def KatsevichFiltering(Proj, ProjScale, DecWidth, DecHeigh, ScanR, StdDis, HelicP,
                       FilterCoeFF, DeltaAngle, FilteringMode, hits=None):
    """KatsevichFiltering.m, the `useGPU == false` branch (:40-288). Proj has MATLAB's shape
    (YL, ZL, ProjNumber); returns FProj of the same shape. `hits` (a dict), if given, counts the
    branches taken by the forward-rebin clamp and the backward-rebin ladder."""
    hits = {} if hits is None else hits

    def hit(k):
        hits[k] = hits.get(k, 0) + 1
    RebinFactor = 1.3                                       # :20
    ParaCoef = FilterCoeFF                                  # :21
    YL, ZL, ProjNumber = Proj.shape                         # :33
    DeltaL = 2 * PI / ProjScale                             # :40
    DeltaU = DecWidth / YL
    DeltaV = DecHeigh / ZL
    HalfZ = (ZL + 1) / 2
    HalfY = (YL + 1) / 2
    y = (np.arange(1, YL + 1) - HalfY) * DeltaU             # :46
    z = (np.arange(1, ZL + 1) - HalfZ) * DeltaV

    # ---- Step 1: derivative (:52-95) ----
    GF = Proj.copy()
    for ProjIndex in range(2, ProjNumber - 1 + 1):
        GF[:, :, ProjIndex - 1] = (Proj[:, :, ProjIndex + 1 - 1] -
                                   Proj[:, :, ProjIndex - 1 - 1]) / (2 * DeltaL)
    GF[:, :, 1 - 1] = GF[:, :, 2 - 1]
    GF[:, :, ProjNumber - 1] = GF[:, :, ProjNumber - 1 - 1]

    for Yindex in range(3, YL - 2 + 1):                     # :63-67
        coef = (StdDis ** 2 + (y[Yindex - 1]) ** 2) / (2 * DeltaU * StdDis)
        GF[Yindex - 1, :, :] = (GF[Yindex - 1, :, :] +
                                (Proj[Yindex + 1 - 1, :, :] - Proj[Yindex - 1 - 1, :, :]) * coef)
    temp = Proj[3 - 1, :, :] - Proj[1 - 1, :, :]            # :69-73
    for Yindex in (1, 2):
        coef = (StdDis ** 2 + (y[Yindex - 1]) ** 2) / (2 * DeltaU * StdDis)
        GF[Yindex - 1, :, :] = GF[Yindex - 1, :, :] + temp * coef
    temp = Proj[YL - 1, :, :] - Proj[YL - 2 - 1, :, :]      # :74-78
    for Yindex in (YL - 1, YL):
        coef = (StdDis ** 2 + (y[Yindex - 1]) ** 2) / (2 * DeltaU * StdDis)
        GF[Yindex - 1, :, :] = GF[Yindex - 1, :, :] + temp * coef

    Y = np.repeat(y[:, None], ProjNumber, axis=1)           # :82 ndgrid(y, 1:ProjNumber)
    Y = Y.reshape(YL, 1, ProjNumber)                        # :83
    coef = 1.0 / (2 * DeltaV * StdDis)                      # :84
    for Zindex in range(3, ZL - 2 + 1):                     # :85-88
        temp = Y * (Proj[:, Zindex + 1 - 1:Zindex + 1, :] - Proj[:, Zindex - 1 - 1:Zindex - 1, :])
        GF[:, Zindex - 1:Zindex, :] = GF[:, Zindex - 1:Zindex, :] + z[Zindex - 1] * temp * coef
    temp = Y * (Proj[:, 3 - 1:3, :] - Proj[:, 1 - 1:1, :])  # :90-92
    GF[:, 1 - 1:1, :] = GF[:, 1 - 1:1, :] + z[1 - 1] * coef * temp
    GF[:, 2 - 1:2, :] = GF[:, 2 - 1:2, :] + z[2 - 1] * coef * temp
    temp = Y * (Proj[:, ZL - 1:ZL, :] - Proj[:, ZL - 2 - 1:ZL - 2, :])  # :93-95
    GF[:, ZL - 1 - 1:ZL - 1, :] = GF[:, ZL - 1 - 1:ZL - 1, :] + z[ZL - 1 - 1] * coef * temp
    GF[:, ZL - 1:ZL, :] = GF[:, ZL - 1:ZL, :] + z[ZL - 1] * coef * temp

    # ---- Step 2: kappa-line resampling and pre-weight (:102-153) ----
    AngleRange = 2 * PI - DeltaAngle
    QQ = math.ceil(ZL * RebinFactor * 0.5)
    AL = 2 * QQ + 1
    Y = y
    Nata = np.arange(1, QQ + 1) * AngleRange / (QQ - 1)     # :107
    Nata = np.concatenate([-Nata[::-1], [0.0], Nata])       # :109
    FilterCoef = np.ones(QQ) * ParaCoef
    if FilteringMode == 2:
        FilterCoef = np.concatenate([FilterCoef, [0.0], FilterCoef])
    else:
        FilterCoef = np.concatenate([1 - FilterCoef, [0.0], FilterCoef])
    AA = np.sin(FilterCoef * Nata) - FilterCoef * np.sin(Nata)
    BB = FilterCoef - 1 + np.cos(FilterCoef * Nata) - FilterCoef * np.cos(Nata)
    CC = np.sin((1 - FilterCoef) * Nata) - np.sin(Nata) + np.sin(FilterCoef * Nata)
    CC[QQ + 1 - 1] = 1
    InDs = Nata * HelicP * StdDis * AA / (2 * PI * ScanR * CC)   # :121
    Rato = Nata * HelicP * BB / (2 * PI * ScanR * CC)            # :123
    Rato[QQ + 1 - 1] = HelicP / (2 * PI * ScanR)
    AZCor = InDs[:, None][:, np.zeros(YL, dtype=int)] + np.outer(Rato, Y)  # :126 (column x row)

    ConvRes = np.zeros((ProjNumber, AL, YL))                # :130
    for Aindex in range(1, AL + 1):
        for tempindex in range(1, YL + 1):
            tempV = AZCor[Aindex - 1, tempindex - 1] / DeltaV + HalfZ
            if tempV < 1.01:
                hit("rebin_clamp_low")
                ConvRes[:, Aindex - 1, tempindex - 1] = GF[tempindex - 1, 1 - 1, :]
            elif tempV > ZL:
                hit("rebin_clamp_high")
                ConvRes[:, Aindex - 1, tempindex - 1] = GF[tempindex - 1, ZL - 1, :]
            else:
                tpUpv = math.ceil(tempV)
                tpLwv = tpUpv - 1
                ConvRes[:, Aindex - 1, tempindex - 1] = (
                    GF[tempindex - 1, tpUpv - 1, :] * (tempV - tpLwv) +
                    GF[tempindex - 1, tpLwv - 1, :] * (tpUpv - tempV))
    coef = StdDis / np.sqrt(StdDis ** 2 + Y[None, :][np.zeros(AL, dtype=int), :] ** 2 + AZCor ** 2)
    for ProjIndex in range(1, ProjNumber + 1):              # :151-153
        ConvRes[ProjIndex - 1, :, :] = ConvRes[ProjIndex - 1, :, :] * coef

    # ---- Step 3: Hilbert transform, post-weight (:160-183) ----
    nn = 2 ** (nextpow2(YL) + 1)
    nn2 = 2 * nn
    HS = CreateHSP(nn, 1)
    tempHS = HS
    HS = np.zeros(nn2)
    HS[1 - 1:nn // 2] = tempHS[nn // 2 + 1 - 1:nn]
    HS[nn + nn // 2 + 1 - 1:nn2] = tempHS[1 - 1:nn // 2]
    FFT_F = np.fft.fft(HS)
    # the loop over ConvRes's ProjNumber*AL rows (:170-176); every row gets the same
    # fft(row, nn2) -> .* FFT_F -> real(ifft) -> -first YL, done here on all rows at once
    rows = ConvRes.reshape(ProjNumber * AL, YL)
    FFT_S = np.fft.fft(rows, nn2, axis=1)
    TempData = np.real(np.fft.ifft(FFT_S * FFT_F[None, :], axis=1))
    ConvRes = (-TempData[:, :YL]).reshape(ProjNumber, AL, YL)
    for ProjIndex in range(1, ProjNumber + 1):              # :181-183
        ConvRes[ProjIndex - 1, :, :] = ConvRes[ProjIndex - 1, :, :] / coef

    # ---- Step 4: backward rebin (:191-287) ----
    FProj = GF.copy()
    for Yindex in range(1, YL + 1):
        zmax = -DecHeigh
        zmin = DecHeigh
        MAXI = 1
        MINI = AL
        for tpindex in range(1, AL + 1):
            if AZCor[tpindex - 1, Yindex - 1] > zmax:
                zmax = AZCor[tpindex - 1, Yindex - 1]
                MAXI = tpindex
            if AZCor[tpindex - 1, Yindex - 1] < zmin:
                zmin = AZCor[tpindex - 1, Yindex - 1]
                MINI = tpindex
        BeginAL = 0
        EndAL = 0
        BeginCoef = 0
        EndCoef = 0
        for Zindex in range(1, ZL + 1):
            CurrZ = (Zindex - HalfZ) * DeltaV
            if CurrZ < zmin:
                hit("below_all_lines")
                BeginAL = MINI
                EndAL = MINI
                BeginCoef = 0.5
                EndCoef = 0.5
            elif CurrZ > zmax:
                hit("above_all_lines")
                BeginAL = MAXI
                EndAL = MAXI
                BeginCoef = 0.5
                EndCoef = 0.5
            else:
                deltamaxB = DecHeigh
                deltamaxE = DecHeigh
                for tpindex in range(1, AL + 1):
                    a = AZCor[tpindex - 1, Yindex - 1]
                    if a > CurrZ and a - CurrZ < deltamaxE:
                        deltamaxE = a - CurrZ
                        EndAL = tpindex
                    if a < CurrZ and CurrZ - a < deltamaxB:
                        deltamaxB = CurrZ - a
                        BeginAL = tpindex
                if not ((EndAL == BeginAL + 1) or (EndAL == BeginAL)):
                    hit("crossing_fixup")
                    Sign_Dis = CurrZ - Rato[QQ + 1 - 1] * y[Yindex - 1]
                    if Sign_Dis > 0:
                        if BeginAL < QQ + 1:
                            BeginAL = EndAL - 1
                            deltamaxB = CurrZ - AZCor[BeginAL - 1, Yindex - 1]
                        elif EndAL < QQ + 1:
                            EndAL = BeginAL + 1
                            deltamaxE = AZCor[EndAL - 1, Yindex - 1] - CurrZ
                        elif EndAL < BeginAL:
                            BeginAL = EndAL - 1
                            deltamaxB = CurrZ - AZCor[BeginAL - 1, Yindex - 1]
                        else:
                            EndAL = BeginAL + 1
                            deltamaxE = AZCor[EndAL - 1, Yindex - 1] - CurrZ
                    else:
                        if BeginAL > QQ + 1:
                            BeginAL = EndAL - 1
                            deltamaxB = CurrZ - AZCor[BeginAL - 1, Yindex - 1]
                        elif EndAL > QQ + 1:
                            EndAL = BeginAL + 1
                            deltamaxE = AZCor[EndAL - 1, Yindex - 1] - CurrZ
                        elif EndAL > BeginAL:
                            BeginAL = EndAL - 1
                            deltamaxB = CurrZ - AZCor[BeginAL - 1, Yindex - 1]
                        else:
                            EndAL = BeginAL + 1
                            deltamaxE = AZCor[EndAL - 1, Yindex - 1] - CurrZ
                BeginCoef = deltamaxE / (deltamaxE + deltamaxB)
                EndCoef = deltamaxB / (deltamaxE + deltamaxB)
            assert 1 <= BeginAL <= AL and 1 <= EndAL <= AL  # MATLAB would raise here
            FProj[Yindex - 1, Zindex - 1, :] = (ConvRes[:, BeginAL - 1, Yindex - 1] * BeginCoef +
                                                ConvRes[:, EndAL - 1, Yindex - 1] * EndCoef)
    return FProj


def _run_both(O, s, proj, mode=None, hits=None):
    fp = oracle_filter_params(O, s)
    if mode is not None:
        fp.FilteringMode = mode
    ref = O.katsevich_filter(fp, proj)
    Proj = np.ascontiguousarray(proj.transpose(2, 1, 0))    # MATLAB Proj(YL, ZL, P)
    got = KatsevichFiltering(Proj, float(s.views_per_turn), s.DecWidth, s.DecHeigh, s.ScanR,
                             s.StdDis, s.HelicP, s.filter_coeff, s.delta, fp.FilteringMode, hits)
    return got.transpose(2, 1, 0), ref


@pytest.mark.parametrize("name,mode", [("tiny", 0), ("tiny", 2), ("c1", 0)])
def test_oracle_filter_matches_matlab_transliteration(oracle_mod, name, mode):
    from ctrecon_b200.geometry import config, small_config
    O = oracle_mod
    s = small_config() if name == "tiny" else config("c1")
    proj = O.project_ellipsoids(oracle_geom(O, s), s.ellipsoids())
    hits = {}
    got, ref = _run_both(O, s, proj, mode, hits)
    scale = np.abs(ref).max()
    rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    mx = float(np.abs(got - ref).max())
    print(f"{name} FilteringMode {mode}: rel RMSE {rel:.2e}, max-abs {mx:.2e} of {scale:.3e}; "
          f"branches {hits}")
    # FFT round-off (about 1e-16 per term) against the exact direct sum
    assert rel < 1e-12
    assert mx < 1e-11 * scale


@pytest.mark.parametrize("fc", [0.2, 0.8])
def test_transliteration_on_noise_reaches_every_rebin_branch(oracle_mod, fc):
    """Random projections (every derivative and rebin weight non-trivial) on a geometry whose
    kappa lines leave the detector at both ends (pitch 1.3x the height rule) and cross inside it
    (FilterCoeFF 0.2 / 0.8): the forward-rebin clamps (:135-138) and the backward rebin's
    crossing fix-up (:243-276) are all taken, and the two restatements still agree."""
    from ctrecon_b200.geometry import small_config
    O = oracle_mod
    s = small_config(views_per_turn=60, turns=1, filter_coeff=fc, pitch_ratio=1.3)
    proj = np.random.default_rng(5).standard_normal(s.proj_shape)
    hits = {}
    got, ref = _run_both(O, s, proj, None, hits)
    print(f"branches {hits}")
    assert float(np.linalg.norm(got - ref) / np.linalg.norm(ref)) < 1e-12
    for k in ("rebin_clamp_low", "rebin_clamp_high", "crossing_fixup"):
        assert hits.get(k, 0) > 0, f"branch {k} not exercised: {hits}"
