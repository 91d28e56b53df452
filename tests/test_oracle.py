"""Pins of the FP64 oracle (CPU only).

* the backprojector restatement is bit-identical to the reference's own KatsevichBkProj.cpp
  (compiled unchanged into oracle/_ref) -- live, and through the committed golden vectors;
* the geometry sizing reproduces the constants recorded in KatsevichFiltering_GPU.cu:997;
* the filter's direct Toeplitz sum equals the reference's circular FFT convolution
  (KatsevichFiltering.m:160-176) with the CreateHSP.m kernel;
* derivative stencils and edge rules (KatsevichFiltering.m:52-95) on fields with known
  derivatives; the PI-line solve satisfies its defining equation and the helix symmetry.
"""
import os

import numpy as np
import pytest

from conftest import oracle_filter_params, oracle_geom

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_geometry_kat(oracle_mod):
    d = np.load(os.path.join(GOLDEN, "geometry_kat.npz"))
    R, D, H, ObjR, YL, ZL = d["inputs"]
    got = oracle_mod.geometry_sizing(R, D, H, ObjR, int(YL), int(ZL))
    # KatsevichFiltering_GPU.cu:997 records 16 significant digits
    np.testing.assert_allclose(got, d["recorded"], rtol=2e-15, atol=0)
    np.testing.assert_array_equal(got, d["computed"])


def test_oracle_bp_equals_reference_golden(oracle_mod):
    f = np.load(os.path.join(GOLDEN, "filter_tiny.npz"))
    b = np.load(os.path.join(GOLDEN, "bkproj_ref_tiny.npz"))
    g = oracle_mod.bp_geom(b["locus"], b["detector"], b["object"], honour_extras=False)
    img = np.full(b["image"].shape, float(b["sentinel"]))
    oracle_mod.bkproj(g, f["fproj"], img)
    assert np.array_equal(img, b["image"])
    assert np.any(b["image"] == b["sentinel"])  # untouched voxels exist and are kept


def test_oracle_filter_golden(oracle_mod):
    f = np.load(os.path.join(GOLDEN, "filter_tiny.npz"))
    a = f["params"]
    fp = oracle_mod.filter_params(ProjScale=a[0], DecWidth=a[1], DecHeigh=a[2], ScanR=a[3],
                                  StdDis=a[4], HelicP=a[5], FilterCoeFF=a[6], DeltaAngle=a[7],
                                  FilteringMode=int(a[8]), YL=int(a[9]), ZL=int(a[10]),
                                  ProjNumber=int(a[11]))
    out = oracle_mod.katsevich_filter(fp, f["proj"])
    assert np.array_equal(out, f["fproj"])


def _edge_geometries():
    from ctrecon_b200.geometry import small_config
    base = small_config(YL=40, ZL=8, views_per_turn=100, turns=2.5, NX=16, NY=16, NZ=12)
    out = [base]
    # volume taller than the helix travel: voxels with Bindex < 0, == 0, == P-2, Tindex > P-1
    out.append(base.with_(NZ=20, voxel=(2 * base.ObjR / 16, 2 * base.ObjR / 16, 3.0)))
    return out


@pytest.mark.parametrize("case", range(4))
def test_oracle_bp_equals_reference_live(oracle_mod, case):
    O = oracle_mod
    if not O.ref_available():
        pytest.skip("oracle/_ref not built (needs the CTRecon sources)")
    s = _edge_geometries()[case % 2]
    locus = s.locus()
    if case >= 2:  # ProjBeginIndex != 1 and a non-integer ProjCtr (FunctionKat_v6.m:103)
        locus[4] = 3.0
        locus[5] = locus[4] + s.P - 1
        locus[6] = s.ProjCtr + 1.5
    rng = np.random.default_rng(case)
    fproj = rng.standard_normal(s.proj_shape)
    # honour_extras=False: exactly KatsevichBkProj.cpp (2*ObjR/N voxels, (N-1)/2 centres)
    g = O.bp_geom(locus, s.detector(), s.object(), honour_extras=False)
    img = np.full(s.vol_shape, -3.5)
    img, n, touched = O.bkproj(g, fproj, img, want_touched=True)
    ref = np.full(s.vol_shape, -3.5)
    geom = {"Locus": np.array(locus), "Detector": np.array(s.detector()),
            "Object": np.array(s.object())}
    O.ref_bkproj(geom, fproj, ref)
    assert np.array_equal(img, ref)
    assert n > 0 and touched.sum() > 0


def test_oracle_endpoint_cases_exercised(oracle_mod):
    """The tall-volume geometry reaches every branch of KatsevichBkProj.cpp:187-234."""
    s = _edge_geometries()[1]
    g = oracle_geom(oracle_mod, s)
    t = oracle_mod.pi_table(g)
    P = s.P
    B, T, v = t["B"], t["T"], t["valid"]
    bidx = (np.floor(B[v])).astype(int)
    tidx = (np.floor(T[v])).astype(int) + 1
    assert np.any(bidx < 0) and np.any(bidx == 0) and np.any(bidx > 0)
    assert np.any(tidx > P - 1) and np.any(tidx < P - 1)
    assert np.any(~v & (np.abs(B) < 1e9))  # voxels skipped by the PI rule (:180)


def _createhsp(nn):
    # CreateHSP.m:11-23 (rectangle window), 1-based loops mapped to 0-based indices
    PI = 3.14159265358979
    HS = np.ones(nn)
    C = nn / 2 + 1
    HS[0] = 0
    for i in range(2, nn + 1):
        if i == C:
            HS[i - 1] = 0
            continue
        HS[i - 1] = 2 * np.sin(PI * (i - C) / 2) ** 2 / (PI * (i - C))
    return HS


@pytest.mark.parametrize("YL", [5, 16, 33, 64, 100, 257])
def test_toeplitz_equals_reference_fft_convolution(oracle_mod, YL):
    nn = 2 ** (int(np.ceil(np.log2(YL))) + 1)
    nn2 = 2 * nn
    temp = _createhsp(nn)
    HS = np.zeros(nn2)  # KatsevichFiltering.m:163-166
    HS[: nn // 2] = temp[nn // 2: nn]
    HS[nn + nn // 2:] = temp[: nn // 2]
    F = np.fft.fft(HS)
    rng = np.random.default_rng(YL)
    rows = rng.standard_normal((7, YL))
    fft_out = np.real(np.fft.ifft(np.fft.fft(rows, nn2, axis=1) * F, axis=1))[:, :YL]
    h = oracle_mod.hilbert_taps(YL)
    i = np.arange(YL)
    T = h[(i[:, None] - i[None, :]) + YL - 1]
    direct = rows @ T.T
    np.testing.assert_allclose(direct, fft_out, rtol=0, atol=1e-12 * np.abs(fft_out).max())


def test_derivative_stencils_linear_field(oracle_mod, tiny_scan):
    """GF of p(u, v, lambda) = a*y + b*z + c*lambda is the chain rule applied exactly,
    also in the edge rows/columns (two-cell differences, :69-78, :89-95) and the end
    views (:58-59)."""
    O, s = oracle_mod, tiny_scan
    fp = oracle_filter_params(O, s)
    P, ZL, YL = s.proj_shape
    dU, dV = s.DecWidth / YL, s.DecHeigh / ZL
    dL = 2 * 3.14159265358979 / s.views_per_turn
    y = (np.arange(1, YL + 1) - (YL + 1) / 2) * dU
    z = (np.arange(1, ZL + 1) - (ZL + 1) / 2) * dV
    a, b, c = 0.3, -0.7, 1.9
    lam = np.arange(P) * dL
    proj = a * y[None, None, :] + b * z[None, :, None] + c * lam[:, None, None]
    D = s.StdDis
    want = c + a * (D ** 2 + y[None, :] ** 2) / D + b * (y[None, :] * z[:, None]) / D
    for p in (0, 1, P // 2, P - 2, P - 1):
        gf, _, _ = O.filter_view_stages(fp, proj, p)
        np.testing.assert_allclose(gf, want, rtol=1e-11, atol=1e-11)


def test_pisegment_defining_equation_and_symmetry(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(3)
    PI = 3.14159265358979
    for _ in range(200):
        r = 0.19 * np.sqrt(rng.random())
        ph = 2 * np.pi * rng.random()
        x, y, z = r * np.cos(ph), r * np.sin(ph), rng.uniform(-2, 2)
        sb, st = O.pisegment(x, y, z)
        # the chord from the helix point at sb to the one at st passes through the voxel:
        # both helix points and (x, y, z) are collinear (normalised units R = P = 1)
        a = np.array([np.cos(sb), np.sin(sb), sb / (2 * PI)])
        bb = np.array([np.cos(st), np.sin(st), st / (2 * PI)])
        q = np.array([x, y, z])
        cr = np.cross(bb - a, q - a)
        assert np.linalg.norm(cr) < 1e-5
        assert 0 < st - sb < 2 * PI
        sb2, st2 = O.pisegment(x, y, z + 1.0)
        assert abs((sb2 - sb) - 2 * PI) < 1e-6 and abs((st2 - st) - 2 * PI) < 1e-6
