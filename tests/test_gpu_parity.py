"""Parity of the CUDA path with the FP64 oracle, called through the C ABI (needs a B200).

Tolerances: the filter computes in FP32 (Hilbert sum in FP32, BF16x3 or TF32 on the tensor
cores), the backprojector interpolates and accumulates in FP32, the PI line is FP64. The
bar of the whole chain against the FP64 oracle is a relative RMSE of 1e-4 over the voxels
the reference writes; untouched voxels must keep their values bit for bit.
"""
import os

import numpy as np
import pytest

from conftest import max_abs, oracle_filter_params, oracle_geom, rel_rmse

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SENTINEL = 7.25


@pytest.fixture(scope="module")
def torch_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def ctx(torch_mod):
    import ctrecon_b200 as ct
    c = ct.Context(0)
    yield c
    c.close()


def _scan(name):
    from ctrecon_b200.geometry import config, small_config
    return small_config() if name == "tiny" else config(name)


@pytest.fixture(scope="module")
def tiny_case(oracle_mod):
    s = _scan("tiny")
    O = oracle_mod
    g = oracle_geom(O, s)
    proj = O.project_ellipsoids(g, s.ellipsoids())
    fproj = O.katsevich_filter(oracle_filter_params(O, s), proj)
    img, n, touched = O.bkproj(g, fproj, np.full(s.vol_shape, SENTINEL), want_touched=True)
    return dict(s=s, proj=proj, fproj=fproj, img=img, n=n, touched=touched.astype(bool))


@pytest.fixture(scope="module")
def c1_case(oracle_mod):
    s = _scan("c1")
    O = oracle_mod
    g = oracle_geom(O, s)
    proj = O.project_ellipsoids(g, s.ellipsoids())
    fproj = O.katsevich_filter(oracle_filter_params(O, s), proj)
    img, n, touched = O.bkproj(g, fproj, np.full(s.vol_shape, SENTINEL), want_touched=True)
    return dict(s=s, proj=proj, fproj=fproj, img=img, n=n, touched=touched.astype(bool))


def test_phantom_projector_matches_oracle(ctx, torch_mod, tiny_case):
    torch = torch_mod
    s = tiny_case["s"]
    d = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
    ctx.phantom_dev(s.geom_struct(), s.ellipsoids(), d)
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    assert rel_rmse(got, tiny_case["proj"]) < 1e-6


@pytest.mark.parametrize("case", ["tiny", "c1"])
def test_filter_matches_oracle(ctx, tiny_case, c1_case, case):
    import ctrecon_b200 as ct
    c = tiny_case if case == "tiny" else c1_case
    s = c["s"]
    out = ctx.filter_host(ct.scan_filter_params(s), c["proj"])
    err = rel_rmse(out, c["fproj"])
    print(f"filter {case}: rel RMSE {err:.3e} max-abs {max_abs(out, c['fproj']):.3e}")
    assert err < 1e-5


@pytest.mark.parametrize("mode,bound", [("bf16x3", 5e-5), ("tf32", 5e-3)])
@pytest.mark.parametrize("case", ["tiny", "c1"])
def test_filter_tensor_core_matches_oracle(torch_mod, tiny_case, c1_case, case, mode, bound):
    """Toeplitz-GEMM Hilbert on tcgen05: BF16x3 must stay near FP32; TF32 is reported."""
    import ctrecon_b200 as ct
    c = tiny_case if case == "tiny" else c1_case
    s = c["s"]
    m = ct.HILBERT_BF16X3 if mode == "bf16x3" else ct.HILBERT_TF32
    with ct.Context(0, hilbert=m) as cx:
        out = cx.filter_host(ct.scan_filter_params(s), c["proj"])
    err = rel_rmse(out, c["fproj"])
    print(f"filter {case} {mode}: rel RMSE {err:.3e} max-abs {max_abs(out, c['fproj']):.3e}")
    assert err < bound


@pytest.mark.parametrize("mode,bound", [("bf16x3", 5e-5), ("tf32", 5e-3)])
@pytest.mark.parametrize("zl,yl", [(200, 96), (260, 64)])
def test_filter_tensor_core_two_halves(torch_mod, oracle_mod, zl, yl, mode, bound):
    """Detectors with more than 256 kappa rows per view (AL = 261, 339): the tensor-core
    Hilbert splits a view's rows into two N-halves accumulated in TMEM columns [0, 256) and
    [256, 512); must agree with the FP64 oracle like the one-half form."""
    import ctrecon_b200 as ct
    from ctrecon_b200.geometry import small_config
    s = small_config(name="tall", YL=yl, ZL=zl, views_per_turn=120, turns=2.2, NX=24, NY=24,
                     NZ=8)
    O = oracle_mod
    proj = O.project_ellipsoids(oracle_geom(O, s), s.ellipsoids())
    ref = O.katsevich_filter(oracle_filter_params(O, s), proj)
    m = ct.HILBERT_BF16X3 if mode == "bf16x3" else ct.HILBERT_TF32
    with ct.Context(0, hilbert=m) as cx:
        out = cx.filter_host(ct.scan_filter_params(s), proj)
    err = rel_rmse(out, ref)
    print(f"filter {zl}x{yl} (AL {2 * int(np.ceil(0.65 * zl)) + 1}) {mode}: rel RMSE {err:.3e}")
    assert err < bound


@pytest.mark.parametrize("mode,bound", [("bf16x3", 5e-5), ("tf32", 5e-3)])
@pytest.mark.parametrize("yl,zl,chunk", [(300, 16, 2048), (130, 40, 7), (736, 64, 100)])
def test_filter_tensor_core_forms_agree(torch_mod, oracle_mod, yl, zl, chunk, mode, bound):
    """The parity-split persistent form (default) and the single-pass form of the tensor-core
    Hilbert, each against the FP64 oracle and against each other, on ragged shapes: 300 columns
    (each parity's 192 outputs padded to two 128-row blocks), 130 columns with 53 kappa rows per
    view (four views per tile) in chunks of 7 views (partial view groups), and the c2 detector
    in chunks of 100 views."""
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import small_config
    s = small_config(name="ragged", YL=yl, ZL=zl, views_per_turn=90, turns=1.3, NX=24, NY=24,
                     NZ=8)
    O = oracle_mod
    proj = O.project_ellipsoids(oracle_geom(O, s), s.ellipsoids())
    ref = O.katsevich_filter(oracle_filter_params(O, s), proj)
    m = ct.HILBERT_BF16X3 if mode == "bf16x3" else ct.HILBERT_TF32
    out = {}
    for form in (_lib.TC_PARITY_SPLIT, _lib.TC_SINGLE_PASS):
        with ct.Context(0, hilbert=m) as cx:
            cx.set_option(_lib.OPT_TC_FORM, form)
            cx.set_option(_lib.OPT_FILTER_CHUNK, chunk)
            out[form] = cx.filter_host(ct.scan_filter_params(s), proj)
        err = rel_rmse(out[form], ref)
        print(f"filter {zl}x{yl} {mode} form {form}: rel RMSE {err:.3e}")
        assert err < bound
        assert np.all(np.isfinite(out[form]))
    d = rel_rmse(out[_lib.TC_PARITY_SPLIT], out[_lib.TC_SINGLE_PASS])
    print(f"  forms differ by {d:.2e}")
    assert d < bound


@pytest.mark.parametrize("yl,zl,chunk", [(300, 16, 2048), (300, 40, 7), (256, 16, 100),
                                          (736, 64, 33), (132, 8, 5), (130, 40, 7),
                                          (256, 80, 9), (160, 132, 40)])
@pytest.mark.parametrize("mode", ["fp32", "bf16x3", "tf32"])
def test_k1_forms_bit_identical(torch_mod, oracle_mod, yl, zl, chunk, mode):
    """The staged K1 (tensor copies of 32-column strips, views walked in order, default) and
    the per-view K1 write the same kappa rows bit for bit, so the filtered projections of every
    Hilbert form agree exactly; both against the FP64 oracle. Shapes: ragged strips (300 and
    132 columns: a partial last strip and zero-padded columns), chunks of 7, 33 and 5 views
    (runs of one view, and chunks with fewer views than runs), eight detector rows (half of
    them under the v stencil's edge rule), 40 rows, 64 rows and the c2 detector width (the
    short shape: 4 rows and 6 kappa lines a warp), 80 rows (105 kappa lines: the tall shape, 8
    rows and 11 lines a warp), 132 rows (173 kappa lines: warp 0 takes a second block of rows,
    the last four), and 130 columns, where the staged form does not apply (rows of 520 bytes)
    and both settings run the per-view form."""
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import small_config
    s = small_config(name="ragged", YL=yl, ZL=zl, views_per_turn=90, turns=1.3, NX=24, NY=24,
                     NZ=8)
    O = oracle_mod
    proj = O.project_ellipsoids(oracle_geom(O, s), s.ellipsoids())
    ref = O.katsevich_filter(oracle_filter_params(O, s), proj)
    m = {"fp32": ct.HILBERT_FP32, "bf16x3": ct.HILBERT_BF16X3, "tf32": ct.HILBERT_TF32}[mode]
    bound = {"fp32": 1e-5, "bf16x3": 1e-4, "tf32": 2e-3}[mode]
    out = {}
    for form in (_lib.K1_STAGED, _lib.K1_PER_VIEW):
        with ct.Context(0, hilbert=m) as cx:
            cx.set_option(_lib.OPT_K1_FORM, form)
            assert cx.get_option(_lib.OPT_K1_FORM) == form
            cx.set_option(_lib.OPT_FILTER_CHUNK, chunk)
            out[form] = cx.filter_host(ct.scan_filter_params(s), proj)
        err = rel_rmse(out[form], ref)
        print(f"filter {zl}x{yl} {mode} K1 form {form}: rel RMSE {err:.3e}")
        assert err < bound
    assert np.array_equal(out[_lib.K1_STAGED], out[_lib.K1_PER_VIEW])


def test_chain_c1_bf16x3_matches_oracle(torch_mod, c1_case):
    import ctrecon_b200 as ct
    s = c1_case["s"]
    img = np.full(s.vol_shape, SENTINEL)
    with ct.Context(0, hilbert=ct.HILBERT_BF16X3) as cx:
        cx.recon_host(ct.scan_filter_params(s), s.geom_struct(), c1_case["proj"], img)
    t = c1_case["touched"]
    assert np.array_equal(img[~t], c1_case["img"][~t])
    err = rel_rmse(img, c1_case["img"], t)
    print(f"chain c1 bf16x3: rel RMSE {err:.3e}")
    assert err < 1e-4


def test_filter_device_path_equals_host_path(ctx, torch_mod, tiny_case):
    import ctrecon_b200 as ct
    torch = torch_mod
    s = tiny_case["s"]
    p = ct.scan_filter_params(s)
    d_in = torch.from_numpy(tiny_case["proj"].astype(np.float32)).cuda()
    d_out = torch.empty_like(d_in)
    ctx.filter_dev(p, d_in, d_out)
    torch.cuda.synchronize()
    host = ctx.filter_host(p, tiny_case["proj"])
    assert np.array_equal(d_out.cpu().numpy().astype(np.float64), host)


def test_filter_in_place_alias(ctx, tiny_case):
    """The MATLAB caller passes FProj sharing Proj's buffer (KatsevichFiltering.m:37)."""
    import ctrecon_b200 as ct
    s = tiny_case["s"]
    buf = tiny_case["proj"].copy()
    ctx.filter_host(ct.scan_filter_params(s), buf, buf)
    assert rel_rmse(buf, tiny_case["fproj"]) < 1e-5


@pytest.mark.parametrize("case", ["tiny", "c1"])
def test_pi_table_matches_oracle(ctx, torch_mod, oracle_mod, case):
    torch = torch_mod
    s = _scan(case)
    nbytes = ctx.pi_table_bytes(s.geom_struct())
    d_tab = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ctx.pi_dev(s.geom_struct(), d_tab, d_cnt)
    torch.cuda.synchronize()
    rec = d_tab.cpu().numpy().view(np.int32).reshape(-1, 4)
    bi, ti = rec[:, 0], rec[:, 2]
    bf, tf = rec[:, 1].view(np.float32), rec[:, 3].view(np.float32)
    valid = bi != 0x7FFFFFFF
    o = oracle_mod.pi_table(oracle_geom(oracle_mod, s))
    ov = o["valid"].ravel()
    assert np.array_equal(valid, ov)
    B = bi[valid] + bf[valid].astype(np.float64)
    T = ti[valid] + tf[valid].astype(np.float64)
    assert np.max(np.abs(B - o["B"].ravel()[ov])) < 1e-4
    assert np.max(np.abs(T - o["T"].ravel()[ov])) < 1e-4
    lb = np.maximum(1, bi[valid])
    le = np.minimum(ti[valid] + 1, s.P - 2)
    n_gpu = int(d_cnt.item())
    assert n_gpu == int(np.sum(le - lb + 1))
    n_orc = int(np.sum(o["loop_end"].ravel()[ov] - o["loop_begin"].ravel()[ov] + 1))
    assert abs(n_gpu - n_orc) <= max(2, n_orc * 1e-7)


def test_pi_table_alignment_is_checked(ctx, torch_mod):
    """The PI table holds 16-byte records: a caller's table that is not 16-byte aligned is
    refused by every entry point that takes one, before any work is enqueued."""
    import ctrecon_b200 as ct
    torch = torch_mod
    s = _scan("tiny")
    g = s.geom_struct()
    nbytes = ctx.pi_table_bytes(g)
    d_buf = torch.zeros(nbytes + 16, dtype=torch.uint8, device="cuda")
    bad = d_buf[4:4 + nbytes]
    assert bad.data_ptr() % 16 == 4
    d_f = torch.zeros(s.proj_shape, dtype=torch.float32, device="cuda")
    img = torch.full(s.vol_shape, SENTINEL, dtype=torch.float32, device="cuda")
    with pytest.raises(ct.CtreconError, match="16-byte aligned"):
        ctx.pi_dev(g, bad)
    with pytest.raises(ct.CtreconError, match="16-byte aligned"):
        ctx.bkproj_dev(g, d_f, img, d_pitab=bad)
    with pytest.raises(ct.CtreconError, match="16-byte aligned"):
        ctx.tune_bkproj(g, d_f, img, d_pitab=bad)
    torch.cuda.synchronize()
    assert int(d_buf.sum().item()) == 0 and bool(torch.all(img == SENTINEL))
    # an aligned table of the same buffer works
    good = d_buf[16:16 + nbytes]
    ctx.pi_dev(g, good)
    torch.cuda.synchronize()


def test_bkproj_matches_oracle_tiny(ctx, tiny_case):
    s = tiny_case["s"]
    img = np.full(s.vol_shape, SENTINEL)
    ctx.bkproj_host(s.geom_struct(), tiny_case["fproj"], img)
    t = tiny_case["touched"]
    assert np.array_equal(img[~t], tiny_case["img"][~t])  # untouched voxels keep their value
    assert not np.any(img[t] == SENTINEL)
    err = rel_rmse(img, tiny_case["img"], t)
    print(f"bkproj tiny: rel RMSE {err:.3e}")
    assert err < 2e-5


def test_bkproj_matches_reference_golden(ctx):
    """Against the reference's own KatsevichBkProj.cpp output (golden vectors)."""
    f = np.load(os.path.join(GOLDEN, "filter_tiny.npz"))
    b = np.load(os.path.join(GOLDEN, "bkproj_ref_tiny.npz"))
    geom = {"Locus": b["locus"], "Detector": b["detector"], "Object": b["object"]}
    img = np.full(b["image"].shape, float(b["sentinel"]))
    ctx.bkproj_host(geom, np.ascontiguousarray(f["fproj"]), img)
    t = b["image"] != b["sentinel"]
    assert np.array_equal(img[~t], b["image"][~t])
    assert rel_rmse(img, b["image"], t) < 2e-5


def test_chain_c1_matches_oracle(ctx, c1_case):
    """The whole chain at the CPU-runnable configuration, through the fused host call."""
    import ctrecon_b200 as ct
    s = c1_case["s"]
    img = np.full(s.vol_shape, SENTINEL)
    ctx.recon_host(ct.scan_filter_params(s), s.geom_struct(), c1_case["proj"], img)
    t = c1_case["touched"]
    assert np.array_equal(img[~t], c1_case["img"][~t])
    err = rel_rmse(img, c1_case["img"], t)
    print(f"chain c1: rel RMSE {err:.3e} max-abs {max_abs(img, c1_case['img'], t):.3e}")
    assert err < 1e-4


def test_mex_modules_in_place(ctx, tiny_case):
    """The MEX entry points through the standalone harness, as the MATLAB drivers call them
    (KatsevichFiltering.m:37-38 then FunctionKat_v6.m:110-113)."""
    from ctrecon_b200 import _lib
    from ctrecon_b200.mexharness import MexModule
    s = tiny_case["s"]
    mf = MexModule(os.path.join(_lib.MEX_DIR, "KatsevichFiltering_GPU.so"))
    mb = MexModule(os.path.join(_lib.MEX_DIR, "KatsevichBkProj_GPU.so"))
    proj = tiny_case["proj"].copy()
    fproj = proj.copy()
    mf.call([proj] + list(s.filter_args()) + [fproj])
    assert rel_rmse(fproj, tiny_case["fproj"]) < 1e-5
    img = np.full(s.vol_shape, SENTINEL)
    mb.call([s.geom_struct(), fproj, img])
    t = tiny_case["touched"]
    assert np.array_equal(img[~t], tiny_case["img"][~t])
    assert rel_rmse(img, tiny_case["img"], t) < 3e-5
