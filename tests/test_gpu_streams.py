"""Ordering of the device work of one context (needs a B200).

* Several scan geometries used one after the other on one context, on a non-blocking stream
  and without host synchronisation in between, must give exactly the images that separate
  contexts give: a geometry change must never touch tables that queued kernels still read.
* The host (MEX-equivalent) calls pipeline their copies on their own streams; with pinned host
  buffers the copies overlap the kernels, with pageable ones they do not. Both must give the
  same bits. The host backprojection accumulates view windows as they arrive: equal to the
  one-pass backprojection up to the order of the FP32 sums.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _scans():
    from ctrecon_b200.geometry import small_config
    return [small_config(name="s0", YL=96, ZL=16, views_per_turn=200, turns=3, NX=48, NY=48,
                         NZ=16, seed=11),
            small_config(name="s1", YL=64, ZL=8, NX=32, NY=40, NZ=12, seed=12),
            small_config(name="s2", YL=136, ZL=24, views_per_turn=240, turns=2.5, NX=56,
                         NY=56, NZ=10, seed=13)]


@pytest.mark.parametrize("hilbert", ["fp32", "bf16x3"])
def test_interleaved_geometries_on_one_context(torch_mod, hilbert):
    torch = torch_mod
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    mode = {"fp32": _lib.HILBERT_FP32, "bf16x3": _lib.HILBERT_BF16X3}[hilbert]
    scans = _scans()
    projs = []
    with ct.Context(0) as cx:
        for s in scans:
            d = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
            cx.phantom_dev(s.geom_struct(), s.ellipsoids(), d)
            projs.append(d)
        torch.cuda.synchronize()
    # one scan per fresh context, synchronised
    want = []
    for s, d in zip(scans, projs):
        with ct.Context(0, hilbert=mode) as cx:
            f = torch.empty_like(d)
            cx.filter_dev(ct.scan_filter_params(s), d, f)
            img = torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
            cx.bkproj_dev(s.geom_struct(), f, img)
            torch.cuda.synchronize()
            want.append(img.cpu().numpy())
    # all scans on one context, twice round, queued on a side stream with no waits
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream), ct.Context(0, hilbert=mode) as cx:
        imgs = []
        for _ in range(2):
            imgs = []
            for s, d in zip(scans, projs):
                f = torch.empty_like(d)
                cx.filter_dev(ct.scan_filter_params(s), d, f)
                img = torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
                cx.bkproj_dev(s.geom_struct(), f, img)
                imgs.append(img)
        stream.synchronize()
        for s, img, w in zip(scans, imgs, want):
            assert np.array_equal(img.cpu().numpy(), w), s.name


def test_host_calls_pinned_equal_pageable(torch_mod):
    torch = torch_mod
    import ctrecon_b200 as ct
    from ctrecon_b200.geometry import config
    s = config("c1")  # 2160 views: the host calls move them in several chunks
    with ct.Context(0) as cx:
        d = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
        cx.phantom_dev(s.geom_struct(), s.ellipsoids(), d)
        torch.cuda.synchronize()
        proj = d.cpu().numpy().astype(np.float64)
        p = ct.scan_filter_params(s)
        # pageable
        f_pg = cx.filter_host(p, proj)
        img_pg = np.full(s.vol_shape, 7.25)
        cx.bkproj_host(s.geom_struct(), f_pg, img_pg)
        rec_pg = np.full(s.vol_shape, 7.25)
        cx.recon_host(p, s.geom_struct(), proj, rec_pg)
        # pinned
        proj_pin = torch.from_numpy(proj).pin_memory()
        f_pin = torch.empty_like(proj_pin).pin_memory()
        img_pin = torch.full(s.vol_shape, 7.25, dtype=torch.float64).pin_memory()
        rec_pin = torch.full(s.vol_shape, 7.25, dtype=torch.float64).pin_memory()
        cx.filter_host(p, proj_pin.numpy(), f_pin.numpy())
        cx.bkproj_host(s.geom_struct(), f_pin.numpy(), img_pin.numpy())
        cx.recon_host(p, s.geom_struct(), proj_pin.numpy(), rec_pin.numpy())
        assert np.array_equal(f_pin.numpy(), f_pg)
        assert np.array_equal(img_pin.numpy(), img_pg)
        assert np.array_equal(rec_pin.numpy(), rec_pg)
        # the chain through the host equals filter then backprojection through the host; the
        # host backprojection sums its views in windows (as their upload completes), which only
        # reorders the FP32 sums of a voxel
        written = img_pg != 7.25
        assert np.array_equal(written, rec_pg != 7.25)
        rel = np.linalg.norm(rec_pg[written] - img_pg[written]) / np.linalg.norm(img_pg[written])
        print(f"windowed vs one-pass host backprojection: rel diff {rel:.2e}")
        assert rel < 1e-6


@pytest.mark.parametrize("cfg", ["c1", "tiny"])
def test_recon_host_conversion_forms_equal(torch_mod, cfg):
    """The host calls convert their FP64 inputs to FP32 either with host threads
    (CTRECON_OPT_HOST_THREADS > 0, default: slots of 64 views copied up as they are converted)
    or on the device (0), and the filter's results for a pageable array come down in FP32 and
    are widened by host threads; the casts round alike and widening is exact, so
    ctrecon_recon_host_f64's image, ctrecon_filter_host_f64's FProj and ctrecon_bkproj_host_f64's
    image are the same bit for bit, for thread counts that do and do not divide a slot, pinned
    and pageable arrays, on repeated calls."""
    torch = torch_mod
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import config, small_config
    s = config("c1") if cfg == "c1" else small_config(name="tiny")
    with ct.Context(0) as cx:
        assert cx.get_option(_lib.OPT_HOST_THREADS) == -1
        d = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
        cx.phantom_dev(s.geom_struct(), s.ellipsoids(), d)
        torch.cuda.synchronize()
        proj = d.cpu().numpy().astype(np.float64)
        proj_pin = torch.from_numpy(proj).pin_memory().numpy()
        p = ct.scan_filter_params(s)
        out, fout, bout = {}, {}, {}
        f_pin = torch.empty(proj.shape, dtype=torch.float64).pin_memory().numpy()
        for th in (0, -1, 1, 3, 7, 16):
            cx.set_option(_lib.OPT_HOST_THREADS, th)
            assert cx.get_option(_lib.OPT_HOST_THREADS) == th
            for src in (proj, proj_pin):
                for _ in range(2):
                    img = np.full(s.vol_shape, 7.25)
                    cx.recon_host(p, s.geom_struct(), src, img)
                    out.setdefault(th, img)
                    assert np.array_equal(img, out[th]), th
            for f in (np.empty_like(proj), f_pin):
                for _ in range(2):
                    f[...] = -1.0
                    cx.filter_host(p, proj_pin if f is f_pin else proj, f)
                    fout.setdefault(th, f.copy())
                    assert np.array_equal(f, fout[th]), th
                    img = np.full(s.vol_shape, 7.25)
                    cx.bkproj_host(s.geom_struct(), f, img)
                    bout.setdefault(th, img)
                    assert np.array_equal(img, bout[th]), th
        for th in out:
            assert np.array_equal(out[th], out[0]), th
            assert np.array_equal(fout[th], fout[0]), th
            assert np.array_equal(bout[th], bout[0]), th
        with pytest.raises(_lib.CtreconError):
            cx.set_option(_lib.OPT_HOST_THREADS, -2)


def test_host_bkproj_fifth_form(torch_mod):
    """The host backprojection accumulates ~2048-view windows; with the fifth form each
    window's cell records are built for that window only."""
    torch = torch_mod
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import config
    s = config("c1")
    with ct.Context(0) as cx:
        d = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
        cx.phantom_dev(s.geom_struct(), s.ellipsoids(), d)
        torch.cuda.synchronize()
        f = cx.filter_host(ct.scan_filter_params(s), d.cpu().numpy().astype(np.float64))
        imgs = {}
        for var in (100, 10):
            cx.set_option(_lib.OPT_BP_VARIANT, var)
            img = np.full(s.vol_shape, 7.25)
            cx.bkproj_host(s.geom_struct(), f, img)
            imgs[var] = img
    written = imgs[100] != 7.25
    assert np.array_equal(written, imgs[10] != 7.25)
    rel = np.linalg.norm(imgs[10][written] - imgs[100][written]) / np.linalg.norm(imgs[100][written])
    print(f"host backprojection, fifth form vs first form: rel diff {rel:.2e}")
    assert rel < 1e-6


@pytest.mark.parametrize("hilbert", ["fp32", "bf16x3", "tf32"])
def test_filter_chunk_size_does_not_change_the_result(torch_mod, hilbert):
    """The filter works through the views in chunks (CTRECON_OPT_FILTER_CHUNK, default 2048) with
    a kappa-row buffer sized to the call; every view is filtered independently, so any chunk
    size -- one that does not divide the view count, one larger than it -- gives the same bits."""
    torch = torch_mod
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import config
    mode = {"fp32": _lib.HILBERT_FP32, "bf16x3": _lib.HILBERT_BF16X3,
            "tf32": _lib.HILBERT_TF32}[hilbert]
    s = config("c1")  # 2160 views
    with ct.Context(0, hilbert=mode) as cx:
        assert cx.get_option(_lib.OPT_FILTER_CHUNK) == 2048
        d = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
        cx.phantom_dev(s.geom_struct(), s.ellipsoids(), d)
        p = ct.scan_filter_params(s)
        outs = []
        for chunk in (2048, 97, 5000):
            cx.set_option(_lib.OPT_FILTER_CHUNK, chunk)
            f = torch.full_like(d, 7.25)
            cx.filter_dev(p, d, f)
            outs.append(f)
        torch.cuda.synchronize()
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
    assert not bool(torch.any(outs[0] == 7.25))
