"""The autotuner (ctrecon_tune_bkproj, ctrecon_batch_tune, the tuning table) on a B200.

Tuning times every candidate backprojector form on the caller's data; whatever it picks, the
image must be exactly what that form computes on its own, the table must survive a save/load
round trip, and CTRECON_BP_AUTO must use it.
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


def test_tune_single_scan_and_table(torch_mod, tmp_path):
    torch = torch_mod
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import config
    s = config("c1")
    g = s.geom_struct()
    with ct.Context(0) as cx:
        d_proj = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
        cx.phantom_dev(g, s.ellipsoids(), d_proj)
        d_f = torch.empty_like(d_proj)
        cx.filter_dev(ct.scan_filter_params(s), d_proj, d_f)
        img_t = torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
        res = cx.tune_bkproj(g, d_f, img_t)
        torch.cuda.synchronize()
        print("tuning:", res)
        best = res["best_variant"]
        assert best in res["ms"] and res["best_ms"] > 0
        assert res["best_ms"] == min(v for v in res["ms"].values() if v >= 0)
        # the tuned image is the chosen form's image
        cx.set_option(_lib.OPT_BP_VARIANT, best)
        img_b = torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
        cx.bkproj_dev(g, d_f, img_b)
        torch.cuda.synchronize()
        assert torch.equal(img_t, img_b)
        # AUTO uses the table
        cx.set_option(_lib.OPT_BP_VARIANT, _lib.BP_AUTO)
        img_a = torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
        cx.bkproj_dev(g, d_f, img_a)
        torch.cuda.synchronize()
        assert torch.equal(img_a, img_b)
        path = str(tmp_path / "tune.txt")
        cx.tune_save(path)
    text = open(path).read()
    assert f" {best} " in text
    with ct.Context(0) as cx2:
        cx2.tune_load(path)
        cx2.set_option(_lib.OPT_BP_VARIANT, _lib.BP_AUTO)
        d_f2 = d_f.clone()
        img_l = torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
        cx2.bkproj_dev(g, d_f2, img_l)
        torch.cuda.synchronize()
        assert torch.equal(img_l, img_b)
        with pytest.raises(ct.CtreconError):
            cx2.set_option(_lib.OPT_BP_VARIANT, 42)


def test_batch_tune_keeps_results(torch_mod):
    torch = torch_mod
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import small_config
    scans = [small_config(name="t0"),
             small_config(name="t1", YL=80, ZL=12, views_per_turn=150, turns=2.5, NX=40, NY=36,
                          NZ=12, seed=3)]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream), ct.Context(0) as cx:
        projs, fprojs, imgs = [], [], []
        for s in scans:
            d = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
            cx.phantom_dev(s.geom_struct(), s.ellipsoids(), d)
            projs.append(d)
            fprojs.append(torch.empty_like(d))
            imgs.append(torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda"))
        b = ct.Batch(cx, scans)
        res = b.tune(projs, fprojs, imgs, stream=stream)
        print("batch tuning:", res)
        per_scan = res["per_scan"]
        assert len(per_scan) == len(scans) and all(v in res["ms"] for v in per_scan)
        assert res["best_ms"] > 0 and res["best_variant"] in per_scan
        # a graph-replayed run with the tuned forms equals single scans with each scan's form
        for _ in range(3):
            b.run(projs, fprojs, imgs, stream=stream, use_graph=True)
        singles = []
        for s, d, v in zip(scans, projs, per_scan):
            cx.set_option(_lib.OPT_BP_VARIANT, v)
            f = torch.empty_like(d)
            cx.filter_dev(ct.scan_filter_params(s), d, f)
            img = torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
            cx.bkproj_dev(s.geom_struct(), f, img)
            singles.append(img)
        stream.synchronize()
        for a, w in zip(imgs, singles):
            assert torch.equal(a, w)
        b.close()
