"""Batched reconstruction of uneven scans (one persistent backprojection launch, CUDA graph).

The batch runs the same per-tile code as the single-scan path, so every scan's image must
equal the one-at-a-time result exactly, in the eager first run and in graph replays.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scans():
    from ctrecon_b200.geometry import small_config
    return [small_config(name="b0"),
            small_config(name="b1", YL=80, ZL=12, views_per_turn=150, turns=2.5, NX=40, NY=36,
                         NZ=12, seed=3),
            small_config(name="b2", YL=48, ZL=8, views_per_turn=120, turns=4, NX=24, NY=24,
                         NZ=20, seed=4)]


@pytest.mark.parametrize("variant", [0, 2, 5, 7, 10, 12])
def test_batch_equals_single_scans(variant):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    scans = _scans()
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream), ct.Context(0) as cx:
        cx.set_option(_lib.OPT_BP_VARIANT, variant)
        projs, singles = [], []
        for s in scans:
            d = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
            cx.phantom_dev(s.geom_struct(), s.ellipsoids(), d)
            projs.append(d)
            f = torch.empty_like(d)
            cx.filter_dev(ct.scan_filter_params(s), d, f)
            img = torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
            cx.bkproj_dev(s.geom_struct(), f, img)
            singles.append(img)
        b = ct.Batch(cx, scans)
        b.set_variant(variant)
        fprojs = [torch.empty_like(d) for d in projs]
        for rnd in range(3):  # eager, captured, replayed
            imgs = [torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
                    for s in scans]
            b.run(projs, fprojs, imgs, use_graph=True)
            stream.synchronize()
            for s, a, ref in zip(scans, imgs, singles):
                assert torch.equal(a, ref), f"{s.name} run {rnd}"
        counts = b.updates()
        assert all(c > 0 for c in counts)
        b.close()


def test_batch_with_per_scan_forms():
    """Scans with different backprojector forms: one persistent launch per form, every image
    equal to its single-scan backprojection with that form, eager and replayed."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    scans = _scans()
    forms = [10, 2, 9][:len(scans)]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream), ct.Context(0) as cx:
        projs, singles = [], []
        for s, v in zip(scans, forms):
            cx.set_option(_lib.OPT_BP_VARIANT, v)
            d = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
            cx.phantom_dev(s.geom_struct(), s.ellipsoids(), d)
            projs.append(d)
            f = torch.empty_like(d)
            cx.filter_dev(ct.scan_filter_params(s), d, f)
            img = torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
            cx.bkproj_dev(s.geom_struct(), f, img)
            singles.append(img)
        b = ct.Batch(cx, scans)
        b.set_variants(forms)
        assert b.variants() == forms
        fprojs = [torch.empty_like(d) for d in projs]
        for rnd in range(3):
            imgs = [torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
                    for s in scans]
            b.run(projs, fprojs, imgs, use_graph=True)
            stream.synchronize()
            for s, a, ref in zip(scans, imgs, singles):
                assert torch.equal(a, ref), f"{s.name} run {rnd}"
        b.close()
