"""PI-line solvers and the learned initialiser on the GPU.

* Newton (closed-form derivative), followed by the bisection replayed from its root, gives the
  bisection arbiter's PI records bit for bit on every voxel (c2 included: 6.7e7 voxels);
* the network's loss gradient from the CUDA training kernel equals the FP64 CPU reference
  (oracle/pinet_oracle.py) at the same parameters;
* after training on the GPU, the BF16 inference kernel matches the FP64 forward pass, and the
  learned start saves Newton iterations while giving the bisection's PI records bit for bit.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _pi(ctx, torch, scan, solver):
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    ctx.set_option(_lib.OPT_PI_SOLVER, solver)
    g = ct.bp_geom(scan.geom_struct())
    d_tab = torch.empty(ctx.pi_table_bytes(g), dtype=torch.uint8, device="cuda")
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    d_its = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = _lib.lib().ctrecon_pi_dev_stats(ctx.handle, torch.cuda.current_stream().cuda_stream,
                                         ctypes.byref(g), d_tab.data_ptr(), d_cnt.data_ptr(),
                                         d_its.data_ptr())
    _lib.check(st, ctx.handle)
    torch.cuda.synchronize()
    rec = d_tab.cpu().numpy().view(np.int32).reshape(-1, 4)
    valid = rec[:, 0] != 0x7FFFFFFF
    return dict(rec=rec, valid=valid, count=int(d_cnt.item()), iters=int(d_its.item()))


def _same_records(a, b, what):
    """The PI records (Bindex, B fraction, Tindex - 1, T fraction) of two solvers, bit for bit."""
    diff = np.any(a["rec"] != b["rec"], axis=1)
    assert not diff.any(), f"{what}: {int(diff.sum())} voxels' records differ from bisection"
    assert a["count"] == b["count"]


@pytest.mark.parametrize("case", ["tiny", "c1", "c2"])
def test_newton_matches_bisection(torch_mod, case):
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import config, small_config
    s = small_config() if case == "tiny" else config(case)
    with ct.Context(0) as cx:
        bis = _pi(cx, torch_mod, s, _lib.PI_BISECT)
        newt = _pi(cx, torch_mod, s, _lib.PI_NEWTON)
    _same_records(newt, bis, f"{case} Newton")
    n = int(bis["valid"].sum())
    print(f"{case}: records identical over {n} voxels; chord evaluations/voxel bisection "
          f"{bis['iters'] / n:.2f}, Newton + replay {newt['iters'] / n:.2f}")
    assert newt["iters"] < bis["iters"] / 3


def test_pinet_gradient_matches_fp64_reference(torch_mod):
    torch = torch_mod
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    import pinet_oracle as PO
    L = _lib.lib()
    n = L.ctrecon_pinet_num_params()
    assert n == PO.n_params()
    rng = np.random.default_rng(5)
    theta = np.zeros(n)
    o = 0
    for i in range(5):
        fi, fo = PO.SIZES[i], PO.SIZES[i + 1]
        theta[o: o + fo * fi] = rng.uniform(-1, 1, fo * fi) * np.sqrt(3.0 / fi)
        o += fo * fi
        theta[o: o + fo] = rng.uniform(-0.1, 0.1, fo)
        o += fo
    theta32 = theta.astype(np.float32)
    B = 1000
    X = np.column_stack([rng.random(B), np.cos(2 * np.pi * rng.random(B)),
                         np.sin(2 * np.pi * rng.random(B))]).astype(np.float32)
    Y = rng.uniform(-1, 1, (B, 2)).astype(np.float32)
    with ct.Context(0) as cx:
        st = L.ctrecon_pinet_set_params(cx.handle, theta32.ctypes.data_as(
            ctypes.POINTER(ctypes.c_float)), n, 0.25)
        _lib.check(st, cx.handle)
        dX, dY = torch.from_numpy(X).cuda(), torch.from_numpy(Y).cuda()
        dG = torch.zeros(n, dtype=torch.float32, device="cuda")
        dL = torch.zeros(1, dtype=torch.float32, device="cuda")
        st = L.ctrecon_pinet_loss_grad(cx.handle, torch.cuda.current_stream().cuda_stream,
                                       dX.data_ptr(), dY.data_ptr(), B, dG.data_ptr(),
                                       dL.data_ptr())
        _lib.check(st, cx.handle)
        torch.cuda.synchronize()
    loss_ref, g_ref = PO.loss_and_grad(theta32.astype(np.float64), X.astype(np.float64),
                                       Y.astype(np.float64))
    g = dG.cpu().numpy().astype(np.float64)
    rel = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    print(f"gradient rel. error {rel:.2e}, loss {float(dL.item()):.6f} vs {loss_ref:.6f}")
    assert abs(float(dL.item()) - loss_ref) < 1e-4 * max(1.0, loss_ref)
    assert rel < 1e-4


def test_pinet_training_inference_and_gain(torch_mod):
    torch = torch_mod
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import config
    import pinet_oracle as PO
    L = _lib.lib()
    s = config("c1")
    with ct.Context(0) as cx:
        loss = ctypes.c_float()
        st = L.ctrecon_pinet_train(cx.handle, torch.cuda.current_stream().cuda_stream, 1 << 18,
                                   4096, 6, s.ObjR / s.ScanR * 1.05, 7, ctypes.byref(loss))
        _lib.check(st, cx.handle)
        print(f"training loss {loss.value:.3e}")
        assert loss.value < 2e-3
        n = L.ctrecon_pinet_num_params()
        theta = np.zeros(n, np.float32)
        _lib.check(L.ctrecon_pinet_get_params(cx.handle, theta.ctypes.data_as(
            ctypes.POINTER(ctypes.c_float)), n), cx.handle)
        # BF16 inference kernel against the FP64 forward pass with the same (rounded) weights
        rng = np.random.default_rng(9)
        m = 4096
        r = 0.2 * np.sqrt(rng.random(m))
        psi = 2 * np.pi * rng.random(m)
        X = np.column_stack([4 * r, np.cos(psi), np.sin(psi)]).astype(np.float32)
        dX = torch.from_numpy(X).cuda()
        dO = torch.zeros((m, 2), dtype=torch.float32, device="cuda")
        _lib.check(L.ctrecon_pinet_predict(cx.handle, torch.cuda.current_stream().cuda_stream,
                                           dX.data_ptr(), m, dO.data_ptr()), cx.handle)
        torch.cuda.synchronize()
        out_ref, _, _ = PO.forward(theta.astype(np.float64), X.astype(np.float64))
        err = np.abs(dO.cpu().numpy() - out_ref).max()
        print(f"inference max |BF16 kernel - FP64 forward| = {err:.3e}")
        assert err < 0.05
        # the learned start in each network mode (per voxel FP32 / packed BF16, and the
        # screw-symmetry grid): same records as the arbiter, fewer Newton steps than the plain start
        bis = _pi(cx, torch, s, _lib.PI_BISECT)
        newt = _pi(cx, torch, s, _lib.PI_NEWTON)
        lrn = {}
        for name, mode in (("voxel-fp32", _lib.PINET_VOXEL_FP32),
                           ("voxel-bf16", _lib.PINET_VOXEL_BF16), ("grid", _lib.PINET_GRID)):
            cx.set_option(_lib.OPT_PINET_MODE, mode)
            lrn[name] = _pi(cx, torch, s, _lib.PI_LEARNED)
    nv = int(bis["valid"].sum())
    for name, r in lrn.items():
        _same_records(r, bis, f"learned start ({name})")
        print(f"Newton iterations/voxel: plain start {newt['iters'] / nv:.2f}, learned start "
              f"({name}) {r['iters'] / nv:.2f}")
        assert r["iters"] < newt["iters"]
    # the grid interpolates the same network: as good a start as evaluating it per voxel
    assert lrn["grid"]["iters"] <= 1.02 * lrn["voxel-fp32"]["iters"]
    # and its points are refined by the FP64 Newton solve, so a voxel's interpolated start is
    # within the 1e-6 rad at which Newton accepts: one Newton evaluation and the replayed
    # bisection's final one per voxel (2.00 measured at c1)
    assert lrn["grid"]["iters"] <= 2.1 * nv


@pytest.mark.parametrize("name", ["c1", "c2s", "ragged"])
def test_backprojector_variants_agree(torch_mod, name):
    """Every tiled form (0, 1: per-cell records; 2-4: second form; 5-9: per-cell records
    staged by producer warps; 10-12: per-cell records copied from device memory) against the
    first form; variant 10 also in windows of 300 views (valid voxels zeroed, then every
    window accumulated); the first, second and fifth forms also against the FP64 oracle.
    c1's 16-row detector sends most tiles through the direct-read fallback, c2s's 64 rows
    almost none; "ragged" has partial tiles in x, y and z (45 x 37 x 13 voxels)."""
    torch = torch_mod
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import config
    if name == "ragged":  # partial tiles in x, y and z; footprints on the cell path
        from ctrecon_b200.geometry import small_config
        s = small_config(name="ragged", YL=200, ZL=48, views_per_turn=120, turns=2.5, NX=45,
                         NY=37, NZ=13, voxel=(0.5, 0.5, 0.5), seed=5)
    else:
        s = config(name)
    outs = {}
    with ct.Context(0) as cx:
        g = s.geom_struct()
        d_proj = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
        cx.phantom_dev(g, s.ellipsoids(), d_proj)
        d_f = torch.empty_like(d_proj)
        cx.filter_dev(ct.scan_filter_params(s), d_proj, d_f)
        for var in (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 100):
            cx.set_option(_lib.OPT_BP_VARIANT, var)
            d_img = torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
            cx.bkproj_dev(g, d_f, d_img)
            torch.cuda.synchronize()
            outs[var] = d_img.cpu().numpy().astype(np.float64)
        cx.set_option(_lib.OPT_BP_VARIANT, 10)
        cx.set_option(_lib.OPT_BP_WINDOW, 300)
        d_img = torch.full(s.vol_shape, 7.25, dtype=torch.float32, device="cuda")
        cx.bkproj_dev(g, d_f, d_img)
        torch.cuda.synchronize()
        outs["10w"] = d_img.cpu().numpy().astype(np.float64)
        fproj = d_f.cpu().numpy().astype(np.float64)
    ref = outs[100]
    for var in (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, "10w"):
        assert np.array_equal(outs[var] == 7.25, ref == 7.25)  # same untouched voxels
        rel = np.linalg.norm(outs[var] - ref) / np.linalg.norm(ref)
        print(f"{name}: variant {var} vs first form: rel diff {rel:.2e}")
        assert rel < 1e-6
    # and each form against the FP64 oracle (KatsevichBkProj.cpp restated, bit for bit) on the
    # same filtered projections
    import oracle as O
    g = O.bp_geom(s.locus(), s.detector(), s.object(), honour_extras=True)
    orc, _, touched = O.bkproj(g, fproj, np.full(s.vol_shape, 7.25), want_touched=True)
    t = touched.astype(bool)
    for var in (100, 2, 10, 12, "10w"):
        assert np.array_equal(outs[var][~t], orc[~t]), f"variant {var}: untouched voxels"
        rel = np.linalg.norm(outs[var][t] - orc[t]) / np.linalg.norm(orc[t])
        mx = np.abs(outs[var][t] - orc[t]).max()
        print(f"{name}: variant {var} vs FP64 oracle: rel RMSE {rel:.2e}, max-abs {mx:.2e}")
        assert rel < 1e-5
