"""The benchmarked forms against the FP64 oracle on central blocks of the benchmark scans.

Scans: c2 (512 x 512 x 256 at 0.4 mm, 64 x 736 detector, 9280 views, Poisson noise) and c3
(512^3, 128 x 1024 detector, 13824 views), both projected on the device by the FP64 analytic
projector. The oracle (FP64) filters the views a central 48^3 block needs and backprojects the
block with orc_bkproj, which equals the reference's KatsevichBkProj.cpp bit for bit.

* Backprojector alone: every form the autotuner picks from -- the fifth form (variants 10 and 12:
  cell records in device memory, footprints brought in by tensor copies) -- and the second form
  (variant 2, the default before tuning) and the first form (100), each fed the oracle's own
  filtered views rounded to FP32, against the oracle's block. 87 % (c2) and 96 % (c3) of the
  block's tile-views take the fifth form's tensor-copy path, the rest (footprints reaching the
  top or bottom detector row) its direct reads (counted in tests/test_footprint.py).
* Whole chain on the device, as the benchmark runs it: the full scan filtered on the GPU, the PI
  lines solved, the block backprojected by variant 12, in the plain form (FP32 Hilbert,
  bisection) and the mixed + learned form (BF16x3 Hilbert, the learned start on its grid, Newton,
  bisection replay), against the oracle's chain.
Bars: relative RMSE over the voxels the reference writes, 1e-5 for FP32 arithmetic and 1e-4 for
BF16x3 + learned (the metric's bar); max-abs is printed; the voxels the reference leaves alone
keep their value bit for bit.
"""
import numpy as np
import pytest

from conftest import central_block, max_abs, oracle_filter_params, rel_rmse

pytestmark = pytest.mark.gpu

SENTINEL = -5.5
N = 48


@pytest.fixture(scope="module")
def torch_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module", params=["c2", "c3"])
def block_case(request, torch_mod, oracle_mod):
    torch = torch_mod
    import ctrecon_b200 as ct
    from ctrecon_b200.geometry import config
    O = oracle_mod
    s = config(request.param)
    locus, det, obj, lo, hi = central_block(O, s, N)
    ctx = ct.Context(0)
    d_proj = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
    ctx.phantom_dev(s.geom_struct(), s.ellipsoids(), d_proj, photons=s.photons or 0.0,
                    seed=s.seed)
    torch.cuda.synchronize()
    # the oracle's filter of views lo-1 .. hi (the outer two only as derivative neighbours)
    a, b = max(0, lo - 1), min(s.P, hi + 1)
    proj_b = d_proj[a:b].cpu().numpy().astype(np.float64)
    fp = oracle_filter_params(O, s)
    fp.ProjNumber = b - a
    ref_f = np.ascontiguousarray(O.katsevich_filter(fp, proj_b)[lo - a:hi - a])
    gb = O.bp_geom(locus, det, obj, honour_extras=True)
    ref_img, n_upd, touched = O.bkproj(gb, ref_f, np.full((N, N, N), SENTINEL),
                                       want_touched=True)
    block = {"Locus": np.array(locus), "Detector": np.array(det), "Object": np.array(obj)}
    yield dict(s=s, ctx=ctx, d_proj=d_proj, lo=lo, hi=hi, block=block, ref_f=ref_f,
               ref_img=ref_img, touched=touched.astype(bool), n_upd=n_upd)
    ctx.close()


def _bp(torch, ctx, block, d_f, variant, solver=None):
    from ctrecon_b200 import _lib
    ctx.set_option(_lib.OPT_BP_VARIANT, variant)
    if solver is not None:
        ctx.set_option(_lib.OPT_PI_SOLVER, solver)
    d_img = torch.full((N, N, N), SENTINEL, dtype=torch.float32, device="cuda")
    ctx.bkproj_dev(block, d_f, d_img)
    torch.cuda.synchronize()
    return d_img.cpu().numpy().astype(np.float64)


def _check(name, got, c, bound):
    t = c["touched"]
    ref = c["ref_img"]
    assert t.sum() > 0.3 * t.size
    assert np.array_equal(got[~t], ref[~t]), f"{name}: voxels outside the PI set changed"
    err, mx = rel_rmse(got, ref, t), max_abs(got, ref, t)
    print(f"{c['s'].name} block {name}: rel RMSE {err:.2e}, max-abs {mx:.2e} "
          f"(of {np.abs(ref[t]).max():.3e}), {int(t.sum())} voxels, {c['n_upd']} updates")
    assert err < bound, (name, err)


@pytest.mark.parametrize("variant", [12, 10, 2, 100])
def test_block_backprojector_forms_match_oracle(torch_mod, block_case, variant):
    torch = torch_mod
    from ctrecon_b200 import _lib
    c = block_case
    d_f = torch.from_numpy(c["ref_f"].astype(np.float32)).cuda()
    got = _bp(torch, c["ctx"], c["block"], d_f, variant, _lib.PI_BISECT)
    # FP32 filtered input (one rounding) and FP32 interpolation / accumulation
    _check(f"backprojector variant {variant}", got, c, 1e-5)


@pytest.mark.parametrize("form", ["plain", "mixed_learned"])
def test_block_chain_matches_oracle(torch_mod, block_case, form):
    torch = torch_mod
    import ctypes
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    c = block_case
    s, ctx = c["s"], c["ctx"]
    if form == "plain":
        ctx.set_option(_lib.OPT_HILBERT, _lib.HILBERT_FP32)
        solver, bound = _lib.PI_BISECT, 1e-5
    else:
        ctx.set_option(_lib.OPT_HILBERT, _lib.HILBERT_BF16X3)
        loss = ctypes.c_float()
        _lib.check(_lib.lib().ctrecon_pinet_train(
            ctx.handle, torch.cuda.current_stream().cuda_stream, 1 << 19, 4096, 6,
            s.ObjR / s.ScanR * 1.05, 11, ctypes.byref(loss)), ctx.handle)
        ctx.set_option(_lib.OPT_PINET_MODE, _lib.PINET_GRID)
        solver, bound = _lib.PI_LEARNED, 1e-4
    d_f = torch.empty_like(c["d_proj"])
    ctx.filter_dev(ct.scan_filter_params(s), c["d_proj"], d_f)
    got = _bp(torch, ctx, c["block"], d_f[c["lo"]:c["hi"]].contiguous(), 12, solver)
    ctx.set_option(_lib.OPT_HILBERT, _lib.HILBERT_FP32)
    del d_f
    _check(f"chain {form}", got, c, bound)
