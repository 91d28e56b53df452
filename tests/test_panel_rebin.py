"""Arc-to-flat detector rebin (rebinToPanel.m:1-36).

CPU: the C oracle (oracle/katsevich_oracle.c::orc_rebin_to_panel) against a literal Python
transcription of the MATLAB loop (1-based indices, the clamps in the reference's order).
GPU: the library's FP64 kernel equals the oracle bit for bit; the FP32 kernel within 1e-6.
"""
import math

import numpy as np
import pytest

CASES = [  # (det_num, centre index 0-based, cell width, source-to-detector distance)
    (9, 4.0, 1.0, 1000.0),          # symmetric, odd: the centre column lands on a cell centre
    (16, 7.5, 1.0, 946.0),          # symmetric, even
    (33, 13.25, 1.0239, 946.0),     # off-centre (the larger half-fan sets the panel width)
    (64, 40.6, 0.8, 600.0),
]


def _matlab_transcription(proj, c, w, D):
    """rebinToPanel.m, statement by statement, on MATLAB-shaped (det_num, det_hei, prj_num)."""
    detNum, detHei, prjNum = proj.shape
    oneFanAngle = math.atan(w / 2 / D) * 2.0
    largerAngle = max((c + 0.5) * oneFanAngle, (detNum - 1 - c + 0.5) * oneFanAngle)
    detWidth = math.tan(largerAngle) * D * 2
    newDetCellWidth = detWidth / detNum
    out = np.zeros(proj.shape)
    for ii in range(1, detNum + 1):
        fanAngle = math.atan((ii - (detNum + 1) / 2) * newDetCellWidth / D)
        idx = fanAngle / oneFanAngle + c + 1
        lowIdx = math.floor(idx)
        higIdx = math.ceil(idx)
        if lowIdx < 1:
            lowIdx = 1
        if higIdx < 1:
            continue
        if lowIdx > detNum:
            continue
        if higIdx > detNum:
            higIdx = detNum
        lowVal = proj[lowIdx - 1, :, :]
        higVal = proj[higIdx - 1, :, :]
        out[ii - 1, :, :] = lowVal * (higIdx - idx) + higVal * (idx - lowIdx)
    return out, detWidth


def _input(n, seed=0):
    return np.random.default_rng(seed).standard_normal((3, 4, n))  # (prj_num, det_hei, det_num)


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_the_matlab_loop(oracle_mod, case):
    n, c, w, D = case
    proj = _input(n)
    out, width = oracle_mod.rebin_to_panel(proj, c, w, D)
    ref, ref_width = _matlab_transcription(np.transpose(proj), c, w, D)
    assert width == ref_width
    assert np.array_equal(out, np.transpose(ref))
    if n == 9:  # the reference's quirk: the centre column sits exactly on a cell centre
        assert np.all(out[:, :, 4] == 0)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_gpu_panel_rebin_matches_oracle(oracle_mod, case):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctrecon_b200 as ct
    n, c, w, D = case
    proj = _input(n, seed=n)
    ref, ref_width = oracle_mod.rebin_to_panel(proj, c, w, D)
    with ct.Context(0) as cx:
        d64 = torch.from_numpy(proj).cuda()
        o64 = torch.empty_like(d64)
        width = cx.rebin_to_panel_dev(d64, c, w, D, o64)
        d32 = d64.float()
        o32 = torch.empty_like(d32)
        cx.rebin_to_panel_dev(d32, c, w, D, o32)
        torch.cuda.synchronize()
        got64, got32 = o64.cpu().numpy(), o32.cpu().numpy().astype(np.float64)
    assert width == ref_width
    assert np.array_equal(got64, ref)
    err = np.linalg.norm(got32 - ref) / np.linalg.norm(ref)
    print(f"panel rebin N={n}: FP32 rel. error {err:.2e}")
    assert err < 1e-6
