"""Failure detection on the GPU without a GPU fault (needs a B200).

Every pipelined kernel bounds its mbarrier waits; a wait that gives up records a code in the
context's device error word and returns, so a stalled pipeline becomes CTRECON_ERR_TIMEOUT on
the host instead of a hung GPU. The self-test entry point runs that wait (tc_util.cuh:
mbar_wait) on a barrier nothing ever arrives on, with a 50 ms limit: it must give up, be
reported, and leave the context usable.
"""
import ctypes
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_is_reported():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import small_config
    L = _lib.lib()
    with ct.Context(0) as cx:
        t0 = time.perf_counter()
        rc = L.ctrecon_selftest_bounded_wait(cx.handle, None, 50)
        dt = time.perf_counter() - t0
        msg = L.ctrecon_last_error(cx.handle).decode()
        print(f"self-test: status {rc} after {dt * 1e3:.0f} ms: {msg}")
        assert rc == _lib.ERR_TIMEOUT
        assert "code 99" in msg
        assert dt < 5.0
        # out-of-range limits are argument errors, not launches
        assert L.ctrecon_selftest_bounded_wait(cx.handle, None, 0) == _lib.ERR_INVALID_ARGUMENT
        # the context is still usable: a reconstruction runs and reports no error
        s = small_config()
        d = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
        cx.phantom_dev(s.geom_struct(), s.ellipsoids(), d)
        f = torch.empty_like(d)
        cx.filter_dev(ct.scan_filter_params(s), d, f)
        img = torch.zeros(s.vol_shape, dtype=torch.float32, device="cuda")
        cx.bkproj_dev(s.geom_struct(), f, img)
        torch.cuda.synchronize()
        assert np.isfinite(img.cpu().numpy()).all() and float(img.abs().sum()) > 0
