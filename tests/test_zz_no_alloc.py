"""The filter entry point that allocates nothing (collected last on purpose).

ctrecon_filter_noalloc_dev_f32 serves callers that cannot call cudaMalloc (a plug-in whose host
application owns every device allocation, a real-time loop that forbids allocation after
start-up): its tables and scratch live in a fixed device array of the library. This test calls
it through the C ABI, twice in a row (the second call reuses the array the first one left
behind), and compares both results with the regular ctrecon_filter_dev_f32 on the same input,
within the filter tolerance of the other parity tests. It checks that the device's free memory
does not move across calls once the array and the kernels are loaded, that a scan too large for
the fixed array is refused with a clear error instead of running, and that a stream under
capture is refused without breaking the capture.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_noalloc_filter_matches_allocating_filter_twice():
    torch = _cuda()
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import config, small_config

    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    cases = []
    for s in (small_config(), config("c1")):
        p = ct.scan_filter_params(s)
        d_proj = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
        with ct.Context(0) as cx:
            cx.phantom_dev(s.geom_struct(), s.ellipsoids(), d_proj)
            d_ref = torch.empty_like(d_proj)
            cx.filter_dev(p, d_proj, d_ref)
        torch.cuda.synchronize()
        ref = d_ref.cpu().numpy().astype(np.float64)
        del d_ref
        cases.append((s, p, d_proj, torch.empty_like(d_proj), ref))

    def call(p, d_proj, d_out):
        st = L.ctrecon_filter_noalloc_dev_f32(stream, ctypes.byref(p), d_proj.data_ptr(),
                                              d_out.data_ptr())
        assert st == _lib.OK, L.ctrecon_last_error(None)
        assert L.ctrecon_last_error(None) == b"", "a successful call leaves no error message"

    for rnd in range(2):
        for s, p, d_proj, d_out, ref in cases:
            d_out.fill_(float("nan"))
            call(p, d_proj, d_out)
            torch.cuda.synchronize()
            out = d_out.cpu().numpy().astype(np.float64)
            assert np.all(np.isfinite(out)), f"{s.name} call {rnd}: unwritten outputs"
            err = _rel(out, ref)
            print(f"no-alloc filter {s.name} call {rnd}: rel diff {err:.3e}")
            assert err < 1e-5

    # once the array and the kernels are loaded, calls take no device memory at all
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for s, p, d_proj, d_out, ref in cases + cases[:1]:
        call(p, d_proj, d_out)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, f"device free memory moved by {free0 - free1} bytes across calls"


def test_noalloc_filter_rejects_scans_beyond_its_scratch():
    torch = _cuda()
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import config

    L = _lib.lib()
    # 2048 x 256 detector: the tables alone (19 MB) exceed the 16 MiB array
    p = ct.scan_filter_params(config("c5").with_(YL=2048, pitch_u=0.375))
    small = torch.zeros(16, dtype=torch.float32, device="cuda")
    st = L.ctrecon_filter_noalloc_dev_f32(torch.cuda.current_stream().cuda_stream,
                                          ctypes.byref(p), small.data_ptr(),
                                          small.data_ptr() + 4)
    assert st == _lib.ERR_UNSUPPORTED
    msg = L.ctrecon_last_error(None).decode()
    assert "too large" in msg and "16777216" in msg


def test_noalloc_filter_refuses_a_capturing_stream():
    torch = _cuda()
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import small_config

    L = _lib.lib()
    s = small_config()
    p = ct.scan_filter_params(s)
    d_proj = torch.zeros(s.proj_shape, dtype=torch.float32, device="cuda")
    d_out = torch.full_like(d_proj, 3.0)
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=side):
        st = L.ctrecon_filter_noalloc_dev_f32(side.cuda_stream, ctypes.byref(p),
                                              d_proj.data_ptr(), d_out.data_ptr())
        d_out.add_(1.0)  # the capture itself goes on: this op is recorded
    assert st == _lib.ERR_UNSUPPORTED
    assert b"captured" in L.ctrecon_last_error(None)
    g.replay()
    torch.cuda.synchronize()
    assert bool((d_out == 4.0).all()), "the refused call enqueued work or broke the capture"
    del g
