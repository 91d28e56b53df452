"""FilteringMode 1 of the reference's driver (FunctionKat_v6.m:86-90): FProj is the mean of the
filters with FilterCoeFF and 1 - FilterCoeFF. Against two device filters and against the FP64
oracle's two filters averaged (bound 1e-5, the FP32 filter's bar)."""
import numpy as np
import pytest

from conftest import oracle_filter_params, rel_rmse

pytestmark = pytest.mark.gpu


def test_filter_mode1(oracle_mod):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctrecon_b200 as ct
    from ctrecon_b200.geometry import small_config
    s = small_config(filter_coeff=0.3)
    O = oracle_mod
    proj = O.project_ellipsoids(O.bp_geom(s.locus(), s.detector(), s.object()), s.ellipsoids())
    fp0 = oracle_filter_params(O, s)
    fp1 = oracle_filter_params(O, s)
    fp1.FilterCoeFF = 1.0 - fp0.FilterCoeFF
    want = 0.5 * (O.katsevich_filter(fp0, proj) + O.katsevich_filter(fp1, proj))
    p = ct.scan_filter_params(s)
    q = ct.scan_filter_params(s)
    q.filter_coeff = 1.0 - p.filter_coeff
    with ct.Context(0) as cx:
        d = torch.from_numpy(proj.astype(np.float32)).cuda()
        out = torch.empty_like(d)
        cx.filter_mode1_dev(p, d, out)
        a, b = torch.empty_like(d), torch.empty_like(d)
        cx.filter_dev(p, d, a)
        cx.filter_dev(q, d, b)
        torch.cuda.synchronize()
        assert torch.equal(out, (a + b) / 2)
        got = out.cpu().numpy()
    err = rel_rmse(got, want)
    print(f"FilteringMode 1 (tau {p.filter_coeff}): rel RMSE {err:.2e}")
    assert err < 1e-5
