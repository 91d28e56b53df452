"""The analytic projectors against the reference's own projector, CreateProjSlice.cpp:26-141,
compiled unchanged from the CTRecon sources against the project's mex.h shim (oracle/_ref).

CreateProjSlice projects its built-in head phantom (CreateProjSlice.cpp:13-24, in units of the
object radius) for one source angle onto a flat detector through the rotation axis, as
FunctionKat_v6.m:73 calls it. The same rays are the oracle's projector (and the library's FP64
CUDA projector, csrc/phantom.cu) with StdDis = ScanR, which puts the flat detector through the
axis, and the head phantom written as ellipsoids rotated about z.

CPU: the oracle's projector against the reference on every view of a short scan.
GPU (marked): csrc/phantom.cu (FP64 arithmetic, FP32 output) against the reference.
"""
import numpy as np
import pytest

PI = 3.14159265358979  # CreateProjSlice.cpp:12


def _scan():
    """A normalised scan in the driver's units (FunctionKat_v6.m:49-57): ObjR = 1, ScanR = 5,
    a 300 x 40 detector (the driver's TestKatsevich size), 768 views per turn; views far from
    the centre of the helix so that the source height is not 0."""
    from ctrecon_b200.geometry import katsevich_sizing
    R, H, YL, ZL, Ps, P = 5.0, 1.1, 300, 40, 768, 48
    DW, DH, _ = katsevich_sizing(R, R, H, 1.0, YL, ZL)
    locus = [R, R, H, float(Ps), 1.0, float(P), -150.5]
    detector = [DW, float(YL), DH, float(ZL), (YL - 1) / 2.0, (ZL - 1) / 2.0]
    obj = [1.0, 8.0, 8.0, 8.0]
    return locus, detector, obj


def _reference_views(O, locus, detector):
    R, _, H, Ps, beg, end, ctr = locus
    DW, YL, DH, ZL = detector[:4]
    out = []
    for p in range(int(end - beg + 1)):
        theta = (p + int(beg) - ctr) * (2 * PI / Ps)  # the projectors' own view angle
        out.append(O.ref_create_proj_slice(theta, R, H, int(YL), int(ZL), DW, DH))
    return np.stack(out)


@pytest.fixture(scope="module")
def ref_views(oracle_mod):
    O = oracle_mod
    if not O.ref_projslice_available():
        pytest.skip("oracle/_ref not built (needs the CTRecon sources)")
    locus, detector, obj = _scan()
    return _reference_views(O, locus, detector)


def test_oracle_projector_matches_reference_head_phantom(oracle_mod, ref_views):
    O = oracle_mod
    locus, detector, obj = _scan()
    got = O.project_ellipsoids(O.bp_geom(locus, detector, obj), O.head_phantom_ellipsoids())
    ref = ref_views
    assert got.shape == ref.shape
    assert np.count_nonzero(ref) > 0.5 * ref.size  # the phantom fills most of the detector
    rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    mx = float(np.abs(got - ref).max())
    print(f"oracle projector vs CreateProjSlice.cpp: rel RMSE {rel:.2e}, max-abs {mx:.2e} "
          f"of {np.abs(ref).max():.3f}")
    assert rel < 1e-12
    assert mx < 1e-10 * np.abs(ref).max()


@pytest.mark.gpu
def test_cuda_projector_matches_reference_head_phantom(oracle_mod, ref_views):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctrecon_b200 as ct
    locus, detector, obj = _scan()
    geom = {"Locus": np.array(locus), "Detector": np.array(detector), "Object": np.array(obj)}
    d = torch.empty(ref_views.shape, dtype=torch.float32, device="cuda")
    with ct.Context(0) as cx:
        cx.phantom_dev(geom, oracle_mod.head_phantom_ellipsoids(), d)
        torch.cuda.synchronize()
    got = d.cpu().numpy().astype(np.float64)
    ref = ref_views
    rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    mx = float(np.abs(got - ref).max())
    print(f"phantom.cu vs CreateProjSlice.cpp: rel RMSE {rel:.2e}, max-abs {mx:.2e}")
    # FP64 arithmetic, FP32 storage: one rounding of each line integral
    assert rel < 1e-7
    assert mx < 2e-7 * np.abs(ref).max()
