"""The reference's data files (ProjectionData.m, ReconImage.m) through the library's native
readers and writers, checked byte for byte against the numpy restatement of the MATLAB code
(oracle/formats_oracle.py). Host only: no GPU needed."""
import os

import numpy as np
import pytest

from ctrecon_b200 import CtreconError
from ctrecon_b200.formats import ProjectionData, ReconImage
import formats_oracle as F  # oracle/ is on the path (conftest.py)


def _proj(order=(1, 2, 3), seed=0):
    rng = np.random.default_rng(seed)
    U, V, P = 7, 3, 5
    sizes = {"U": U, "V": V, "P": P}
    shape = tuple(reversed([sizes["UVP"[o - 1]] for o in order]))
    return ProjectionData(source_to_center=600.0, source_to_detector=1200.0, det_reso_u=U,
                          det_reso_v=V, det_pixel_u=0.8, det_pixel_v=0.8, det_center_u=3.0,
                          det_center_v=1.0, is_arc=False, start_angle_deg=12.5, start_z=-3.0,
                          pitch=37.98, total_views=P, views_per_turn=4,
                          projection=rng.standard_normal(shape), storage_order=order)


def _proj_header(p):
    vals = (p.source_to_center, p.source_to_detector, p.det_reso_u, p.det_reso_v,
            p.det_pixel_u, p.det_pixel_v, p.det_center_u, p.det_center_v, float(p.is_arc),
            p.start_angle_deg, p.start_z, p.pitch, p.total_views, p.views_per_turn)
    return dict(zip(F.PROJ_FIELDS, vals))


@pytest.mark.parametrize("order", [(1, 2, 3), (2, 1, 3), (3, 1, 2), (1, 3, 2), (2, 3, 1),
                                   (3, 2, 1)])
def test_projection_file_bytes_and_round_trip(tmp_path, order):
    p = _proj(order)
    ours, ref = str(tmp_path / "ours.prj"), str(tmp_path / "ref.prj")
    p.write(ours)
    F.write(ref, _proj_header(p), F.PROJ_FIELDS, p.projection, order)
    assert open(ours, "rb").read() == open(ref, "rb").read()
    q = ProjectionData.read(ref)
    assert q.storage_order == order and q.total_views == 5 and not q.is_arc
    assert np.array_equal(q.projection, p.projection)
    h, data, o = F.read(ours, F.PROJ_FIELDS, F.proj_count)
    assert h == _proj_header(p) and tuple(o) == order


def test_storage_orders_describe_the_same_projections(tmp_path):
    base = _proj((1, 2, 3), seed=3)
    uvp = base.projection                     # numpy (P, V, U)
    m = np.transpose(uvp)                     # MATLAB U x V x P
    for order in [(2, 1, 3), (3, 1, 2), (3, 2, 1)]:
        perm = [o - 1 for o in order]
        stored = np.ascontiguousarray(np.transpose(np.transpose(m, perm)))
        p = _proj(order)
        p.projection = stored
        path = str(tmp_path / f"o{order}.prj")
        p.write(path)
        assert np.array_equal(ProjectionData.read(path).uvp(), uvp)


def test_image_file_bytes_and_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    img = rng.standard_normal((6, 5, 4))      # backprojector layout (NX, NY, NZ), z fastest
    r = ReconImage.from_bkproj(img, (0.5, 0.5, 0.25))
    ours, ref = str(tmp_path / "ours.img"), str(tmp_path / "ref.img")
    r.write(ours)
    hdr = dict(zip(F.IMG_FIELDS, (*r.reso, *r.pixel, *r.ctr_idx, *r.center)))
    F.write(ref, hdr, F.IMG_FIELDS, img, (3, 2, 1))
    assert open(ours, "rb").read() == open(ref, "rb").read()
    q = ReconImage.read(ref)
    assert q.reso == (6, 5, 4) and q.storage_order == (3, 2, 1)
    assert np.array_equal(q.image, img)
    assert np.array_equal(q.xyz(), np.ascontiguousarray(np.transpose(img)))


def test_derived_geometry_follows_the_callbacks():
    p = _proj()
    ang = p.view_angles()
    assert np.allclose(ang, np.arange(5) * 2 * np.pi / 4 + 12.5 / 180 * np.pi)
    assert np.allclose(p.z_shifts(), np.arange(5) / 4 * 37.98 - 3.0)
    x, y, z = p.detector_xyz()
    assert np.allclose(x, (np.arange(1, 8) - 4.0) * 0.8)
    assert np.allclose(y, -600.0)
    assert np.allclose(z, (np.arange(1, 4) - 2.0) * 0.8)
    p.is_arc = True
    x, y, _ = p.detector_xyz()
    a = (np.arange(1, 8) - 4.0) * 0.8 / 1200.0
    assert np.allclose(x, np.sin(a) * 1200.0) and np.allclose(y, 600.0 - 1200.0 * np.cos(a))


def test_bad_files_are_refused(tmp_path):
    p = _proj()
    path = str(tmp_path / "a.prj")
    p.write(path)
    with open(path, "r+b") as f:
        f.truncate(os.path.getsize(path) - 8)
    with pytest.raises(CtreconError, match="does not match its header"):
        ProjectionData.read(path)
    # the native writer refuses a storage order that is not a permutation
    import ctypes
    from ctrecon_b200 import _lib
    h = _lib.ProjFileHeader()
    h.det_reso_u, h.det_reso_v, h.total_views = 2, 2, 2
    h.storage_order[:] = [1, 1, 3]
    data = np.zeros(8)
    rc = _lib.lib().ctrecon_projfile_write(os.fsencode(str(tmp_path / "b.prj")), ctypes.byref(h),
                                            data.ctypes.data_as(_lib._dp))
    assert rc == _lib.ERR_INVALID_ARGUMENT
    assert b"storage order" in _lib.lib().ctrecon_last_error(None)
    with pytest.raises(CtreconError, match="cannot open"):
        ReconImage.read(str(tmp_path / "missing.img"))
