"""The reference's data files: ``ProjectionData`` (ProjectionData.m) and ``ReconImage``
(ReconImage.m), read and written through the library's native readers
(``ctrecon_projfile_*``, ``ctrecon_imgfile_*``).

MATLAB stores the arrays column-major; here they are numpy arrays in C order with the axes
reversed (a MATLAB ``U x V x P`` projection is a numpy ``(P, V, U)`` array), the layout the
rest of the package uses. The derived geometry (view angles, z shifts, detector-cell
coordinates) follows the classes' callbacks.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import ImgFileHeader, ProjFileHeader, check, lib

_AXES_P = "UVP"
_AXES_I = "XYZ"


def _shape_of(order, sizes: dict, names: str):
    """numpy shape (C order) of data stored with MATLAB dims [names[order[0]-1], ...]."""
    dims = [sizes[names[int(o) - 1]] for o in order]
    return tuple(reversed(dims))


def _to_canonical(a: np.ndarray, order) -> np.ndarray:
    """Permute an array stored in `order` (MATLAB dims) to the canonical 1 2 3 order,
    returned as numpy axes (3, 2, 1)."""
    m = np.transpose(a)  # numpy view in MATLAB dim order
    perm = [list(map(int, order)).index(k) for k in (1, 2, 3)]
    return np.ascontiguousarray(np.transpose(np.transpose(m, perm)))


@dataclass
class ProjectionData:
    """ProjectionData.m:1-176: scan description and projections (defaults as its constructor)."""
    source_to_center: float = 538.0
    source_to_detector: float = 946.0
    det_reso_u: int = 888
    det_reso_v: int = 64
    det_pixel_u: float = 1.0239
    det_pixel_v: float = 1.0963
    det_center_u: float = 443.75
    det_center_v: float = 31.5
    is_arc: bool = True
    start_angle_deg: float = 0.0
    start_z: float = 0.0
    pitch: float = 0.0
    total_views: int = 984
    views_per_turn: int = 984
    projection: np.ndarray = field(default=None, repr=False)  # numpy, stored order
    storage_order: tuple = (1, 2, 3)

    # ---- files -----------------------------------------------------------------------------
    @classmethod
    def read(cls, path: str) -> "ProjectionData":
        h = ProjFileHeader()
        check(lib().ctrecon_projfile_read(os.fsencode(path), ctypes.byref(h), None, 0), None)
        n = int(h.det_reso_u * h.det_reso_v * h.total_views)
        buf = np.empty(n, dtype=np.float64)
        check(lib().ctrecon_projfile_read(os.fsencode(path), ctypes.byref(h),
                                          buf.ctypes.data_as(_lib._dp), n), None)
        order = tuple(int(o) for o in h.storage_order)
        sizes = {"U": int(h.det_reso_u), "V": int(h.det_reso_v), "P": int(h.total_views)}
        return cls(h.source_to_center, h.source_to_detector, int(h.det_reso_u),
                   int(h.det_reso_v), h.det_pixel_u, h.det_pixel_v, h.det_center_u,
                   h.det_center_v, bool(h.is_arc), h.start_angle_deg, h.start_z, h.pitch,
                   int(h.total_views), int(h.views_per_turn),
                   buf.reshape(_shape_of(order, sizes, _AXES_P)), order)

    def write(self, path: str):
        h = ProjFileHeader(self.source_to_center, self.source_to_detector, self.det_reso_u,
                           self.det_reso_v, self.det_pixel_u, self.det_pixel_v,
                           self.det_center_u, self.det_center_v, float(self.is_arc),
                           self.start_angle_deg, self.start_z, self.pitch, self.total_views,
                           self.views_per_turn, (ctypes.c_double * 3)(*self.storage_order))
        data = np.ascontiguousarray(self.projection, dtype=np.float64)
        sizes = {"U": self.det_reso_u, "V": self.det_reso_v, "P": self.total_views}
        if data.shape != _shape_of(self.storage_order, sizes, _AXES_P):
            raise ValueError(f"projection shape {data.shape} does not match the header")
        check(lib().ctrecon_projfile_write(os.fsencode(path), ctypes.byref(h),
                                           data.ctypes.data_as(_lib._dp)), None)

    def uvp(self) -> np.ndarray:
        """The projections as numpy (P, V, U), the layout of the Katsevich entry points."""
        return _to_canonical(self.projection, self.storage_order)

    # ---- derived geometry (ProjectionData.m:349-372) ----------------------------------------
    def view_angles(self) -> np.ndarray:
        return (np.arange(self.total_views) * 2 * math.pi / self.views_per_turn
                + self.start_angle_deg / 180 * math.pi)

    def z_shifts(self) -> np.ndarray:
        return ((self.view_angles() - self.start_angle_deg / 180 * math.pi) / (2 * math.pi)
                * self.pitch + self.start_z)

    def detector_xyz(self):
        """Cell coordinates (xds, yds, zds) in the source frame of view 0."""
        k = np.arange(1, self.det_reso_u + 1) - (self.det_center_u + 1)
        if self.is_arc:
            a = k * self.det_pixel_u / self.source_to_detector
            x = np.sin(a) * self.source_to_detector
            y = self.source_to_center - self.source_to_detector * np.cos(a)
        else:
            x = k * self.det_pixel_u
            y = np.full(self.det_reso_u, self.source_to_center - self.source_to_detector)
        z = (np.arange(1, self.det_reso_v + 1) - self.det_center_v - 1) * self.det_pixel_v
        return x, y, z


@dataclass
class ReconImage:
    """ReconImage.m:1-117: a reconstructed volume and its sampling (defaults as its constructor)."""
    reso: tuple = (512, 512, 64)
    pixel: tuple = (0.9766, 0.9766, 0.9766)
    ctr_idx: tuple = (255.5, 255.5, 31.5)
    center: tuple = (0.0, 0.0, 0.0)
    image: np.ndarray = field(default=None, repr=False)  # numpy, stored order
    storage_order: tuple = (1, 2, 3)

    @classmethod
    def read(cls, path: str) -> "ReconImage":
        h = ImgFileHeader()
        check(lib().ctrecon_imgfile_read(os.fsencode(path), ctypes.byref(h), None, 0), None)
        reso = tuple(int(v) for v in h.reso)
        n = reso[0] * reso[1] * reso[2]
        buf = np.empty(n, dtype=np.float64)
        check(lib().ctrecon_imgfile_read(os.fsencode(path), ctypes.byref(h),
                                         buf.ctypes.data_as(_lib._dp), n), None)
        order = tuple(int(o) for o in h.storage_order)
        sizes = dict(zip(_AXES_I, reso))
        return cls(reso, tuple(h.pixel), tuple(h.ctr_idx), tuple(h.center),
                   buf.reshape(_shape_of(order, sizes, _AXES_I)), order)

    def write(self, path: str):
        d3 = lambda v: (ctypes.c_double * 3)(*v)
        h = ImgFileHeader(d3(self.reso), d3(self.pixel), d3(self.ctr_idx), d3(self.center),
                          d3(self.storage_order))
        data = np.ascontiguousarray(self.image, dtype=np.float64)
        if data.shape != _shape_of(self.storage_order, dict(zip(_AXES_I, self.reso)), _AXES_I):
            raise ValueError(f"image shape {data.shape} does not match the header")
        check(lib().ctrecon_imgfile_write(os.fsencode(path), ctypes.byref(h),
                                          data.ctypes.data_as(_lib._dp)), None)

    def xyz(self) -> np.ndarray:
        """The volume as numpy (Z, Y, X) -- MATLAB X x Y x Z."""
        return _to_canonical(self.image, self.storage_order)

    @classmethod
    def from_bkproj(cls, img_xyz_zfast: np.ndarray, voxel) -> "ReconImage":
        """Wrap a backprojector image (numpy (NX, NY, NZ), z fastest: KatsevichBkProj.cpp:264)
        as a ReconImage stored in order Z Y X (its bytes unchanged)."""
        nx, ny, nz = img_xyz_zfast.shape
        return cls((nx, ny, nz), tuple(voxel), ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2),
                   (0.0, 0.0, 0.0), np.ascontiguousarray(img_xyz_zfast), (3, 2, 1))
