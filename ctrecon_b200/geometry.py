"""Helical scan configurations and the reference's argument packing.

``HelicalScan`` holds one helical cone-beam geometry in millimetres and derives the
arguments the reference's entry points take:

* ``filter_args()`` -- the 13 scalar inputs of ``KatsevichFiltering_GPU``
  (``KatsevichFiltering_GPU.cu:939-959``; caller ``KatsevichFiltering.m:38``);
* ``geom_struct()`` -- the ``geom`` struct of ``KatsevichBkProj`` with its fields
  ``Locus``, ``Detector``, ``Object`` (``FunctionKat_v6.m:110-112``).

Detector sizing follows the reference's own rules (``FunctionKat_v6.m:49-57``) run
backwards: for a detector of ``YL x ZL`` cells at a given pitch the field-of-view radius
is the largest ``ObjR`` that the width rule (one-column margin) allows, and the helical
pitch is a fraction of the largest pitch the height rule allows (the Tam-Danielson window).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Optional, Sequence

import numpy as np


def katsevich_sizing(ScanR, StdDis, HelicP, ObjR, YL, ZL, pi=3.1415926):
    """Detector sizing of ``FunctionKat_v6.m:49-57`` -> (DecWidth, DecHeigh, delta).

    ``pi`` defaults to the driver's own constant (``FunctionKat_v6.m:49``)."""
    U_HelicP = HelicP / ObjR
    U_ScanR = ScanR / ObjR
    U_DW = 2 * (U_ScanR / (U_ScanR ** 2 - 1) ** 0.5) * YL / (YL - 2)
    delta = 2 * math.acos(ObjR / ScanR)
    coef = (2 * pi - delta) / (2 * pi * (1 - math.cos(delta)))
    U_DH = 2 * coef * U_HelicP * ZL / (ZL - 2)
    return U_DW * StdDis / U_ScanR, U_DH * StdDis / U_ScanR, delta


@dataclass
class HelicalScan:
    name: str
    ScanR: float            # source-to-axis distance (mm)
    StdDis: float           # source-to-detector distance (mm)
    YL: int                 # detector columns (u)
    ZL: int                 # detector rows (v)
    pitch_u: float          # column pitch (mm)
    pitch_v: float          # row pitch (mm)
    views_per_turn: int     # ProjScale
    turns: float
    pitch_ratio: float      # helical pitch / largest pitch of the height rule
    NX: int
    NY: int
    NZ: int
    voxel: Optional[Sequence[float]] = None  # (dx, dy, dz); None -> 2*ObjR/N
    obj_r_cap: float = 120.0
    n_ellipsoids: int = 10
    seed: int = 1000
    photons: Optional[float] = None          # Poisson noise: incident photons per ray
    filter_coeff: float = 0.5                # FilterCoeFF (tau); 0.5 = standard Katsevich
    filtering_mode: int = 0
    ellipsoid_radius_frac: float = 0.8       # centres within this fraction of the FOV radius

    # ---- derived quantities ----------------------------------------------------------
    @property
    def DecWidth(self) -> float:
        return self.YL * self.pitch_u

    @property
    def DecHeigh(self) -> float:
        return self.ZL * self.pitch_v

    @property
    def ObjR(self) -> float:
        t = self.DecWidth * (self.YL - 2) / (2 * self.StdDis * self.YL)
        return min(self.obj_r_cap, self.ScanR * t / math.sqrt(1 + t * t))

    @property
    def delta(self) -> float:
        return 2 * math.acos(self.ObjR / self.ScanR)

    @property
    def HelicP(self) -> float:
        d = self.delta
        coef = (2 * math.pi - d) / (2 * math.pi * (1 - math.cos(d)))
        Hmax = self.DecHeigh * (self.ZL - 2) / self.ZL * self.ScanR / (2 * coef * self.StdDis)
        return self.pitch_ratio * Hmax

    @property
    def P(self) -> int:
        return int(round(self.views_per_turn * self.turns))

    @property
    def ProjCtr(self) -> float:
        return (self.P + 1) / 2.0

    @property
    def voxel_size(self):
        if self.voxel is not None:
            return tuple(float(v) for v in self.voxel)
        return (2 * self.ObjR / self.NX, 2 * self.ObjR / self.NY, 2 * self.ObjR / self.NZ)

    # ---- argument packing --------------------------------------------------------------
    def filter_args(self):
        """(ProjScale, DecWidth, DecHeigh, ScanR, StdDis, HelicP, FilterCoeFF, DeltaAngle,
        FilteringMode, YL, ZL, ProjNumber) -- inputs 2..13 of KatsevichFiltering_GPU."""
        return (float(self.views_per_turn), self.DecWidth, self.DecHeigh, self.ScanR,
                self.StdDis, self.HelicP, self.filter_coeff, self.delta,
                float(self.filtering_mode), float(self.YL), float(self.ZL), float(self.P))

    def locus(self):
        return [self.ScanR, self.StdDis, self.HelicP, float(self.views_per_turn), 1.0,
                float(self.P), self.ProjCtr]

    def detector(self):
        return [self.DecWidth, float(self.YL), self.DecHeigh, float(self.ZL),
                (self.YL - 1) / 2.0, (self.ZL - 1) / 2.0]

    def object(self):
        dx, dy, dz = self.voxel_size
        return [self.ObjR, float(self.NX), float(self.NY), float(self.NZ), dx, dy, dz]

    def geom_struct(self) -> dict:
        """The ``geom`` struct of FunctionKat_v6.m:110-112 (field order matters)."""
        return {"Locus": np.array(self.locus()), "Detector": np.array(self.detector()),
                "Object": np.array(self.object())}

    @property
    def proj_shape(self):
        return (self.P, self.ZL, self.YL)

    @property
    def vol_shape(self):
        return (self.NX, self.NY, self.NZ)

    # ---- synthetic phantom -------------------------------------------------------------
    def ellipsoids(self) -> np.ndarray:
        """Seeded random ellipsoids: rows (cx, cy, cz, a, b, c, phi, theta, psi, density).

        Centres are area-uniform in a disc of ``ellipsoid_radius_frac`` x the FOV radius
        and uniform in the volume's z-span; semi-axes U[5, 60] mm (scaled down with the
        FOV when it is smaller than 120 mm); ZXZ Euler angles uniform; density
        U[-0.2, 1.0]."""
        rng = np.random.default_rng(self.seed)
        n = self.n_ellipsoids
        fov = min(self.ObjR, self.obj_r_cap)
        scale = min(1.0, fov / 120.0)
        r = self.ellipsoid_radius_frac * fov * np.sqrt(rng.random(n))
        phi0 = 2 * np.pi * rng.random(n)
        zspan = self.NZ * self.voxel_size[2]
        cz = (rng.random(n) - 0.5) * zspan
        axes = (5 + 55 * rng.random((n, 3))) * scale
        ang = np.stack([2 * np.pi * rng.random(n), np.pi * rng.random(n),
                        2 * np.pi * rng.random(n)], axis=1)
        dens = -0.2 + 1.2 * rng.random(n)
        return np.column_stack([r * np.cos(phi0), r * np.sin(phi0), cz, axes, ang, dens])

    def with_(self, **kw) -> "HelicalScan":
        return replace(self, **kw)


# ---- the benchmark configurations ------------------------------------------------------
def config(name: str) -> HelicalScan:
    """The five workloads: c1 CPU-runnable plain, c2 plain FP32 at 512^2x256,
    c3 mixed-precision filter, c5 learned PI initialiser at 1024^3 (c4 is the batch of
    uneven scans, see :func:`batch_configs`)."""
    if name == "c1":
        return HelicalScan("c1", 600.0, 1200.0, 256, 16, 1.0, 1.0, 720, 3, 0.9,
                           256, 256, 64, voxel=(0.5, 0.5, 0.5), n_ellipsoids=10, seed=1001)
    if name == "c2":
        return HelicalScan("c2", 600.0, 1200.0, 736, 64, 0.8, 0.8, 1160, 8, 0.9,
                           512, 512, 256, voxel=(0.4, 0.4, 0.4), n_ellipsoids=40, seed=1002,
                           photons=1e5)
    if name == "c2s":
        # a slab of c2 for profiling captures: same detector, pitch and voxels, 2 turns,
        # 32 slices (the per-voxel PI coverage is that of c2)
        return HelicalScan("c2s", 600.0, 1200.0, 736, 64, 0.8, 0.8, 1160, 2, 0.9,
                           512, 512, 32, voxel=(0.4, 0.4, 0.4), n_ellipsoids=40, seed=1012,
                           photons=1e5)
    if name == "c3":
        return HelicalScan("c3", 600.0, 1200.0, 1024, 128, 0.8, 0.8, 2304, 6, 0.9,
                           512, 512, 512, voxel=None, n_ellipsoids=40, seed=1003)
    if name == "c3s":
        # a slab of c3 for profiling captures: same detector, pitch and voxels, 1.25 turns,
        # 32 slices (FP32 projections 1.5 GB, above L2)
        return HelicalScan("c3s", 600.0, 1200.0, 1024, 128, 0.8, 0.8, 2304, 1.25, 0.9,
                           512, 512, 32, voxel=(0.46875, 0.46875, 0.46875), n_ellipsoids=40,
                           seed=1013)
    if name == "c5":
        return HelicalScan("c5", 600.0, 1200.0, 1536, 256, 0.5, 0.5, 2000, 10, 0.9,
                           1024, 1024, 1024, voxel=None, n_ellipsoids=40, seed=1005)
    raise KeyError(name)


def batch_configs(n: int = 16, seed: int = 1004):
    """c4: ``n`` helical scans of uneven size (volumes 128^3 .. 512x512x192, detectors
    32-96 rows x 384-896 columns, 600-1600 views/turn, 2-8 turns, pitch ratio 0.5-1.0,
    10-60 ellipsoids each). The volume is sized to fit inside the helix travel."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        ZL = int(rng.integers(32, 97))
        YL = int(rng.integers(384, 897))
        Ps = int(rng.integers(600, 1601))
        turns = int(rng.integers(2, 9))
        ratio = float(0.5 + 0.5 * rng.random())
        nx = int(rng.integers(128, 513))
        nz = int(rng.integers(128, 193))
        s = HelicalScan(f"c4_{i}", 600.0, 1200.0, YL, ZL, 0.8, 0.8, Ps, turns, ratio,
                        nx, nx, nz, voxel=None, n_ellipsoids=int(rng.integers(10, 61)),
                        seed=seed * 100 + i)
        # voxel pitch: 2*ObjR/N in x,y; z shrunk so the volume lies inside the helix minus
        # ~0.6 pitch at each end
        dxy = 2 * s.ObjR / nx
        zmax = max(0.5 * (turns - 1.2) * s.HelicP, 4 * dxy)
        dz = min(dxy, 2 * zmax / nz)
        out.append(s.with_(voxel=(dxy, dxy, dz)))
    return out


def small_config(name: str = "tiny", **kw) -> HelicalScan:
    """Small geometries for tests (seconds on the CPU oracle)."""
    base = dict(name=name, ScanR=600.0, StdDis=1200.0, YL=64, ZL=8, pitch_u=2.0, pitch_v=2.0,
                views_per_turn=180, turns=3, pitch_ratio=0.9, NX=32, NY=32, NZ=16,
                voxel=None, n_ellipsoids=6, seed=7)
    base.update(kw)
    return HelicalScan(**base)
