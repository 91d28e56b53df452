"""The staged footprint of the fourth and fifth backprojector forms covers every cell a voxel
of the tile reads (CPU emulation in FP32, no GPU).

ctrecon_b200/csrc/bp_tile4.cuh: the producer bounds a tile's footprint on the detector from
the four corner columns of the tile and its first / last slice, with a slack of kFootMargin
cells; a consumer thread reads, for the voxel at detector position (u, v), the cell record at
(rint(u - 1/2), rint(v - 1/2)) of that footprint. If a voxel's cell fell outside the staged
cells the read would land in another view's records, so the rule is checked here over whole
tiles and many views, with the smallest slack reported: it must stay far above the FP32
rounding differences between the two computations (~1e-3 cells).
"""
import numpy as np
import pytest

from ctrecon_b200.geometry import config, small_config

F = np.float32
MARGIN = F(0.0625)  # kFootMargin


def _views(s, stride):
    g = s.geom_struct()
    R, SD, HP, PS, PB, PE, PC = g["Locus"]
    P = int(PE - PB + 1)
    p = np.arange(0, P, stride)
    th = (p + PB - PC) * (2 * np.pi / PS)  # build_bp_plan: FP64, then rounded
    return p, np.cos(th).astype(F), np.sin(th).astype(F), (HP * th / (2 * np.pi)).astype(F)


def _check(s, n_tiles, view_stride, seed=0):
    g = s.geom_struct()
    R, SD = F(g["Locus"][0]), g["Locus"][1]
    DW, YL, DH, ZL, HalfY, HalfZ = g["Detector"]
    YL, ZL = int(YL), int(ZL)
    ObjR, NX, NY, NZ, dx, dy, dz = g["Object"]
    NX, NY, NZ = int(NX), int(NY), int(NZ)
    DdU, DdV = F(SD / (DW / YL)), F(SD / (DH / ZL))
    HalfY, HalfZ = F(HalfY), F(HalfZ)
    HalfYm, HalfZm = HalfY - F(0.5), HalfZ - F(0.5)
    xc = ((np.arange(NX) - (NX - 1) / 2) * dx).astype(F)
    yc = ((np.arange(NY) - (NY - 1) / 2) * dy).astype(F)
    zc = ((np.arange(NZ) - (NZ - 1) / 2) * dz).astype(F)
    dzf = F(dz)
    _, c, sn, sz = _views(s, view_stride)
    rng = np.random.default_rng(seed)
    tiles = [(bx, by, bz) for bx in range(0, NX, 16) for by in range(0, NY, 16)
             for bz in range(0, NZ, 8)]
    pick = rng.choice(len(tiles), size=min(n_tiles, len(tiles)), replace=False)
    slack, n_cell = np.inf, 0
    for t in pick:
        bx, by, bz = tiles[t]
        x1, y1, z1 = min(bx + 16, NX) - 1, min(by + 16, NY) - 1, min(bz + 8, NZ) - 1
        # producer: corner bounds (one lane per view)
        umin = np.full(c.shape, np.inf, F); umax = np.full(c.shape, -np.inf, F)
        vmin = np.full(c.shape, np.inf, F); vmax = np.full(c.shape, -np.inf, F)
        ok = np.ones(c.shape, bool)
        for cx in (xc[bx], xc[x1]):
            for cy in (yc[by], yc[y1]):
                fen = R - (cx * c + cy * sn)
                ok &= fen > F(1e-3) * R
                inv = F(1) / fen
                u = (cy * c - cx * sn) * DdU * inv + HalfY
                va = (zc[bz] - sz) * DdV * inv + HalfZ
                vb = (zc[z1] - sz) * DdV * inv + HalfZ
                umin = np.minimum(umin, u); umax = np.maximum(umax, u)
                vmin = np.minimum(vmin, np.minimum(va, vb)); vmax = np.maximum(vmax, np.maximum(va, vb))
        u0 = np.floor(umin - MARGIN).astype(np.int64); u1 = np.floor(umax + MARGIN).astype(np.int64) + 1
        v0 = np.floor(vmin - MARGIN).astype(np.int64); v1 = np.floor(vmax + MARGIN).astype(np.int64) + 1
        cell = ok & (u0 >= 0) & (u1 <= YL - 1) & (v0 >= 0) & (v1 <= ZL - 1)
        if not cell.any():
            continue
        n_cell += int(cell.sum())
        cc, ss, zz = c[cell], sn[cell], sz[cell]
        cu0, cu1, cv0, cv1 = u0[cell], u1[cell], v0[cell], v1[cell]
        # consumers: every voxel column and slice of the tile
        X = xc[bx:x1 + 1][:, None, None]
        Y = yc[by:y1 + 1][None, :, None]
        fen = R - (X * cc + Y * ss)
        YY = Y * cc - X * ss
        inv = F(1) / fen
        kv = DdV * inv
        um = ((YY * DdU).astype(np.float64) * inv + HalfYm).astype(F)  # fmaf
        dz0 = zc[bz] - zz
        lo_u = um - (cu0 - F(0.5)); hi_u = (cu1 - F(0.5)) - um  # rint(um) in [u0, u1 - 1]
        slack = min(slack, float(lo_u.min()), float(hi_u.min()))
        for k in range(z1 - bz + 1):
            dzk = (np.float64(k) * dzf + dz0).astype(F)
            vm = (dzk.astype(np.float64) * kv + HalfZm).astype(F)
            lo_v = vm - (cv0 - F(0.5)); hi_v = (cv1 - F(0.5)) - vm
            slack = min(slack, float(lo_v.min()), float(hi_v.min()))
    return slack, n_cell


@pytest.mark.parametrize("name", ["c1", "c2s", "c3", "c5", "fine", "thin"])
def test_footprint_covers_every_cell_read(name):
    if name == "fine":  # 0.5 mm voxels, few views per turn
        s = small_config(name="fine", YL=200, ZL=48, views_per_turn=120, turns=2.5, NX=64,
                         NY=48, NZ=24, voxel=(0.5, 0.5, 0.5), seed=5)
    elif name == "thin":  # anisotropic voxels, low pitch
        s = small_config(name="thin", YL=96, ZL=40, NX=40, NY=40, NZ=24, pitch_ratio=0.6,
                         voxel=(0.8, 0.8, 0.3), seed=6)
    else:
        s = config(name)
    slack, n = _check(s, n_tiles=24, view_stride=7)
    print(f"{name}: {n} tile-views on the cell path, smallest slack {slack:.4f} cells")
    assert n > 0
    assert slack > 0.03  # the margin less the worst FP32 difference, with room to spare


def _tile_view_paths(s, B, T, valid):
    """For every 16 x 16 x 8 tile of scan s and every view of the tile's PI range (the union of
    its voxels' [floor(B), ceil(T)]), whether the fifth form brings the footprint in with a
    tensor copy (inside the detector, and a box of at most 64 x 32 cells) or reads the view
    directly. Returns (tile-views on the copy path, all tile-views)."""
    g = s.geom_struct()
    R, SD = F(g["Locus"][0]), g["Locus"][1]
    DW, YL, DH, ZL, HalfY, HalfZ = g["Detector"]
    YL, ZL = int(YL), int(ZL)
    ObjR, NX, NY, NZ, dx, dy, dz = g["Object"]
    NX, NY, NZ = int(NX), int(NY), int(NZ)
    DdU, DdV = F(SD / (DW / YL)), F(SD / (DH / ZL))
    HalfY, HalfZ = F(HalfY), F(HalfZ)
    xc = ((np.arange(NX) - (NX - 1) / 2) * dx).astype(F)
    yc = ((np.arange(NY) - (NY - 1) / 2) * dy).astype(F)
    zc = ((np.arange(NZ) - (NZ - 1) / 2) * dz).astype(F)
    p_all, c_all, s_all, z_all = _views(s, 1)
    copy = total = 0
    for bx in range(0, NX, 16):
        for by in range(0, NY, 16):
            for bz in range(0, NZ, 8):
                x1, y1, z1 = min(bx + 16, NX) - 1, min(by + 16, NY) - 1, min(bz + 8, NZ) - 1
                v = valid[bx:x1 + 1, by:y1 + 1, bz:z1 + 1]
                if not v.any():
                    continue
                p0 = max(0, int(np.floor(B[bx:x1 + 1, by:y1 + 1, bz:z1 + 1][v].min())))
                p1 = min(len(p_all) - 1, int(np.ceil(T[bx:x1 + 1, by:y1 + 1, bz:z1 + 1][v].max())))
                c, sn, sz = c_all[p0:p1 + 1], s_all[p0:p1 + 1], z_all[p0:p1 + 1]
                umin = np.full(c.shape, np.inf, F); umax = np.full(c.shape, -np.inf, F)
                vmin = np.full(c.shape, np.inf, F); vmax = np.full(c.shape, -np.inf, F)
                for cx in (xc[bx], xc[x1]):
                    for cy in (yc[by], yc[y1]):
                        inv = F(1) / (R - (cx * c + cy * sn))
                        u = (cy * c - cx * sn) * DdU * inv + HalfY
                        va = (zc[bz] - sz) * DdV * inv + HalfZ
                        vb = (zc[z1] - sz) * DdV * inv + HalfZ
                        umin = np.minimum(umin, u); umax = np.maximum(umax, u)
                        vmin = np.minimum(vmin, np.minimum(va, vb))
                        vmax = np.maximum(vmax, np.maximum(va, vb))
                u0 = np.floor(umin - MARGIN).astype(np.int64)
                u1 = np.floor(umax + MARGIN).astype(np.int64) + 1
                v0 = np.floor(vmin - MARGIN).astype(np.int64)
                v1 = np.floor(vmax + MARGIN).astype(np.int64) + 1
                bw = (u1 - u0 + 3) & ~3
                bh = (v1 - v0 + 1) & ~1
                ok = ((u0 >= 0) & (u1 <= YL - 1) & (v0 >= 0) & (v1 <= ZL - 1) &
                      (bw <= 64) & (bh <= 32))
                copy += int(ok.sum())
                total += ok.size
    return copy, total


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_central_block_takes_the_tensor_copy_path(oracle_mod, name):
    """The central 48^3 blocks of tests/test_gpu_blocks.py: most of their tile-views go through
    the fifth form's tensor copies (c2 87 %, c3 96 %; the rest are views whose footprint reaches
    the top or bottom detector row), so that test checks that path against the oracle."""
    from conftest import central_block
    O = oracle_mod
    s = config(name)
    locus, det, obj, lo, hi = central_block(O, s, 48)
    blk = s.with_(NX=48, NY=48, NZ=48, voxel=tuple(obj[4:7]), obj_r_cap=obj[0])
    pit = O.pi_table(O.bp_geom(s.locus(), s.detector(), obj, honour_extras=True))
    copy, total = _tile_view_paths(blk, pit["B"], pit["T"], pit["valid"])
    print(f"{name} central block: {copy} of {total} tile-views on the tensor-copy path "
          f"({copy / total:.1%})")
    assert copy >= 0.85 * total
