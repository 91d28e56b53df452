"""Test infrastructure (oracle): numpy restatement of the reference's file writers and readers,
used only by tests/ as the checker for the library's native file code.

ProjectionData.m:113-131 (WriteFile) and :133-163 (ReadFile); ReconImage.m:60-82 and :84-117.
MATLAB `fwrite(fid, x, 'double')` writes x's elements column-major as native (little-endian)
doubles; a numpy array in C order with the MATLAB axes reversed has the same bytes.
"""
import numpy as np

PROJ_FIELDS = ("SourceToCenterDistance", "SourceToDetectorDistance", "DetResoU", "DetResoV",
               "DetPixelSizeU", "DetPixelSizeV", "DetCntIdxU", "DetCntIdxV", "IsArcDetector",
               "StartSourceAngle", "StartSourceZPos", "Pitch", "TotalProjectionNumber",
               "ProjectionNumberPerTurn")  # ProjectionData.m:115-130, in write order
IMG_FIELDS = ("resoX", "resoY", "resoZ", "pixelSizeX", "pixelSizeY", "pixelSizeZ", "ctrIdxX",
              "ctrIdxY", "ctrIdxZ", "imgCenterX", "imgCenterY", "imgCenterZ")  # ReconImage.m:62-76


def write(path, header: dict, fields, data: np.ndarray, order):
    with open(path, "wb") as f:
        f.write(np.array([header[k] for k in fields], dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(data, dtype="<f8").tobytes())
        f.write(np.array(order, dtype="<f8").tobytes())


def read(path, fields, count):
    raw = np.fromfile(path, dtype="<f8")
    nh = len(fields)
    header = dict(zip(fields, raw[:nh].tolist()))
    n = count(header)
    return header, raw[nh:nh + n], raw[nh + n:nh + n + 3]


def proj_count(h):  # ProjectionData.m:149
    return int(h["DetResoU"] * h["DetResoV"] * h["TotalProjectionNumber"])


def img_count(h):  # ReconImage.m:102
    return int(h["resoX"] * h["resoY"] * h["resoZ"])
