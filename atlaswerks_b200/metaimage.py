"""MetaImage (.mha / .mhd) and NRRD (.nhdr) volumes without ITK.

The reference reads and writes its images and deformation fields through
ITK (Base/ApplicationUtils.cxx: LoadImageITK, SaveImageITK, SaveHFieldITK);
its regression fixtures are MetaImage files with the data inline
(ElementDataFile = LOCAL) and NRRD headers with a detached raw file.
These functions cover that subset: 3D, float32, little-endian, scalar
images and 3-component vector fields (ElementNumberOfChannels = 3, the
components interleaved per voxel, as an ITK vector image stores them).

Arrays are [nz, ny, nx] (x fastest); vector fields are planar [3, nz, ny, nx]
here and interleaved on disk. Spacing and origin are (x, y, z).
"""
from __future__ import annotations

import os
import re
from typing import Sequence, Tuple

import numpy as np

Vec3 = Tuple[float, float, float]


def _header(data: bytes):
    hdr, pos = {}, 0
    while True:
        end = data.index(b"\n", pos)
        line = data[pos:end].decode("latin-1").strip()
        pos = end + 1
        k, _, v = line.partition("=")
        hdr[k.strip()] = v.strip()
        if k.strip() == "ElementDataFile":
            return hdr, pos


def read_mha(path: str):
    """Returns (array, spacing): a scalar volume [nz, ny, nx] or a vector
    field [3, nz, ny, nx], float32. Data inline (LOCAL) or in the file the
    header names next to it."""
    with open(path, "rb") as f:
        data = f.read()
    hdr, pos = _header(data)
    if hdr.get("ElementType") != "MET_FLOAT":
        raise ValueError(f"{path}: only MET_FLOAT volumes are supported")
    if hdr.get("BinaryDataByteOrderMSB", "False").lower() == "true":
        raise ValueError(f"{path}: big-endian data is not supported")
    dims = [int(x) for x in hdr["DimSize"].split()]
    if len(dims) != 3:
        raise ValueError(f"{path}: only 3D volumes are supported")
    ch = int(hdr.get("ElementNumberOfChannels", "1"))
    sp = tuple(float(x) for x in hdr.get("ElementSpacing", "1 1 1").split())
    n = dims[0] * dims[1] * dims[2] * ch
    if hdr["ElementDataFile"] == "LOCAL":
        raw = np.frombuffer(data[pos:pos + 4 * n], dtype="<f4")
    else:
        raw = np.fromfile(os.path.join(os.path.dirname(path), hdr["ElementDataFile"]), dtype="<f4",
                          count=n)
    if raw.size != n:
        raise ValueError(f"{path}: expected {n} floats, found {raw.size}")
    if ch == 1:
        return raw.reshape(dims[2], dims[1], dims[0]).astype(np.float32), sp
    if ch != 3:
        raise ValueError(f"{path}: only scalar or 3-component volumes are supported")
    a = raw.reshape(dims[2], dims[1], dims[0], 3)
    return np.ascontiguousarray(np.moveaxis(a, -1, 0), dtype=np.float32), sp


def write_mha(path: str, a: np.ndarray, spacing: Sequence[float] = (1.0, 1.0, 1.0),
              origin: Sequence[float] = (0.0, 0.0, 0.0)) -> None:
    """Writes a scalar volume [nz, ny, nx] or a vector field [3, nz, ny, nx]
    (stored interleaved, 3 channels) as MetaImage with the data inline."""
    a = np.asarray(a, dtype=np.float32)
    if a.ndim == 4 and a.shape[0] == 3:
        ch, (nz, ny, nx) = 3, a.shape[1:]
        payload = np.ascontiguousarray(np.moveaxis(a, 0, -1), dtype="<f4")
    elif a.ndim == 3:
        ch, (nz, ny, nx) = 1, a.shape
        payload = np.ascontiguousarray(a, dtype="<f4")
    else:
        raise ValueError("expected [nz, ny, nx] or [3, nz, ny, nx]")
    lines = ["ObjectType = Image", "NDims = 3", "BinaryData = True",
             "BinaryDataByteOrderMSB = False", "CompressedData = False",
             "TransformMatrix = 1 0 0 0 1 0 0 0 1",
             "Offset = " + " ".join(repr(float(o)) for o in origin),
             "CenterOfRotation = 0 0 0", "AnatomicalOrientation = RAI",
             "ElementSpacing = " + " ".join(repr(float(s)) for s in spacing),
             f"DimSize = {nx} {ny} {nz}"]
    if ch > 1:
        lines.append(f"ElementNumberOfChannels = {ch}")
    lines += ["ElementType = MET_FLOAT", "ElementDataFile = LOCAL"]
    with open(path, "wb") as f:
        f.write(("\n".join(lines) + "\n").encode("latin-1"))
        f.write(payload.tobytes())


def read_nhdr(path: str):
    """NRRD header with a detached raw float32 file: (array, spacing)."""
    hdr = {}
    for line in open(path, "r", encoding="latin-1"):
        if ":" in line and not line.startswith("#"):
            k, _, v = line.partition(":")
            hdr[k.strip()] = v.strip()
    if hdr.get("type") not in ("float", "float32"):
        raise ValueError(f"{path}: only float volumes are supported")
    dims = [int(x) for x in hdr["sizes"].split()]
    dirs = re.findall(r"\(([^)]*)\)", hdr.get("space directions", "(1,0,0) (0,1,0) (0,0,1)"))
    sp = tuple(float(d.split(",")[i]) for i, d in enumerate(dirs))
    raw = os.path.join(os.path.dirname(path), hdr["data file"])
    arr = np.fromfile(raw, dtype="<f4").reshape(dims[2], dims[1], dims[0])
    return arr.astype(np.float32), sp


def rescale_intensities(a: np.ndarray) -> np.ndarray:
    """The ImagePreprocessor's intensity window to [0, 1]
    (Array3DUtils::rescaleElements): (a - min) * (1 / (max - min)), the
    difference in float, the product in double."""
    mn, mx = float(a.min()), float(a.max())
    scale = (1.0 - 0.0) / (mx - mn)
    return ((a - np.float32(mn)).astype(np.float64) * scale).astype(np.float32)
