"""Minimal readers for the reference's test volumes: MetaImage (.mha,
ElementDataFile = LOCAL) and NRRD headers (.nhdr) with a detached raw file,
float32 little-endian, 3D. Returns (array [nz, ny, nx] float32, spacing
(sx, sy, sz))."""
import os
import re

import numpy as np


def read_mha(path):
    with open(path, "rb") as f:
        data = f.read()
    hdr = {}
    pos = 0
    while True:
        end = data.index(b"\n", pos)
        line = data[pos:end].decode("latin-1").strip()
        pos = end + 1
        k, _, v = line.partition("=")
        hdr[k.strip()] = v.strip()
        if k.strip() == "ElementDataFile":
            break
    dims = [int(x) for x in hdr["DimSize"].split()]
    sp = tuple(float(x) for x in hdr.get("ElementSpacing", "1 1 1").split())
    assert hdr["ElementType"] == "MET_FLOAT" and hdr["ElementDataFile"] == "LOCAL"
    n = dims[0] * dims[1] * dims[2]
    arr = np.frombuffer(data[pos:pos + 4 * n], dtype="<f4").reshape(dims[2], dims[1], dims[0])
    return arr.astype(np.float32), sp


def read_nhdr(path):
    hdr = {}
    for line in open(path, "r", encoding="latin-1"):
        if ":" in line and not line.startswith("#"):
            k, _, v = line.partition(":")
            hdr[k.strip()] = v.strip()
    dims = [int(x) for x in hdr["sizes"].split()]
    dirs = re.findall(r"\(([^)]*)\)", hdr["space directions"])
    sp = tuple(float(d.split(",")[i]) for i, d in enumerate(dirs))
    raw = os.path.join(os.path.dirname(path), hdr["data file"])
    arr = np.fromfile(raw, dtype="<f4").reshape(dims[2], dims[1], dims[0])
    return arr.astype(np.float32), sp


def rescale_intensities(a):
    """The ImagePreprocessor's intensity window to [0, 1]
    (Array3DUtils::rescaleElements): (a - min) * (1 / (max - min)), the
    difference in float, the product in double."""
    mn, mx = float(a.min()), float(a.max())
    scale = (1.0 - 0.0) / (mx - mn)
    return ((a - np.float32(mn)).astype(np.float64) * scale).astype(np.float32)
