"""MetaImage (.mhd + .raw) reading and writing for volumes in the image3d layout.

The reference reads and writes MetaImage through VTK (header/interface_imp.hxx:34-90,
672-712). DimSize and ElementSpacing list the fastest axis first; image3d's fastest
axis is k, so a volume v[i, j, k] of shape (X, Y, Z) is stored with DimSize Z Y X.
"""
from __future__ import annotations

import os

import numpy as np

_TYPES = {"MET_UCHAR": np.uint8, "MET_CHAR": np.int8, "MET_USHORT": np.uint16,
          "MET_SHORT": np.int16, "MET_UINT": np.uint32, "MET_INT": np.int32,
          "MET_FLOAT": np.float32, "MET_DOUBLE": np.float64}
_NAMES = {np.dtype(v): k for k, v in _TYPES.items()}


def write(path_base: str, vol: np.ndarray, spacing=(1.0, 1.0, 1.0)) -> str:
    """Writes <path_base>.mhd and <path_base>.raw; returns the .mhd path."""
    vol = np.ascontiguousarray(vol)
    X, Y, Z = vol.shape
    raw = path_base + ".raw"
    with open(path_base + ".mhd", "w") as f:
        f.write("ObjectType = Image\nNDims = 3\nBinaryData = True\n"
                "BinaryDataByteOrderMSB = False\n"
                f"DimSize = {Z} {Y} {X}\n"
                f"ElementSpacing = {spacing[2]!r} {spacing[1]!r} {spacing[0]!r}\n"
                f"ElementType = {_NAMES[vol.dtype]}\n"
                f"ElementDataFile = {os.path.basename(raw)}\n")
    vol.astype(vol.dtype.newbyteorder("<"), copy=False).tofile(raw)
    return path_base + ".mhd"


def read(path: str):
    """(volume[i, j, k], spacing (hx, hy, hz)) of a little-endian MetaImage file."""
    hdr = {}
    with open(path, "rb") as f:
        while True:
            line = f.readline()
            if not line:
                break
            text = line.decode("latin-1").strip()
            if "=" not in text:
                continue
            k, v = (s.strip() for s in text.split("=", 1))
            hdr[k] = v
            if k == "ElementDataFile":
                offset = f.tell()
                break
    dims = [int(x) for x in hdr["DimSize"].split()]
    while len(dims) < 3:
        dims.append(1)
    sp = [float(x) for x in hdr.get("ElementSpacing", "1 1 1").split()]
    while len(sp) < 3:
        sp.append(1.0)
    dt = np.dtype(_TYPES[hdr["ElementType"]]).newbyteorder("<")
    n = dims[0] * dims[1] * dims[2]
    if hdr["ElementDataFile"] == "LOCAL":
        data = np.fromfile(path, dtype=dt, count=n, offset=offset)
    else:
        data = np.fromfile(os.path.join(os.path.dirname(path), hdr["ElementDataFile"]),
                           dtype=dt, count=n)
    vol = data.reshape(dims[2], dims[1], dims[0])
    return vol, (sp[2], sp[1], sp[0])
