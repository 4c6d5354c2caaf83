"""ImageStack's `.tmp` raw image files (src/FileTMP.cpp:13-38 describes the format).

A file is a header of five native 32-bit integers — width, height, frames, channels and a
type code — followed by the samples, channel by channel, then frame by frame, row by row,
as values of the coded type.  Loading converts every sample to float32, as ImageStack
stores all images; saving converts float32 samples with a C cast.  Arrays here are planar
float32: (channels, frames, height, width), or (channels, height, width) for one frame,
the layout every entry point of this package takes.
"""
from __future__ import annotations

import numpy as np

# type codes of src/FileTMP.cpp:13 and the names its save accepts (:86-123)
TYPES = {0: np.float32, 1: np.float64, 2: np.uint8, 3: np.int8, 4: np.uint16, 5: np.int16,
         6: np.uint32, 7: np.int32, 8: np.uint64, 9: np.int64}
NAMES = {"float": 0, "float32": 0, "double": 1, "float64": 1, "uint8": 2, "unsigned char": 2,
         "int8": 3, "char": 3, "uint16": 4, "unsigned short": 4, "int16": 5, "short": 5,
         "uint32": 6, "unsigned int": 6, "int32": 7, "int": 7, "uint64": 8, "int64": 9}


def load_tmp(path: str) -> np.ndarray:
    """Read a .tmp file into a planar float32 array ((c, h, w) for one frame)."""
    with open(path, "rb") as f:
        head = np.fromfile(f, dtype=np.int32, count=5)
        if head.size != 5:
            raise ValueError("%s: file ended before end of header" % path)
        w, h, frames, channels, code = (int(x) for x in head)
        if code not in TYPES:
            raise ValueError("%s: unknown type code %d" % (path, code))
        if min(w, h, frames, channels) < 0:
            raise ValueError("%s: negative size in header" % path)
        n = w * h * frames * channels
        data = np.fromfile(f, dtype=TYPES[code], count=n)
        if data.size != n:
            raise ValueError("%s: unexpected end of file" % path)
    im = data.astype(np.float32).reshape(channels, frames, h, w)
    return im[:, 0] if frames == 1 else im


def save_tmp(path: str, image: np.ndarray, type: str = "float32") -> None:
    """Write a planar array ((c, h, w) or (c, f, h, w)) as a .tmp file of the named type."""
    if type not in NAMES:
        raise ValueError("unknown .tmp type %r" % type)
    code = NAMES[type]
    im = np.asarray(image, dtype=np.float32)
    if im.ndim == 3:
        im = im[:, None]
    if im.ndim != 4:
        raise ValueError("expected a (c, h, w) or (c, f, h, w) array")
    channels, frames, h, w = im.shape
    with open(path, "wb") as f:
        np.array([w, h, frames, channels, code], dtype=np.int32).tofile(f)
        data = im if code == 0 else im.astype(TYPES[code])
        np.ascontiguousarray(data).tofile(f)
