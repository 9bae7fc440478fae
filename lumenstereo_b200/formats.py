"""File formats either side of the stereo path (host side, numpy).

* PFM: ``read_pfm`` follows the reference's loadPFM
  (tools/compare_opencv.cpp:50-83): grayscale "Pf" files only, width, height
  and scale as whitespace-separated text, one separator byte, then float32
  rows stored bottom-up, little-endian when the scale is negative (byte-swapped
  otherwise).  A file that does not parse reads as None (the reference returns
  an empty Mat).  ``write_pfm`` writes that layout little-endian.
* PGM: binary 8-bit "P5" images (the synthetic workloads' image files).
* PLY: ``export_ply`` / ``export_ply_ascii`` follow exportPLY / exportPLY_ASCII
  (src/point_cloud.cpp:57-127): the same header, then per point x, y, z
  float32 and red, green, blue uint8 (15 bytes, little-endian) or one text
  line "x y z r g b" with floats in the "%g" form of a C++ stream.
"""
from __future__ import annotations

import re
from typing import Optional

import numpy as np

_PLY_HEADER = ("ply\nformat {fmt} 1.0\nelement vertex {n}\nproperty float x\nproperty float y\n"
               "property float z\nproperty uchar red\nproperty uchar green\nproperty uchar blue\n"
               "end_header\n")


def read_pfm(path: str) -> Optional[np.ndarray]:
    with open(path, "rb") as f:
        data = f.read()
    m = re.match(rb"\s*(\S+)\s+([+-]?\d+)\s+([+-]?\d+)\s+(\S+)", data)
    if not m or m.group(1) != b"Pf":
        return None
    w, h = int(m.group(2)), int(m.group(3))
    try:
        scale = float(m.group(4))
    except ValueError:
        return None
    if w <= 0 or h <= 0:
        return None
    start = m.end() + 1                      # the single separator byte
    n = w * h * 4
    if len(data) < start + n:
        return None
    img = np.frombuffer(data, dtype="<f4" if scale < 0 else ">f4", count=w * h, offset=start)
    return np.ascontiguousarray(img.reshape(h, w)[::-1].astype(np.float32))


def write_pfm(path: str, img: np.ndarray) -> None:
    img = np.asarray(img, np.float32)
    if img.ndim != 2:
        raise ValueError("PFM: one-channel images only")
    h, w = img.shape
    with open(path, "wb") as f:
        f.write(b"Pf\n%d %d\n-1.0\n" % (w, h))
        f.write(np.ascontiguousarray(img[::-1]).astype("<f4").tobytes())


def read_pgm(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        data = f.read()
    toks, pos = [], 0
    while len(toks) < 4 and pos < len(data):       # magic, width, height, maxval
        c = data[pos:pos + 1]
        if c.isspace():
            pos += 1
        elif c == b"#":                              # a comment runs to the end of its line
            nl = data.find(b"\n", pos)
            pos = len(data) if nl < 0 else nl + 1
        else:
            end = pos
            while end < len(data) and not data[end:end + 1].isspace() and data[end:end + 1] != b"#":
                end += 1
            toks.append(data[pos:end])
            pos = end
    if len(toks) < 4 or toks[0] != b"P5" or not all(t.isdigit() for t in toks[1:]):
        raise ValueError(f"{path}: not a binary PGM")
    w, h, maxval = (int(t) for t in toks[1:])
    if maxval > 255:
        raise ValueError(f"{path}: 16-bit PGM")
    pos += 1                                         # the single byte after maxval
    if len(data) < pos + w * h:
        raise ValueError(f"{path}: truncated")
    return np.frombuffer(data, np.uint8, count=w * h, offset=pos).reshape(h, w).copy()


def write_pgm(path: str, img: np.ndarray) -> None:
    img = np.asarray(img)
    if img.dtype != np.uint8 or img.ndim != 2:
        raise ValueError("PGM: 8-bit one-channel images only")
    with open(path, "wb") as f:
        f.write(b"P5\n%d %d\n255\n" % (img.shape[1], img.shape[0]))
        f.write(np.ascontiguousarray(img).tobytes())


def _split_points(points):
    """(xyz [n, 3] float32, rgb [n, 3] uint8) from a pair or from records
    with x, y, z, r, g, b fields."""
    if isinstance(points, tuple):
        xyz, rgb = points
    else:
        xyz = np.stack([points["x"], points["y"], points["z"]], axis=1)
        rgb = np.stack([points["r"], points["g"], points["b"]], axis=1)
    return np.asarray(xyz, np.float32).reshape(-1, 3), np.asarray(rgb, np.uint8).reshape(-1, 3)


def export_ply(points, path: str, binary: bool = True) -> bool:
    if not binary:
        return export_ply_ascii(points, path)
    xyz, rgb = _split_points(points)
    rec = np.empty(len(xyz), dtype=[("xyz", "<f4", 3), ("rgb", "u1", 3)])
    rec["xyz"], rec["rgb"] = xyz, rgb
    try:
        with open(path, "wb") as f:
            f.write(_PLY_HEADER.format(fmt="binary_little_endian", n=len(xyz)).encode())
            f.write(rec.tobytes())
    except OSError:
        return False
    return True


def export_ply_ascii(points, path: str) -> bool:
    xyz, rgb = _split_points(points)
    try:
        with open(path, "w") as f:
            f.write(_PLY_HEADER.format(fmt="ascii", n=len(xyz)))
            f.writelines("%g %g %g %d %d %d\n" % (float(p[0]), float(p[1]), float(p[2]), c[0], c[1], c[2])
                         for p, c in zip(xyz, rgb.astype(int)))
    except OSError:
        return False
    return True
