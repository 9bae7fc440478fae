"""Host file formats (lumenstereo_b200.formats): PFM as the reference's loadPFM
reads it (tools/compare_opencv.cpp:50-83), binary PGM, and PLY as
exportPLY / exportPLY_ASCII write it (src/point_cloud.cpp:57-127)."""
import struct

import numpy as np

from lumenstereo_b200 import POINT_DTYPE, formats

PLY_HEAD = ("ply\nformat {} 1.0\nelement vertex {}\nproperty float x\nproperty float y\nproperty float z\n"
            "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n")


def test_pfm_round_trip_and_layout(tmp_path):
    img = np.arange(12, dtype=np.float32).reshape(3, 4) * np.float32(0.25) - 1
    img[1, 2] = np.inf
    formats.write_pfm(str(tmp_path / "a.pfm"), img)
    raw = (tmp_path / "a.pfm").read_bytes()
    assert raw.startswith(b"Pf\n4 3\n-1.0\n")
    # rows are stored bottom-up
    assert raw[-16:] == img[0].astype("<f4").tobytes()
    back = formats.read_pfm(str(tmp_path / "a.pfm"))
    assert back.dtype == np.float32 and np.array_equal(back, img)


def test_pfm_big_endian_and_rejects(tmp_path):
    img = np.array([[1.5, -2.0], [3.25, 1e-3]], np.float32)
    body = np.ascontiguousarray(img[::-1]).astype(">f4").tobytes()
    (tmp_path / "be.pfm").write_bytes(b"Pf 2 2 1.0\n" + body)          # positive scale: big-endian
    assert np.array_equal(formats.read_pfm(str(tmp_path / "be.pfm")), img)
    (tmp_path / "rgb.pfm").write_bytes(b"PF\n2 2\n-1.0\n" + body * 3)   # colour PFM: not read
    assert formats.read_pfm(str(tmp_path / "rgb.pfm")) is None
    (tmp_path / "short.pfm").write_bytes(b"Pf\n2 2\n-1.0\n" + body[:10])
    assert formats.read_pfm(str(tmp_path / "short.pfm")) is None
    (tmp_path / "zero.pfm").write_bytes(b"Pf\n0 2\n-1.0\n")
    assert formats.read_pfm(str(tmp_path / "zero.pfm")) is None


def test_pgm_round_trip_and_comments(tmp_path):
    img = (np.arange(35).reshape(5, 7) * 7).astype(np.uint8)
    formats.write_pgm(str(tmp_path / "a.pgm"), img)
    assert (tmp_path / "a.pgm").read_bytes() == b"P5\n7 5\n255\n" + img.tobytes()
    assert np.array_equal(formats.read_pgm(str(tmp_path / "a.pgm")), img)
    (tmp_path / "c.pgm").write_bytes(b"P5\n# made here\n7 # width\n5\n255\n" + img.tobytes())
    assert np.array_equal(formats.read_pgm(str(tmp_path / "c.pgm")), img)


def _points():
    rec = np.zeros(3, POINT_DTYPE)
    rec["x"], rec["y"], rec["z"] = [0.1, -2.5, 1e-7], [1234567.0, 0.0, -0.0], [3.0, 99.99999, 1.0 / 3.0]
    rec["r"], rec["g"], rec["b"] = [255, 0, 12], [1, 2, 3], [200, 100, 0]
    return rec


def test_ply_binary_bytes(tmp_path):
    rec = _points()
    assert formats.export_ply(rec, str(tmp_path / "p.ply"))
    exp = PLY_HEAD.format("binary_little_endian", 3).encode()
    for p in rec:
        exp += struct.pack("<fffBBB", p["x"], p["y"], p["z"], p["r"], p["g"], p["b"])
    assert (tmp_path / "p.ply").read_bytes() == exp
    # the (xyz, rgb) form writes the same file
    xyz = np.stack([rec["x"], rec["y"], rec["z"]], 1)
    rgb = np.stack([rec["r"], rec["g"], rec["b"]], 1)
    assert formats.export_ply((xyz, rgb), str(tmp_path / "q.ply"))
    assert (tmp_path / "q.ply").read_bytes() == exp


def test_ply_ascii_text(tmp_path):
    assert formats.export_ply(_points(), str(tmp_path / "a.ply"), binary=False)
    # a C++ stream prints a float (promoted to double) like printf "%g"
    exp = PLY_HEAD.format("ascii", 3) + ("0.1 1.23457e+06 3 255 1 200\n"
                                         "-2.5 0 100 0 2 100\n"
                                         "1e-07 -0 0.333333 12 3 0\n")
    assert (tmp_path / "a.ply").read_text() == exp
    assert not formats.export_ply(_points(), str(tmp_path / "no" / "dir.ply"))
