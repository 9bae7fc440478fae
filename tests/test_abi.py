"""The C-ABI library loads and exports every symbol include/lumen_sgbm.h
declares; pure host entry points behave like the reference (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

from lumenstereo_b200 import StereoParams, _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        if not hdr.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", hdr)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(lumen_\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_loads():
    assert os.path.exists(_lib.LIB_PATH), "build liblumen_sgbm.so first"
    _lib.lib()


def test_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 20
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"symbols declared in include/*.h but not exported: {missing}"


def test_params_default_matches_python():
    c = _lib.CParams()
    _lib.lib().lumen_stereo_params_default(C.byref(c))
    assert StereoParams.from_c(c) == StereoParams()


@pytest.mark.parametrize("kw,valid", [
    ({}, True), ({"blockSize": 4}, False), ({"blockSize": 0}, False),
    ({"minDisparity": 100, "maxDisparity": 50}, False), ({"minDisparity": -1}, False),
    ({"P1": 100, "P2": 50}, False), ({"uniquenessRatio": 101}, False)])
def test_is_valid_c_matches_python(kw, valid):
    p = StereoParams(**kw)
    assert bool(_lib.lib().lumen_stereo_params_is_valid(C.byref(p.to_c()))) == valid == p.isValid()


def test_auto_penalties_c():
    c = StereoParams(blockSize=7).to_c()
    _lib.lib().lumen_stereo_params_auto_penalties(C.byref(c), 3)
    assert (c.P1, c.P2) == (8 * 3 * 49, 32 * 3 * 49)


def test_null_arguments_are_invalid():
    lib = _lib.lib()
    assert lib.lumen_sgbm_create(None, None) == _lib.ERR_INVALID_ARGUMENT
    assert lib.lumen_sgbm_set_params(None, None) == _lib.ERR_INVALID_ARGUMENT
    assert lib.lumen_sgbm_destroy(None) == _lib.OK
    assert "NULL" in _lib.last_error() or _lib.last_error() == ""


def test_depth_entry_points_check_arguments_before_the_device():
    """Argument errors of the depth / colour / point-cloud entry points are
    reported before any CUDA call (so they hold without a device too)."""
    lib = _lib.lib()
    bad = _lib.ERR_INVALID_ARGUMENT
    fake = 1 << 20                       # never dereferenced: the checks fail first
    lut = (C.c_uint8 * 768)()
    # no output at all / NULL input / empty size
    assert lib.lumen_disparity_to_depth_color_device(fake, 4, 4, 0, 1.0, 1.0, 0.0, None, 0, 0.5, 10.0, lut,
                                                     None, 0, None) == bad
    assert lib.lumen_disparity_to_depth_device(None, 4, 4, 0, 1.0, 1.0, 0.0, fake, 0, None) == bad
    assert lib.lumen_disparity_to_depth_device(fake, 0, 4, 0, 1.0, 1.0, 0.0, fake, 0, None) == bad
    # colours without a table; strides below the packed row or not a multiple of the element
    assert lib.lumen_disparity_to_depth_color_device(fake, 4, 4, 0, 1.0, 1.0, 0.0, None, 0, 0.5, 10.0, None,
                                                     fake, 0, None) == bad
    assert lib.lumen_disparity_to_depth_device(fake, 4, 4, 6, 1.0, 1.0, 0.0, fake, 0, None) == bad
    assert lib.lumen_disparity_to_depth_device(fake, 4, 4, 9, 1.0, 1.0, 0.0, fake, 0, None) == bad
    assert lib.lumen_depth_colorize_device(fake, 4, 4, 0, 0.5, 10.0, lut, fake, 11, None) == bad
    assert lib.lumen_depth_colorize_device(fake, 4, 4, 0, 0.5, 10.0, None, fake, 0, None) == bad
    # points: unaligned record buffer, missing offsets, bad colour stride
    pts = fake + 8
    assert lib.lumen_depth_to_points_device(fake, 4, 4, 0, None, 0, 1.0, 1.0, 0.0, 0.0, pts, fake, None) == bad
    assert lib.lumen_depth_to_points_device(fake, 4, 4, 0, None, 0, 1.0, 1.0, 0.0, 0.0, fake, None, None) == bad
    assert lib.lumen_depth_to_points_device(fake, 4, 4, 0, fake, 5, 1.0, 1.0, 0.0, 0.0, fake, fake, None) == bad
    n = C.c_int(-1)
    assert lib.lumen_depth_to_points(None, 4, 4, 0, None, 0, 1.0, 1.0, 0.0, 0.0, fake, C.byref(n)) == bad
    assert n.value == -1
    assert "stride" in _lib.last_error() or "NULL" in _lib.last_error()
