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
