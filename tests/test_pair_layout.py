"""Schedule 6's host-shared index arithmetic (lumenstereo_b200/csrc/pair_layout.h)
checked by a host program (tests/cpp/pair_layout_test.cpp), and the four-sweep
decomposition itself restated in numpy against the oracle's 8-path volume:
{LR, TLBR} and {RL, BRTL} over rows, {TB, TRBL} and {BT, BLTR} over columns,
each path starting at L = C where its predecessor leaves the image."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from lumenstereo_b200 import MatchingCostMode, StereoParams, synth
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_pair_layout_host_checks(tmp_path):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "pair_layout_test"
    subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "lumenstereo_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "pair_layout_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr


def test_pair_handoff_protocol_host_model(tmp_path):
    """Worker threads standing for any number of resident CTAs run the bands
    in ticket order with the kernel's publish / bounded-wait protocol: every
    band finishes and consumes only published pixels."""
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "pair_progress_test"
    subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-pthread", "-I",
                    os.path.join(ROOT, "lumenstereo_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "pair_progress_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr


def _step(Lp, C, P1, p2):
    """src/sgbm_kernels.cu:338-360 on one pixel (uint16 wrap)."""
    a = Lp.astype(np.int64)
    mp = int(a.min())
    b = np.concatenate([[0xFFFF], (a[:-1] + P1) & 0xFFFF])
    c = np.concatenate([(a[1:] + P1) & 0xFFFF, [0xFFFF]])
    m = np.minimum(np.minimum(a, b), np.minimum(c, np.full_like(a, (mp + p2) & 0xFFFF)))
    return (C + m - mp) & 0xFFFF


def _four_sweeps(cost, img, P1, P2, cs):
    H, W, D = cost.shape
    C = (cost.astype(np.int64) * cs) & 0xFFFF
    total = np.zeros((H, W, D), np.int64)

    def xy(s, u, v):
        return [(u, v), (W - 1 - u, H - 1 - v), (W - 1 - v, u), (v, H - 1 - u)][s]

    def p2(cur, prev):
        return max(P1 + 1, P2 * 8 // max(8, abs(int(cur) - int(prev))))

    for s in range(4):
        Ws, Hs = (W, H) if s < 2 else (H, W)
        above = None
        for v in range(Hs):
            row = []
            LH = None
            for u in range(Ws):
                x, y = xy(s, u, v)
                if u == 0:
                    LH = C[y, x].copy()
                else:
                    px, py = xy(s, u - 1, v)
                    LH = _step(LH, C[y, x], P1, p2(img[y, x], img[py, px]))
                if u == 0 or v == 0:
                    LD = C[y, x].copy()
                else:
                    px, py = xy(s, u - 1, v - 1)
                    LD = _step(above[u - 1], C[y, x], P1, p2(img[y, x], img[py, px]))
                row.append(LD)
                total[y, x] = (total[y, x] + LH + LD) & 0xFFFF
            above = row
    return total


@pytest.mark.parametrize("w,h,kw", [(23, 17, dict(maxDisparity=16)),
                                    (13, 29, dict(maxDisparity=24, matchingCostMode=MatchingCostMode.Census)),
                                    (16, 11, dict(maxDisparity=8, blockSize=19))])   # uint16 wrap
def test_four_sweep_decomposition_matches_oracle(w, h, kw):
    left, right = synth.random_pair(w, h, 5)
    p = StereoParams(numDirections=8, speckleWindowSize=0, **kw)
    _, inter = oracle.sgbm({k: int(v) for k, v in p.__dict__.items()}, left, right, intermediates=True)
    cs = p.blockSize ** 2 if p.matchingCostMode == MatchingCostMode.SAD else \
        max(1, p.blockSize ** 2 * 2 * p.preFilterCap // 255)
    agg = _four_sweeps(inter["cost"], inter["gray_left"], p.P1, p.P2, cs)
    assert np.array_equal(agg, inter["agg"].astype(np.int64))
