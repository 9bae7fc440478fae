"""The oracle (oracle/sgbm_oracle.c) pinned on the CPU:

* against the golden fixtures produced by the reference's own CUDA kernels
  (tests/golden/*.npz, made by tests/golden/make_golden.py on a GPU);
* against the reference's own known-answer tests that hold for this path
  (remap vs cv::remap, tests/test_rectification.cpp:189-265 of the reference)
  and cv2.cvtColor for the BGR->gray step;
* against an independent pure-Python restatement of the recurrence on tiny
  inputs (two restatements written separately must agree bit for bit).
"""
import glob
import json
import os

import numpy as np
import pytest

from tests.conftest import params_dict

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


# ---------------------------------------------------------------- identities
def test_census_cost_identity():
    for h in range(25):
        assert (h * 255 + 12) // 24 == (85 * h + 4) >> 3


def test_umulhi_division_exact():
    """sum/count == umulhi(sum, ceil(2^32/count)) over every SAD window sum
    (count <= 441 for blockSize <= 21, each term <= 254)."""
    for c in range(2, 442):
        m = (2 ** 32 + c - 1) // c
        s = np.arange(0, c * 254 + 1, dtype=np.uint64)
        assert np.array_equal((s * np.uint64(m)) >> np.uint64(32), s // np.uint64(c)), c


# ------------------------------------------------------- reference KATs (cv2)
def test_bgr2gray_matches_cv2_all_colours(oracle_mod):
    cv2 = pytest.importorskip("cv2")
    v = np.arange(256 ** 3, dtype=np.uint32)
    img = np.stack([v & 255, (v >> 8) & 255, v >> 16], -1).astype(np.uint8).reshape(4096, 4096, 3)
    assert np.array_equal(oracle_mod.bgr2gray(img), cv2.cvtColor(img, cv2.COLOR_BGR2GRAY))


def test_remap_identity_matches_cv2(oracle_mod):
    """test_rectification.cpp:189-224: identity map, GPU == cv::remap exactly."""
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(1)
    src = rng.integers(0, 255, (480, 640), dtype=np.uint8)
    my, mx = np.mgrid[0:480, 0:640].astype(np.float32)
    ref = cv2.remap(src, mx, my, cv2.INTER_LINEAR)
    assert np.array_equal(oracle_mod.remap(src, mx, my), ref)


def test_remap_half_pixel_within_one(oracle_mod):
    """test_rectification.cpp:226-265: +0.5 px map, |GPU - cv::remap| <= 1."""
    cv2 = pytest.importorskip("cv2")
    xs = np.arange(100)
    src = np.tile((xs * 255 // 100).astype(np.uint8), (100, 1))
    my, mx = np.mgrid[0:100, 0:100].astype(np.float32)
    mx += 0.5
    my += 0.5
    ref = cv2.remap(src, mx, my, cv2.INTER_LINEAR)
    diff = np.abs(oracle_mod.remap(src, mx, my).astype(int) - ref.astype(int))
    assert diff.max() <= 1


# --------------------------------------- independent pure-Python restatement
def py_cost_census(L, R, D, minD):
    H, W = L.shape

    def census(img):
        out = np.zeros((H, W), np.uint32)
        for y in range(2, H - 2):
            for x in range(2, W - 2):
                bits, b = 0, 0
                for dy in range(-2, 3):
                    for dx in range(-2, 3):
                        if dx == 0 and dy == 0:
                            continue
                        if img[y + dy, x + dx] >= img[y, x]:
                            bits |= 1 << b
                        b += 1
                out[y, x] = bits
        return out

    cl, cr = census(L), census(R)
    cost = np.full((H, W, D), 255, np.uint8)
    for y in range(2, H - 2):
        for x in range(2, W - 2):
            for d in range(D):
                rx = x - minD - d
                if 2 <= rx < W - 2:
                    h = bin(int(cl[y, x]) ^ int(cr[y, rx])).count("1")
                    cost[y, x, d] = (h * 255 + 12) // 24
    return cost


def py_aggregate(cost, img, P1, P2, cs, paths):
    H, W, D = cost.shape
    agg = np.zeros((H, W, D), np.int64)
    steps = [(1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, -1), (-1, 1), (1, -1)]
    for k, (sx, sy) in enumerate(steps):
        if not (paths >> k) & 1:
            continue
        for y in range(H):
            for x in range(W):
                px, py = x - sx, y - sy
                if not (0 <= px < W and 0 <= py < H):  # line start
                    L = [(int(c) * cs) & 0xFFFF for c in cost[y, x]]
                    cx, cy = x, y
                    while 0 <= cx < W and 0 <= cy < H:
                        if (cx, cy) != (x, y):
                            g = abs(int(img[cy, cx]) - int(img[cy - sy, cx - sx]))
                            p2 = max(P1 + 1, P2 * 8 // max(8, g))
                            mp = min(L)
                            new = []
                            for d in range(D):
                                c0 = L[d]
                                c1 = (L[d - 1] + P1) & 0xFFFF if d > 0 else 0xFFFF
                                c2 = (L[d + 1] + P1) & 0xFFFF if d < D - 1 else 0xFFFF
                                c3 = (mp + p2) & 0xFFFF
                                C = (int(cost[cy, cx, d]) * cs) & 0xFFFF
                                new.append((C + min(c0, c1, c2, c3) - mp) & 0xFFFF)
                            L = new
                        agg[cy, cx] += L
                        cx += sx
                        cy += sy
    return (agg & 0xFFFF).astype(np.uint16)


def py_wta(agg, minD, UR):
    H, W, D = agg.shape
    out = np.zeros((H, W), np.int16)
    for y in range(H):
        for x in range(W):
            v = [int(a) for a in agg[y, x]]
            mn, sec, bd = 0xFFFF, 0xFFFF, 0
            for d, c in enumerate(v):
                if c < mn:
                    sec, mn, bd = mn, c, d
                elif c < sec:
                    sec = c
            if UR > 0 and sec != 0xFFFF and sec <= mn + (mn * UR) // 100:
                out[y, x] = -1
                continue
            sub = np.float32(bd)
            if 0 < bd < D - 1:
                c0, c1, c2 = (np.float32(v[bd - 1]), np.float32(v[bd]), np.float32(v[bd + 1]))
                den = np.float32(2.0) * (c0 + c2 - np.float32(2.0) * c1)
                if abs(den) > np.float32(1e-6):
                    dl = np.float32((c0 - c2) / den)
                    dl = max(np.float32(-1.0), min(np.float32(1.0), dl))
                    sub = np.float32(sub + dl)
            out[y, x] = int(np.float32((sub + np.float32(minD)) * np.float32(16.0)))
    return out


@pytest.mark.parametrize("paths", [0x0F, 0xFF])
def test_oracle_matches_python_restatement(oracle_mod, paths):
    from lumenstereo_b200.synth import random_pair
    L, R = random_pair(14, 11, seed=3, shift=3)
    D, minD = 7, 1
    p = params_dict(minDisparity=minD, maxDisparity=minD + D, matchingCostMode=1,
                    numDirections=8 if paths == 0xFF else 4, speckleWindowSize=0,
                    uniquenessRatio=10, P1=8, P2=40)
    disp, inter = oracle_mod.sgbm(p, L, R, intermediates=True)
    cost = py_cost_census(L, R, D, minD)
    assert np.array_equal(inter["cost"], cost)
    cs = max(1, (25 * 2 * 31) // 255)
    agg = py_aggregate(cost, L, 8, 40, cs, paths)
    assert np.array_equal(inter["agg"], agg)
    assert np.array_equal(inter["disp_wta"], py_wta(agg, minD, 10))


def test_oracle_wraps_uint16(oracle_mod):
    """Large penalties / costScale make the uint16 sums wrap; the C oracle and
    the Python restatement must wrap identically."""
    from lumenstereo_b200.synth import random_pair
    L, R = random_pair(9, 8, seed=4, shift=2)
    p = params_dict(maxDisparity=5, matchingCostMode=1, numDirections=8, blockSize=21,
                    preFilterCap=63, P1=30000, P2=60000, speckleWindowSize=0)
    _, inter = oracle_mod.sgbm(p, L, R, intermediates=True)
    cs = max(1, (21 * 21 * 2 * 63) // 255)
    cost = py_cost_census(L, R, 5, 0)
    agg = py_aggregate(cost, L, 30000, 60000, cs, 0xFF)
    assert np.array_equal(inter["agg"], agg)


def test_oracle_thread_count_independent(oracle_mod):
    from lumenstereo_b200.synth import random_pair
    L, R = random_pair(96, 40, seed=9, shift=5)
    p = params_dict(maxDisparity=32, numDirections=8, speckleWindowSize=50)
    oracle_mod.set_threads(1)
    a = oracle_mod.sgbm(p, L, R)
    oracle_mod.set_threads(os.cpu_count() or 4)
    b = oracle_mod.sgbm(p, L, R)
    assert np.array_equal(a, b)


def test_oracle_errors(oracle_mod):
    L = np.zeros((8, 8), np.uint8)
    with pytest.raises(RuntimeError):
        oracle_mod.sgbm(params_dict(minDisparity=10, maxDisparity=10), L, L)
    with pytest.raises(RuntimeError):
        oracle_mod.sgbm(params_dict(maxDisparity=513), L, L)


def test_median_positive_upper_median(oracle_mod):
    d = np.array([[5, -1, 7], [0, 9, 3], [-1, -1, 8]], np.int16)
    out = oracle_mod.median3x3(d)
    # centre: positives {5,7,9,3,8} -> sorted 3,5,7,8,9 -> [5//2] = 7
    assert out[1, 1] == 7
    # corner (0,0): {5,9} -> [1] = 9
    assert out[0, 0] == 9
    z = np.array([[-1, 0], [0, -1]], np.int16)
    assert np.array_equal(oracle_mod.median3x3(z), z)


# ------------------------------------------------------------ golden vectors
def golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: os.path.basename(p))
def test_oracle_matches_reference_golden(oracle_mod, path):
    g = np.load(path)
    meta = json.loads(str(g["meta"]))
    p = meta["params"]
    disp, inter = oracle_mod.sgbm(p, g["left"], g["right"], intermediates=True,
                                  path_mask=meta.get("path_mask", 0))
    for key in ("pref_left", "pref_right", "census_left", "census_right", "cost", "agg"):
        if key in g.files:
            assert np.array_equal(inter[key], g[key]), key
    # 1/16-px maps: the reference divides with --use_fast_math; allow the
    # documented 1/16 px on <= 0.01% of pixels (plus one pixel for tiny cases).
    # The reference's speckle filter races (src/sgbm_kernels.cu:979-1013), so
    # maps after it are reported, not compared, when the filter is on.
    keys = [("disp_wta", inter["disp_wta"]), ("disp_right", inter["disp_right"])]
    if p["speckleWindowSize"] > 0:
        diff = int((disp != g["disp"]).sum())
        print(f"{meta['name']}: {diff} of {disp.size} pixels differ after the racy speckle filter")
    else:
        keys += [("disp_lr", inter["disp_lr"]), ("disp", disp)]
    for key, ours in keys:
        if key not in g.files:
            continue
        ref = g[key]
        bad = ours != ref
        assert np.all(np.abs(ours.astype(int) - ref.astype(int))[bad] <= 1), key
        assert bad.sum() <= max(1, int(1e-4 * bad.size)), (key, int(bad.sum()))
