"""CUDA path vs the oracle (bit-exact integer stages, 1/16-px subpixel
tolerance), through the C ABI.  Mirrors the reference's SGBM tests
(tests/test_sgbm.cpp:163-406) and adds the value checks they lack.

Tolerance for 1/16-px maps: the CUDA path divides with --use_fast_math like
the reference; the oracle divides in IEEE single precision, so a pixel may
differ by 1 (= 1/16 px) on at most 0.01% of pixels (one pixel for tiny maps).
Against the reference's own kernels (oracle/_ref) the maps must be identical.
"""
import os
import zlib

import numpy as np
import pytest

from lumenstereo_b200 import (MatchingCostMode, StereoException, StereoParams, StereoSGBM,
                              TimeoutException,
                              bgr_to_gray, kSgbmMaxDisparityRange, rectify_image_gpu, synth)
from tests.conftest import params_dict

pytestmark = pytest.mark.gpu

SUBPIX_FRAC = 1e-4


def assert_subpix_close(ours, ref, what=""):
    bad = ours != ref
    assert np.all(np.abs(ours.astype(int) - ref.astype(int))[bad] <= 1), what
    assert bad.sum() <= max(1, int(SUBPIX_FRAC * bad.size)), (what, int(bad.sum()))


def to_params(d):
    d = dict(d)
    d["matchingCostMode"] = MatchingCostMode(d["matchingCostMode"])
    return StereoParams(**d)


def run_ours(pdict, left, right, path_mask=0, schedule=0):
    p = to_params(pdict)
    h, w = left.shape[:2]
    D = p.maxDisparity - p.minDisparity
    with StereoSGBM(p) as s:
        s.retain_intermediates(True)
        if path_mask:
            s.set_debug_paths(path_mask)
        if schedule:
            s.set_schedule(schedule)
        disp = s.compute(left, right)
        inter = dict(cost=s.intermediate("cost", (h, w, D), np.uint8),
                     agg=s.intermediate("agg", (h, w, D), np.uint16),
                     disp_wta=s.intermediate("disp_wta", (h, w), np.int16),
                     disp_right=s.intermediate("disp_right", (h, w), np.int16),
                     disp_lr=s.intermediate("disp_lr", (h, w), np.int16))
        if p.matchingCostMode == MatchingCostMode.Census:
            inter["census_left"] = s.intermediate("census_left", (h, w), np.uint32)
            inter["census_right"] = s.intermediate("census_right", (h, w), np.uint32)
        else:
            inter["pref_left"] = s.intermediate("pref_left", (h, w), np.uint8)
            inter["pref_right"] = s.intermediate("pref_right", (h, w), np.uint8)
    return disp, inter


def compare_all(pdict, left, right, oracle_mod, path_mask=0, schedule=0):
    disp, ours = run_ours(pdict, left, right, path_mask, schedule)
    ref_disp, ref = oracle_mod.sgbm(pdict, left, right, intermediates=True, path_mask=path_mask)
    for key in ("census_left", "census_right", "pref_left", "pref_right", "cost", "agg"):
        if key in ours:
            assert np.array_equal(ours[key], ref[key]), key
    # integer WTA (first strict minimum) from the bit-exact volume
    assert np.array_equal(np.argmin(ours["agg"], axis=2), np.argmin(ref["agg"], axis=2))
    assert_subpix_close(ours["disp_wta"], ref["disp_wta"], "disp_wta")
    assert_subpix_close(ours["disp_right"], ref["disp_right"], "disp_right")
    assert_subpix_close(ours["disp_lr"], ref["disp_lr"], "disp_lr")
    assert_subpix_close(disp, ref_disp, "disp")
    return disp


CASES = {
    "census_4path_d32": (64, 48, dict(maxDisparity=32, matchingCostMode=1)),
    "sad_8path_d64": (96, 64, dict(maxDisparity=64, numDirections=8)),
    "census_8path_d45_min3": (72, 40, dict(minDisparity=3, maxDisparity=48, matchingCostMode=1,
                                           numDirections=8)),
    "sad_4path_bs3_ur0_nolr": (60, 44, dict(maxDisparity=24, blockSize=3, uniquenessRatio=0,
                                            disp12MaxDiff=-1)),
    "sad_8path_bs7_speckle": (80, 36, dict(maxDisparity=40, blockSize=7, numDirections=8,
                                           speckleWindowSize=100, speckleRange=2)),
    "census_d290_tail": (330, 20, dict(maxDisparity=290, matchingCostMode=1, numDirections=8)),
    "sad_d512": (600, 10, dict(maxDisparity=512, numDirections=8)),
    "census_d192": (260, 30, dict(maxDisparity=192, matchingCostMode=1, numDirections=8)),
    "sad_d1": (30, 20, dict(maxDisparity=1)),
    "sad_d2_odd_w": (31, 17, dict(maxDisparity=2, numDirections=8)),
    "census_wrap_bs21": (40, 30, dict(maxDisparity=16, matchingCostMode=1, blockSize=21,
                                      preFilterCap=63, P1=30000, P2=60000, numDirections=8)),
    "sad_wrap_bs19": (48, 32, dict(maxDisparity=16, blockSize=19, numDirections=8)),
    "sad_wide_bs11_cap127": (64, 40, dict(maxDisparity=24, blockSize=11, preFilterCap=127,
                                          numDirections=8)),
    "sad_bs0": (40, 20, dict(maxDisparity=8, blockSize=0)),
    "census_tiny_5x3": (5, 3, dict(maxDisparity=4, matchingCostMode=1, numDirections=8)),
    "sad_tiny_2x2": (2, 2, dict(maxDisparity=3, numDirections=8)),
    "sad_minD20_ur15": (90, 30, dict(minDisparity=20, maxDisparity=52, uniquenessRatio=15,
                                     numDirections=8)),
    "census_minD100_wide": (120, 16, dict(minDisparity=100, maxDisparity=164,
                                          matchingCostMode=1)),
    # widths divisible by 4: the 5x5 SAD kernel stages right rows a word at a time
    # (Dp 128 with minDisparity, 192, 256 with a partial last quad, 320 with one
    # column-sum buffer), tiles running past both image edges and 70 rows (3 row tiles)
    "sad_minD5_d128_w4": (136, 70, dict(minDisparity=5, maxDisparity=133, numDirections=8)),
    "sad_d192_w4": (200, 40, dict(maxDisparity=192, numDirections=8)),
    "sad_minD7_d250_w4": (264, 36, dict(minDisparity=7, maxDisparity=257)),
    "sad_d300_w4": (324, 24, dict(maxDisparity=300, numDirections=8)),
}


@pytest.mark.parametrize("schedule", [1, 4, 6])
@pytest.mark.parametrize("name", sorted(CASES))
def test_parity_small(name, schedule, oracle_mod):
    w, h, over = CASES[name]
    if w * h >= 2048:
        left, right, _ = synth.make_pair(synth.PairSpec(w, h, 4, 1, max(2, 0.3 * min(w, 300)), 2.0,
                                                        zlib.crc32(name.encode()) % 1000))
    else:
        left, right = synth.random_pair(w, h, seed=zlib.crc32(name.encode()) % 1000, shift=1)
    compare_all(params_dict(speckleWindowSize=0, **over) if "speckle" not in name
                else params_dict(**over), left, right, oracle_mod, schedule=schedule)


@pytest.mark.parametrize("rows", [8, 16])
@pytest.mark.parametrize("D", [40, 128, 150, 290, 512])
def test_parity_schedule4_rows(D, rows, oracle_mod):
    """The lockstep row-band sweeps (schedule 4) at both band heights reproduce
    the oracle bit for bit, both cost modes, 4 and 8 paths, odd image sizes
    (several bands per sweep, a partial last band)."""
    left, right, _ = synth.make_pair(synth.PairSpec(131, 53, 4, 1, min(D - 1, 40), 2.0, 80 + D))
    for mode, nd in ((0, 8), (1, 4), (1, 8)):
        pd = params_dict(maxDisparity=D, numDirections=nd, matchingCostMode=mode,
                         speckleWindowSize=0)
        with StereoSGBM(to_params(pd)) as s:
            s.set_schedule(4)
            s.set_tuning(32, rows)
            s.retain_intermediates(True)
            disp = s.compute(left, right)
            agg = s.intermediate("agg", (53, 131, D), np.uint16)
            used = s.get_tuning()
        assert used[0] == 4, used
        ref_disp, ref = oracle_mod.sgbm(pd, left, right, intermediates=True)
        assert np.array_equal(agg, ref["agg"]), (mode, nd)
        assert_subpix_close(disp, ref_disp)


@pytest.mark.parametrize("rows", [8, 16, 32])
@pytest.mark.parametrize("D,team", [(40, 8), (128, 8), (40, 16), (128, 16), (150, 16), (200, 16), (256, 16),
                                    (290, 16)])
def test_parity_schedule4_lane_teams(D, team, rows, oracle_mod):
    """Rows as lane teams (8 or 16 lanes for 64/128 padded disparities, 16 for
    192/256; the batched launches' form) in the plain call, pinned through
    set_tuning: bit for bit equal to the oracle, partial last bands included."""
    left, right, _ = synth.make_pair(synth.PairSpec(131, 75, 4, 1, min(D - 1, 40), 2.0, 280 + D))
    for mode, nd in ((0, 8), (1, 4)):
        pd = params_dict(maxDisparity=D, numDirections=nd, matchingCostMode=mode,
                         speckleWindowSize=0)
        with StereoSGBM(to_params(pd)) as s:
            s.set_schedule(4)
            s.set_tuning(team, rows)
            s.retain_intermediates(True)
            disp = s.compute(left, right)
            agg = s.intermediate("agg", (75, 131, D), np.uint16)
            used = s.get_tuning()
        # 32 rows of 256+ disparities exceed the shared memory: 16-row bands then
        assert tuple(used) == (4, team, rows) or (rows == 32 and used[0] == 4), used
        ref_disp, ref = oracle_mod.sgbm(pd, left, right, intermediates=True)
        assert np.array_equal(agg, ref["agg"]), (mode, nd)
        assert_subpix_close(disp, ref_disp)


def test_parity_schedule4_wide_image(oracle_mod):
    """A row longer than the exchange ring (kWK = 64 pixels) exercises the
    exporter's back-pressure waits between bands."""
    left, right, _ = synth.make_pair(synth.PairSpec(700, 40, 4, 1, 30, 2.0, 99))
    for nd in (4, 8):
        pd = params_dict(maxDisparity=48, numDirections=nd, speckleWindowSize=0)
        with StereoSGBM(to_params(pd)) as s:
            s.set_schedule(4)
            s.retain_intermediates(True)
            disp = s.compute(left, right)
            agg = s.intermediate("agg", (40, 700, 48), np.uint16)
        ref_disp, ref = oracle_mod.sgbm(pd, left, right, intermediates=True)
        assert np.array_equal(agg, ref["agg"]), nd
        assert_subpix_close(disp, ref_disp)


@pytest.mark.parametrize("D,size", [(40, (131, 53)), (64, (40, 200)), (128, (97, 150)), (150, (160, 70)),
                                    (200, (230, 16)), (290, (330, 41))])
@pytest.mark.parametrize("census", [False, True])
def test_parity_schedule6_pair_sweeps(D, size, census, oracle_mod):
    """Four lag-free sweeps (schedule 6: {LR, TLBR}, {RL, BRTL} over rows,
    {TB, TRBL}, {BT, BLTR} over columns) reproduce the oracle's summed volume
    bit for bit; without retained intermediates the selection sums the four
    partial volumes itself and the maps still match.  Sizes cover wider and
    taller images than bands (both ticket orders) and a single-band sweep."""
    w, h = size
    left, right, _ = synth.make_pair(synth.PairSpec(w, h, 4, 1, min(D - 1, 40), 2.0, 90 + D + w))
    pd = params_dict(maxDisparity=D, numDirections=8, speckleWindowSize=0, matchingCostMode=int(census))
    ref_disp, ref = oracle_mod.sgbm(pd, left, right, intermediates=True)
    with StereoSGBM(to_params(pd)) as s:
        s.set_schedule(6)
        s.retain_intermediates(True)
        disp = s.compute(left, right)
        agg = s.intermediate("agg", (h, w, D), np.uint16)
        assert s.get_tuning()[0] == 6
        assert s.get_tuning_columns() == 24   # untuned: the column sweeps in their own launch
    assert np.array_equal(agg, ref["agg"])
    assert_subpix_close(disp, ref_disp)
    with StereoSGBM(to_params(pd)) as s:
        s.set_schedule(6)
        assert np.array_equal(s.compute(left, right), disp)


@pytest.mark.parametrize("D,size,lanes,rows",
                         [(D, size, lanes, rows)
                          for D, size in [(40, (131, 53)), (64, (40, 200)), (128, (97, 150)), (100, (700, 90))]
                          for lanes, rows in [(8, 24), (8, 32)]] +
                         [(D, size, 16, rows) for D, size in [(150, (160, 70)), (290, (330, 61))] for rows in (24, 32)])
def test_parity_schedule6_configurations(D, size, lanes, rows, oracle_mod):
    """Every schedule-6 configuration the autotuner can pick (24- and 32-row
    bands) reproduces the
    oracle's summed volume bit for bit, both cost modes, partial last bands
    included."""
    w, h = size
    left, right, _ = synth.make_pair(synth.PairSpec(w, h, 4, 1, min(D - 1, 40), 2.0, 300 + D + w))
    for census in (0, 1):
        pd = params_dict(maxDisparity=D, numDirections=8, speckleWindowSize=0, matchingCostMode=census)
        ref_disp, ref = oracle_mod.sgbm(pd, left, right, intermediates=True)
        with StereoSGBM(to_params(pd)) as s:
            s.set_schedule(6)
            s.set_tuning(lanes, rows)
            s.retain_intermediates(True)
            disp = s.compute(left, right)
            agg = s.intermediate("agg", (h, w, D), np.uint16)
            assert s.get_tuning() == (6, lanes, rows), s.get_tuning()
        assert np.array_equal(agg, ref["agg"]), (census, lanes, rows)
        assert_subpix_close(disp, ref_disp)


@pytest.mark.parametrize("D,size,lanes,rows,cols",
                         [(D, size, 8, rows, cols)
                          for D, size in [(40, (131, 53)), (128, (97, 150)), (100, (700, 90)), (64, (40, 200))]
                          for rows, cols in [(16, 16), (16, 24), (16, 32), (24, 24), (24, 32)]] +
                         [(D, size, 16, 16, cols) for D, size in [(150, (160, 70)), (290, (330, 61))]
                          for cols in (16, 24, 32)])
def test_parity_schedule6_column_launch(D, size, lanes, rows, cols, oracle_mod):
    """The column sweeps as a launch of their own beside the row sweeps' (with
    their own band height, on a second stream): the summed volume equals the
    oracle's bit for bit, both cost modes, partial last bands included."""
    w, h = size
    left, right, _ = synth.make_pair(synth.PairSpec(w, h, 4, 1, min(D - 1, 40), 2.0, 400 + D + w))
    for census in (0, 1):
        pd = params_dict(maxDisparity=D, numDirections=8, speckleWindowSize=0, matchingCostMode=census)
        ref_disp, ref = oracle_mod.sgbm(pd, left, right, intermediates=True)
        with StereoSGBM(to_params(pd)) as s:
            s.set_schedule(6)
            s.set_tuning(lanes, rows)
            s.set_tuning_columns(cols)
            s.retain_intermediates(True)
            disp = s.compute(left, right)
            agg = s.intermediate("agg", (h, w, D), np.uint16)
            assert s.get_tuning() == (6, lanes, rows), s.get_tuning()
            assert s.get_tuning_columns() == cols
            # and one launch of all four sweeps gives the same maps
            s.set_tuning_columns(0)
            assert np.array_equal(s.compute(left, right), disp)
            assert s.get_tuning_columns() == 0
        assert np.array_equal(agg, ref["agg"]), (census, lanes, rows, cols)
        assert_subpix_close(disp, ref_disp)


@pytest.mark.parametrize("D,size", [(40, (131, 53)), (64, (40, 200)), (128, (97, 150)), (150, (160, 70)),
                                    (290, (330, 41)), (16, (700, 9))])
def test_parity_schedule6_four_paths(D, size, oracle_mod):
    """4 paths through schedule 6 (LR, RL, TB, BT, one path a sweep, no band
    hand-offs): the summed volume equals the oracle's bit for bit, both cost
    modes, wider and taller images than a band, partial last bands."""
    w, h = size
    left, right, _ = synth.make_pair(synth.PairSpec(w, h, 4, 1, min(D - 1, 40), 2.0, 500 + D + w))
    for census in (0, 1):
        pd = params_dict(maxDisparity=D, numDirections=4, speckleWindowSize=0, matchingCostMode=census)
        ref_disp, ref = oracle_mod.sgbm(pd, left, right, intermediates=True)
        with StereoSGBM(to_params(pd)) as s:
            s.set_schedule(6)
            s.retain_intermediates(True)
            disp = s.compute(left, right)
            agg = s.intermediate("agg", (h, w, D), np.uint16)
            assert s.get_tuning()[0] == 6
        assert np.array_equal(agg, ref["agg"]), census
        assert_subpix_close(disp, ref_disp)
        with StereoSGBM(to_params(pd)) as s:   # the default picks it too, without retained volumes
            assert np.array_equal(s.compute(left, right), disp)


def test_schedule6_matches_schedule4_full_size():
    """1920x1080 D128 SAD and Census, 8 paths: the four-partial selection of
    schedule 6 gives schedule 4's maps (no intermediates retained)."""
    for wl in ("1920x1080_d128_sad_8path", "1920x1080_d128_census_8path"):
        w = synth.WORKLOADS[wl]
        left, right, _ = synth.make_pair(w.pair)
        p = StereoParams(maxDisparity=w.max_disparity, numDirections=8, speckleWindowSize=0,
                         matchingCostMode=MatchingCostMode.Census if w.census else MatchingCostMode.SAD)
        outs = []
        for schedule in (4, 6):
            with StereoSGBM(p) as s:
                s.set_schedule(schedule)
                outs.append(s.compute(left, right))
                assert s.get_tuning()[0] == schedule
        assert np.array_equal(outs[0], outs[1]), wl


@pytest.mark.parametrize("schedule", [4, 6])
def test_fused_sweep_timeout_reports_error(schedule):
    """A device-side wait that runs out ends the launch with a timeout status,
    not a hang: one wait of a band that imports through the global ring is
    made unsatisfiable and the wait limit is cut, so the launch gives up
    quickly; the handle then recovers."""
    left, right = synth.random_pair(300, 64, seed=3)
    p = StereoParams(maxDisparity=64, numDirections=8, speckleWindowSize=0)
    with StereoSGBM(p) as s:
        s.set_schedule(schedule)
        s.set_wait_limit(1 << 14)
        s.stall_test(True)
        with pytest.raises(TimeoutException):
            s.compute(left, right)
        s.stall_test(False)
        s.set_wait_limit(0)
        ref = s.compute(left, right)
    with StereoSGBM(p) as s:
        s.set_schedule(1)
        assert np.array_equal(s.compute(left, right), ref)


def test_autotune_and_cache(tmp_path):
    torch = pytest.importorskip("torch")
    left, right, _ = synth.make_pair(synth.PairSpec(320, 180, 5, 4, 40, 2.0, 90))
    p = StereoParams(maxDisparity=64, numDirections=8, speckleWindowSize=0)
    dl = torch.from_numpy(left).cuda()
    dr = torch.from_numpy(right).cuda()
    with StereoSGBM(p) as s:
        ref = s.compute(left, right).copy()
        rep = s.autotune(dl.data_ptr(), dr.data_ptr(), 320, 180)
        assert "best schedule=" in rep
        assert np.array_equal(s.compute(left, right), ref)  # uses the tuned choice
        tuned = (s.get_tuning(), s.get_tuning_columns())
        path = str(tmp_path / "tune.txt")
        s.save_tuning(path)
    with StereoSGBM(p) as s2:
        s2.load_tuning(path)
        assert np.array_equal(s2.compute(left, right), ref)
        assert (s2.get_tuning(), s2.get_tuning_columns()) == tuned   # the column launch included
    lines = open(path).read().split()
    assert len(lines) == 5   # key schedule lanes rows column-rows
    # a cache written before the column launch existed (four fields) still loads: one launch
    old = tmp_path / "old.txt"
    old.write_text(" ".join(lines[:3] + ["16"]) + "\n")
    with StereoSGBM(p) as s3:
        s3.load_tuning(str(old))
        assert np.array_equal(s3.compute(left, right), ref)
        if int(lines[1]) == 6:
            assert s3.get_tuning_columns() == 0


@pytest.mark.parametrize("k", range(8))
def test_parity_single_path(k, oracle_mod):
    left, right = synth.random_pair(70, 45, seed=40 + k, shift=4)
    for mode in (0, 1):
        compare_all(params_dict(maxDisparity=40, numDirections=8, matchingCostMode=mode,
                                speckleWindowSize=0), left, right, oracle_mod, path_mask=1 << k)


def test_parity_color_input(oracle_mod):
    """SGBMTest.ColorInput (tests/test_sgbm.cpp:194-218) plus values: BGR is
    converted on the device like cv::cvtColor(COLOR_BGR2GRAY)."""
    rng = np.random.default_rng(7)
    left = rng.integers(0, 256, (48, 64, 3), dtype=np.uint8)
    right = np.roll(left, -3, axis=1)
    p = params_dict(maxDisparity=32, speckleWindowSize=0)
    disp, _ = run_ours(p, left, right)
    ref = oracle_mod.sgbm(p, left, right)
    assert disp.dtype == np.int16 and disp.shape == (48, 64)
    assert_subpix_close(disp, ref, "color")


def test_bgr_to_gray_matches_oracle(oracle_mod):
    rng = np.random.default_rng(8)
    img = rng.integers(0, 256, (123, 77, 3), dtype=np.uint8)
    assert np.array_equal(bgr_to_gray(img), oracle_mod.bgr2gray(img))


def test_compute_basic_shifted_rectangles():
    """SGBMTest.ComputeBasic (tests/test_sgbm.cpp:163-192)."""
    left = np.zeros((100, 100), np.uint8)
    right = np.zeros((100, 100), np.uint8)
    left[30:71, 30:71] = 128
    right[30:71, 25:66] = 128
    with StereoSGBM(StereoParams(maxDisparity=32, blockSize=5, numDirections=4)) as s:
        disp = s.compute(left, right)
        assert disp.shape == left.shape and disp.dtype == np.int16
        assert s.getLastComputeTimeMs() > 0


def test_different_sizes_and_disparities(oracle_mod):
    """SGBMTest.DifferentSizes / DifferentDisparities (tests/test_sgbm.cpp:220-281),
    one handle reused across sizes (buffers grow)."""
    rng = np.random.default_rng(3)
    with StereoSGBM(StereoParams(maxDisparity=32, numDirections=4, speckleWindowSize=0)) as s:
        for (h, w) in [(48, 64), (96, 128), (240, 320), (480, 640), (48, 64)]:
            left = rng.integers(0, 255, (h, w), dtype=np.uint8)
            right = rng.integers(0, 255, (h, w), dtype=np.uint8)
            disp = s.compute(left, right)
            assert disp.shape == (h, w)
            if h <= 96:
                assert_subpix_close(disp, oracle_mod.sgbm(params_dict(maxDisparity=32,
                                                                      speckleWindowSize=0),
                                                          left, right))
    left = rng.integers(0, 255, (240, 320), dtype=np.uint8)
    right = rng.integers(0, 255, (240, 320), dtype=np.uint8)
    for md in (32, 64, 96, 128):
        with StereoSGBM(StereoParams(maxDisparity=md, numDirections=4)) as s:
            assert s.compute(left, right).shape == (240, 320)


def test_empty_input():
    with StereoSGBM(StereoParams()) as s:
        with pytest.raises(StereoException):
            s.compute(np.zeros((0, 0), np.uint8), np.zeros((0, 0), np.uint8))


def test_size_mismatch():
    with StereoSGBM(StereoParams()) as s:
        with pytest.raises(StereoException):
            s.compute(np.zeros((100, 100), np.uint8), np.zeros((100, 200), np.uint8))


def test_disparity_range_exceeds_gpu_limit():
    rng = np.random.default_rng(0)
    img = rng.integers(0, 255, (64, 64), dtype=np.uint8)
    with StereoSGBM(StereoParams(minDisparity=0, maxDisparity=kSgbmMaxDisparityRange + 32)) as s:
        with pytest.raises(StereoException):
            s.compute(img, img)
    with StereoSGBM(StereoParams(minDisparity=10, maxDisparity=10)) as s:
        with pytest.raises(StereoException):
            s.compute(img, img)


@pytest.mark.parametrize("wl", ["640x480_d64_census_4path", "1920x1080_d128_census_8path"])
def test_schedules_agree_full_size(wl):
    """Per-direction kernels and the fused sweeps give identical volumes and maps."""
    w = synth.WORKLOADS[wl]
    left, right, _ = synth.make_pair(w.pair)
    p = StereoParams(maxDisparity=w.max_disparity, numDirections=w.num_directions,
                     matchingCostMode=MatchingCostMode.Census if w.census else MatchingCostMode.SAD,
                     speckleWindowSize=0)
    outs = []
    for schedule in (1, 4, 6):
        with StereoSGBM(p) as s:
            s.set_schedule(schedule)
            s.retain_intermediates(True)
            d = s.compute(left, right)
            agg = s.intermediate("agg", left.shape + (w.max_disparity,), np.uint16)
            outs.append((d, agg))
    for k in (1, 2):
        assert np.array_equal(outs[0][1], outs[k][1]), k
        assert np.array_equal(outs[0][0], outs[k][0]), k


def test_deterministic_and_handle_reuse():
    left, right, _ = synth.make_pair(synth.PairSpec(200, 120, 5, 4, 40, 2.0, 77))
    p = StereoParams(maxDisparity=48, numDirections=8, matchingCostMode=MatchingCostMode.Census)
    with StereoSGBM(p) as s:
        a = s.compute(left, right).copy()
        b = s.compute(left, right).copy()
    with StereoSGBM(p) as s2:
        c = s2.compute(left, right)
    assert np.array_equal(a, b) and np.array_equal(a, c)


def test_compute_device_matches_host():
    torch = pytest.importorskip("torch")
    left, right, _ = synth.make_pair(synth.PairSpec(256, 96, 5, 4, 40, 2.0, 78))
    p = StereoParams(maxDisparity=64, numDirections=8)
    with StereoSGBM(p) as s:
        host = s.compute(left, right)
        dl = torch.from_numpy(left).cuda()
        dr = torch.from_numpy(right).cuda()
        out = torch.empty((96, 256), dtype=torch.int16, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        s.compute_device(dl.data_ptr(), dr.data_ptr(), 256, 96, out.data_ptr(), stream=stream)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), host)


def test_remap_known_answers(oracle_mod):
    """RectificationTest.GPUvsOpenCV / BilinearInterpolation
    (tests/test_rectification.cpp:189-265) and bit-exactness vs the oracle."""
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(1)
    src = rng.integers(0, 255, (480, 640), dtype=np.uint8)
    my, mx = np.mgrid[0:480, 0:640].astype(np.float32)
    assert np.array_equal(rectify_image_gpu(src, mx, my), cv2.remap(src, mx, my, cv2.INTER_LINEAR))
    g = np.tile((np.arange(100) * 255 // 100).astype(np.uint8), (100, 1))
    my2, mx2 = np.mgrid[0:100, 0:100].astype(np.float32)
    mx2 += 0.5
    my2 += 0.5
    ours = rectify_image_gpu(g, mx2, my2)
    assert np.abs(ours.astype(int) - cv2.remap(g, mx2, my2, cv2.INTER_LINEAR).astype(int)).max() <= 1
    # random sub-pixel maps, gray and BGR: identical to the oracle
    for ch in (1, 3):
        img = rng.integers(0, 256, (90, 120) if ch == 1 else (90, 120, 3), dtype=np.uint8)
        mxr = (rng.random((90, 120)) * 130 - 5).astype(np.float32)
        myr = (rng.random((90, 120)) * 100 - 5).astype(np.float32)
        assert np.array_equal(rectify_image_gpu(img, mxr, myr), oracle_mod.remap(img, mxr, myr))


# ---------------------------------------------------------------------------
# The reference's own CUDA pipeline (oracle/_ref) at the benchmark sizes.
# ---------------------------------------------------------------------------
def _ref_or_skip(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference tree at build time)")


@pytest.mark.parametrize("wl", ["640x480_d64_census_4path", "1920x1080_d128_sad_8path",
                                "1920x1080_d128_census_8path", "2880x1988_d290_census_8path"])
def test_parity_vs_reference_kernels_full_size(wl, oracle_mod):
    _ref_or_skip(oracle_mod)
    w = synth.WORKLOADS[wl]
    left, right, gt = synth.make_pair(w.pair)
    p = params_dict(maxDisparity=w.max_disparity, matchingCostMode=int(w.census),
                    numDirections=w.num_directions, speckleWindowSize=0)
    ref_disp, ref, _ = oracle_mod.ref_sgbm(p, left, right, intermediates=False)
    # 0: the untuned default the bench runs; 4 and 6: the fused sweeps it picks
    # (4 paths: schedule 4; 8 paths: schedule 6); 1: the per-direction fallback
    for schedule in (0, 1, 4, 6):
        ours, inter = run_ours_light(p, left, right, schedule)
        assert np.array_equal(ours, ref_disp), schedule
    # sanity: the scene's disparities are recovered
    v = ours > 0
    assert v.mean() > 0.5
    assert np.median(np.abs(ours[v] / 16.0 - gt[v])) < 1.0


def run_ours_light(pdict, left, right, schedule=0):
    p = to_params(pdict)
    with StereoSGBM(p) as s:
        if schedule:
            s.set_schedule(schedule)
        return s.compute(left, right), None


def test_parity_vs_reference_kernels_intermediates(oracle_mod):
    """Every checkpoint against the reference kernels on the 640x480 workload."""
    _ref_or_skip(oracle_mod)
    w = synth.WORKLOADS["640x480_d64_census_4path"]
    left, right, _ = synth.make_pair(w.pair)
    for mode, nd, ur in ((1, 4, 10), (0, 8, 0), (1, 8, 0)):
        p = params_dict(maxDisparity=64, matchingCostMode=mode, numDirections=nd,
                        uniquenessRatio=ur, speckleWindowSize=0)
        ref_disp, ref, _ = oracle_mod.ref_sgbm(p, left, right, intermediates=True)
        for schedule in (0, 1, 4, 6):
            disp, ours = run_ours(p, left, right, schedule=schedule)
            for key in ("cost", "agg", "disp_wta", "disp_right", "disp_lr"):
                assert np.array_equal(ours[key], ref[key]), (mode, nd, key, schedule)
            assert np.array_equal(disp, ref_disp)


@pytest.mark.parametrize("wl", ["1920x1080_d128_sad_8path", "1920x1080_d128_census_8path"])
def test_parity_vs_reference_kernels_volume_full_size(wl, oracle_mod):
    """The summed aggregated volume of the default 8-path schedule (four
    partial volumes summed mod 2^16 in the selection) and every map after it
    against the reference kernels' agg volume and maps at 1920x1080 D128."""
    _ref_or_skip(oracle_mod)
    w = synth.WORKLOADS[wl]
    left, right, _ = synth.make_pair(w.pair)
    p = params_dict(maxDisparity=w.max_disparity, matchingCostMode=int(w.census),
                    numDirections=w.num_directions, speckleWindowSize=0)
    ref_disp, ref, _ = oracle_mod.ref_sgbm(p, left, right, intermediates=True)
    for schedule in (0, 6):
        disp, ours = run_ours(p, left, right, schedule=schedule)
        for key in ("cost", "agg", "disp_wta", "disp_right", "disp_lr"):
            assert np.array_equal(ours[key], ref[key]), (wl, key, schedule)
        assert np.array_equal(disp, ref_disp), schedule


def test_remap_vs_reference_kernel(oracle_mod):
    _ref_or_skip(oracle_mod)
    rng = np.random.default_rng(2)
    for ch in (1, 3):
        img = rng.integers(0, 256, (200, 300) if ch == 1 else (200, 300, 3), dtype=np.uint8)
        mx = (rng.random((200, 300)) * 320 - 10).astype(np.float32)
        my = (rng.random((200, 300)) * 220 - 10).astype(np.float32)
        assert np.array_equal(rectify_image_gpu(img, mx, my), oracle_mod.ref_remap(img, mx, my))


@pytest.mark.parametrize("schedule", [2, 3, 5, 7, -1])
def test_retired_schedules_rejected(schedule):
    """Only 0 (automatic), 1, 4 and 6 are schedules; the others are refused
    before any device work."""
    with StereoSGBM(StereoParams()) as s:
        with pytest.raises(StereoException):
            s.set_schedule(schedule)
