"""StereoParams / limits API (mirrors tests/test_sgbm.cpp:28-75 of the reference)."""
from lumenstereo_b200 import (MatchingCostMode, StereoParams, kSgbmMaxDisparityRange,
                              middleburyMatcherMaxDisparity)


def test_default_values():
    p = StereoParams()
    assert p.minDisparity == 0
    assert p.maxDisparity == 128
    assert p.blockSize == 5
    assert p.P1 == 200 and p.P2 == 800
    assert p.preFilterCap == 31
    assert p.uniquenessRatio == 10
    assert p.disp12MaxDiff == 1
    assert p.speckleWindowSize == 100 and p.speckleRange == 32
    assert p.useGPU and p.useSharedMemory
    assert p.numDirections == 4
    assert p.matchingCostMode == MatchingCostMode.SAD
    assert p.isValid()


def test_invalid_block_size():
    p = StereoParams()
    for bs in (4, 0, -1):
        p.blockSize = bs
        assert not p.isValid()


def test_invalid_disparity():
    p = StereoParams(minDisparity=100, maxDisparity=50)
    assert not p.isValid()
    p = StereoParams(minDisparity=-10, maxDisparity=128)
    assert not p.isValid()


def test_invalid_penalties():
    assert not StereoParams(P1=100, P2=50).isValid()


def test_invalid_uniqueness():
    assert not StereoParams(uniquenessRatio=-1).isValid()
    assert not StereoParams(uniquenessRatio=101).isValid()


def test_auto_penalties():
    p = StereoParams(blockSize=5)
    p.autoComputePenalties(1)
    assert p.P1 == 8 * 1 * 5 * 5
    assert p.P2 == 32 * 1 * 5 * 5
    assert p.P2 > p.P1


def test_limits():
    assert kSgbmMaxDisparityRange == 512
    assert middleburyMatcherMaxDisparity(290) == 290
    assert middleburyMatcherMaxDisparity(0) == 96
    assert middleburyMatcherMaxDisparity(-5, 64) == 64
    assert middleburyMatcherMaxDisparity(1000) == 512


def test_roundtrip_c_struct():
    p = StereoParams(minDisparity=3, maxDisparity=77, numDirections=8,
                     matchingCostMode=MatchingCostMode.Census, useGPU=False)
    q = StereoParams.from_c(p.to_c())
    assert q == p
