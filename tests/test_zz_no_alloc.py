"""lumen_census_cost_noalloc: the Census cost volume for callers that cannot
allocate device memory (a real-time loop that must not take cudaMalloc's
implicit device synchronisation, a plugin host whose pool owns all device
memory, work built inside a stream capture).  Its only intermediate lives in a
fixed array inside the library, so the test checks that two calls in a row
(the second smaller and with a different disparity range, so the array still
holds the first call's descriptors) each give exactly the cost volume of the
ordinary entry point, lumen_sgbm_compute.  Cost volumes are integers: the
tolerance is zero.

This file is collected last on purpose: it runs on its own in a fresh process
and after every other test."""
import ctypes as C

import numpy as np
import pytest

from lumenstereo_b200 import MatchingCostMode, StereoParams, StereoSGBM, _lib, synth


def _cost_via_compute(left, right, min_d, max_d):
    """Cost volume [H][W][D] from the ordinary (allocating) pipeline."""
    h, w = left.shape
    p = StereoParams(minDisparity=min_d, maxDisparity=max_d, numDirections=4,
                     matchingCostMode=MatchingCostMode.Census, speckleWindowSize=0)
    with StereoSGBM(p) as s:
        s.retain_intermediates(True)
        s.compute(left, right)
        return s.intermediate("cost", (h, w, max_d - min_d), np.uint8)


def test_no_alloc_rejects_oversized_images():
    lib = _lib.lib()
    cap = int(lib.lumen_census_cost_noalloc_max_pixels())
    assert cap == 1 << 21
    w = 4096
    h = cap // w + 1
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    st = lib.lumen_census_cost_noalloc(dummy, dummy, w, h, 0, 64, dummy, 64, None)
    assert st == _lib.ERR_OUT_OF_BUDGET
    assert "scratch" in _lib.last_error()


@pytest.mark.gpu
def test_no_alloc_matches_compute_two_calls():
    import torch

    assert torch.cuda.is_available()
    lib = _lib.lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    cases = [  # (pair spec, minDisparity, maxDisparity, cost_stride)
        (synth.PairSpec(1920, 1080, 8, 4, 100, 2.0, 11), 0, 128, 128),
        (synth.PairSpec(640, 480, 5, 4, 60, 2.0, 12), 7, 83, 80),
    ]
    for spec, min_d, max_d, stride in cases:
        left, right, _ = synth.make_pair(spec)
        h, w = left.shape
        D = max_d - min_d
        dl = torch.from_numpy(left).to(dev)
        dr = torch.from_numpy(right).to(dev)
        dcost = torch.full((h, w, stride), 0xA5, dtype=torch.uint8, device=dev)
        st = lib.lumen_census_cost_noalloc(dl.data_ptr(), dr.data_ptr(), w, h, min_d, max_d,
                                           dcost.data_ptr(), stride, stream.cuda_stream)
        assert st == _lib.OK, _lib.last_error()
        stream.synchronize()
        ours = dcost.cpu().numpy()
        ref = _cost_via_compute(left, right, min_d, max_d)
        assert np.array_equal(ours[:, :, :D], ref), (w, h, D)
        assert not ours[:, :, D:].any(), "padding entries must be 0"
