"""lumen_census_cost_noalloc: the Census cost volume for callers that cannot
allocate device memory (a real-time loop that must not take cudaMalloc's
implicit device synchronisation, a plugin host whose pool owns all device
memory).  Its only intermediate lives in a fixed array inside the library, so
the GPU test makes two calls in a row (the second smaller and with another
disparity range, so the array still holds the first call's descriptors) and
checks each against the oracle's Census cost volume and against the cost
volume of the ordinary entry point, lumen_sgbm_compute.  Cost volumes are
integers: the tolerance is zero.  It also checks that, once the library's
device code is loaded, the calls take no device memory.

The file name makes pytest collect it after every other test file, so a run
that stops at the first failure has run everything else before it.  The test
needs nothing from the other tests: it passes alone in a fresh process and
after them."""
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


def test_no_alloc_rejects_before_launching():
    """Size, alignment and range errors come back before anything touches the
    (here fake) device pointers."""
    lib = _lib.lib()
    cap = int(lib.lumen_census_cost_noalloc_max_pixels())
    assert cap == 1 << 21
    w = 4096
    h = cap // w + 1
    dummy = C.c_void_p(16)  # never dereferenced: every check comes first
    st = lib.lumen_census_cost_noalloc(dummy, dummy, w, h, 0, 64, dummy, 64, None)
    assert st == _lib.ERR_OUT_OF_BUDGET
    assert "scratch" in _lib.last_error()
    st = lib.lumen_census_cost_noalloc(dummy, dummy, 64, 64, 0, 64, C.c_void_p(24), 64, None)
    assert st == _lib.ERR_INVALID_ARGUMENT
    assert "aligned" in _lib.last_error()
    st = lib.lumen_census_cost_noalloc(dummy, dummy, 64, 64, 2100, 2164, dummy, 64, None)
    assert st == _lib.ERR_INVALID_ARGUMENT
    st = lib.lumen_census_cost_noalloc(dummy, dummy, 64, 64, 0, 64, dummy, 72, None)
    assert st == _lib.ERR_INVALID_ARGUMENT


@pytest.mark.gpu
def test_no_alloc_matches_compute_two_calls():
    import torch

    from oracle import oracle

    assert torch.cuda.is_available()
    lib = _lib.lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    # A first call loads the library's device code on this device; with lazy
    # module loading that is when the driver commits the fixed scratch array
    # (its 16 MiB show up once in the free-memory count).  Calls after it must
    # take no device memory at all.
    tiny = torch.zeros((16, 16), dtype=torch.uint8, device=dev)
    tiny_cost = torch.zeros((16, 16, 16), dtype=torch.uint8, device=dev)
    assert lib.lumen_census_cost_noalloc(tiny.data_ptr(), tiny.data_ptr(), 16, 16, 0, 16,
                                         tiny_cost.data_ptr(), 16, stream.cuda_stream) == _lib.OK
    stream.synchronize()
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
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        st = lib.lumen_census_cost_noalloc(dl.data_ptr(), dr.data_ptr(), w, h, min_d, max_d,
                                           dcost.data_ptr(), stride, stream.cuda_stream)
        assert st == _lib.OK, _lib.last_error()
        stream.synchronize()
        assert torch.cuda.mem_get_info(dev)[0] == free_before, "the call took device memory"
        ours = dcost.cpu().numpy()
        assert np.array_equal(ours[:, :, :D], oracle.census_cost(left, right, min_d, max_d)), \
            (w, h, D)
        assert np.array_equal(ours[:, :, :D], _cost_via_compute(left, right, min_d, max_d)), \
            (w, h, D)
        assert not ours[:, :, D:].any(), "padding entries must be 0"
