"""Either side of the disparity map (the next rows after the hot path):
disparity -> depth (disparityToDepthGPU, src/depth_map.cu:74-102) and the
rectification maps generated on the device (cv::initUndistortRectifyMap, the
calls of src/calibration.cpp:253-266).

CPU: the oracle's numpy restatement of the maps is pinned to maps OpenCV made
(tests/golden/maps/rectify_maps.npz, written by tests/golden/maps/make_rectify_maps.py).
GPU: the device maps agree with those within one float ulp (double on the
device, float storage; OpenCV accumulates along the row) and rectify an image
to the same bytes as OpenCV's maps; the device depth agrees
with the IEEE float32 restatement within 4 ulp (the division is the
fast-math one, like the reference's build)."""
import os

import numpy as np
import pytest

from oracle import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "maps", "rectify_maps.npz")


def _cams():
    z = np.load(GOLD)
    w, h = int(z["width"]), int(z["height"])
    for c in range(2):
        for cam in (0, 1):
            yield (w, h, z[f"c{c}_K{cam}"], z[f"c{c}_D{cam}"], z[f"c{c}_R{cam}"], z[f"c{c}_P{cam}"],
                   z[f"c{c}_map{cam}x"], z[f"c{c}_map{cam}y"])


def test_oracle_maps_match_opencv():
    for w, h, K, D, R, P, mx, my in _cams():
        ox, oy = oracle.rectify_maps(K, D, R, P, w, h)
        assert np.abs(ox - mx).max() <= 1e-3 and np.abs(oy - my).max() <= 1e-3


@pytest.mark.gpu
def test_device_maps_match_opencv():
    """Device maps within one float ulp of OpenCV's, and an image rectified
    through them identical to one rectified through OpenCV's maps."""
    torch = pytest.importorskip("torch")
    from lumenstereo_b200 import rectify_image_gpu, rectify_maps_device
    rng = np.random.Generator(np.random.PCG64(31))
    for w, h, K, D, R, P, mx, my in _cams():
        dx = torch.empty((h, w), dtype=torch.float32, device="cuda")
        dy = torch.empty((h, w), dtype=torch.float32, device="cuda")
        rectify_maps_device(K, D, R, P, w, h, dx.data_ptr(), dy.data_ptr())
        torch.cuda.synchronize()
        gx, gy = dx.cpu().numpy(), dy.cpu().numpy()
        ulp_x = np.abs(gx.view(np.int32).astype(np.int64) - mx.view(np.int32))
        ulp_y = np.abs(gy.view(np.int32).astype(np.int64) - my.view(np.int32))
        assert ulp_x.max() <= 1 and ulp_y.max() <= 1, (int(ulp_x.max()), int(ulp_y.max()))
        img = rng.integers(0, 256, (h, w), dtype=np.uint8)
        ours = rectify_image_gpu(img, gx, gy)
        theirs = rectify_image_gpu(img, mx, my)
        assert np.array_equal(ours, theirs), int((ours != theirs).sum())


@pytest.mark.gpu
def test_device_depth_matches_restatement():
    torch = pytest.importorskip("torch")
    from lumenstereo_b200 import disparity_to_depth_device
    rng = np.random.Generator(np.random.PCG64(5))
    disp = rng.integers(-20, 290 * 16, (123, 257)).astype(np.int16)
    disp[0, :10] = [-1, 0, 1, 2, 16, -16, 32767, 5, 0, -32768]
    for f, b, doffs in ((1400.0, 0.12, 0.0), (3997.684, 0.19395, 131.111), (800.0, 0.3, -3.0)):
        dd = torch.from_numpy(disp).cuda()
        out = torch.empty(disp.shape, dtype=torch.float32, device="cuda")
        disparity_to_depth_device(dd.data_ptr(), disp.shape[1], disp.shape[0], f, b, out.data_ptr(), doffs)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        ref = oracle.disparity_to_depth(disp, f, b, doffs)
        assert np.array_equal(got == 0, ref == 0)
        nz = ref != 0
        ulp = np.abs(got[nz].view(np.int32) - ref[nz].view(np.int32))
        assert ulp.max() <= 4, ulp.max()


@pytest.mark.gpu
def test_served_calibration_from_params():
    """A served calibration registered from camera matrices (maps generated on
    the device) gives the plain path's result on the same maps."""
    torch = pytest.importorskip("torch")
    from lumenstereo_b200 import StereoParams, StereoRectifier, StereoServer, StereoSGBM, rectify_maps_device, synth
    z = np.load(GOLD)
    w, h = int(z["width"]), int(z["height"])
    cam = {k: z[f"c0_{k}"] for k in ("K0", "D0", "R0", "P0", "K1", "D1", "R1", "P1")}
    maps = []
    for i in (0, 1):
        dx = torch.empty((h, w), dtype=torch.float32, device="cuda")
        dy = torch.empty((h, w), dtype=torch.float32, device="cuda")
        rectify_maps_device(cam[f"K{i}"], cam[f"D{i}"], cam[f"R{i}"], cam[f"P{i}"], w, h, dx.data_ptr(), dy.data_ptr())
        torch.cuda.synchronize()
        maps += [dx.cpu().numpy(), dy.cpu().numpy()]
    left, right, _ = synth.make_pair(synth.PairSpec(w, h, 4, 1, 20, 2.0, 77))
    p = StereoParams(maxDisparity=32, numDirections=8, speckleWindowSize=0)
    rl, rr = StereoRectifier(w, h, *maps).rectify(left, right)
    with StereoSGBM(p) as s:
        ref = s.compute(rl, rr)
    with StereoServer(budget_bytes=256 << 20) as srv:
        srv.set_calibration_params(7, w, h, cam["K0"], cam["D0"], cam["R0"], cam["P0"],
                                   cam["K1"], cam["D1"], cam["R1"], cam["P1"])
        out, _ = srv.wait(srv.submit(p, left, right, calib_id=7))
    assert np.array_equal(out, ref)
