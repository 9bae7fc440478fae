"""The consumers of the disparity map: colour-coded depth (colorizeDepthKernel,
src/depth_map.cu:104-142, here fused with disparityToDepthKernel into one
pass) and the point cloud (depthToPointCloud, src/point_cloud.cpp:11-55).

CPU: the numpy restatements in the oracle against plain per-pixel loops of the
reference's expressions.  GPU: the device colours against the oracle's index
(the division is the fast-math one, like the reference's build: an index may
differ by one only where the ramp value lies within 1e-3 of an integer); the
fused pass's depth equals the depth-only pass bit for bit; the point cloud is
bit-exact (double arithmetic on both sides, raster order, row offsets)."""
import math

import numpy as np
import pytest

from oracle import oracle


def _depth_field(shape, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    z = rng.uniform(-1.0, 25.0, shape).astype(np.float32)
    flat = z.reshape(-1)
    special = [0.0, -0.0, np.nan, np.inf, -np.inf, 0.5, 10.0, 20.0, 20.000002, 100.0, 100.00001, 1e-30]
    flat[:len(special)] = special[:flat.size]
    flat[rng.integers(0, flat.size, flat.size // 10)] = 0.0
    return z


def _index_loop(z, lo, hi):
    f32 = np.float32
    out = np.zeros(z.shape, np.int32)
    for i, d in np.ndenumerate(z):
        if d <= 0 or d > f32(hi) * f32(2):
            continue
        n = (d - f32(lo)) / (f32(hi) - f32(lo))
        n = f32(1.0) if math.isnan(n) else n     # fminf(1, NaN) = 1
        n = max(f32(0.0), min(f32(1.0), n))
        out[i] = int(f32(f32(1.0) - n) * f32(255.0))
    return out


def test_color_index_restatement_matches_loop():
    z = _depth_field((9, 13), 3)
    with np.errstate(invalid="ignore", over="ignore"):
        for lo, hi in ((0.5, 10.0), (2.0, 3.0), (0.0, 120.0)):
            assert np.array_equal(oracle.depth_color_index(z, lo, hi), _index_loop(z, lo, hi))


def test_point_cloud_restatement_matches_loop():
    z = _depth_field((7, 11), 4)
    rng = np.random.Generator(np.random.PCG64(5))
    bgr = rng.integers(0, 256, (7, 11, 3), dtype=np.uint8)
    fx, fy, cx, cy = 1234.5, 1229.25, 5.3, 3.1
    for color in (bgr, None, bgr[:6]):
        xyz, rgb = oracle.depth_to_point_cloud(z, color, fx, fy, cx, cy)
        exp = []
        for v in range(z.shape[0]):
            for u in range(z.shape[1]):
                Z = z[v, u]
                if Z <= 0 or Z > 100.0:
                    continue
                X = np.float32((u - cx) * float(Z) / fx)
                Y = np.float32((v - cy) * float(Z) / fy)
                c = (255, 255, 255) if color is None or color.shape[:2] != z.shape else tuple(color[v, u][::-1])
                exp.append((X, Y, Z) + c)
        exp = np.array(exp, dtype=object)
        assert len(xyz) == len(exp)
        got = np.concatenate([xyz.astype(object), rgb.astype(object)], axis=1)
        for a, b in zip(got, exp):
            assert all((x == y) or (isinstance(x, float) and math.isnan(x) and math.isnan(y))
                       for x, y in zip(a, b)), (a, b)


def _index_lut():
    """a table whose first channel is the index itself"""
    i = np.arange(256)
    return np.stack([i, 255 - i, (i * 37) & 255], axis=1).astype(np.uint8)


def _check_indices(got, z, lo, hi):
    ref = oracle.depth_color_index(z, lo, hi)
    diff = got != ref
    if diff.any():
        ramp = oracle.depth_color_ramp(z[diff], lo, hi)
        assert np.all(np.abs(got[diff] - ref[diff]) == 1)
        assert np.all(np.abs(ramp - np.round(ramp)) < 1e-3), ramp
    assert diff.mean() <= 1e-3


@pytest.mark.gpu
def test_device_colorize_matches_restatement():
    torch = pytest.importorskip("torch")
    from lumenstereo_b200 import depth_colorize_device
    lut = _index_lut()
    z = _depth_field((67, 301), 6)
    for lo, hi in ((0.5, 10.0), (1.0, 1.5), (0.0, 30.0)):
        dz = torch.from_numpy(z).cuda()
        rgb = torch.full((67, 301, 3), 7, dtype=torch.uint8, device="cuda")
        depth_colorize_device(dz.data_ptr(), 301, 67, rgb.data_ptr(), lut, lo, hi)
        torch.cuda.synchronize()
        out = rgb.cpu().numpy()
        got = out[..., 0].astype(np.int32)
        assert np.array_equal(out, lut[got])
        with np.errstate(invalid="ignore", over="ignore"):
            _check_indices(got, z, lo, hi)


@pytest.mark.gpu
def test_device_fused_depth_color_matches_two_passes():
    torch = pytest.importorskip("torch")
    from lumenstereo_b200 import disparity_to_depth_color_device, disparity_to_depth_device
    rng = np.random.Generator(np.random.PCG64(7))
    H, W = 131, 517
    disp = rng.integers(-40, 256 * 16, (H, W)).astype(np.int16)
    disp[0, :6] = [-1, 0, 1, 16, 32767, -32768]
    lut = _index_lut()
    dd = torch.from_numpy(disp).cuda()
    for f, b, doffs, lo, hi in ((1400.0, 0.12, 0.0, 0.5, 10.0), (3997.684, 0.19395, 131.111, 1.0, 6.0)):
        ref_depth = torch.empty((H, W), dtype=torch.float32, device="cuda")
        disparity_to_depth_device(dd.data_ptr(), W, H, f, b, ref_depth.data_ptr(), doffs)
        depth = torch.empty((H, W), dtype=torch.float32, device="cuda")
        rgb = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda")
        rgb_only = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda")
        disparity_to_depth_color_device(dd.data_ptr(), W, H, f, b, depth.data_ptr(), rgb.data_ptr(), lut, lo, hi,
                                        doffs)
        disparity_to_depth_color_device(dd.data_ptr(), W, H, f, b, 0, rgb_only.data_ptr(), lut, lo, hi, doffs)
        torch.cuda.synchronize()
        z = ref_depth.cpu().numpy()
        assert np.array_equal(depth.cpu().numpy().view(np.int32), z.view(np.int32))
        out = rgb.cpu().numpy()
        assert np.array_equal(out, rgb_only.cpu().numpy())
        got = out[..., 0].astype(np.int32)
        assert np.array_equal(out, lut[got])
        _check_indices(got, z, lo, hi)


@pytest.mark.gpu
def test_device_point_cloud_bit_exact():
    torch = pytest.importorskip("torch")
    from lumenstereo_b200 import POINT_DTYPE, depth_to_points_device
    rng = np.random.Generator(np.random.PCG64(8))
    for (H, W) in ((97, 1283), (1, 5), (300, 33)):
        z = _depth_field((H, W), 9 + W)
        z[H // 2] = 0.0                       # an empty row
        bgr = rng.integers(0, 256, (H, W, 3), dtype=np.uint8)
        fx, fy, cx, cy = 1733.74, 1731.5, W / 2 - 0.37, H / 2 + 0.81
        dz = torch.from_numpy(z).cuda()
        db = torch.from_numpy(bgr).cuda()
        for color in (bgr, None):
            pts = torch.full((H * W * 16,), 0xAB, dtype=torch.uint8, device="cuda")
            offs = torch.full((H + 1,), -5, dtype=torch.int32, device="cuda")
            depth_to_points_device(dz.data_ptr(), W, H, fx, fy, cx, cy, pts.data_ptr(), offs.data_ptr(),
                                   db.data_ptr() if color is not None else 0)
            torch.cuda.synchronize()
            off = offs.cpu().numpy()
            xyz, rgb = oracle.depth_to_point_cloud(z, color, fx, fy, cx, cy)
            n = int(off[H])
            assert n == len(xyz)
            keep = ~((z <= 0) | (z > 100))
            assert np.array_equal(np.diff(off), keep.sum(axis=1))
            rec = pts.cpu().numpy()[:n * 16].view(POINT_DTYPE)
            got = np.stack([rec["x"], rec["y"], rec["z"]], axis=1)
            nan = np.isnan(xyz)                  # NaN depths stay points; NaN payloads may differ
            assert np.array_equal(np.isnan(got), nan)
            assert np.array_equal(got[~nan].view(np.int32), xyz[~nan].view(np.int32))
            assert np.array_equal(np.stack([rec["r"], rec["g"], rec["b"]], axis=1), rgb)
            assert not rec["pad"].any()


@pytest.mark.gpu
def test_host_point_cloud_matches_oracle():
    from lumenstereo_b200 import depth_to_point_cloud
    z = _depth_field((45, 77), 10)
    rng = np.random.Generator(np.random.PCG64(11))
    bgr = rng.integers(0, 256, (45, 77, 3), dtype=np.uint8)
    K = np.array([[901.5, 0, 38.2], [0, 899.25, 21.7], [0, 0, 1]])
    for color in (bgr, None, bgr[:40]):
        rec = depth_to_point_cloud(z, K, color)
        xyz, rgb = oracle.depth_to_point_cloud(z, color, 901.5, 899.25, 38.2, 21.7)
        got = np.stack([rec["x"], rec["y"], rec["z"]], axis=1)
        nan = np.isnan(xyz)
        assert np.array_equal(np.isnan(got), nan)
        assert np.array_equal(got[~nan].view(np.int32), xyz[~nan].view(np.int32))
        assert np.array_equal(np.stack([rec["r"], rec["g"], rec["b"]], axis=1), rgb)


# ---------------------------------------------------------------------------
# The reference's own depth and colour kernels (oracle/_ref).
# ---------------------------------------------------------------------------
def _ref_or_skip():
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference tree at build time)")


@pytest.mark.gpu
def test_depth_and_colour_vs_reference_kernels():
    """disparityToDepthKernel and colorizeDepthKernel (src/depth_map.cu:74-142)
    against the depth-only pass, the colour-only pass and the fused pass, with
    the reference's own colour table passed as the caller's table: depth bit
    for bit, colours byte for byte.  Depth fields hold no NaN (a disparity map
    never gives one; the reference's clamp of NaN under fast math is not part
    of the comparison)."""
    _ref_or_skip()
    torch = pytest.importorskip("torch")
    from lumenstereo_b200 import (depth_colorize_device, disparity_to_depth_color_device,
                                  disparity_to_depth_device)
    lut = oracle.ref_turbo_table()
    rng = np.random.Generator(np.random.PCG64(21))
    H, W = 257, 611
    disp = rng.integers(-40, 300 * 16, (H, W)).astype(np.int16)
    disp[0, :6] = [-1, 0, 1, 16, 32767, -32768]
    dd = torch.from_numpy(disp).cuda()
    for f, b, doffs, lo, hi in ((1400.0, 0.12, 0.0, 0.5, 10.0), (3997.684, 0.19395, 131.111, 1.0, 6.0),
                                (2000.0, 0.3, -3.5, 0.2, 3.0)):
        ref_z = oracle.ref_depth(disp, f, b, doffs)
        ref_rgb = oracle.ref_colorize(ref_z, lo, hi)
        z = torch.empty((H, W), dtype=torch.float32, device="cuda")
        disparity_to_depth_device(dd.data_ptr(), W, H, f, b, z.data_ptr(), doffs)
        z2 = torch.empty((H, W), dtype=torch.float32, device="cuda")
        rgb = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda")
        disparity_to_depth_color_device(dd.data_ptr(), W, H, f, b, z2.data_ptr(), rgb.data_ptr(), lut, lo, hi,
                                        doffs)
        rgb2 = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda")
        depth_colorize_device(torch.from_numpy(ref_z).cuda().data_ptr(), W, H, rgb2.data_ptr(), lut, lo, hi)
        torch.cuda.synchronize()
        assert np.array_equal(z.cpu().numpy().view(np.int32), ref_z.view(np.int32)), (f, b, doffs)
        assert np.array_equal(z2.cpu().numpy().view(np.int32), ref_z.view(np.int32)), (f, b, doffs)
        assert np.array_equal(rgb.cpu().numpy(), ref_rgb), (f, b, doffs, lo, hi)
        assert np.array_equal(rgb2.cpu().numpy(), ref_rgb), (f, b, doffs, lo, hi)
    # a depth field with values below, inside and far above the colour range
    zf = _depth_field((93, 177), 22)
    zf = np.ascontiguousarray(np.where(np.isnan(zf), np.float32(0.0), zf), np.float32)
    h2, w2 = zf.shape
    for lo, hi in ((0.5, 10.0), (1.0, 1.5), (0.0, 30.0)):
        out = torch.empty((h2, w2, 3), dtype=torch.uint8, device="cuda")
        depth_colorize_device(torch.from_numpy(zf).cuda().data_ptr(), w2, h2, out.data_ptr(), lut, lo, hi)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), oracle.ref_colorize(zf, lo, hi)), (lo, hi)
