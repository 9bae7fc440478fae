"""Seeded synthetic stereo pairs (the benchmark inputs).

The reference measures on Middlebury scenes that are not available here, so
every workload is a seeded synthetic pair with the same shapes and value
ranges: a fractal value-noise texture (4 octaves, 0-255) over a Voronoi
partition into slanted planes ``d = a*x + b*y + c`` clipped to the ground-truth
range; the right image is the left forward-warped by ``x_r = x - d`` with a
z-buffer (larger disparity, i.e. nearer, wins), holes filled with fresh noise,
then gain U(0.9, 1.1), offset U(-10, 10) and Gaussian noise, clipped to uint8.

Everything is drawn from ``numpy.random.PCG64(seed)``, so a (config, seed)
pair gives the same bytes on every machine.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass(frozen=True)
class PairSpec:
    width: int
    height: int
    n_planes: int
    d_lo: float
    d_hi: float
    sigma: float
    seed: int
    low_texture_frac: float = 0.0


@dataclass(frozen=True)
class Workload:
    """One benchmark configuration: the pair recipe plus matcher settings."""
    name: str
    pair: PairSpec
    max_disparity: int
    census: bool
    num_directions: int
    extra: dict = field(default_factory=dict)


# The three single-pair configurations (640x480 / 1920x1080 / 2880x1988).
WORKLOADS = {
    "640x480_d64_census_4path": Workload(
        "640x480_d64_census_4path", PairSpec(640, 480, 6, 4, 60, 2.0, 1), 64, True, 4),
    "1920x1080_d128_sad_8path": Workload(
        "1920x1080_d128_sad_8path", PairSpec(1920, 1080, 12, 8, 124, 3.0, 2), 128, False, 8),
    "1920x1080_d128_census_8path": Workload(
        "1920x1080_d128_census_8path", PairSpec(1920, 1080, 12, 8, 124, 3.0, 2), 128, True, 8),
    "2880x1988_d290_census_8path": Workload(
        "2880x1988_d290_census_8path", PairSpec(2880, 1988, 20, 10, 280, 3.0, 3, 0.3), 290, True, 8),
}

# Size classes of the mixed batch / served stream: (W, H, maxDisparity).
MIX_SIZES = [(640, 480, 64), (1280, 720, 128), (1920, 1080, 128), (2880, 1988, 192)]


def _value_noise(rng: np.random.Generator, w: int, h: int, octaves: int = 4,
                 base_cell: int = 16) -> np.ndarray:
    """Fractal value noise in [0, 1): lattice values, smoothstep-bilinear."""
    out = np.zeros((h, w), dtype=np.float64)
    amp, total = 1.0, 0.0
    cell = float(base_cell)
    ys = np.arange(h, dtype=np.float64)
    xs = np.arange(w, dtype=np.float64)
    for _ in range(octaves):
        gh = int(np.ceil(h / cell)) + 2
        gw = int(np.ceil(w / cell)) + 2
        lat = rng.random((gh, gw))
        fy, fx = ys / cell, xs / cell
        iy, ix = np.floor(fy).astype(np.int64), np.floor(fx).astype(np.int64)
        ty, tx = fy - iy, fx - ix
        ty = ty * ty * (3 - 2 * ty)
        tx = tx * tx * (3 - 2 * tx)
        a = lat[iy][:, ix]
        b = lat[iy][:, ix + 1]
        c = lat[iy + 1][:, ix]
        d = lat[iy + 1][:, ix + 1]
        top = a + (b - a) * tx[None, :]
        bot = c + (d - c) * tx[None, :]
        out += amp * (top + (bot - top) * ty[:, None])
        total += amp
        amp *= 0.5
        cell = max(cell / 2.0, 1.0)
    return out / total


def make_pair(spec: PairSpec):
    """Return (left u8[H,W], right u8[H,W], gt_disparity f32[H,W])."""
    rng = np.random.Generator(np.random.PCG64(spec.seed))
    w, h = spec.width, spec.height
    tex = _value_noise(rng, w, h)
    tex = (tex - tex.min()) / max(tex.max() - tex.min(), 1e-12)

    # Voronoi cells, one slanted plane each.
    k = spec.n_planes
    sx = rng.uniform(0, w, k)
    sy = rng.uniform(0, h, k)
    c = rng.uniform(spec.d_lo, spec.d_hi, k)
    span = spec.d_hi - spec.d_lo
    a = rng.uniform(-0.25, 0.25, k) * span / w
    b = rng.uniform(-0.25, 0.25, k) * span / h
    low = rng.random(k) < spec.low_texture_frac
    yy, xx = np.mgrid[0:h, 0:w]
    best = np.full((h, w), np.inf)
    label = np.zeros((h, w), dtype=np.int64)
    for i in range(k):
        dist = (xx - sx[i]) ** 2 + (yy - sy[i]) ** 2
        m = dist < best
        best[m] = dist[m]
        label[m] = i
    gt = a[label] * (xx - sx[label]) + b[label] * (yy - sy[label]) + c[label]
    gt = np.clip(gt, spec.d_lo, spec.d_hi)

    if low.any():
        mean = tex.mean()
        lm = low[label]
        tex = np.where(lm, mean + (tex - mean) / 8.0, tex)
    left = np.clip(np.rint(tex * 255.0), 0, 255).astype(np.uint8)

    # Forward warp with a z-buffer: key = (quantised d, source index), max wins.
    xr = np.rint(xx - gt).astype(np.int64)
    ok = (xr >= 0) & (xr < w)
    tgt = (yy * w + xr)[ok]
    src = (yy * w + xx)[ok]
    dq = np.rint(gt[ok] * 1024.0).astype(np.int64)
    key = (dq << 32) | src
    zbuf = np.full(h * w, -1, dtype=np.int64)
    np.maximum.at(zbuf, tgt, key)
    filled = zbuf >= 0
    fresh = _value_noise(rng, w, h)
    fresh = (fresh - fresh.min()) / max(fresh.max() - fresh.min(), 1e-12)
    right = np.rint(fresh.reshape(-1) * 255.0)
    right[filled] = left.reshape(-1)[zbuf[filled] & 0xFFFFFFFF]
    right = right.reshape(h, w)

    gain = rng.uniform(0.9, 1.1)
    offset = rng.uniform(-10.0, 10.0)
    noise = rng.normal(0.0, spec.sigma, (h, w))
    right = np.clip(np.rint(gain * right + offset + noise), 0, 255).astype(np.uint8)
    return left, right, gt.astype(np.float32)


def workload_pair(name: str):
    wl = WORKLOADS[name]
    return make_pair(wl.pair)


def mix_item(seed: int):
    """One pair of the mixed-size batch / served stream, drawn from ``seed``:
    returns (PairSpec, maxDisparity, census, num_directions)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w, h, dmax = MIX_SIZES[int(rng.integers(0, len(MIX_SIZES)))]
    census = bool(rng.integers(0, 2))
    ndir = 8 if rng.integers(0, 2) else 4
    planes = max(4, (w * h) // 150000)
    spec = PairSpec(w, h, planes, 4, dmax - 4, 2.0, seed)
    return spec, dmax, census, ndir


def calibration_maps(calib_id: int, w: int, h: int):
    """Rectification maps of a synthetic calibration (seed 500 + calib_id):
    focal length f ~ U(1000, 2000) px, principal point at the centre, radial
    distortion k1 ~ U(-0.1, 0.1), and per camera a rectifying rotation with
    angles ~ U(-2, 2) degrees about each axis.  For every rectified pixel the
    map holds the raw pixel it samples, the pinhole model with one radial
    term: ray K^-1 (u, v, 1), rotated by R^T, projected, distorted by
    (1 + k1 r^2) and mapped through K.  Returns float32 HxW arrays
    (map0x, map0y, map1x, map1y), the inputs of StereoRectifier."""
    rng = np.random.Generator(np.random.PCG64(500 + calib_id))
    f = rng.uniform(1000.0, 2000.0)
    k1 = rng.uniform(-0.1, 0.1)
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    u, v = np.meshgrid(np.arange(w, dtype=np.float64), np.arange(h, dtype=np.float64))
    x, y = (u - cx) / f, (v - cy) / f
    maps = []
    for _ in range(2):
        ax, ay, az = np.deg2rad(rng.uniform(-2.0, 2.0, 3))
        rx = np.array([[1, 0, 0], [0, np.cos(ax), -np.sin(ax)], [0, np.sin(ax), np.cos(ax)]])
        ry = np.array([[np.cos(ay), 0, np.sin(ay)], [0, 1, 0], [-np.sin(ay), 0, np.cos(ay)]])
        rz = np.array([[np.cos(az), -np.sin(az), 0], [np.sin(az), np.cos(az), 0], [0, 0, 1]])
        rt = (rz @ ry @ rx).T
        X = rt[0, 0] * x + rt[0, 1] * y + rt[0, 2]
        Y = rt[1, 0] * x + rt[1, 1] * y + rt[1, 2]
        Z = rt[2, 0] * x + rt[2, 1] * y + rt[2, 2]
        xp, yp = X / Z, Y / Z
        d = 1.0 + k1 * (xp * xp + yp * yp)
        maps += [(f * xp * d + cx).astype(np.float32), (f * yp * d + cy).astype(np.float32)]
    return tuple(maps)


def random_pair(w: int, h: int, seed: int, shift: int = 7):
    """Small random pair for unit tests: right = left shifted by ``shift`` px
    plus noise (cheap, no scene model)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    left = rng.integers(0, 256, (h, w), dtype=np.uint8)
    right = np.roll(left, -shift, axis=1).astype(np.int32)
    right += rng.integers(-6, 7, (h, w))
    return left, np.clip(right, 0, 255).astype(np.uint8)
