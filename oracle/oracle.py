"""ctypes bindings to the test-only checkers.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py, never by the product package.

* ``liboracle.so``  -- C restatement of the reference's SGBM path (sgbm_oracle.c)
* ``_ref/libref_sgbm.so`` -- the reference's own CUDA kernels with a host
  driver that restates src/sgbm_gpu.cu (needs a GPU; optional).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import astuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

PATH_NAMES = ["LR", "RL", "TB", "BT", "TLBR", "BRTL", "TRBL", "BLTR"]


class OracleParams(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "minDisparity", "maxDisparity", "blockSize", "P1", "P2", "preFilterCap",
        "uniquenessRatio", "disp12MaxDiff", "speckleWindowSize", "speckleRange", "useGPU",
        "useSharedMemory", "numDirections", "matchingCostMode")]


class OracleIntermediates(C.Structure):
    _fields_ = [("gray_left", C.c_void_p), ("gray_right", C.c_void_p),
                ("pref_left", C.c_void_p), ("pref_right", C.c_void_p),
                ("census_left", C.c_void_p), ("census_right", C.c_void_p),
                ("cost", C.c_void_p), ("agg", C.c_void_p), ("disp_wta", C.c_void_p),
                ("disp_right", C.c_void_p), ("disp_lr", C.c_void_p)]


class RefDump(C.Structure):
    _fields_ = [("pref_left", C.c_void_p), ("pref_right", C.c_void_p),
                ("census_left", C.c_void_p), ("census_right", C.c_void_p),
                ("cost", C.c_void_p), ("agg", C.c_void_p), ("disp_wta", C.c_void_p),
                ("disp_right", C.c_void_p), ("disp_lr", C.c_void_p)]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def build():
    """Build liboracle.so (and _ref when the reference tree is present)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        _LIB.oracle_sgbm_compute.restype = C.c_int
        _LIB.oracle_sgbm_compute.argtypes = [C.POINTER(OracleParams), C.c_void_p, C.c_void_p,
                                             C.c_int, C.c_int, C.c_int, C.c_void_p,
                                             C.POINTER(OracleIntermediates), C.c_uint]
        _LIB.oracle_max_threads.restype = C.c_int
    return _LIB


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_sgbm.so"))


def ref():
    global _REF
    if _REF is None:
        _REF = C.CDLL(os.path.join(HERE, "_ref", "libref_sgbm.so"))
        _REF.ref_sgbm_run.restype = C.c_int
        _REF.ref_sgbm_run.argtypes = [C.POINTER(OracleParams), C.c_void_p, C.c_void_p, C.c_int,
                                      C.c_int, C.c_void_p, C.POINTER(RefDump), C.c_uint, C.c_int,
                                      C.POINTER(C.c_float)]
        _REF.ref_remap_run.restype = C.c_int
        _REF.ref_last_error.restype = C.c_char_p
    return _REF


def to_params(p) -> OracleParams:
    """From any object with the StereoParams field names (or a dict)."""
    get = (lambda k: p[k]) if isinstance(p, dict) else (lambda k: getattr(p, k))
    vals = []
    for name, _ in OracleParams._fields_:
        v = get(name)
        vals.append(int(v))
    return OracleParams(*vals)


def set_threads(n: int):
    lib().oracle_set_threads(int(n))


def max_threads() -> int:
    return lib().oracle_max_threads()


def sgbm(params, left: np.ndarray, right: np.ndarray, intermediates: bool = False,
         path_mask: int = 0):
    """Full pipeline. Returns disparity (int16 HxW), or (disparity, dict)."""
    left = np.ascontiguousarray(left)
    right = np.ascontiguousarray(right)
    h, w = left.shape[:2]
    ch = 1 if left.ndim == 2 else left.shape[2]
    p = to_params(params)
    D = p.maxDisparity - p.minDisparity
    out = np.zeros((h, w), np.int16)
    inter = None
    arrs = {}
    if intermediates:
        arrs = dict(
            gray_left=np.zeros((h, w), np.uint8), gray_right=np.zeros((h, w), np.uint8),
            pref_left=np.zeros((h, w), np.uint8), pref_right=np.zeros((h, w), np.uint8),
            census_left=np.zeros((h, w), np.uint32), census_right=np.zeros((h, w), np.uint32),
            cost=np.zeros((h, w, max(D, 1)), np.uint8), agg=np.zeros((h, w, max(D, 1)), np.uint16),
            disp_wta=np.zeros((h, w), np.int16), disp_right=np.zeros((h, w), np.int16),
            disp_lr=np.zeros((h, w), np.int16))
        inter = OracleIntermediates(*[_ptr(arrs[f]) for f, _ in OracleIntermediates._fields_])
    rc = lib().oracle_sgbm_compute(C.byref(p), _ptr(left), _ptr(right), w, h, ch, _ptr(out),
                                   C.byref(inter) if inter is not None else None, path_mask)
    if rc != 0:
        raise RuntimeError(f"oracle_sgbm_compute failed with status {rc}")
    return (out, arrs) if intermediates else out


def census_cost(left: np.ndarray, right: np.ndarray, min_disparity: int, max_disparity: int):
    """Census stage alone: descriptors of both gray images
    (src/sgbm_kernels.cu:217-245) and the uint8 cost volume [H][W][D]
    (src/sgbm_kernels.cu:250-286)."""
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    h, w = left.shape
    D = max_disparity - min_disparity
    cl = np.zeros((h, w), np.uint32)
    cr = np.zeros((h, w), np.uint32)
    lib().oracle_census5x5(_ptr(left), _ptr(cl), w, h)
    lib().oracle_census5x5(_ptr(right), _ptr(cr), w, h)
    cost = np.zeros((h, w, D), np.uint8)
    lib().oracle_cost_census(_ptr(cl), _ptr(cr), _ptr(cost), w, h, D, min_disparity)
    return cost


def remap(src: np.ndarray, mapx: np.ndarray, mapy: np.ndarray) -> np.ndarray:
    src = np.ascontiguousarray(src)
    h, w = mapx.shape
    ch = 1 if src.ndim == 2 else src.shape[2]
    dst = np.zeros_like(src)
    lib().oracle_remap(_ptr(src), _ptr(np.ascontiguousarray(mapx, np.float32)),
                       _ptr(np.ascontiguousarray(mapy, np.float32)), _ptr(dst), w, h, ch)
    return dst


def bgr2gray(bgr: np.ndarray) -> np.ndarray:
    bgr = np.ascontiguousarray(bgr)
    h, w = bgr.shape[:2]
    g = np.zeros((h, w), np.uint8)
    lib().oracle_bgr2gray(_ptr(bgr), _ptr(g), w, h, C.c_size_t(w * 3))
    return g


def median3x3(disp: np.ndarray) -> np.ndarray:
    disp = np.ascontiguousarray(disp, np.int16)
    h, w = disp.shape
    out = np.zeros_like(disp)
    lib().oracle_median3x3(_ptr(disp), _ptr(out), w, h)
    return out


def speckle(disp: np.ndarray, max_speckle: int, max_diff: int) -> np.ndarray:
    disp = np.array(disp, np.int16, copy=True)
    h, w = disp.shape
    lib().oracle_speckle(_ptr(disp), w, h, int(max_speckle), int(max_diff))
    return disp


def ref_sgbm(params, left: np.ndarray, right: np.ndarray, intermediates: bool = False,
             path_mask: int = 0, repeats: int = 1):
    """The reference's CUDA pipeline on the GPU (gray input).  Returns
    (disparity, dict of intermediates, best device ms)."""
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    h, w = left.shape
    p = to_params(params)
    D = p.maxDisparity - p.minDisparity
    out = np.zeros((h, w), np.int16)
    arrs = {}
    dump = None
    if intermediates:
        arrs = dict(pref_left=np.zeros((h, w), np.uint8), pref_right=np.zeros((h, w), np.uint8),
                    census_left=np.zeros((h, w), np.uint32),
                    census_right=np.zeros((h, w), np.uint32),
                    cost=np.zeros((h, w, D), np.uint8), agg=np.zeros((h, w, D), np.uint16),
                    disp_wta=np.zeros((h, w), np.int16), disp_right=np.zeros((h, w), np.int16),
                    disp_lr=np.zeros((h, w), np.int16))
        dump = RefDump(*[_ptr(arrs[f]) for f, _ in RefDump._fields_])
    ms = C.c_float(0.0)
    rc = ref().ref_sgbm_run(C.byref(p), _ptr(left), _ptr(right), w, h, _ptr(out),
                            C.byref(dump) if dump is not None else None, path_mask, repeats,
                            C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"ref_sgbm_run failed ({rc}): {ref().ref_last_error()!r}")
    return out, arrs, ms.value


def ref_depth(disp: np.ndarray, focal: float, baseline: float, doffs: float = 0.0) -> np.ndarray:
    """The reference's disparityToDepthKernel (src/depth_map.cu:74-102) on the GPU."""
    disp = np.ascontiguousarray(disp, np.int16)
    h, w = disp.shape
    out = np.zeros((h, w), np.float32)
    rc = ref().ref_depth_run(_ptr(disp), _ptr(out), w, h, C.c_float(focal), C.c_float(baseline),
                             C.c_float(doffs))
    if rc != 0:
        raise RuntimeError(f"ref_depth_run failed ({rc}): {ref().ref_last_error()!r}")
    return out


def ref_colorize(depth: np.ndarray, min_depth: float, max_depth: float) -> np.ndarray:
    """The reference's colorizeDepthKernel (src/depth_map.cu:104-142) on the
    GPU: H x W x 3 bytes in R, G, B order."""
    depth = np.ascontiguousarray(depth, np.float32)
    h, w = depth.shape
    out = np.zeros((h, w, 3), np.uint8)
    rc = ref().ref_colorize_run(_ptr(depth), _ptr(out), w, h, C.c_float(min_depth),
                                C.c_float(max_depth))
    if rc != 0:
        raise RuntimeError(f"ref_colorize_run failed ({rc}): {ref().ref_last_error()!r}")
    return out


def ref_turbo_table() -> np.ndarray:
    """The reference's colour table (src/depth_map.cu:18-64) as 256 x 3 (R, G, B)."""
    out = np.zeros((256, 3), np.uint8)
    rc = ref().ref_turbo_table(_ptr(out))
    if rc != 0:
        raise RuntimeError(f"ref_turbo_table failed ({rc}): {ref().ref_last_error()!r}")
    return out


def ref_remap(src: np.ndarray, mapx: np.ndarray, mapy: np.ndarray) -> np.ndarray:
    src = np.ascontiguousarray(src)
    h, w = mapx.shape
    ch = 1 if src.ndim == 2 else src.shape[2]
    dst = np.zeros_like(src)
    rc = ref().ref_remap_run(_ptr(src), _ptr(np.ascontiguousarray(mapx, np.float32)),
                             _ptr(np.ascontiguousarray(mapy, np.float32)), _ptr(dst), w, h, ch)
    if rc != 0:
        raise RuntimeError(f"ref_remap_run failed ({rc})")
    return dst


def disparity_to_depth(disp: np.ndarray, focal: float, baseline: float, doffs: float = 0.0) -> np.ndarray:
    """disparityToDepthKernel (src/depth_map.cu:74-102) in IEEE float32:
    f * B / (d / 16 + doffs) for d > 0 and a positive denominator, else 0."""
    d = disp.astype(np.float32) / np.float32(16.0)
    denom = d + np.float32(doffs)
    fb = np.float32(focal) * np.float32(baseline)
    with np.errstate(divide="ignore", invalid="ignore"):
        z = fb / denom
    return np.where((disp > 0) & (denom > 0), z, np.float32(0.0)).astype(np.float32)


def depth_color_index(depth: np.ndarray, min_depth: float, max_depth: float) -> np.ndarray:
    """colorizeDepthKernel's index (src/depth_map.cu:121-133) in IEEE float32:
    0 for z <= 0 or z > 2 max, else int((1 - clamp((z - min)/(max - min))) * 255)
    with C's fminf/fmaxf NaN rules."""
    z = depth.astype(np.float32)
    lo, hi = np.float32(min_depth), np.float32(max_depth)
    with np.errstate(divide="ignore", invalid="ignore"):
        n = (z - lo) / (hi - lo)
    n = np.fmax(np.float32(0), np.fmin(np.float32(1), n))
    n = np.float32(1) - n
    idx = (n * np.float32(255)).astype(np.int32)
    bad = (z <= 0) | (z > hi * np.float32(2))
    return np.where(bad, 0, idx).astype(np.int32)


def depth_color_ramp(depth: np.ndarray, min_depth: float, max_depth: float) -> np.ndarray:
    """The pre-truncation value (1 - clamp(...)) * 255 of depth_color_index,
    float64, for locating pixels that sit on an index boundary."""
    z = depth.astype(np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        n = (z - min_depth) / (max_depth - min_depth)
    return (1.0 - np.fmax(0.0, np.fmin(1.0, n))) * 255.0


def depth_to_point_cloud(depth: np.ndarray, bgr, fx: float, fy: float, cx: float, cy: float):
    """depthToPointCloud (src/point_cloud.cpp:11-55): pixels with 0 < Z <= 100
    (NaN kept) in raster order, X = (float)((u - cx) Z / fx), Y likewise in v,
    both in float64; colour (r, g, b) from a BGR image of the same size, else
    white.  Returns (xyz float32 [n, 3], rgb uint8 [n, 3])."""
    z = depth.astype(np.float32)
    keep = ~((z <= 0) | (z > np.float32(100)))
    v, u = np.nonzero(keep)                  # raster order
    Z = z[v, u]
    X = ((u.astype(np.float64) - cx) * Z.astype(np.float64) / fx).astype(np.float32)
    Y = ((v.astype(np.float64) - cy) * Z.astype(np.float64) / fy).astype(np.float32)
    if bgr is not None and bgr.shape[:2] == depth.shape:
        rgb = bgr[v, u][:, ::-1].astype(np.uint8)
    else:
        rgb = np.full((len(Z), 3), 255, np.uint8)
    return np.stack([X, Y, Z], axis=1), np.ascontiguousarray(rgb)


def rectify_maps(K, dist, R, P, width: int, height: int):
    """The maps of cv::initUndistortRectifyMap (CV_32FC1), restated in float64
    numpy from the published pinhole + Brown-Conrady model: the ray
    (P[:, :3] R)^-1 (u, v, 1), projected, distorted by (k1, k2, p1, p2, k3) and
    mapped through K."""
    K = np.asarray(K, np.float64).reshape(3, 3)
    R = np.asarray(R, np.float64).reshape(3, 3)
    P = np.asarray(P, np.float64).reshape(3, 4)
    k = np.zeros(5) if dist is None else np.concatenate([np.asarray(dist, np.float64).ravel(), np.zeros(5)])[:5]
    iR = np.linalg.inv(P[:, :3] @ R)
    u, v = np.meshgrid(np.arange(width, dtype=np.float64), np.arange(height, dtype=np.float64))
    X = iR[0, 0] * u + iR[0, 1] * v + iR[0, 2]
    Y = iR[1, 0] * u + iR[1, 1] * v + iR[1, 2]
    Z = iR[2, 0] * u + iR[2, 1] * v + iR[2, 2]
    x, y = X / Z, Y / Z
    x2, y2 = x * x, y * y
    r2, xy2 = x2 + y2, 2 * x * y
    s = 1 + ((k[4] * r2 + k[1]) * r2 + k[0]) * r2
    xd = x * s + k[2] * xy2 + k[3] * (r2 + 2 * x2)
    yd = y * s + k[2] * (r2 + 2 * y2) + k[3] * xy2
    return ((K[0, 0] * xd + K[0, 2]).astype(np.float32), (K[1, 1] * yd + K[1, 2]).astype(np.float32))
