"""lumenstereo_b200 -- B200-native SGBM stereo matching.

Python mirror of LumenStereo's public C++ API for the stereo path
(include/stereo/stereo_params.h, sgbm_limits.h, sgbm_gpu.h, rectification.h,
common.h of the reference), over the C ABI in include/lumen_sgbm.h:

    params = StereoParams(maxDisparity=64, numDirections=8)
    sgbm = StereoSGBM(params)
    disparity = sgbm.compute(left, right)      # int16, 1/16 px, -1 invalid

Errors follow the reference: StereoException for empty input, size mismatch
and bad disparity ranges; CudaException (with ``error_code``) for CUDA
failures.  Arrays are numpy; device tensors (torch) go through
``compute_device``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields
from enum import IntEnum

import numpy as np

from . import _lib

__all__ = ["MatchingCostMode", "StereoParams", "StereoSGBM", "StereoBatch", "StereoServer", "StereoRectifier",
           "StereoException", "CudaException", "kSgbmMaxDisparityRange",
           "middleburyMatcherMaxDisparity", "rectify_image_gpu", "bgr_to_gray",
           "disparity_to_depth_device", "rectify_maps_device"]

# include/stereo/sgbm_limits.h:9
kSgbmMaxDisparityRange = 512


def middleburyMatcherMaxDisparity(calibNumDisparities: int, fallbackWhenMissing: int = 96) -> int:
    """include/stereo/sgbm_limits.h:11-22."""
    ndisp = calibNumDisparities if calibNumDisparities > 0 else fallbackWhenMissing
    return kSgbmMaxDisparityRange if ndisp > kSgbmMaxDisparityRange else ndisp


class MatchingCostMode(IntEnum):
    """include/stereo/stereo_params.h:20-23."""
    SAD = 0
    Census = 1


@dataclass
class StereoParams:
    """include/stereo/stereo_params.h:57-104 (same fields, defaults and checks)."""
    minDisparity: int = 0
    maxDisparity: int = 128
    blockSize: int = 5
    P1: int = 200
    P2: int = 800
    preFilterCap: int = 31
    uniquenessRatio: int = 10
    disp12MaxDiff: int = 1
    speckleWindowSize: int = 100
    speckleRange: int = 32
    useGPU: bool = True
    useSharedMemory: bool = True
    numDirections: int = 4
    matchingCostMode: MatchingCostMode = MatchingCostMode.SAD

    def autoComputePenalties(self, numChannels: int = 1) -> None:
        self.P1 = 8 * numChannels * self.blockSize * self.blockSize
        self.P2 = 32 * numChannels * self.blockSize * self.blockSize

    def isValid(self) -> bool:
        if self.blockSize < 1 or self.blockSize % 2 == 0:
            return False
        if self.minDisparity < 0:
            return False
        if self.maxDisparity <= self.minDisparity:
            return False
        if self.P2 <= self.P1:
            return False
        if self.uniquenessRatio < 0 or self.uniquenessRatio > 100:
            return False
        return True

    def to_c(self) -> _lib.CParams:
        return _lib.CParams(*[int(getattr(self, n)) for n in _lib.PARAM_FIELDS])

    @classmethod
    def from_c(cls, c: _lib.CParams) -> "StereoParams":
        vals = {n: getattr(c, n) for n in _lib.PARAM_FIELDS}
        vals["useGPU"] = bool(vals["useGPU"])
        vals["useSharedMemory"] = bool(vals["useSharedMemory"])
        vals["matchingCostMode"] = MatchingCostMode(vals["matchingCostMode"])
        return cls(**vals)

    def replace(self, **kw) -> "StereoParams":
        d = {f.name: getattr(self, f.name) for f in fields(self)}
        d.update(kw)
        return StereoParams(**d)


class StereoException(RuntimeError):
    """include/stereo/common.h:105-110."""


class CudaException(RuntimeError):
    """include/stereo/common.h:31-48 (``error_code`` carries the status)."""

    def __init__(self, msg: str, error_code: int = _lib.ERR_CUDA):
        super().__init__(msg)
        self.error_code = error_code


class TimeoutException(CudaException):
    """A bounded device-side wait gave up (LUMEN_ERR_TIMEOUT)."""


class OutOfBudgetException(StereoException):
    """A request does not fit the device-memory budget (LUMEN_ERR_OUT_OF_BUDGET)."""


def _check(status: int) -> None:
    if status == _lib.OK:
        return
    msg = _lib.last_error()
    if status in (_lib.ERR_INVALID_ARGUMENT, _lib.ERR_RANGE_EXCEEDS_LIMIT):
        raise StereoException(msg)
    if status == _lib.ERR_OUT_OF_BUDGET:
        raise OutOfBudgetException(msg)
    if status == _lib.ERR_TIMEOUT:
        raise TimeoutException(msg, status)
    raise CudaException(msg, status)


def _image_view(img: np.ndarray):
    """(array, channels, row stride) for a uint8 HxW or HxWx3 image whose rows
    are contiguous; copies otherwise."""
    if img.dtype != np.uint8:
        raise StereoException("input images must be uint8")
    if img.ndim == 3 and img.shape[2] == 1:
        img = img[:, :, 0]
    if img.ndim == 2:
        ch = 1
    elif img.ndim == 3 and img.shape[2] == 3:
        ch = 3
    else:
        raise StereoException("input images must be gray (HxW) or BGR (HxWx3)")
    inner_ok = (img.strides[-1] == 1) and (ch == 1 or img.strides[1] == 3)
    if not inner_ok or img.strides[0] < img.shape[1] * ch:
        img = np.ascontiguousarray(img)
    return img, ch, img.strides[0]


class StereoSGBM:
    """include/stereo/sgbm_gpu.h:29-91."""

    def __init__(self, params: StereoParams | None = None):
        self._h = C.c_void_p()
        p = (params or StereoParams()).to_c()
        _check(_lib.lib().lumen_sgbm_create(C.byref(p), C.byref(self._h)))

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib().lumen_sgbm_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def setParams(self, params: StereoParams) -> None:
        p = params.to_c()
        _check(_lib.lib().lumen_sgbm_set_params(self._h, C.byref(p)))

    def getParams(self) -> StereoParams:
        c = _lib.CParams()
        _check(_lib.lib().lumen_sgbm_get_params(self._h, C.byref(c)))
        return StereoParams.from_c(c)

    def compute(self, left: np.ndarray, right: np.ndarray,
                disparity: np.ndarray | None = None) -> np.ndarray:
        """StereoSGBM::compute (src/sgbm_gpu.cu:147-195): returns (or fills)
        an int16 HxW disparity map in 1/16 px, -1 = invalid."""
        left = np.asarray(left)
        right = np.asarray(right)
        if left.size == 0 or right.size == 0:
            raise StereoException("Input images are empty")
        if left.shape[:2] != right.shape[:2]:
            raise StereoException("Left and right images must have same size")
        left, ch, stride = _image_view(left)
        right, chr_, stride_r = _image_view(right)
        if ch != chr_:
            raise StereoException("Left and right images must have the same channel count")
        if stride_r != stride:
            right = np.ascontiguousarray(right)
            left = np.ascontiguousarray(left)
            stride = left.strides[0]
        h, w = left.shape[:2]
        if disparity is None or disparity.shape != (h, w) or disparity.dtype != np.int16:
            disparity = np.empty((h, w), np.int16)
        elif disparity.strides[1] != 2:
            raise StereoException("disparity output must have contiguous rows")
        _check(_lib.lib().lumen_sgbm_compute(
            self._h, left.ctypes.data, right.ctypes.data, w, h, stride, ch,
            disparity.ctypes.data, disparity.strides[0]))
        return disparity

    def compute_device(self, left_ptr: int, right_ptr: int, width: int, height: int,
                       out_ptr: int, channels: int = 1, in_stride: int = 0, out_stride: int = 0,
                       stream: int = 0) -> None:
        """Asynchronous compute on device buffers (raw CUDA pointers, e.g.
        ``tensor.data_ptr()``) on ``stream`` (a cudaStream_t as int)."""
        _check(_lib.lib().lumen_sgbm_compute_device(
            self._h, left_ptr, right_ptr, width, height, in_stride, channels, out_ptr,
            out_stride, stream or None))  # 0 / None: the default stream

    def _timings(self):
        t = (C.c_float * 4)()
        _check(_lib.lib().lumen_sgbm_get_timings(self._h, t))
        return list(t)

    def getLastComputeTimeMs(self) -> float:
        return self._timings()[0]

    def getCostComputeTimeMs(self) -> float:
        return self._timings()[1]

    def getAggregationTimeMs(self) -> float:
        return self._timings()[2]

    def getPostProcessTimeMs(self) -> float:
        return self._timings()[3]

    # ---- diagnostics (no counterpart in the reference API) ----
    def set_debug_paths(self, mask: int) -> None:
        _check(_lib.lib().lumen_sgbm_debug_set_paths(self._h, mask))

    def set_schedule(self, schedule: int) -> None:
        _check(_lib.lib().lumen_sgbm_set_schedule(self._h, schedule))

    def set_wait_limit(self, spins: int = 0) -> None:
        """Iteration limit of the device-side waits (0 = default)."""
        _check(_lib.lib().lumen_sgbm_debug_set_wait_limit(self._h, spins))

    def stall_test(self, enable: bool = True) -> None:
        """Make one device-side wait of schedules 4 and 6 unsatisfiable (failure-path test)."""
        _check(_lib.lib().lumen_sgbm_debug_stall_test(self._h, 1 if enable else 0))

    def set_tuning(self, lanes_per_pixel: int = 0, warps_per_block: int = 0) -> None:
        """Pin the fused-sweep configuration (0, 0 = automatic)."""
        _check(_lib.lib().lumen_sgbm_set_tuning(self._h, lanes_per_pixel, warps_per_block))

    def set_tuning_columns(self, rows_per_band: int = -1) -> None:
        """Schedule 6 with 8 paths: the column sweeps in a launch of their own
        with this many rows per band (16, 24, 32), 0 for one launch of all four
        sweeps, -1 automatic."""
        _check(_lib.lib().lumen_sgbm_set_tuning_columns(self._h, rows_per_band))

    def get_tuning_columns(self) -> int:
        """Rows per band of the column sweeps' own launch in the last compute (0: none)."""
        r = C.c_int(0)
        _check(_lib.lib().lumen_sgbm_get_tuning_columns(self._h, C.byref(r)))
        return r.value

    def get_tuning(self):
        """(schedule, lanes per pixel, warps per block) the last compute used."""
        out = (C.c_int * 3)()
        _check(_lib.lib().lumen_sgbm_get_tuning(self._h, out))
        return tuple(out)

    def autotune(self, left_ptr: int, right_ptr: int, width: int, height: int,
                 channels: int = 1, in_stride: int = 0, repeats: int = 2) -> str:
        """Time every aggregation schedule/configuration on device buffers and
        keep the fastest for this workload; returns the per-candidate report."""
        buf = C.create_string_buffer(4096)
        _check(_lib.lib().lumen_sgbm_autotune(self._h, left_ptr, right_ptr, width, height,
                                              in_stride, channels, repeats, buf, 4096))
        return buf.value.decode()

    def save_tuning(self, path: str) -> None:
        _check(_lib.lib().lumen_sgbm_tuning_save(self._h, path.encode()))

    def load_tuning(self, path: str) -> None:
        _check(_lib.lib().lumen_sgbm_tuning_load(self._h, path.encode()))

    def enable_trace(self, enable: bool = True) -> None:
        """Record the band timeline of the row-band sweeps (schedules 4 and 6)."""
        _check(_lib.lib().lumen_sgbm_debug_trace(self._h, int(enable)))

    def trace(self) -> np.ndarray:
        """Band timeline of the last traced launch, one row per band ticket.
        Schedule 4 (ticket 2*band + sweep): [first row at the middle pixel ns,
        last row at the middle pixel ns, end ns, sm << 48 | import polls << 32
        | export polls << 16 | row waits].  Schedule 6 (its ticket order):
        [rows start the first pixel ns, rows finish the middle pixel ns, rows
        finish the row ns, sm << 32 | sweep << 16 | 1]."""
        lib = _lib.lib()
        n = C.c_size_t(0)
        _check(lib.lumen_sgbm_debug_trace_copy(self._h, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 4), dtype=np.uint64)
        if n.value:
            _check(lib.lumen_sgbm_debug_trace_copy(self._h, out.ctypes.data, n.value, C.byref(n)))
        return out[: n.value].reshape(-1, 4)

    def launch_count(self) -> int:
        """Kernels this handle has enqueued so far."""
        return int(_lib.lib().lumen_sgbm_debug_launch_count(self._h))

    def timings(self):
        """[total, cost, aggregation, select+post] device ms of the last compute."""
        return self._timings()

    def retain_intermediates(self, enable: bool = True) -> None:
        _check(_lib.lib().lumen_sgbm_debug_retain(self._h, 1 if enable else 0))

    def intermediate(self, which: str, shape, dtype) -> np.ndarray:
        ids = {"pref_left": 0, "pref_right": 1, "census_left": 2, "census_right": 3,
               "cost": 4, "agg": 5, "disp_wta": 6, "disp_right": 7, "disp_lr": 8,
               "gray_left": 9, "gray_right": 10}
        out = np.empty(shape, dtype)
        _check(_lib.lib().lumen_sgbm_debug_copy(self._h, ids[which], out.ctypes.data, out.nbytes))
        return out


class StereoBatch:
    """Batched form of StereoSGBM.compute_device: many pairs (device buffers,
    their own sizes and parameters) per run, one persistent aggregation launch
    per kernel class, optionally replayed from a CUDA graph
    (lumen_sgbm_batch_* in include/lumen_sgbm.h)."""

    def __init__(self, rows_per_band: int = 0, use_graph: bool = False, budget_bytes: int = 0,
                 schedule: int = 0):
        self._h = C.c_void_p()
        _check(_lib.lib().lumen_sgbm_batch_create(C.byref(self._h)))
        self.set_options(rows_per_band, use_graph, budget_bytes)
        if schedule:
            self.set_schedule(schedule)

    def set_schedule(self, schedule: int = 0) -> None:
        """Aggregation of the batch: 6 (four lag-free sweeps), 4 (two wavefront
        sweeps) or 0 (automatic: 6 until the autotuner picks)."""
        _check(_lib.lib().lumen_sgbm_batch_set_schedule(self._h, schedule))

    def config(self):
        """(schedule, rows per band) the next run uses."""
        sc, r = C.c_int(0), C.c_int(0)
        _check(_lib.lib().lumen_sgbm_batch_config(self._h, C.byref(sc), C.byref(r)))
        return sc.value, r.value

    def set_options(self, rows_per_band: int = 0, use_graph: bool = False, budget_bytes: int = 0) -> None:
        _check(_lib.lib().lumen_sgbm_batch_set_options(self._h, rows_per_band, int(use_graph), budget_bytes))

    def add(self, params: StereoParams, left_ptr: int, right_ptr: int, width: int, height: int,
            out_ptr: int) -> None:
        c = params.to_c()
        _check(_lib.lib().lumen_sgbm_batch_add(self._h, C.byref(c), left_ptr, right_ptr, width, height,
                                               out_ptr))

    def clear(self) -> None:
        _check(_lib.lib().lumen_sgbm_batch_clear(self._h))

    def run(self, stream: int = 0) -> None:
        _check(_lib.lib().lumen_sgbm_batch_run(self._h, stream))

    def sync(self, stream: int = 0) -> None:
        _check(_lib.lib().lumen_sgbm_batch_sync(self._h, stream))

    def autotune(self, stream: int = 0, repeats: int = 2):
        """Times the batch with schedule 6 at 16, 24 and 32 rows per band and
        schedule 4 at 4, 8 and 16 (only the schedule set_schedule pinned, if
        any) and keeps the fastest: (rows, ms per run); config() gives the
        schedule."""
        r, ms = C.c_int(0), C.c_float(0)
        _check(_lib.lib().lumen_sgbm_batch_autotune(self._h, stream, repeats, C.byref(r), C.byref(ms)))
        return r.value, ms.value

    def info(self):
        nb, ng, nl = C.c_size_t(0), C.c_int(0), C.c_ulonglong(0)
        _check(_lib.lib().lumen_sgbm_batch_info(self._h, C.byref(nb), C.byref(ng), C.byref(nl)))
        return {"device_bytes": nb.value, "groups": ng.value, "launches": nl.value}

    def close(self) -> None:
        if self._h:
            _lib.lib().lumen_sgbm_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class StereoServer:
    """Served form: a request loop with continuous batching over a device
    arena of ``budget_bytes`` (lumen_server_* in include/lumen_sgbm.h).

        with StereoServer(budget_bytes=8 << 30) as srv:
            srv.set_calibration(3, w, h, m0x, m0y, m1x, m1y)   # resident maps
            rid = srv.submit(params, left, right, calib_id=3)   # returns at once
            disparity, info = srv.wait(rid)                     # info: latency_ms, ...
    """

    def __init__(self, budget_bytes: int = 40 << 30, max_batch_pairs: int = 32, rows_per_band: int = 16,
                 max_inflight: int = 2, watchdog_ms: int = 60000, spin_limit: int = 0,
                 plain_fallback: bool = True, schedule: int = 6):
        o = _lib.CServerOptions()
        _lib.lib().lumen_server_options_default(C.byref(o))
        o.device_budget_bytes = budget_bytes
        o.max_batch_pairs = max_batch_pairs
        o.rows_per_band = rows_per_band
        o.max_inflight = max_inflight
        o.watchdog_ms = watchdog_ms
        o.spin_limit = spin_limit
        o.plain_fallback = 1 if plain_fallback else 0
        o.schedule = schedule
        self._h = C.c_void_p()
        self._outs = {}
        _check(_lib.lib().lumen_server_create(C.byref(o), C.byref(self._h)))

    def set_calibration(self, calib_id: int, width: int, height: int, map0x=None, map0y=None,
                        map1x=None, map1y=None) -> None:
        maps = [None if m is None else np.ascontiguousarray(m, dtype=np.float32)
                for m in (map0x, map0y, map1x, map1y)]
        for m in maps:
            if m is not None and m.shape != (height, width):
                raise StereoException("maps must be height x width float32")
        ptrs = [None if m is None else m.ctypes.data for m in maps]
        _check(_lib.lib().lumen_server_set_calibration(self._h, calib_id, width, height, *ptrs))

    def set_calibration_params(self, calib_id: int, width: int, height: int, K0, D0, R0, P0, K1, D1, R1,
                               P1) -> None:
        """Registers a calibration from its camera matrices; both cameras'
        maps are generated on the device."""
        arrs = []
        for a, n in ((K0, 9), (D0, 5), (R0, 9), (P0, 12), (K1, 9), (D1, 5), (R1, 9), (P1, 12)):
            v = np.zeros(n) if a is None else np.asarray(a, np.float64).ravel()
            if v.size < n:
                v = np.concatenate([v, np.zeros(n - v.size)])
            arrs.append(np.ascontiguousarray(v[:n]))
        _check(_lib.lib().lumen_server_set_calibration_params(self._h, calib_id, width, height,
                                                              *[a.ctypes.data for a in arrs]))

    def submit(self, params: StereoParams, left: np.ndarray, right: np.ndarray, calib_id: int = -1,
               out: np.ndarray | None = None) -> int:
        """Queues a gray uint8 pair (copied before returning); returns its id."""
        left = np.ascontiguousarray(left, dtype=np.uint8)
        right = np.ascontiguousarray(right, dtype=np.uint8)
        if left.ndim != 2 or left.shape != right.shape:
            raise StereoException("Left and right images must have the same size")
        h, w = left.shape
        if out is None:
            out = np.empty((h, w), np.int16)
        c = params.to_c()
        rid = C.c_ulonglong(0)
        _check(_lib.lib().lumen_server_submit(self._h, C.byref(c), calib_id, left.ctypes.data,
                                              right.ctypes.data, w, h, out.ctypes.data, C.byref(rid)))
        self._outs[rid.value] = out
        return rid.value

    def wait(self, request_id: int, timeout_ms: int = -1):
        """(disparity, info) of a request; raises the request's error."""
        info = _lib.CRequestInfo()
        info.status = -1  # stays -1 when the wait itself runs out (the id is kept)
        st = _lib.lib().lumen_server_wait(self._h, request_id, timeout_ms, C.byref(info))
        if st != _lib.OK and info.status != -1:
            self._outs.pop(request_id, None)
        _check(st)
        out = self._outs.pop(request_id)
        return out, {"latency_ms": info.latency_ms, "queue_ms": info.queue_ms, "device_ms": info.device_ms,
                     "batch_pairs": info.batch_pairs, "batch_id": info.batch_id}

    def debug_fail_batches(self, n: int) -> None:
        """Failure injection (tests): the next ``n`` batch launches fail on
        the host before any device work."""
        _check(_lib.lib().lumen_server_debug_fail_batches(self._h, n))

    def stats(self) -> dict:
        s = _lib.CServerStats()
        _check(_lib.lib().lumen_server_get_stats(self._h, C.byref(s)))
        return {n: getattr(s, n) for n, _ in _lib.CServerStats._fields_}

    def close(self) -> None:
        if self._h:
            _lib.lib().lumen_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class StereoRectifier:
    """include/stereo/rectification.h:41-84.  Maps are CV_32FC1 float32 HxW
    arrays (map0x, map0y for the left camera, map1x, map1y for the right);
    without maps the pair is treated as pre-rectified."""

    def __init__(self, width: int, height: int, map0x=None, map0y=None, map1x=None, map1y=None):
        self._h = C.c_void_p()
        self._maps = [None if m is None else np.ascontiguousarray(m, np.float32)
                      for m in (map0x, map0y, map1x, map1y)]
        ptrs = [None if m is None else m.ctypes.data for m in self._maps]
        _check(_lib.lib().lumen_rectifier_create(width, height, *ptrs, C.byref(self._h)))
        self.width, self.height = width, height

    def isPreRectified(self) -> bool:
        return bool(_lib.lib().lumen_rectifier_is_pre_rectified(self._h))

    def rectify(self, left_raw: np.ndarray, right_raw: np.ndarray):
        l = np.ascontiguousarray(left_raw, np.uint8)
        r = np.ascontiguousarray(right_raw, np.uint8)
        ch = 1 if l.ndim == 2 else l.shape[2]
        ol = np.empty_like(l)
        orr = np.empty_like(r)
        _check(_lib.lib().lumen_rectifier_rectify(self._h, l.ctypes.data, r.ctypes.data, ch,
                                                  ol.ctypes.data, orr.ctypes.data))
        return ol, orr

    def rectify_device(self, left_ptr: int, right_ptr: int, channels: int, out_left_ptr: int,
                       out_right_ptr: int, stream: int = 0) -> None:
        _check(_lib.lib().lumen_rectifier_rectify_device(
            self._h, left_ptr, right_ptr, channels, out_left_ptr, out_right_ptr, stream or None))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib().lumen_rectifier_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rectify_image_gpu(src: np.ndarray, map_x: np.ndarray, map_y: np.ndarray) -> np.ndarray:
    """rectifyImageGPU (src/rectification.cu:354-411)."""
    s = np.ascontiguousarray(src, np.uint8)
    ch = 1 if s.ndim == 2 else s.shape[2]
    h, w = map_x.shape
    mx = np.ascontiguousarray(map_x, np.float32)
    my = np.ascontiguousarray(map_y, np.float32)
    dst = np.empty_like(s)
    _check(_lib.lib().lumen_remap(s.ctypes.data, mx.ctypes.data, my.ctypes.data, dst.ctypes.data,
                                  w, h, ch))
    return dst


def bgr_to_gray(bgr: np.ndarray) -> np.ndarray:
    """Device BGR -> gray, BT.601 15-bit fixed point (cv::cvtColor semantics)."""
    b = np.ascontiguousarray(bgr, np.uint8)
    h, w = b.shape[:2]
    g = np.empty((h, w), np.uint8)
    _check(_lib.lib().lumen_bgr_to_gray(b.ctypes.data, b.strides[0], g.ctypes.data, w, h))
    return g


def disparity_to_depth_device(disp_ptr: int, width: int, height: int, focal_px: float, baseline: float,
                              depth_ptr: int, disparity_offset_px: float = 0.0, stream: int = 0) -> None:
    """disparityToDepthGPU (include/stereo/depth_map.h): packed device int16
    disparity (1/16 px) -> packed device float32 depth, f * B / (d/16 + doffs)."""
    _check(_lib.lib().lumen_disparity_to_depth_device(disp_ptr, width, height, 0, focal_px, baseline,
                                                      disparity_offset_px, depth_ptr, 0, stream))


def turbo_lut() -> np.ndarray:
    """A 256 x 3 RGB colour table: OpenCV's COLORMAP_TURBO (the map the
    reference's host colorizeDepth applies, src/depth_map.cu:189-203), taken
    from cv2 at run time."""
    import cv2
    ramp = np.arange(256, dtype=np.uint8).reshape(256, 1)
    return np.ascontiguousarray(cv2.applyColorMap(ramp, cv2.COLORMAP_TURBO).reshape(256, 3)[:, ::-1])


def _lut_bytes(lut) -> np.ndarray:
    t = np.ascontiguousarray(turbo_lut() if lut is None else lut, dtype=np.uint8)
    if t.size != 768:
        raise StereoException("colour table must hold 256 triplets")
    return t.reshape(768)


def disparity_to_depth_color_device(disp_ptr: int, width: int, height: int, focal_px: float, baseline: float,
                                    depth_ptr: int, rgb_ptr: int, lut=None, min_depth: float = 0.5,
                                    max_depth: float = 10.0, disparity_offset_px: float = 0.0,
                                    stream: int = 0) -> None:
    """disparityToDepthKernel + colorizeDepthKernel (src/depth_map.cu:74-142)
    fused: packed device int16 disparity -> packed float32 depth (depth_ptr 0:
    not stored) and packed 3-byte colours (rgb_ptr 0: none).  `lut`: 256 x 3
    uint8 table (default turbo_lut())."""
    t = _lut_bytes(lut) if rgb_ptr else None
    _check(_lib.lib().lumen_disparity_to_depth_color_device(
        disp_ptr, width, height, 0, focal_px, baseline, disparity_offset_px, depth_ptr or None, 0,
        min_depth, max_depth, None if t is None else t.ctypes.data, rgb_ptr or None, 0, stream))


def depth_colorize_device(depth_ptr: int, width: int, height: int, rgb_ptr: int, lut=None,
                          min_depth: float = 0.5, max_depth: float = 10.0, stream: int = 0) -> None:
    """colorizeDepthGPU (include/stereo/depth_map.h:53-56): packed device
    float32 depth -> packed 3-byte colours through a 256 x 3 table."""
    t = _lut_bytes(lut)
    _check(_lib.lib().lumen_depth_colorize_device(depth_ptr, width, height, 0, min_depth, max_depth,
                                                  t.ctypes.data, rgb_ptr, 0, stream))


POINT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("r", "u1"), ("g", "u1"), ("b", "u1"),
                        ("pad", "u1")])


def depth_to_points_device(depth_ptr: int, width: int, height: int, fx: float, fy: float, cx: float,
                           cy: float, points_ptr: int, row_offsets_ptr: int, bgr_ptr: int = 0,
                           stream: int = 0) -> None:
    """depthToPointCloud (src/point_cloud.cpp:11-55) on the device: packed
    float32 depth (and packed BGR colours, 0: white) -> POINT_DTYPE records in
    raster order at points_ptr (room for width*height, 16-byte aligned);
    row_offsets_ptr receives height + 1 int32 offsets, the last one the
    number of points."""
    _check(_lib.lib().lumen_depth_to_points_device(depth_ptr, width, height, 0, bgr_ptr or None, 0, fx, fy,
                                                   cx, cy, points_ptr, row_offsets_ptr, stream))


def depth_to_point_cloud(depth: np.ndarray, K, color: np.ndarray = None) -> np.ndarray:
    """depthToPointCloud(depth, color, params) (include/stereo/point_cloud.h:
    39-43) with host arrays: float32 depth, K the 3x3 intrinsics (params.K0),
    an optional BGR image used when its size matches.  Returns POINT_DTYPE
    records in raster order (the reference's std::vector<Point3D>)."""
    z = np.ascontiguousarray(depth, dtype=np.float32)
    if z.ndim != 2:
        raise StereoException("depth must be a one-channel image")
    k = np.asarray(K, np.float64).reshape(3, 3)
    h, w = z.shape
    bgr = None
    if color is not None and color.shape[:2] == z.shape and color.ndim == 3 and color.shape[2] == 3:
        bgr = np.ascontiguousarray(color, dtype=np.uint8)
    out = np.empty(h * w, POINT_DTYPE)
    n = C.c_int(0)
    _check(_lib.lib().lumen_depth_to_points(z.ctypes.data, w, h, 0, None if bgr is None else bgr.ctypes.data, 0,
                                            k[0, 0], k[1, 1], k[0, 2], k[1, 2], out.ctypes.data,
                                            C.byref(n)))
    return out[:n.value].copy()


def rectify_maps_device(K, dist, R, P, width: int, height: int, map_x_ptr: int, map_y_ptr: int,
                        stream: int = 0) -> None:
    """cv::initUndistortRectifyMap (CV_32FC1) for one camera, on the device."""
    k = np.ascontiguousarray(K, dtype=np.float64).reshape(9)
    r = np.ascontiguousarray(R, dtype=np.float64).reshape(9)
    p = np.ascontiguousarray(P, dtype=np.float64).reshape(12)
    d = None if dist is None else np.ascontiguousarray(np.asarray(dist, np.float64).ravel()[:5])
    if d is not None and d.size < 5:
        d = np.concatenate([d, np.zeros(5 - d.size)])
    _check(_lib.lib().lumen_rectify_maps_device(k.ctypes.data, None if d is None else d.ctypes.data,
                                                r.ctypes.data, p.ctypes.data, width, height,
                                                map_x_ptr, map_y_ptr, stream))
