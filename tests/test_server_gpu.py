"""Served form (lumen_server_*): every request's disparity map is the same
whether it runs alone or batched with others that arrive while it is queued
or on the GPU, and equals the plain path on the same pair (StereoRectifier +
StereoSGBM.compute for calibrated requests); admission never holds more
arena bytes than the budget; invalid and oversized requests are rejected at
submit while the server keeps serving; device-side wait limits and the host
watchdog turn into per-request TIMEOUT statuses without faulting anything.
Disparity maps are integers (1/16 px): the tolerance is zero."""
import numpy as np
import pytest

from lumenstereo_b200 import (MatchingCostMode, OutOfBudgetException, StereoException, StereoParams,
                              StereoRectifier, StereoServer, StereoSGBM, TimeoutException, synth)

pytestmark = pytest.mark.gpu

# (w, h, calibration id or -1, params)
MIX = [
    (160, 96, -1, dict(maxDisparity=48, numDirections=8, matchingCostMode=MatchingCostMode.Census)),
    (131, 53, 0, dict(maxDisparity=64, numDirections=4)),
    (200, 120, 1, dict(maxDisparity=128, numDirections=8)),
    (96, 40, -1, dict(minDisparity=5, maxDisparity=37, numDirections=8, uniquenessRatio=0)),
    (150, 70, 2, dict(maxDisparity=150, numDirections=8, matchingCostMode=MatchingCostMode.Census)),
    (64, 48, -1, dict(maxDisparity=16, numDirections=8, blockSize=19)),  # uint16 wrap
    (310, 20, -1, dict(maxDisparity=290, numDirections=8, matchingCostMode=MatchingCostMode.Census)),
    (640, 480, 3, dict(maxDisparity=64, numDirections=8)),
]


def _requests():
    reqs = []
    for i, (w, h, cid, kw) in enumerate(MIX):
        left, right, _ = synth.make_pair(synth.PairSpec(w, h, 4, 1, min(40, kw["maxDisparity"] - 1), 2.0, 700 + i))
        reqs.append((StereoParams(speckleWindowSize=0, **kw), left, right, cid))
    return reqs


def _register(srv):
    for w, h, cid, _ in MIX:
        if cid >= 0:
            srv.set_calibration(cid, w, h, *synth.calibration_maps(cid, w, h))


def _plain(reqs):
    refs = []
    for (p, left, right, cid), (w, h, _, _) in zip(reqs, MIX):
        if cid >= 0:
            left, right = StereoRectifier(w, h, *synth.calibration_maps(cid, w, h)).rectify(left, right)
        with StereoSGBM(p) as s:
            refs.append(s.compute(left, right))
    return refs


def test_served_results_match_alone_and_plain():
    reqs = _requests()
    refs = _plain(reqs)
    with StereoServer(budget_bytes=1 << 30, max_batch_pairs=4) as srv:
        _register(srv)
        alone = []
        for p, left, right, cid in reqs:  # one at a time: a batch of one each
            out, info = srv.wait(srv.submit(p, left, right, calib_id=cid))
            assert info["batch_pairs"] == 1
            alone.append(out)
        # all at once, twice over: batches of up to 4 mixed requests, the
        # second wave admitted while the first is on the GPU
        ids = [srv.submit(p, l, r, calib_id=c) for p, l, r, c in reqs + reqs]
        mixed = [srv.wait(i) for i in ids]
        st = srv.stats()
    for i, ref in enumerate(refs):
        assert np.array_equal(alone[i], ref), ("alone", i)
        assert np.array_equal(mixed[i][0], ref), ("mixed", i)
        assert np.array_equal(mixed[i + len(refs)][0], ref), ("mixed again", i)
    assert max(info["batch_pairs"] for _, info in mixed) > 1
    assert st["completed"] == 3 * len(reqs) and st["failed"] == 0
    assert st["peak_admitted_bytes"] <= st["budget_bytes"]
    assert st["admitted_bytes"] == 0 and st["queue_depth"] == 0


def test_budget_admission_and_rejections_keep_serving():
    reqs = _requests()[:4]
    refs = _plain(reqs)
    # a budget that holds about one 200x120 D128 request at a time
    with StereoServer(budget_bytes=48 << 20, max_batch_pairs=8, max_inflight=3) as srv:
        _register(srv)
        with pytest.raises(OutOfBudgetException):  # 640x480 D256 cannot fit 48 MiB
            srv.submit(StereoParams(maxDisparity=256), np.zeros((480, 640), np.uint8), np.zeros((480, 640), np.uint8))
        with pytest.raises(StereoException):  # invalid disparity range
            srv.submit(StereoParams(minDisparity=10, maxDisparity=5), reqs[0][1], reqs[0][2])
        with pytest.raises(StereoException):  # calibration id never registered
            srv.submit(reqs[0][0], reqs[0][1], reqs[0][2], calib_id=99)
        ids = [srv.submit(p, l, r, calib_id=c) for p, l, r, c in reqs * 3]
        outs = [srv.wait(i)[0] for i in ids]
        st = srv.stats()
    for k, out in enumerate(outs):
        assert np.array_equal(out, refs[k % len(refs)]), k
    assert st["rejected"] == 3 and st["completed"] == len(ids)
    assert st["peak_admitted_bytes"] <= 48 << 20
    assert st["batches"] >= 2


def test_device_wait_limit_and_watchdog_report_timeouts():
    p = StereoParams(maxDisparity=128, numDirections=8, speckleWindowSize=0)
    left, right, _ = synth.make_pair(synth.PairSpec(640, 480, 4, 1, 60, 2.0, 41))
    # every device-side wait gives up after one poll: the batch reports
    # LUMEN_ERR_TIMEOUT through its status word, the server keeps serving
    # (the plain-call fallback off, so the timeout reaches the caller)
    with StereoServer(budget_bytes=1 << 30, spin_limit=1, plain_fallback=False) as srv:
        ids = [srv.submit(p, left, right) for _ in range(3)]
        errs = 0
        for i in ids:
            try:
                srv.wait(i)
            except TimeoutException:
                errs += 1
        assert errs >= 1
        assert srv.stats()["failed"] == errs
    # a host deadline far below a batch's run time: the requests complete with
    # TIMEOUT while the GPU work finishes in the background
    big_l, big_r, _ = synth.make_pair(synth.PairSpec(1920, 1080, 8, 1, 60, 2.0, 42))
    with StereoServer(budget_bytes=4 << 30, watchdog_ms=1, max_batch_pairs=4, plain_fallback=False) as srv:
        ids = [srv.submit(p, big_l, big_r) for _ in range(4)]
        for i in ids:
            with pytest.raises(TimeoutException):
                srv.wait(i)
        assert srv.stats()["watchdog_expired"] >= 1
    # a wait that runs out keeps the id; the next wait gets the result
    with StereoSGBM(p) as s:
        ref = s.compute(left, right)
    with StereoServer(budget_bytes=1 << 30) as srv:
        rid = srv.submit(p, left, right)
        try:
            out, _ = srv.wait(rid, timeout_ms=0)
        except TimeoutException:
            out, _ = srv.wait(rid)
    assert np.array_equal(out, ref)


def test_plain_call_fallback_on_failed_and_timed_out_batches():
    """A batch whose launch fails on the host (injected) or whose device-side
    waits run out: each of its requests is computed again by the plain call
    and equals the plain result; with the fallback off the failure reaches
    the caller; either way the server keeps serving."""
    reqs = _requests()[:5]
    refs = _plain(reqs)
    with StereoServer(budget_bytes=1 << 30, max_batch_pairs=8) as srv:
        _register(srv)
        srv.debug_fail_batches(1)
        ids = [srv.submit(p, l, r, calib_id=c) for p, l, r, c in reqs]
        outs = [srv.wait(i)[0] for i in ids]
        st = srv.stats()
        assert st["fallbacks"] >= 1 and st["failed"] == 0
        # the next batches run normally again
        again = [srv.wait(srv.submit(p, l, r, calib_id=c))[0] for p, l, r, c in reqs]
        assert srv.stats()["fallbacks"] == st["fallbacks"]
    for k, ref in enumerate(refs):
        assert np.array_equal(outs[k], ref), k
        assert np.array_equal(again[k], ref), k
    # device-side waits that give up after one poll: the plain call (default
    # wait limit) serves every request of those batches
    p = StereoParams(maxDisparity=128, numDirections=8, speckleWindowSize=0)
    left, right, _ = synth.make_pair(synth.PairSpec(640, 480, 4, 1, 60, 2.0, 43))
    with StereoSGBM(p) as s:
        ref = s.compute(left, right)
    with StereoServer(budget_bytes=1 << 30, spin_limit=1) as srv:
        ids = [srv.submit(p, left, right) for _ in range(3)]
        outs = [srv.wait(i)[0] for i in ids]
        st = srv.stats()
    assert all(np.array_equal(o, ref) for o in outs)
    assert st["failed"] == 0 and st["completed"] == 3
    # fallback off: the injected failure is the requests' error
    with StereoServer(budget_bytes=1 << 30, plain_fallback=False) as srv:
        srv.debug_fail_batches(1)
        with pytest.raises(Exception):
            srv.wait(srv.submit(p, left, right))
        out, _ = srv.wait(srv.submit(p, left, right))
        assert np.array_equal(out, ref)
