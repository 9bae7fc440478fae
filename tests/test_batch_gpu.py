"""Batched form (lumen_sgbm_batch_*): every pair of a mixed batch — sizes,
disparity ranges, cost modes, path sets and parameters that wrap uint16 —
gives exactly the disparity map of the plain device call for the same pair,
whether the batch runs as one launch group, is split by a small device-memory
budget into several, or is replayed from a captured CUDA graph.  Disparity maps
are integers (1/16 px): the tolerance is zero."""
import numpy as np
import pytest

from lumenstereo_b200 import MatchingCostMode, StereoBatch, StereoParams, StereoSGBM, synth

pytestmark = pytest.mark.gpu

MIX = [  # (w, h, params)
    (160, 96, dict(maxDisparity=48, numDirections=8, matchingCostMode=MatchingCostMode.Census)),
    (131, 53, dict(maxDisparity=64, numDirections=4)),
    (200, 120, dict(maxDisparity=128, numDirections=8)),
    (96, 40, dict(minDisparity=5, maxDisparity=37, numDirections=8, uniquenessRatio=0)),
    (150, 70, dict(maxDisparity=150, numDirections=8, matchingCostMode=MatchingCostMode.Census)),
    (120, 64, dict(maxDisparity=64, numDirections=8)),
    (64, 48, dict(maxDisparity=16, numDirections=8, blockSize=19)),  # uint16 wrap
    (310, 20, dict(maxDisparity=290, numDirections=8, matchingCostMode=MatchingCostMode.Census)),
]


def _pairs(torch):
    out = []
    for i, (w, h, kw) in enumerate(MIX):
        left, right, _ = synth.make_pair(synth.PairSpec(w, h, 4, 1, min(40, kw["maxDisparity"] - 1), 2.0, 300 + i))
        p = StereoParams(speckleWindowSize=0, **kw)
        out.append((p, torch.from_numpy(left).cuda(), torch.from_numpy(right).cuda(), w, h))
    return out


def _plain(torch, pairs):
    refs = []
    for p, dl, dr, w, h in pairs:
        o = torch.empty((h, w), dtype=torch.int16, device="cuda")
        with StereoSGBM(p) as s:
            s.compute_device(dl.data_ptr(), dr.data_ptr(), w, h, o.data_ptr())
            torch.cuda.synchronize()
        refs.append(o.cpu().numpy())
    return refs


@pytest.mark.parametrize("schedule,rows,graph,budget", [
    (0, 0, False, 0), (6, 24, True, 0), (6, 32, False, 0), (6, 16, True, 48 << 20),
    (4, 4, False, 0), (4, 16, True, 0), (4, 8, True, 24 << 20)])
def test_batch_matches_plain_calls(schedule, rows, graph, budget):
    torch = pytest.importorskip("torch")
    pairs = _pairs(torch)
    refs = _plain(torch, pairs)
    outs = [torch.full((h, w), 0x7ABC, dtype=torch.int16, device="cuda") for _, _, _, w, h in pairs]
    with StereoBatch(rows_per_band=rows, use_graph=graph, budget_bytes=budget, schedule=schedule) as b:
        for (p, dl, dr, w, h), o in zip(pairs, outs):
            b.add(p, dl.data_ptr(), dr.data_ptr(), w, h, o.data_ptr())
        for rep in range(2):  # the second run replays (graph) or reuses the plan
            for o in outs:
                o.fill_(0x7ABC)
            b.run()
            b.sync()
            for i, (o, ref) in enumerate(zip(outs, refs)):
                assert np.array_equal(o.cpu().numpy(), ref), (i, rep)
        info = b.info()
        if budget:
            assert info["groups"] > 4, info  # the small budget splits the larger classes
        assert b.config() == (schedule or 6, rows or (8 if schedule == 4 else 16))
        assert info["launches"] > 0


@pytest.mark.parametrize("schedule,rows,paths", [(4, 4, 4), (4, 8, 4), (6, 16, 8), (6, 24, 8), (6, 16, 4)])
def test_batch_many_wide_pairs(schedule, rows, paths):
    """24 pairs of one class, 2048 px wide and 160 rows tall: the tickets
    exceed the resident CTAs many times over.  Schedule 4: a band can only
    finish while the bands several ring lengths below it run, so the batch is
    cut into chunks whose hand-off window fits them.  Schedule 6: CTAs take
    band after band, of different pairs and sweeps, each waiting only on the
    band above it in its own sweep.  Exact against the plain call."""
    torch = pytest.importorskip("torch")
    pairs = []
    for i in range(24):
        left, right, _ = synth.make_pair(synth.PairSpec(2048, 160, 4, 1, 40, 2.0, 500 + i))
        p = StereoParams(maxDisparity=64, numDirections=paths, speckleWindowSize=0, P2=400 + 100 * (i % 5))
        pairs.append((p, torch.from_numpy(left).cuda(), torch.from_numpy(right).cuda(), 2048, 160))
    refs = _plain(torch, pairs)
    outs = [torch.full((h, w), 0x7ABC, dtype=torch.int16, device="cuda") for _, _, _, w, h in pairs]
    with StereoBatch(rows_per_band=rows, use_graph=True, schedule=schedule) as b:
        for (p, dl, dr, w, h), o in zip(pairs, outs):
            b.add(p, dl.data_ptr(), dr.data_ptr(), w, h, o.data_ptr())
        b.run()
        b.sync()
        for i, (o, ref) in enumerate(zip(outs, refs)):
            assert np.array_equal(o.cpu().numpy(), ref), i
        assert b.info()["groups"] == 1



def test_batch_autotune_keeps_outputs():
    """The batch autotuner picks a band height and the outputs stay exact."""
    torch = pytest.importorskip("torch")
    pairs = _pairs(torch)
    refs = _plain(torch, pairs)
    outs = [torch.zeros((h, w), dtype=torch.int16, device="cuda") for _, _, _, w, h in pairs]
    with StereoBatch(use_graph=True) as b:
        for (p, dl, dr, w, h), o in zip(pairs, outs):
            b.add(p, dl.data_ptr(), dr.data_ptr(), w, h, o.data_ptr())
        rows, ms = b.autotune()
        sched, r2 = b.config()
        assert r2 == rows and ms > 0
        assert (sched, rows) in [(4, 4), (4, 8), (4, 16), (6, 16), (6, 24), (6, 32)]
        for o in outs:
            o.fill_(0)
        b.run()
        b.sync()
    for o, ref in zip(outs, refs):
        assert np.array_equal(o.cpu().numpy(), ref)


@pytest.mark.parametrize("schedule,rows", [(4, 8), (4, 16), (6, 16), (6, 24)])
def test_batch_lane_team_classes(schedule, rows):
    """Groups of four or more pairs run with narrow lane teams per row (8
    lanes for 64/128 padded disparities, 16 for 192-320): every class of them
    (both path sets, uint16 wrap, partial padding, odd sizes) against the
    plain call, which keeps full-warp rows."""
    torch = pytest.importorskip("torch")
    classes = [
        dict(maxDisparity=128, numDirections=8, matchingCostMode=MatchingCostMode.Census),
        dict(maxDisparity=170, numDirections=4),                      # Dp 192, partial
        dict(maxDisparity=256, numDirections=8),                      # Dp 256
        dict(minDisparity=3, maxDisparity=40, numDirections=8, blockSize=19),  # wrap, Dp 64
        dict(maxDisparity=290, numDirections=8, matchingCostMode=MatchingCostMode.Census),  # Dp 320
    ]
    pairs = []
    for c, kw in enumerate(classes):
        for i in range(4):
            w, h = 150 + 17 * i, 60 + 9 * i
            left, right, _ = synth.make_pair(synth.PairSpec(w, h, 4, 1, 30, 2.0, 900 + 10 * c + i))
            p = StereoParams(speckleWindowSize=0, P2=700 + 50 * i, **kw)
            pairs.append((p, torch.from_numpy(left).cuda(), torch.from_numpy(right).cuda(), w, h))
    refs = _plain(torch, pairs)
    outs = [torch.full((h, w), 0x7ABC, dtype=torch.int16, device="cuda") for _, _, _, w, h in pairs]
    with StereoBatch(rows_per_band=rows, use_graph=True, schedule=schedule) as b:
        for (p, dl, dr, w, h), o in zip(pairs, outs):
            b.add(p, dl.data_ptr(), dr.data_ptr(), w, h, o.data_ptr())
        b.run()
        b.sync()
    for i, (o, ref) in enumerate(zip(outs, refs)):
        assert np.array_equal(o.cpu().numpy(), ref), i
