#!/usr/bin/env python
"""Benchmark of the B200 SGBM engine (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl reference]

A step is one full StereoSGBM computation (cost volume, SGM aggregation, WTA,
LR check, median) of one seeded synthetic pair, default the 1920x1080,
maxDisparity=128, SAD + Sobel-x prefilter, 8-path configuration.  ``value`` is
pixel-disparities per second (W*H*D per step) of the whole job with the inputs
resident in HBM; ``e2e`` is the same metric through the host-buffer C-ABI
call (pinned host memory, host<->device copies inside the timed region).

Multi-GPU (torchrun): replicas -- every rank computes its own copy of the
workload on its own GPU, no collective on the data path; value = all ranks'
pixel-disparities / max-over-ranks device time.

``--impl reference`` times the reference's algorithm on the host cores (the C
restatement in oracle/, all threads, a bounded sample of the same workload)
and, when a GPU and oracle/_ref are present, the reference's own CUDA kernels
on the GPU as extra information.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from lumenstereo_b200 import MatchingCostMode, StereoParams, StereoSGBM, synth  # noqa: E402

DEFAULT_WORKLOAD = "1920x1080_d128_sad_8path"
METRIC = "pixel-disparities/s vs HBM roofline"
UNIT = "pd/s"
FLUSH_BYTES = 256 << 20  # > 126 MB L2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(synth.WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--schedule", type=int, default=0, help="aggregation schedule (0 = auto)")
    ap.add_argument("--rows", type=int, default=0,
                    help="rows per band of the fused sweeps with --schedule 3/4 (0 = default)")
    ap.add_argument("--lanes", type=int, default=32,
                    help="lanes per row with --schedule 4 --rows (8/16: lane teams)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="plain", choices=["plain", "batch", "serve", "epilogue", "ops"],
                    help="plain: one pair per call (default); batch: the 64-pair mixed stream; "
                         "serve: Poisson request stream through the served form")
    ap.add_argument("--pairs", type=int, default=0,
                    help="distinct pairs of the mixed stream (batch: 64, serve: 32)")
    ap.add_argument("--requests", type=int, default=200,
                    help="requests per offered rate (--mode serve; 0: 25 s of arrivals, at most 10000)")
    ap.add_argument("--inflight", type=int, default=2, help="batches on the device at once (--mode serve)")
    # the server counts every working byte of a request against its arena (about 10 bytes a
    # pixel-disparity with schedule 6); 120 GiB keeps the cost volumes in flight near 12 GB,
    # inside a 40 GB cost-volume budget
    ap.add_argument("--budget-gib", type=int, default=120, help="device arena of the server, GiB (--mode serve)")
    ap.add_argument("--rates", default="20,50,100,200,300,400", help="offered rates, requests/s (--mode serve)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def replica_rate(local_time: float, units_per_rank: float, world: int, device="cpu"):
    """Whole-job time and rate of `world` independent replicas: every rank
    processed `units_per_rank`; the job's time is the slowest rank's (a MAX
    all-reduce over the process group when world > 1)."""
    t = float(local_time)
    if world > 1:
        import torch
        import torch.distributed as dist
        tt = torch.tensor([t], device=device, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    return t, units_per_rank * world / t


def workload_params(wl) -> StereoParams:
    # StereoParams{} defaults except the configuration's fields and the speckle
    # filter (off: not one of the measured stages, and racy in the reference).
    return StereoParams(maxDisparity=wl.max_disparity, numDirections=wl.num_directions,
                        matchingCostMode=MatchingCostMode.Census if wl.census else MatchingCostMode.SAD,
                        speckleWindowSize=0)


def workload_config(name: str, world: int) -> dict:
    """The `config` object of the JSON line; both arms print the same one."""
    wl = synth.WORKLOADS[name]
    return {"workload": name, "width": wl.pair.width, "height": wl.pair.height,
            "max_disparity": wl.max_disparity,
            "cost": "census" if wl.census else "sad+sobel-x prefilter",
            "paths": wl.num_directions, "params": "StereoParams defaults, speckleWindowSize=0",
            "l2": "256 MiB buffer written before every timed step, outside its events",
            "parallelism": f"replicas x{world}"}


def params_dict(p: StereoParams):
    return {k: int(v) for k, v in p.__dict__.items()}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(workload: str, schedule: int):
    """DRAM bytes per pixel-disparity of the aggregation stage of `schedule` on
    `workload` from the ncu summary committed under profiles/ (None when that
    kernel has no capture)."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(f"{workload}/schedule{schedule}")
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (C restatement of the reference path), all threads
# ---------------------------------------------------------------------------
def cpu_port_rate(p: dict, left, right, budget_s: float = 15.0):
    """pixel-disparities/s of the oracle on a bounded sample of the workload:
    the full pair when it fits the budget, else a band of full-width rows."""
    from oracle import oracle
    H, W = left.shape
    D = p["maxDisparity"] - p["minDisparity"]
    probe_rows = max(8, H // 16)
    t = time.perf_counter()
    oracle.sgbm(p, left[:probe_rows], right[:probe_rows])
    t_probe = time.perf_counter() - t
    est_full = t_probe * H / probe_rows
    if est_full <= budget_s:
        rows = H
        reps = max(1, int(round(budget_s / max(est_full, 1e-3) * 0.6)))
    else:
        rows = max(probe_rows, int(H * budget_s / est_full))
        reps = 1
    t = time.perf_counter()
    for _ in range(reps):
        oracle.sgbm(p, left[:rows], right[:rows])
    dt = time.perf_counter() - t
    sample = f"{reps} x {W}x{rows} rows of the {W}x{H} pair (D={D})"
    return W * rows * D * reps / dt, oracle.max_threads(), sample


def opencv_rate(p: dict, left, right, paths: int):
    """OpenCV StereoSGBM (cv2, host cores) on the same pair: a baseline only
    (a different SGBM formulation), MODE_HH for 8 paths, MODE_HH4 for 4."""
    try:
        import cv2
    except Exception:
        return None
    D = p["maxDisparity"] - p["minDisparity"]
    nd = ((D + 15) // 16) * 16
    m = cv2.StereoSGBM_create(minDisparity=0, numDisparities=nd, blockSize=5, P1=200, P2=800,
                              disp12MaxDiff=1, preFilterCap=31, uniquenessRatio=10,
                              speckleWindowSize=0, speckleRange=0,
                              mode=cv2.StereoSGBM_MODE_HH if paths == 8 else cv2.StereoSGBM_MODE_HH4)
    cv2.setNumThreads(os.cpu_count() or 1)
    m.compute(left, right)
    ts = []
    for _ in range(3):
        t = time.perf_counter()
        m.compute(left, right)
        ts.append(time.perf_counter() - t)
    H, W = left.shape
    return {"value": W * H * D / statistics.median(ts), "unit": UNIT,
            "threads": cv2.getNumThreads(), "numDisparities": nd,
            "mode": "MODE_HH" if paths == 8 else "MODE_HH4"}


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    wl = synth.WORKLOADS[args.workload]
    left, right, gt = synth.make_pair(wl.pair)
    H, W = left.shape
    D = wl.max_disparity
    params = workload_params(wl)
    pd_per_step = W * H * D
    sgbm = StereoSGBM(params)
    if args.schedule:
        sgbm.set_schedule(args.schedule)
        if args.rows:
            sgbm.set_tuning(args.lanes, args.rows)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream
    dl = torch.from_numpy(left).to(dev)
    dr = torch.from_numpy(right).to(dev)
    dout = torch.empty((H, W), dtype=torch.int16, device=dev)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def step():
        sgbm.compute_device(dl.data_ptr(), dr.data_ptr(), W, H, dout.data_ptr(), stream=sptr)

    tune_report = None
    if not args.schedule:
        # autotuner: every schedule / sweep configuration on this pair, outside the timed region
        tune_report = sgbm.autotune(dl.data_ptr(), dr.data_ptr(), W, H, repeats=2)
    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    tuning = sgbm.get_tuning()
    check = dout.cpu().numpy()
    v = check > 0
    quality = {"valid_frac": float(v.mean()),
               "bad2_frac": float(np.mean(np.abs(check[v] / 16.0 - gt[v]) > 2)) if v.any() else None}

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    launches0 = sgbm.launch_count()
    step_ms, agg_ms, cost_ms, sel_ms = [], [], [], []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()  # L2 flush, outside the step's events
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
            t = sgbm.timings()  # waits for this step; stage times from the handle's events
            cost_ms.append(t[1]); agg_ms.append(t[2]); sel_ms.append(t[3])
        torch.cuda.synchronize()
        barrier()
    launches = sgbm.launch_count() - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_s, value = replica_rate(sum(step_ms) / 1e3, pd_per_step * args.steps, world, dev)
    total_ms = total_s * 1e3

    # e2e: host buffers through the C-ABI call (H2D + compute + D2H per step)
    lh = torch.from_numpy(left).pin_memory()
    rh = torch.from_numpy(right).pin_memory()
    oh = torch.empty((H, W), dtype=torch.int16).pin_memory()
    from lumenstereo_b200 import _lib, _check
    lib = _lib.lib()

    def e2e_step():
        _check(lib.lumen_sgbm_compute(sgbm._h, lh.data_ptr(), rh.data_ptr(), W, H, W, 1,
                                      oh.data_ptr(), W * 2))

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    e2e_time = 0.0
    for _ in range(args.steps):
        flush.zero_()  # L2 flush, outside the timed call
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()     # synchronous: H2D, pipeline, D2H
        e2e_time += time.perf_counter() - t0
    e2e_time, e2e_value = replica_rate(e2e_time, pd_per_step * args.steps, world, dev)

    hbm, peak_kind = measured_peaks()
    P = wl.num_directions
    agg_mean = statistics.mean(agg_ms)
    agg_bytes = (P + 2) * pd_per_step          # cost read once per path + agg written once
    achieved = agg_bytes / (agg_mean / 1e3) / 1e9
    traffic_per_pd = profiled_traffic(args.workload, tuning[0])
    pipe_ms = statistics.mean(step_ms)
    pipe_bytes = (P + 5) * pd_per_step         # SGM core model: cost w + P reads, agg w + r
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": workload_config(args.workload, world),
        "schedule": {"requested": args.schedule or "auto", "used": tuning[0],
                     "lanes_per_pixel": tuning[1], "warps_per_block": tuning[2],
                     "column_rows": sgbm.get_tuning_columns()},
        "roofline": {"bound": "hbm", "kernel": "sgm aggregation stage",
                     "achieved": achieved, "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / hbm,
                     "algorithmic_bytes_per_pd": P + 2,
                     "traffic": None if traffic_per_pd is None else traffic_per_pd * pd_per_step,
                     "mean_ms": agg_mean},
        "pipeline_roofline": {"algorithmic_bytes_per_pd": P + 5, "mean_ms": pipe_ms,
                              "achieved": pipe_bytes / (pipe_ms / 1e3) / 1e9, "peak": hbm,
                              "frac": pipe_bytes / (pipe_ms / 1e3) / 1e9 / hbm},
        "stage_ms": {"cost": statistics.mean(cost_ms), "aggregate": agg_mean,
                     "select_post": statistics.mean(sel_ms)},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * W * H,
                "d2h_bytes_per_step": 2 * W * H, "ms_per_step": e2e_time / args.steps * 1e3},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "quality": quality,
        "autotune": tune_report.strip().splitlines() if tune_report else None,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        pdct = params_dict(params)
        try:
            rate, cores, sample = cpu_port_rate(pdct, left, right)
            result["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                                      "sample": sample}
        except Exception as e:  # report, never hide
            result["cpu_baseline"] = {"value": None, "error": repr(e)}
        ocv = opencv_rate(pdct, left, right, P)
        if ocv:
            result["opencv_cpu"] = ocv
    if rank == 0:
        print(json.dumps(result), flush=True)
    sgbm.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    wl = synth.WORKLOADS[args.workload]
    left, right, _ = synth.make_pair(wl.pair)
    H, W = left.shape
    D = wl.max_disparity
    p = params_dict(workload_params(wl))
    from oracle import oracle
    # each step: a bounded sample (full-width band of rows) of ~4 s on the host cores
    probe = max(8, H // 16)
    t = time.perf_counter()
    oracle.sgbm(p, left[:probe], right[:probe])
    est = (time.perf_counter() - t) * H / probe
    rows = H if est <= 4.0 else max(probe, int(H * 4.0 / est))
    for _ in range(args.warmup):
        oracle.sgbm(p, left[:rows], right[:rows])
    t = time.perf_counter()
    for _ in range(args.steps):
        oracle.sgbm(p, left[:rows], right[:rows])
    dt = time.perf_counter() - t
    value = W * rows * D * args.steps / dt
    sample = f"{W}x{rows} rows of the {W}x{H} pair (D={D}) per step"
    res = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u16", "data": "synthetic",
           "config": workload_config(args.workload, world),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": oracle.max_threads(),
                            "kind": "port", "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    # The reference's own CUDA kernels on this GPU (information only).
    try:
        import torch
        if torch.cuda.is_available() and oracle.ref_available():
            _, _, ms = oracle.ref_sgbm(p, left, right, repeats=3)
            res["reference_cuda_gpu"] = {"value": W * H * D / (ms / 1e3), "unit": UNIT,
                                         "ms_per_pair": ms,
                                         "what": "LumenStereo src/sgbm_kernels.cu (sm_100, -O3 "
                                                 "--use_fast_math) with its host sequence; "
                                                 "getLastComputeTimeMs interval"}
    except Exception as e:
        res["reference_cuda_gpu"] = {"error": repr(e)}
    print(json.dumps(res), flush=True)


# ---------------------------------------------------------------------------
# Batched form: the mixed stream of pairs (seeds 100.., sizes 640x480 D64 ..
# 2880x1988 D192, Census/SAD, 4/8 paths) through one StereoBatch against a
# loop of plain device calls on the same GPU; outputs must match bit for bit.
# ---------------------------------------------------------------------------
def run_batch(args):
    import torch
    from lumenstereo_b200 import StereoBatch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    items = [synth.mix_item(100 + i) for i in range(args.pairs or 64)]
    pairs = []
    for spec, dmax, census, ndir in items:
        left, right, _ = synth.make_pair(spec)
        p = StereoParams(maxDisparity=dmax, numDirections=ndir,
                         matchingCostMode=MatchingCostMode.Census if census else MatchingCostMode.SAD,
                         speckleWindowSize=0)
        pairs.append((p, torch.from_numpy(left).to(dev), torch.from_numpy(right).to(dev),
                      spec.width, spec.height))
    pd_total = sum(w * h * p.maxDisparity for p, _, _, w, h in pairs)
    ref = [torch.empty((h, w), dtype=torch.int16, device=dev) for _, _, _, w, h in pairs]
    out = [torch.empty((h, w), dtype=torch.int16, device=dev) for _, _, _, w, h in pairs]
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream
    # plain loop: one handle, parameters switched per pair (buffers grow to the largest)
    plain = StereoSGBM(pairs[0][0])

    def plain_loop():
        for (p, dl, dr, w, h), o in zip(pairs, ref):
            plain.setParams(p)
            plain.compute_device(dl.data_ptr(), dr.data_ptr(), w, h, o.data_ptr(), stream=sptr)

    def timed(fn, reps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for a, b in ev:
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in ev]

    plain_loop()
    torch.cuda.synchronize()
    plain_ms = timed(plain_loop, max(1, args.steps // 2))
    # the library's batch autotuner (rows per band), then graph replay
    batch = StereoBatch(use_graph=True)
    for (p, dl, dr, w, h), o in zip(pairs, out):
        batch.add(p, dl.data_ptr(), dr.data_ptr(), w, h, o.data_ptr())
    best_rows, best_ms = batch.autotune(sptr, repeats=2)
    best_sched, _ = batch.config()
    tune = {"schedule": best_sched, "rows_per_band": best_rows, "ms": best_ms}
    for _ in range(max(args.warmup, 2)):
        batch.run(sptr)
    batch.sync(sptr)
    with ClockSampler(local) as clocks:
        batch_ms = timed(lambda: batch.run(sptr), args.steps)
    batch.sync(sptr)
    exact = all(torch.equal(a, b) for a, b in zip(ref, out))
    info = batch.info()
    # end to end: host images in, host maps out, through the same batch
    host_in = [(dl.cpu().pin_memory(), dr.cpu().pin_memory()) for _, dl, dr, _, _ in pairs]
    host_out = [torch.empty(o.shape, dtype=torch.int16).pin_memory() for o in out]
    h2d = sum(2 * w * h for _, _, _, w, h in pairs)
    d2h = sum(2 * w * h for _, _, _, w, h in pairs)

    def e2e():
        for (hl, hr), (_, dl, dr, _, _) in zip(host_in, pairs):
            dl.copy_(hl, non_blocking=True)
            dr.copy_(hr, non_blocking=True)
        batch.run(sptr)
        for ho, o in zip(host_out, out):
            ho.copy_(o, non_blocking=True)

    e2e()
    torch.cuda.synchronize()
    e2e_ms = timed(e2e, max(1, args.steps // 2))
    value = len(pairs) / (statistics.mean(batch_ms) / 1e3)
    plain_rate = len(pairs) / (statistics.mean(plain_ms) / 1e3)
    res = {"metric": "pairs/s, batched mixed stream", "value": value, "unit": "pairs/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": statistics.mean(batch_ms), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u16", "data": "synthetic",
           "config": {"workload": f"mixed_stream_{len(pairs)}_pairs", "seeds": f"100..{99 + len(pairs)}",
                      "sizes": "640x480 D64, 1280x720 D128, 1920x1080 D128, 2880x1988 D192",
                      "cost": "Census/SAD 50/50", "paths": "4/8", "pixel_disparities": pd_total,
                      "schedule": best_sched, "rows_per_band": best_rows, "graph": True,
                      "groups": info["groups"],
                      "device_bytes": info["device_bytes"]},
           "plain_loop": {"value": plain_rate, "unit": "pairs/s", "ms": statistics.mean(plain_ms)},
           "speedup_vs_plain_loop": value / plain_rate,
           "bit_exact_vs_plain": exact,
           "autotune_ms": tune,
           "pd_per_s": pd_total / (statistics.mean(batch_ms) / 1e3),
           "e2e": {"value": len(pairs) / (statistics.mean(e2e_ms) / 1e3), "unit": "pairs/s",
                   "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
           "gpu_launches": int(info["launches"]),
           "clocks": clocks.summary()}
    if rank == 0:
        print(json.dumps(res), flush=True)
    batch.close()
    plain.close()


# ---------------------------------------------------------------------------
# Served form: Poisson arrivals of requests drawn from a pool of mixed pairs
# (seeds 10000.., each with its calibration id seed % 16 and resident
# rectification maps) through one StereoServer, swept over offered rates;
# latency percentiles per rate, throughput against the plain serial loop
# (rectify + compute per pair through the host-buffer API), and every pool
# pair's served map checked bit-exact against its plain result.
# ---------------------------------------------------------------------------
def run_serve(args):
    import threading
    import torch
    from lumenstereo_b200 import StereoRectifier, StereoServer
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    n_pool = args.pairs or 32
    pool, maps = [], {}
    for i in range(n_pool):
        seed = 10000 + i
        spec, dmax, census, ndir = synth.mix_item(seed)
        left, right, _ = synth.make_pair(spec)
        p = StereoParams(maxDisparity=dmax, numDirections=ndir,
                         matchingCostMode=MatchingCostMode.Census if census else MatchingCostMode.SAD,
                         speckleWindowSize=0)
        key = (seed % 16) * 64 + synth.MIX_SIZES.index((spec.width, spec.height, dmax))
        if key not in maps:
            maps[key] = (spec.width, spec.height, synth.calibration_maps(seed % 16, spec.width, spec.height))
        pool.append((p, left, right, key))
    # plain serial loop: the reference's per-pair calls (rectify, then compute)
    rects = {k: StereoRectifier(w, h, *m) for k, (w, h, m) in maps.items()}
    sgbm = StereoSGBM(pool[0][0])
    refs = []

    def plain_one(item):
        p, left, right, key = item
        rl, rr = rects[key].rectify(left, right)
        sgbm.setParams(p)
        return sgbm.compute(rl, rr)

    for item in pool:
        refs.append(plain_one(item))
    t0 = time.perf_counter()
    for item in pool:
        plain_one(item)
    plain_rate = len(pool) / (time.perf_counter() - t0)
    srv_sched = args.schedule if args.schedule in (4, 6) else 6
    srv = StereoServer(budget_bytes=args.budget_gib << 30, max_batch_pairs=32, rows_per_band=16,
                       max_inflight=args.inflight,
                       schedule=srv_sched)
    for key, (w, h, m) in maps.items():
        srv.set_calibration(key, w, h, *m)
    # warm-up pass, and the bit-exact check of every pool pair
    ids = [srv.submit(p, l, r, calib_id=k) for p, l, r, k in pool]
    exact = all(np.array_equal(srv.wait(i)[0], ref) for i, ref in zip(ids, refs))
    rng = np.random.Generator(np.random.PCG64(10000))
    rates = [float(x) for x in args.rates.split(",") if x]
    sweep = []
    with ClockSampler(local) as clocks:
        for rate in rates:
            # --requests 0: 25 s of arrivals at this rate, at most 10,000 requests
            n = args.requests or int(min(10000, max(200, 25 * rate)))
            gaps = rng.exponential(1.0 / rate, n)
            picks = rng.integers(0, len(pool), n)
            sub = [None] * n
            t_start = time.perf_counter()

            def producer():
                t = t_start
                for k in range(n):
                    t += gaps[k]
                    d = t - time.perf_counter()
                    if d > 0:
                        time.sleep(d)
                    p, l, r, key = pool[picks[k]]
                    sub[k] = (time.perf_counter(), srv.submit(p, l, r, calib_id=key))

            th = threading.Thread(target=producer)
            th.start()
            lat, done_at, bsz = [], [], []
            for k in range(n):
                while sub[k] is None:
                    time.sleep(0.0002)
                ts, rid = sub[k]
                _, info = srv.wait(rid)
                lat.append(info["latency_ms"])
                done_at.append(ts + info["latency_ms"] / 1e3)
                bsz.append(info["batch_pairs"])
            th.join()
            span = max(done_at) - t_start
            st = srv.stats()
            sweep.append({"offered_per_s": rate, "requests": n, "seconds": span,
                          "achieved_pairs_per_s": n / span,
                          "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                          "p999_ms": float(np.percentile(lat, 99.9)), "mean_batch_pairs": float(np.mean(bsz)),
                          "peak_queue_depth": st["peak_queue_depth"]})
    st = srv.stats()
    best = max(sweep, key=lambda r: r["achieved_pairs_per_s"])
    res = {"metric": "served pairs/s with p50/p99 latency", "value": best["achieved_pairs_per_s"],
           "unit": "pairs/s", "n_gpus": world, "steps": sum(r["requests"] for r in sweep), "warmup": len(pool),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16",
           "data": "synthetic",
           "config": {"workload": f"served_stream_pool_{len(pool)}_pairs", "seeds": f"10000..{9999 + len(pool)}",
                      "calibrations": "16 ids (seed % 16), rectified on the device from resident maps",
                      "arrivals": "Poisson",
                      "requests_per_rate": args.requests or "25 s of arrivals, at most 10000",
                      "budget_bytes": args.budget_gib << 30, "max_batch_pairs": 32, "max_inflight": args.inflight,
                      "schedule": srv_sched, "rows_per_band": 16},
           "p50_ms": best["p50_ms"], "p99_ms": best["p99_ms"], "p999_ms": best["p999_ms"],
           "rates": sweep,
           "plain_serial": {"value": plain_rate, "unit": "pairs/s",
                            "path": "StereoRectifier.rectify + StereoSGBM.compute per pair (host buffers)"},
           "speedup_vs_plain_serial": best["achieved_pairs_per_s"] / plain_rate,
           "bit_exact_vs_plain": bool(exact),
           "e2e": {"value": best["achieved_pairs_per_s"], "unit": "pairs/s",
                   "note": "host images in, host maps out: every served request is end to end"},
           "server": {k: int(v) for k, v in st.items()},
           "clocks": clocks.summary()}
    if rank == 0:
        print(json.dumps(res), flush=True)
    srv.close()
    sgbm.close()


# ---------------------------------------------------------------------------
# Either side of the disparity map: disparity -> depth at 1920x1080 and the
# device-generated rectification maps at 2880x1988, against the HBM roofline
# (depth: 2 B read + 4 B written per pixel; maps: 8 B written per pixel).
# ---------------------------------------------------------------------------
def run_epilogue(args):
    """The kernels either side of the disparity map, each timed as a CUDA
    graph of 20 launches (one launch is a few microseconds: a loop of host
    calls would time the host)."""
    import torch
    from lumenstereo_b200 import (depth_colorize_device, depth_to_points_device, disparity_to_depth_color_device,
                                  disparity_to_depth_device, rectify_maps_device)
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    peak, kind = measured_peaks()
    res = {"metric": "GB/s of the depth, colour, point-cloud and map-generation kernels", "unit": "GB/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
           "data": "synthetic", "dtype": "f32", "vs_baseline": None, "peak_gbs": peak, "peak_kind": kind}
    reps = 20

    def timed(fn):
        side = torch.cuda.Stream()
        with torch.cuda.stream(side):
            for _ in range(max(3, args.warmup)):
                fn(side.cuda_stream)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            for _ in range(reps):
                fn(side.cuda_stream)
        g.replay()
        torch.cuda.synchronize()
        cur = torch.cuda.current_stream()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(cur)
        for _ in range(args.steps):
            g.replay()
        b.record(cur)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / (args.steps * reps)

    def entry(name, W, H, ms, bytes_):
        res[name] = {"workload": f"{W}x{H}", "ms": ms, "gbs": bytes_ / ms / 1e6, "frac": bytes_ / ms / 1e6 / peak}

    lut = np.stack([np.arange(256), 255 - np.arange(256), np.arange(256) // 2], axis=1).astype(np.uint8)
    for W, H in ((1920, 1080), (2880, 1988)):
        disp = torch.randint(-16, 128 * 16, (H, W), dtype=torch.int16, device="cuda")
        depth = torch.empty((H, W), dtype=torch.float32, device="cuda")
        rgb = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda")
        tag = f"_{H}p" if H == 1080 else ""
        entry("depth" + tag, W, H, timed(lambda s: disparity_to_depth_device(
            disp.data_ptr(), W, H, 1400.0, 0.12, depth.data_ptr(), 0.0, s)), W * H * 6)
        # depth + colour: fused (2 B in, 4 + 3 B out) against the two passes
        entry("depth_color_fused" + tag, W, H, timed(lambda s: disparity_to_depth_color_device(
            disp.data_ptr(), W, H, 1400.0, 0.12, depth.data_ptr(), rgb.data_ptr(), lut, 0.5, 10.0, 0.0, s)),
            W * H * 9)

        def two(s):
            disparity_to_depth_device(disp.data_ptr(), W, H, 1400.0, 0.12, depth.data_ptr(), 0.0, s)
            depth_colorize_device(depth.data_ptr(), W, H, rgb.data_ptr(), lut, 0.5, 10.0, s)
        entry("depth_color_two_pass" + tag, W, H, timed(two), W * H * 9)
        # point cloud: depth read twice (count, write), colours read, 16 B a point written
        bgr = torch.randint(0, 256, (H, W, 3), dtype=torch.uint8, device="cuda")
        pts = torch.empty((H * W * 16,), dtype=torch.uint8, device="cuda")
        offs = torch.empty((H + 1,), dtype=torch.int32, device="cuda")
        ms = timed(lambda s: depth_to_points_device(depth.data_ptr(), W, H, 1733.7, 1731.5, W / 2, H / 2,
                                                    pts.data_ptr(), offs.data_ptr(), bgr.data_ptr(), s))
        torch.cuda.synchronize()
        n = int(offs[H].item())
        entry("points" + tag, W, H, ms, W * H * (4 + 3) + n * 16)
        res["points" + tag]["points"] = n
    W, H = 2880, 1988
    K = np.array([[1500.0, 0, 1440], [0, 1500.0, 994], [0, 0, 1]])
    R = np.eye(3)
    P = np.hstack([K, np.zeros((3, 1))])
    mx = torch.empty((H, W), dtype=torch.float32, device="cuda")
    my = torch.empty((H, W), dtype=torch.float32, device="cuda")
    entry("maps", W, H, timed(lambda s: rectify_maps_device(K, [0.05, -0.01, 1e-4, -1e-4, 0.0], R, P, W, H,
                                                           mx.data_ptr(), my.data_ptr(), s)), W * H * 8)
    res["value"] = res["depth_color_fused"]["gbs"]
    if rank == 0:
        print(json.dumps(res), flush=True)


def run_ops(args):
    """Issue rate of the packed minima the recurrence can use (the library's
    lumen_debug_op_rates): ns per warp-instruction per SM, and the ratio to
    the two-input __vminu2."""
    import ctypes as C
    import torch
    from lumenstereo_b200 import _check, _lib
    torch.cuda.set_device(0)
    out = (C.c_float * 4)()
    _check(_lib.lib().lumen_debug_op_rates(out))
    names = ["vminu2", "vimin3_u16x2", "viaddmin_u16x2", "iadd"]
    res = {"metric": "ns per warp-instruction per SM", "unit": "ns", "higher_is_better": False,
           "n_gpus": 1, "data": "synthetic", "dtype": "u16x2",
           "ops": {n: float(v) for n, v in zip(names, out)},
           "relative_to_vminu2": {n: float(v) / float(out[0]) for n, v in zip(names, out)}}
    print(json.dumps(res), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "batch":
        run_batch(args)
    elif args.mode == "serve":
        run_serve(args)
    elif args.mode == "epilogue":
        run_epilogue(args)
    elif args.mode == "ops":
        run_ops(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
