"""Generate the golden fixtures in this directory from the reference itself.

Runs LumenStereo's own CUDA kernels (oracle/_ref/libref_sgbm.so, built by
oracle/Makefile from the unmodified reference sources) on small seeded inputs
and stores inputs, parameters, every intermediate and the outputs as
compressed .npz files.  Needs a CUDA GPU; run from the repository root:

    python tests/golden/make_golden.py --out tests/golden

The CPU test tests/test_oracle.py::test_oracle_matches_reference_golden then
pins the C oracle to these files without a GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from lumenstereo_b200 import synth  # noqa: E402

BASE = dict(minDisparity=0, maxDisparity=128, blockSize=5, P1=200, P2=800, preFilterCap=31,
            uniquenessRatio=10, disp12MaxDiff=1, speckleWindowSize=0, speckleRange=32,
            useGPU=1, useSharedMemory=1, numDirections=4, matchingCostMode=0)

# (name, W, H, seed, params overrides, keep the aggregated volume, path mask)
CASES = [
    ("census_4path_d32", 64, 48, 11, dict(maxDisparity=32, matchingCostMode=1), True, 0),
    ("sad_8path_d32", 64, 48, 12, dict(maxDisparity=32, numDirections=8), True, 0),
    ("census_8path_d45_min3", 72, 40, 13,
     dict(minDisparity=3, maxDisparity=48, matchingCostMode=1, numDirections=8), True, 0),
    ("sad_4path_bs3_ur0_nolr", 60, 44, 14,
     dict(maxDisparity=24, blockSize=3, uniquenessRatio=0, disp12MaxDiff=-1), True, 0),
    ("sad_8path_bs7", 80, 36, 15, dict(maxDisparity=40, blockSize=7, numDirections=8), False, 0),
    ("census_path_brtl_only", 50, 30, 16, dict(maxDisparity=20, matchingCostMode=1,
                                               numDirections=8), True, 0x20),
    ("sad_path_trbl_only", 50, 30, 17, dict(maxDisparity=20, numDirections=8), True, 0x40),
    ("census_wrap_bs21", 40, 30, 18, dict(maxDisparity=16, matchingCostMode=1, blockSize=21,
                                          preFilterCap=63, P1=30000, P2=60000,
                                          numDirections=8), True, 0),
    ("sad_wrap_bs19", 48, 32, 19, dict(maxDisparity=16, blockSize=19, numDirections=8), True, 0),
    ("census_d290_tail", 330, 12, 20, dict(maxDisparity=290, matchingCostMode=1,
                                           numDirections=8), False, 0),
    ("sad_d1", 30, 20, 21, dict(maxDisparity=1), True, 0),
    ("census_tiny_5x3", 5, 3, 22, dict(maxDisparity=4, matchingCostMode=1, numDirections=8),
     True, 0),
    ("sad_tiny_2x2", 2, 2, 23, dict(maxDisparity=3, numDirections=8), True, 0),
    ("sad_minD20_ur15", 90, 30, 24, dict(minDisparity=20, maxDisparity=52, uniquenessRatio=15,
                                         numDirections=8), False, 0),
    ("census_speckle", 96, 64, 25, dict(maxDisparity=32, matchingCostMode=1,
                                        speckleWindowSize=100, speckleRange=2), False, 0),
    ("scene_census_4path_d64", 160, 120, 26, dict(maxDisparity=64, matchingCostMode=1), False, 0),
]


def make_inputs(W, H, seed):
    if W * H >= 64 * 32:
        spec = synth.PairSpec(W, H, 4, 2, 0.4 * W if W < 200 else 30, 2.0, seed)
        left, right, _ = synth.make_pair(spec)
        return left, right
    return synth.random_pair(W, H, seed, shift=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    for name, W, H, seed, over, keep_agg, mask in CASES:
        p = dict(BASE, **over)
        left, right = make_inputs(W, H, seed)
        disp, inter, _ = oracle.ref_sgbm(p, left, right, intermediates=True, path_mask=mask)
        arrays = dict(left=left, right=right, disp=disp, disp_wta=inter["disp_wta"],
                      disp_right=inter["disp_right"], disp_lr=inter["disp_lr"],
                      cost=inter["cost"])
        if p["matchingCostMode"] == 1:
            arrays.update(census_left=inter["census_left"], census_right=inter["census_right"])
        else:
            arrays.update(pref_left=inter["pref_left"], pref_right=inter["pref_right"])
        if keep_agg:
            arrays["agg"] = inter["agg"]
        meta = dict(name=name, params=p, path_mask=mask, seed=seed,
                    generator="LumenStereo src/sgbm_kernels.cu via oracle/_ref (sm_100, -O3 "
                              "--use_fast_math)")
        np.savez_compressed(os.path.join(args.out, name + ".npz"), meta=json.dumps(meta),
                            **arrays)
        print(name, "ok", disp.shape)


if __name__ == "__main__":
    main()
