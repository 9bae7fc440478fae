"""Generate tests/golden/maps/rectify_maps.npz: rectification maps made by OpenCV
itself (cv2.stereoRectify + cv2.initUndistortRectifyMap, CV_32FC1), the calls
LumenStereo makes in computeRectification (src/calibration.cpp:230-266), for
two seeded synthetic stereo calibrations at 96x72.  Stores K, D, R, P of
both cameras and the four maps.  Run from the repository root (needs cv2):

    python tests/golden/maps/make_rectify_maps.py
"""
from __future__ import annotations

import os

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rectify_maps.npz")


def calibration(seed: int, w: int, h: int):
    rng = np.random.Generator(np.random.PCG64(500 + seed))
    f = rng.uniform(1000.0, 2000.0) * w / 1920.0
    K = np.array([[f, 0, (w - 1) / 2 + rng.uniform(-3, 3)], [0, f * rng.uniform(0.99, 1.01),
                  (h - 1) / 2 + rng.uniform(-3, 3)], [0, 0, 1]], np.float64)
    D0 = np.array([rng.uniform(-0.1, 0.1), rng.uniform(-0.02, 0.02), rng.uniform(-1e-3, 1e-3),
                   rng.uniform(-1e-3, 1e-3), 0.0])
    D1 = np.array([rng.uniform(-0.1, 0.1), rng.uniform(-0.02, 0.02), rng.uniform(-1e-3, 1e-3),
                   rng.uniform(-1e-3, 1e-3), 0.0])
    rvec = np.deg2rad(rng.uniform(-2.0, 2.0, 3))
    B = rng.uniform(0.05, 0.3)
    return K, D0, K.copy(), D1, rvec, np.array([-B, 0.0, 0.0])


def main():
    import cv2
    w, h = 96, 72
    out = {}
    for cid in range(2):
        K0, D0, K1, D1, rvec, T = calibration(cid, w, h)
        Rm, _ = cv2.Rodrigues(rvec)
        R0, R1, P0, P1, Q, _, _ = cv2.stereoRectify(K0, D0, K1, D1, (w, h), Rm, T,
                                                     flags=cv2.CALIB_ZERO_DISPARITY, alpha=0)
        m0x, m0y = cv2.initUndistortRectifyMap(K0, D0, R0, P0, (w, h), cv2.CV_32FC1)
        m1x, m1y = cv2.initUndistortRectifyMap(K1, D1, R1, P1, (w, h), cv2.CV_32FC1)
        for k, v in dict(K0=K0, D0=D0, R0=R0, P0=P0, K1=K1, D1=D1, R1=R1, P1=P1,
                         map0x=m0x, map0y=m0y, map1x=m1x, map1y=m1y).items():
            out[f"c{cid}_{k}"] = v
    np.savez_compressed(OUT, width=w, height=h, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
