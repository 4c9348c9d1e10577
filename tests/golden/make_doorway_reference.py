"""Generates tests/golden/doorway_reference_64k.npz: the converged image the guiding
measurement's time to relMSE 0.01 is taken against.

The doorway interior (sprout_b200.scenes.doorway) at 1280x720, plain MIS, 65,536 samples per
pixel: 64 frames of 1,024 spp with independent sample seeds, each resolved on the device, summed
in float64 on the host and divided by 64.  The reference renderer cannot render this many
samples on a CPU in reasonable time (60 G paths); the image is cross-checked instead against
the reference's own 320x180 render of the same room (tests/test_doorway_reference.py).  Stored
as float16 (relative rounding 2^-11, far below any relMSE the measurement resolves).

Needs a B200 (about five minutes):

    python tests/golden/make_doorway_reference.py [--out PATH] [--frames 64] [--spp 1024]
"""

from __future__ import annotations

import argparse
import json
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from sprout_b200.render_bench import doorway_frame  # noqa: E402

WIDTH, HEIGHT = 1280, 720
FIRST_SEED = 10000  # sample streams independent of the measurement's renders (seed 0)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--out", default=str(HERE / "doorway_reference_64k.npz"))
    p.add_argument("--frames", type=int, default=64)
    p.add_argument("--spp", type=int, default=1024)
    a = p.parse_args()
    acc = np.zeros((HEIGHT, WIDTH, 3), np.float64)
    device_s = 0.0
    t0 = time.perf_counter()
    for i in range(a.frames):
        img, dev, _ = doorway_frame(WIDTH, HEIGHT, a.spp, None, seed=FIRST_SEED + i)
        acc += img
        device_s += dev
        print(f"frame {i + 1}/{a.frames}: mean {img.mean():.6f}, {dev:.2f} s", flush=True)
    acc /= a.frames
    meta = {"scene": "sprout_b200.scenes.doorway (defaults), plain MIS", "width": WIDTH, "height": HEIGHT,
            "spp": a.frames * a.spp, "frames": a.frames, "spp_per_frame": a.spp,
            "seeds": [FIRST_SEED, FIRST_SEED + a.frames - 1], "accumulation": "float64 sum of resolved frames",
            "device_seconds": round(device_s, 2), "wall_seconds": round(time.perf_counter() - t0, 1),
            "mean": [float(x) for x in acc.mean(axis=(0, 1))]}
    np.savez_compressed(a.out, image=acc.astype(np.float16),
                        meta=np.frombuffer(json.dumps(meta).encode(), np.uint8))
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
