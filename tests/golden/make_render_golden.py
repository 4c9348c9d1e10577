"""Generates tests/golden/cornell_reference.npz with the compiled reference renderer.

Renders the Cornell-box scene of sprout_b200.scenes.cornell through the reference's own C API
(oracle/_ref/ref_render replaying the su_* calls; batch mode, su_create_defaults, i.e. the
Linear tonemapper to linear sRGB) at sizes the tests can compare against.

    python tests/golden/make_render_golden.py
"""

from __future__ import annotations

import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from sprout_b200 import scenes  # noqa: E402

# A homogeneous scattering sphere in place of the metal one (Volumetric material).
MEDIUM = {"color": [0.8, 0.8, 0.8], "attenuation_distance": 0.05, "anisotropy": 0.5}

# name -> (width, height, spp, sphere subdivisions, medium)
CASES = {
    "cornell64_sub3": (64, 64, 4096, 3, None),
    "cornell128_sub6": (128, 128, 2048, 6, None),
    "cornell64_medium": (64, 64, 4096, 4, MEDIUM),
}


def main():
    out = {}
    meta = {"generator": "oracle/_ref/ref_render (reference su_* C API, batch mode)", "cases": {}}
    for name, (w, h, spp, sub, medium) in CASES.items():
        img, timing = oracle.reference_render(
            lambda su: scenes.cornell(su, w, h, sphere_subdivisions=sub, tonemap=True, spp=spp,
                                      medium=medium),
            w, h, 0, progressive=False)
        out[name] = img.astype(np.float32)
        meta["cases"][name] = {"width": w, "height": h, "spp": spp, "sphere_subdivisions": sub,
                               "medium": medium,
                               "render_s": timing["render_s"], "mean": [float(x) for x in img.mean(axis=(0, 1))]}
        print(name, meta["cases"][name])
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    np.savez_compressed(HERE / "cornell_reference.npz", **out)


if __name__ == "__main__":
    main()
