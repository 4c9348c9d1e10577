"""Generates tests/golden/cast_reference.npz from the compiled reference.

Runs the reference's own Builder_SAH(16, 64, 4) + Tree::intersect / Tree::intersect_p
(oracle/_ref/ref_cast, built from the reference sources by oracle/Makefile) on seeded
synthetic inputs and stores its per-ray answers.  The inputs themselves are not stored:
they are regenerated deterministically by sprout_b200.sphere_mesh / random_rays and
tests/cases.edge_rays, and their SHA-256 digests are stored so a test can prove it fed the
same bytes.

    python tests/golden/make_cast_golden.py
"""

from __future__ import annotations

import hashlib
import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

import oracle  # noqa: E402
import sprout_b200 as sb  # noqa: E402
from cases import edge_rays  # noqa: E402

# name -> (mesh subdivision n, random ray count, ray seed, include edge rays)
CASES = {
    "sphere32": (32, 65536, 7, True),
    "sphere128": (128, 16384, 9, True),
    # the cast benchmark's own scene (n = 512, 1,048,576 triangles) and its first rays
    "bench512": (512, 16384, 1, False),
}


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def case_inputs(name):
    n, count, seed, with_edges = CASES[name]
    pos, idx = sb.sphere_mesh(n, 0.1, 1)
    rays = sb.random_rays(count, seed=seed)
    if with_edges:
        rays = np.concatenate([rays, edge_rays(pos, idx)])
    return pos, idx, rays


def main():
    out = {}
    meta = {"generator": "oracle/_ref/ref_cast (reference Builder_SAH(16,64,4) + Tree::intersect/_p)",
            "cases": {}}
    for name in CASES:
        pos, idx, rays = case_inputs(name)
        ref = oracle.reference_cast(pos, idx, rays)
        out[f"{name}_ids"] = ref["ids"]
        out[f"{name}_t"] = ref["t"]
        out[f"{name}_occ"] = ref["occluded"]
        meta["cases"][name] = {
            "mesh_sha256": digest(pos, idx),
            "rays_sha256": digest(rays),
            "num_triangles": int(idx.shape[0]),
            "num_rays": int(rays.shape[0]),
            "hit_fraction": float((ref["ids"] != 0xFFFFFFFF).mean()),
            "reference_slots": ref["timing"]["slots"],
        }
        print(name, meta["cases"][name])
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    np.savez_compressed(HERE / "cast_reference.npz", **out)


if __name__ == "__main__":
    main()
