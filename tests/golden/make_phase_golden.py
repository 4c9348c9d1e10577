"""Generates tests/golden/phase_reference.npz: the reference's Henyey-Greenstein phase function,
its sampling and the anisotropy and similarity-relation scale by depth (material.inl:15-40,
material.cpp:108-140) on seeded inputs, by running oracle/_ref/ref_phase (built by
oracle/Makefile from the reference's sources).

    python tests/golden/make_phase_golden.py
"""

from __future__ import annotations

import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
HARNESS = HERE.parent.parent / "oracle" / "_ref" / "ref_phase"


def main():
    rng = np.random.default_rng(23)
    n = 1000
    g = np.concatenate([rng.uniform(-0.99, 0.99, n - 4), [0.0, 0.0005, -0.0005, 0.9]]).astype(np.float32)
    cos = rng.uniform(-1.0, 1.0, n).astype(np.float32)
    wo = rng.normal(size=(n, 3))
    wo = (wo / np.linalg.norm(wo, axis=1, keepdims=True)).astype(np.float32)
    r = rng.uniform(0.0, 1.0, (n, 2)).astype(np.float32)
    gd = rng.uniform(-0.99, 0.99, 200).astype(np.float32)
    depth = np.arange(200, dtype=np.uint32) % 100
    lines = [f"p {c:.9g} {x:.9g}" for c, x in zip(cos, g)]
    lines += [f"s {w[0]:.9g} {w[1]:.9g} {w[2]:.9g} {a:.9g} {b:.9g} {x:.9g}" for w, (a, b), x in zip(wo, r, g)]
    lines += [f"v {x:.9g} {d}" for x, d in zip(gd, depth)]
    out = subprocess.run([str(HARNESS)], input="\n".join(lines) + "\n", capture_output=True, text=True,
                         check=True).stdout.strip().splitlines()
    vals = [[float(x) for x in line.split()] for line in out]
    np.savez_compressed(HERE / "phase_reference.npz", g=g, cos=cos, wo=wo, r=r, gd=gd, depth=depth,
                        phase=np.array([v[0] for v in vals[:n]], np.float32),
                        sample=np.array(vals[n:2 * n], np.float32),
                        by_depth=np.array(vals[2 * n:], np.float32),
                        source=np.frombuffer(b"oracle/_ref/ref_phase", np.uint8))
    print("wrote", HERE / "phase_reference.npz")


if __name__ == "__main__":
    main()
