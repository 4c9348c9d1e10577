"""Generates tests/golden/attenuation_reference.npz: the reference's medium coefficients
attenuation(attenuation colour, subsurface colour, distance, anisotropy)
(source/core/scene/material/collision_coefficients.inl:50-71) on seeded inputs -- colours over
[0, 1] and past its clamp, distances from 1 mm to 10 m, anisotropies over (-1, 1) -- by running
oracle/_ref/ref_attenuation (built by oracle/Makefile from the reference's sources).

    python tests/golden/make_attenuation_golden.py
"""

from __future__ import annotations

import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
HARNESS = HERE.parent.parent / "oracle" / "_ref" / "ref_attenuation"


def main():
    rng = np.random.default_rng(17)
    n = 2000
    colours = rng.uniform(-0.05, 1.05, (n, 6)).astype(np.float32)
    distance = np.exp(rng.uniform(np.log(1e-3), np.log(10.0), (n, 1))).astype(np.float32)
    g = rng.uniform(-0.999, 0.999, (n, 1)).astype(np.float32)
    inputs = np.concatenate([colours, distance, g], axis=1)
    text = "\n".join(" ".join(f"{x:.9g}" for x in row) for row in inputs) + "\n"
    out = subprocess.run([str(HARNESS)], input=text, capture_output=True, text=True, check=True).stdout
    coefficients = np.array([[float(x) for x in line.split()] for line in out.strip().splitlines()], np.float32)
    assert coefficients.shape == (n, 6)
    np.savez_compressed(HERE / "attenuation_reference.npz", inputs=inputs, mu_a_mu_s=coefficients,
                        source=np.frombuffer(b"oracle/_ref/ref_attenuation: attenuation()", np.uint8))
    print("wrote", HERE / "attenuation_reference.npz")


if __name__ == "__main__":
    main()
