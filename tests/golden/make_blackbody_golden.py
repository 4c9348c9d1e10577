"""Generates tests/golden/blackbody_reference.npz: the reference's spectrum::blackbody
(source/base/spectrum/mapping.cpp:125-147) at the 16 temperatures of Grid_emission's table
(2000 + 200 k kelvin, volumetric_grid.cpp:140-160) and a few beyond, as linear sRGB, by
running oracle/_ref/ref_blackbody (built by oracle/Makefile from the reference's sources).

    python tests/golden/make_blackbody_golden.py
"""

from __future__ import annotations

import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
HARNESS = HERE.parent.parent / "oracle" / "_ref" / "ref_blackbody"


def main():
    kelvin = [2000.0 + 200.0 * k for k in range(16)] + [1500.0, 6500.0, 8000.0, 10000.0]
    out = subprocess.run([str(HARNESS)] + [f"{t:.1f}" for t in kelvin], capture_output=True, text=True,
                         check=True).stdout
    rows = np.array([[float(x) for x in line.split()] for line in out.strip().splitlines()])
    assert rows.shape == (len(kelvin), 4)
    np.savez_compressed(HERE / "blackbody_reference.npz", kelvin=rows[:, 0], srgb=rows[:, 1:].astype(np.float64),
                        source=np.frombuffer(b"oracle/_ref/ref_blackbody: spectrum::blackbody", np.uint8))
    print("wrote", HERE / "blackbody_reference.npz")


if __name__ == "__main__":
    main()
