"""Medium coefficients from colours (sprout_b200/csrc/material.cuh, attenuation: homogeneous
media take theirs from it once, colour grids at every collision) against the reference's
attenuation() on 2,000 seeded inputs (tests/golden/attenuation_reference.npz, made by the
compiled reference through oracle/_ref/ref_attenuation).  The same float arithmetic in the same
order, but the reference's vector log and square root round differently from the C library's,
and mu_a = mu_t (1 - pss) cancels where the albedo is near 1; so each coefficient must agree
within 1e-5 of its channel's total mu_a + mu_s (the largest difference seen is 4.4e-6)."""

import pathlib
import shutil
import subprocess

import numpy as np
import pytest

HERE = pathlib.Path(__file__).resolve().parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_attenuation_matches_reference(tmp_path):
    exe = tmp_path / "attenuation_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", str(HERE / "attenuation_check.cpp"), "-o",
                    str(exe)], check=True)
    ref = np.load(HERE / "golden" / "attenuation_reference.npz")
    text = "\n".join(" ".join(f"{x:.9g}" for x in row) for row in ref["inputs"]) + "\n"
    out = subprocess.run([str(exe)], input=text, capture_output=True, text=True, check=True).stdout
    mine = np.array([[float(x) for x in line.split()] for line in out.strip().splitlines()], np.float32)
    want = ref["mu_a_mu_s"]
    assert mine.shape == want.shape
    total = np.tile(want[:, :3] + want[:, 3:], 2)
    err = np.abs(mine - want) / total
    assert err.max() < 1e-5, (err.max(), ref["inputs"][np.unravel_index(err.argmax(), err.shape)[0]])
