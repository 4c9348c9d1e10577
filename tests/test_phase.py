"""The medium's phase function (sprout_b200/csrc/material.cuh) against the reference's
(tests/golden/phase_reference.npz, made by the compiled reference through oracle/_ref/ref_phase):
Henyey-Greenstein values, the sampled direction's cosine to the forward direction and its pdf
(the frame around it is each renderer's own, so the azimuth is not compared), unit length, and
the anisotropy and similarity-relation scale by depth that the trackers use.  Bounds are float
rounding: the cosine is recomputed from each side's direction (built in its own frame), and
near the forward peak of g = 0.99 one float ulp of the cosine moves the pdf by up to 5e-4
relative."""

import pathlib
import shutil
import subprocess

import numpy as np
import pytest

HERE = pathlib.Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def answers(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    exe = tmp_path_factory.mktemp("phase") / "phase_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", str(HERE / "phase_check.cpp"), "-o", str(exe)],
                   check=True)
    ref = np.load(HERE / "golden" / "phase_reference.npz")
    lines = [f"p {c:.9g} {x:.9g}" for c, x in zip(ref["cos"], ref["g"])]
    lines += [f"s {w[0]:.9g} {w[1]:.9g} {w[2]:.9g} {a:.9g} {b:.9g} {x:.9g}"
              for w, (a, b), x in zip(ref["wo"], ref["r"], ref["g"])]
    lines += [f"v {x:.9g} {d}" for x, d in zip(ref["gd"], ref["depth"])]
    out = subprocess.run([str(exe)], input="\n".join(lines) + "\n", capture_output=True, text=True,
                         check=True).stdout.strip().splitlines()
    vals = [[float(x) for x in line.split()] for line in out]
    n = len(ref["g"])
    return ref, np.array([v[0] for v in vals[:n]]), np.array(vals[n:2 * n]), np.array(vals[2 * n:])


def test_phase_values(answers):
    ref, phase, _, _ = answers
    np.testing.assert_allclose(phase, ref["phase"], rtol=1e-5, atol=0)


def test_phase_sampling(answers):
    ref, _, sample, _ = answers
    want = ref["sample"].astype(np.float64)
    np.testing.assert_allclose(sample[:, 0], want[:, 0], rtol=0, atol=5e-6)   # cosine to the forward direction
    np.testing.assert_allclose(sample[:, 1], want[:, 1], rtol=1e-3, atol=0)   # its pdf
    np.testing.assert_allclose(sample[:, 2], 1.0, atol=2e-6)


def test_anisotropy_and_similarity_relation_by_depth(answers):
    ref, _, _, by_depth = answers
    np.testing.assert_allclose(by_depth, ref["by_depth"], rtol=1e-6, atol=1e-7)
