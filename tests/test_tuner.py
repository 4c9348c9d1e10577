"""The path tracer's online autotuner (sprout_b200/csrc/tuner.hpp): the order in which it tries
wave sizes and traversal occupancies and the shape it keeps, driven with synthetic timings by
a C++ check program."""

import pathlib
import shutil
import subprocess

import pytest

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE.parent / "sprout_b200" / "csrc"


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_tuner_search_order_and_choice(tmp_path):
    exe = tmp_path / "tuner_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", str(CSRC), str(HERE / "tuner_check.cpp"), "-o", str(exe)],
                   check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.count("ok ") == 6, res.stdout
