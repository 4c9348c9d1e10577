"""Host light-tree build: structural invariants checked by a C++ driver (light_tree_check.cpp)
compiled against the library's own builder source."""

import pathlib
import shutil
import subprocess

import pytest

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_light_tree_invariants(tmp_path):
    exe = tmp_path / "light_tree_check"
    subprocess.run(["g++", "-O2", "-std=c++17", str(HERE / "light_tree_check.cpp"),
                    str(ROOT / "sprout_b200" / "csrc" / "light_tree.cpp"), "-o", str(exe)], check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.count("ok ") == 7, res.stdout
