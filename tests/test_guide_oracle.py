"""The CPU restatement of the guiding network (oracle/guide_oracle.py): its analytic gradient
against central finite differences (with BF16 rounding switched off so that small parameter
steps are not rounded away), and its parameter layout against the library's."""

import ctypes
import sys
import pathlib

import numpy as np

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parent.parent))

from oracle import guide_oracle as g  # noqa: E402


def test_parameter_layout_matches_library():
    from sprout_b200 import _lib

    n = ctypes.c_uint32()
    assert _lib.load().spb_guide_parameter_count(ctypes.byref(n)) == 0
    assert n.value == g.num_parameters() == 17192


def test_oracle_gradient_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(g, "bf16", lambda x: np.asarray(x, np.float64))
    rng = np.random.default_rng(0)
    p = g.init_parameters(1).astype(np.float64)
    x = rng.normal(size=(48, 32))
    d = rng.normal(size=(48, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    c = rng.uniform(0, 2, 48)
    grad = g.gradients(p, x, d, c)
    eps = 1e-6
    for idx in rng.choice(g.num_parameters(), 40, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[idx] += eps
        pm[idx] -= eps
        fd = (g.loss(pp, x, d, c) - g.loss(pm, x, d, c)) / (2 * eps)
        assert abs(fd - grad[idx]) < 1e-7 + 1e-5 * abs(fd), (idx, fd, grad[idx])
