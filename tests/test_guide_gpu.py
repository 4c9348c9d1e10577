"""The guiding network's GPU kernels against the CPU restatement (oracle/guide_oracle.py), on
the same parameters and inputs: the forward outputs and the training gradient.

Both use BF16 GEMM operands; the GPU accumulates in FP32 and the oracle in FP64, so an
activation can round to the neighbouring BF16 value now and then.  Tolerances: outputs within
1 % of the output scale; per layer, the gradient's relative L2 error below 2 % and its cosine
to the oracle's above 0.999."""

import ctypes
import pathlib
import sys

import numpy as np
import pytest

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parent.parent))

from oracle import guide_oracle as g  # noqa: E402
from sprout_b200 import _lib  # noqa: E402

pytestmark = pytest.mark.gpu


def batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, 32)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    c = rng.uniform(0.0, 3.0, n).astype(np.float32)
    return x, d, c


@pytest.mark.parametrize("n", [1, 127, 1000])
def test_forward_matches_oracle(n):
    params = g.init_parameters(3)
    x, _, _ = batch(n, 1)
    out = np.zeros((n, 40), np.float32)
    assert _lib.load().spb_guide_forward(params.ctypes.data, x.ctypes.data, n, out.ctypes.data) == 0
    ref, _ = g.forward(params, x)
    assert np.max(np.abs(out - ref)) <= 0.01 * np.max(np.abs(ref))


@pytest.mark.parametrize("n", [129, 4096])
def test_gradients_match_oracle(n):
    params = g.init_parameters(4)
    x, d, c = batch(n, 2)
    grad = np.zeros(g.num_parameters(), np.float32)
    lib = _lib.load()
    assert lib.spb_guide_gradients(params.ctypes.data, x.ctypes.data, d.ctypes.data, c.ctypes.data, n,
                                   grad.ctypes.data) == 0, lib.spb_last_error()
    ref = g.gradients(params, x.astype(np.float64), d.astype(np.float64), c.astype(np.float64))
    k = 0
    for i, o in g.dims():
        for size in (i * o, o):
            a, b = grad[k:k + size].astype(np.float64), ref[k:k + size]
            k += size
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
            cos = a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30)
            assert rel < 0.02 and cos > 0.999, (i, o, size, rel, cos)
