"""CPU restatement of this project's path-guiding network, for tests only: TEST
INFRASTRUCTURE, not product.  The reference renderer has no path guiding, so there is no
reference code to follow; this restates, in float64 numpy, exactly what the GPU kernels in
sprout_b200/csrc/guide.cu compute (the same BF16 rounding of GEMM operands, the same output
mapping and loss), so that their forward outputs and parameter gradients can be checked.

Network (sprout_b200/csrc/guide.cuh): 32 -> 64 -> 64 -> 64 -> 64 (ReLU) -> 40.  Parameters are
packed per layer as W (out x in, row-major) then b (out).  Loss over a batch:
    (1/n) sum_i c_i * (-log q(w_i | x_i)),
q the mixture of 8 vMF lobes given by the outputs (means 4j..4j+2, log-concentrations 4j+3
clamped to [-3, 6], softmax weights from outputs 32..39).
"""

from __future__ import annotations

import numpy as np

INPUTS, WIDTH, OUTPUTS, LOBES, LAYERS = 32, 64, 40, 8, 5
LOG_KAPPA_MIN, LOG_KAPPA_MAX = -3.0, 6.0


def dims():
    return [(INPUTS if l == 0 else WIDTH, OUTPUTS if l == LAYERS - 1 else WIDTH) for l in range(LAYERS)]


def num_parameters():
    return sum(i * o + o for i, o in dims())


def unpack(params):
    """[(W (out, in), b (out,)), ...] views of the packed float32 vector."""
    out, k = [], 0
    for i, o in dims():
        w = params[k:k + i * o].reshape(o, i)
        k += i * o
        b = params[k:k + o]
        k += o
        out.append((w, b))
    return out


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float64."""
    a = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def init_parameters(seed=0):
    """He-style uniform initialisation (the one the renderer uses), float32."""
    rng = np.random.default_rng(seed)
    parts = []
    for i, o in dims():
        lim = np.sqrt(6.0 / i)
        parts += [rng.uniform(-lim, lim, (o, i)).ravel(), np.zeros(o)]
    return np.concatenate(parts).astype(np.float32)


def forward(params, x):
    """Outputs (n, 40) and the BF16 activations fed to each layer."""
    layers = unpack(params)
    a = bf16(x)
    acts = [a]
    for l, (w, b) in enumerate(layers):
        z = a @ bf16(w).T + b.astype(np.float64)
        if l < LAYERS - 1:
            a = bf16(np.maximum(z, 0.0))
            acts.append(a)
        else:
            return z, acts


def mixture(out):
    logits = out[:, 32:40]
    e = np.exp(logits - logits.max(axis=1, keepdims=True))
    w = e / e.sum(axis=1, keepdims=True)
    m = out[:, :32].reshape(-1, LOBES, 4)[:, :, :3]
    lm = np.linalg.norm(m, axis=2, keepdims=True)
    mu = np.where(lm > 1e-10, m / np.maximum(lm, 1e-300), np.array([0.0, 0.0, 1.0]))
    o = out[:, :32].reshape(-1, LOBES, 4)[:, :, 3]
    kappa = np.exp(np.clip(o, LOG_KAPPA_MIN, LOG_KAPPA_MAX))
    return mu, kappa, w, lm[:, :, 0], o


def vmf(mu, kappa, d):
    c = np.einsum("nlk,nk->nl", mu, d)
    return kappa / (2 * np.pi * -np.expm1(-2 * kappa)) * np.exp(kappa * (c - 1.0)), c


def loss(params, x, d, c):
    out, _ = forward(params, x)
    mu, kappa, w, _, _ = mixture(out)
    v, _ = vmf(mu, kappa, d)
    q = (w * v).sum(axis=1)
    return float(np.mean(c * -np.log(q)))


def output_gradients(out, d, c):
    """d loss / d outputs, (n, 40)."""
    n = out.shape[0]
    mu, kappa, w, lm, o = mixture(out)
    v, cos = vmf(mu, kappa, d)
    q = (w * v).sum(axis=1, keepdims=True)
    r = w * v / q
    g = np.zeros_like(out)
    s = (c / n)[:, None]
    g[:, 32:40] = s * (w - r)
    x2 = 2 * kappa
    dlog = 1.0 - x2 / np.expm1(x2) + kappa * (cos - 1.0)
    inside = (o > LOG_KAPPA_MIN) & (o < LOG_KAPPA_MAX)
    gk = s * np.where(inside, -r * dlog, 0.0)
    tang = d[:, None, :] - mu * cos[:, :, None]
    gm = s[:, :, None] * np.where((lm > 1e-10)[:, :, None],
                                  -(r * kappa / np.maximum(lm, 1e-300))[:, :, None] * tang, 0.0)
    gg = g[:, :32].reshape(n, LOBES, 4)
    gg[:, :, :3] = gm
    gg[:, :, 3] = gk
    g[:, :32] = gg.reshape(n, 32)
    return g


def gradients(params, x, d, c):
    """Gradient of the batch loss with respect to the packed parameters (float64)."""
    layers = unpack(params)
    out, acts = forward(params, x)
    dz = output_gradients(out, d, c)
    grads = []
    for l in range(LAYERS - 1, -1, -1):
        w, _ = layers[l]
        a = acts[l]
        grads.append((dz.T @ a, dz.sum(axis=0)))
        if l > 0:
            da = dz @ bf16(w)
            dz = da * (acts[l] > 0)
    grads.reverse()
    return np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
