"""Shared inputs and checks for the cast tests (deterministic, no randomness outside seeds)."""

from __future__ import annotations

import numpy as np

RAY_MAX_T = np.float32(3.4027715434167032e38)  # scene::Ray_max_t, scene_constants.hpp:10
MISS = 0xFFFFFFFF


def _ray(o, d, tmin=0.0, tmax=RAY_MAX_T):
    return np.array([o[0], o[1], o[2], tmin, d[0], d[1], d[2], tmax], np.float32)


def edge_rays(positions, indices):
    """Hand-made rays for the cases the traversal must get right:

    axis-aligned directions (zero components, infinite reciprocals), rays aimed at vertices,
    edge midpoints and centroids (shared-edge ties), rays from a vertex (t = 0 hits), limited
    max_t, min_t past the first hit, min_t > max_t, zero and NaN directions, grazing rays.
    """
    pos = np.asarray(positions, np.float32)
    idx = np.asarray(indices, np.uint32)
    out = []
    axes = np.eye(3, dtype=np.float32)
    for a in range(3):
        for s in (1.0, -1.0):
            d = axes[a] * s
            out.append(_ray((0, 0, 0), d))
            out.append(_ray(-3.0 * d, d))                 # from outside through the centre
            out.append(_ray((0, 0, 0), d, tmax=0.5))      # stops short of the surface
            out.append(_ray(-3.0 * d, d, tmin=3.0))       # skips the near side
            out.append(_ray(-3.0 * d, d, tmin=2.0, tmax=1.0))
    picks = np.linspace(0, len(idx) - 1, 24).astype(np.int64)
    for t in picks:
        a, b, c = pos[idx[t, 0]], pos[idx[t, 1]], pos[idx[t, 2]]
        for target in (a, 0.5 * (a + b), (a + b + c) / 3.0):
            d = (target / np.linalg.norm(target)).astype(np.float32)
            out.append(_ray((0, 0, 0), d))
            out.append(_ray(3.0 * d, -d))
        n = np.cross(b - a, c - a)
        n = (n / np.linalg.norm(n)).astype(np.float32)
        out.append(_ray(a, n))            # leaves from a vertex outward
        out.append(_ray(a, -n))           # enters from a vertex inward (t = 0 candidates)
    out.append(_ray((0, 0, 0), (0, 0, 0)))
    out.append(_ray((0, 0, 0), (np.nan, 0, 1)))
    out.append(_ray((0, 1.15, -3), (0, 0, 1)))     # grazing the displaced surface
    out.append(_ray((1.05, 0, -3), (0, 0, 1)))
    out.append(_ray((0.5, 0.5, 0.5), (1, 1, 1) / np.sqrt(np.float32(3))))
    return np.stack(out).astype(np.float32)


def classify_mismatches(positions, indices, rays, ids_a, t_a, ids_b, t_b, test):
    """Counts disagreements between two closest-hit results that are NOT explained by
    rounding at a triangle edge or an equal-t tie.  ``test(ray, a, b, c)`` is the restated
    triangle test returning (pass, t, u, v).  Returns (explained, unexplained) index lists."""
    pos = np.asarray(positions, np.float32)
    idx = np.asarray(indices, np.uint32)
    explained, unexplained = [], []
    for i in np.nonzero(ids_a != ids_b)[0]:
        ray = rays[i]
        ok = True
        tvals = []
        for tid in (ids_a[i], ids_b[i]):
            if tid == MISS:
                continue
            a, b, c = pos[idx[tid, 0]], pos[idx[tid, 1]], pos[idx[tid, 2]]
            _, t, u, v = test(ray, a, b, c)
            margin = min(u, 1.0 - u, v, 1.0 - u - v)
            if not np.isfinite(t) or margin < -1e-5:
                ok = False
            tvals.append(t)
        if len(tvals) == 2 and abs(tvals[0] - tvals[1]) > 1e-5 * max(1.0, abs(tvals[0])):
            ok = False
        if len(tvals) == 1:
            # one side missed: the other's hit must sit on an edge
            tid = ids_a[i] if ids_a[i] != MISS else ids_b[i]
            a, b, c = pos[idx[tid, 0]], pos[idx[tid, 1]], pos[idx[tid, 2]]
            _, t, u, v = test(ray, a, b, c)
            if min(abs(u), abs(1 - u), abs(v), abs(1 - u - v)) > 1e-5:
                ok = False
        (explained if ok else unexplained).append(int(i))
    return explained, unexplained
