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
    rounding at a triangle edge or an equal-t tie (the checker lives in the oracle package)."""
    import oracle

    return oracle.classify_mismatches(positions, indices, rays, ids_a, t_a, ids_b, t_b, test)
