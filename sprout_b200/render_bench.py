"""Path-tracer measurement: the Cornell scene (sprout_b200.scenes.cornell) rendered through the
su_* C API, timed on the device.

    python -m sprout_b200.render_bench [--size 512] [--spp 64] [--frames 3] [--convergence]

Prints one JSON object: samples/s and rays/s (closest-hit + shadow) per frame, the end-to-end
frame rate seen by the caller (render + postprocess + framebuffer copy to host), optionally
the sample count and device time to reach relMSE 0.01 against a 4096-spp image of this
renderer, and optionally the reference renderer's time for the same frame on the host cores.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import time

import numpy as np

from . import _lib, capi, scenes

CONFIG = ("Cornell box (5 walls, 0.25 m^2 light of radiance 17, 81,920-tri GGX conductor sphere alpha 0.3), "
          "PTMIS max depth 8 (Russian roulette from depth 4)")


def rel_mse(x, r):
    """Mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2)."""
    return float(np.mean((x - r) ** 2 / (r * r + 1e-2)))


def measure(size=512, spp=64, frames=3, convergence=False, cpu_reference=False):
    lib = _lib.load()
    stats = _lib.RenderStats()
    su = capi.SuLibrary()
    out = {"config": f"{CONFIG}, {size}x{size}, {spp} spp"}
    assert su.su_init(False) == 0
    try:
        scenes.cornell(su, size, size, sphere_subdivisions=6, tonemap=True, spp=spp)
        assert su.su_render_frame(0) == 0, su.messages  # scene upload + BVH build + warm-up
        dev, wall = [], []
        for _ in range(frames):
            t0 = time.perf_counter()
            assert su.su_render_frame(0) == 0
            assert su.su_postprocess() == 0
            su.framebuffer(size, size)
            wall.append(time.perf_counter() - t0)
            assert lib.spb_render_last_stats(ctypes.byref(stats)) == 0
            dev.append(stats.device_seconds)
        dev_s = statistics.median(dev)
        rays = stats.extension_rays + stats.shadow_rays
        samples = size * size * spp
        out.update({"msamples_s": round(samples / dev_s / 1e6, 3), "mrays_s": round(rays / dev_s / 1e6, 3),
                    "ms_per_frame": round(1e3 * dev_s, 3), "rays_per_sample": round(rays / samples, 3),
                    "e2e_msamples_s": round(samples / statistics.median(wall) / 1e6, 3),
                    "e2e_note": "su_render_frame + su_postprocess + su_copy_framebuffer to host, wall clock"})
        if convergence:
            assert su.su_create_sampler(4096) == 0
            assert su.su_render_frame(0) == 0 and su.su_postprocess() == 0
            ref = su.framebuffer(size, size)[0][:, :, :3].copy()
            k, reached = 1, None
            while k <= 1024:
                assert su.su_create_sampler(k) == 0
                assert su.su_render_frame(0) == 0 and su.su_postprocess() == 0
                lib.spb_render_last_stats(ctypes.byref(stats))
                e = rel_mse(su.framebuffer(size, size)[0][:, :, :3], ref)
                if e <= 0.01:
                    reached = {"spp": k, "device_seconds": round(stats.device_seconds, 5), "rel_mse": round(e, 5)}
                    break
                k *= 2
            out["time_to_rel_mse_0.01"] = reached
            out["rel_mse_against"] = "4096-spp image of this renderer (plain MIS; no guiding)"
    finally:
        su.su_release()

    if cpu_reference:
        import oracle  # test/baseline infrastructure: times the reference renderer

        if oracle.REF_RENDER.exists():
            _, timing = oracle.reference_render(
                lambda r: scenes.cornell(r, size, size, sphere_subdivisions=6, tonemap=True, spp=spp),
                size, size, 0, progressive=False)
            out["cpu_baseline"] = {"msamples_s": round(size * size * spp / timing["render_s"] / 1e6, 4),
                                   "seconds": round(timing["render_s"], 3), "cores": os.cpu_count(),
                                   "kind": "reference",
                                   "sample": "full frame, the reference's su_render_frame (batch) on all host threads"}
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--size", type=int, default=512)
    p.add_argument("--spp", type=int, default=64)
    p.add_argument("--frames", type=int, default=3)
    p.add_argument("--convergence", action="store_true")
    p.add_argument("--cpu-reference", action="store_true")
    a = p.parse_args()
    print(json.dumps(measure(a.size, a.spp, a.frames, a.convergence, a.cpu_reference)))


if __name__ == "__main__":
    main()
