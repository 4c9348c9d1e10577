"""Path-tracer measurement through the su_* C API, timed on the device.  Four workloads:

* cornell: the Cornell scene (sprout_b200.scenes.cornell), 512x512, 64 spp, max depth 8;
* wavefront: 400 instances of a 5,000-triangle displaced sphere (2,000,000 triangles) lit by
  4,096 emissive triangles through the light tree (sprout_b200.scenes.wavefront), 1920x1080,
  256 spp, max depth 12;
* volume: a 2 m cube of 256^3 fBm density lit by a sphere light and the environment
  (sprout_b200.scenes.volume), a few of 64 seeded views of 256..1024 px, 128 spp, max depth
  32;
* guiding: the doorway interior (sprout_b200.scenes.doorway), 1280x720: sample count and
  device time to relMSE 0.01 for plain MIS and for learned path guiding.

    python -m sprout_b200.render_bench [--scene cornell|wavefront|volume|guiding] [--width 512] [--height 512] [--spp 64]
                                       [--frames 3] [--convergence] [--cpu-reference]

Prints one JSON object: samples/s and rays/s (closest-hit + shadow) per frame, the end-to-end
frame rate seen by the caller (render + postprocess + framebuffer copy to host), optionally
the sample count and device time to reach relMSE 0.01 against a 4096-spp image of this
renderer (the doorway against its 65,536-spp image), and optionally the reference renderer's rate on the host cores (the whole frame for
cornell; a 960x540, 16-spp frame of the same scene for wavefront), its scene preparation timed
apart.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import pathlib
import statistics
import time

import numpy as np

from . import _lib, capi, scenes

SCENES = {
    "cornell": ("Cornell box (5 walls, 0.25 m^2 light of radiance 17, 81,920-tri GGX conductor sphere alpha 0.3), "
                "PTMIS max depth 8 (Russian roulette from depth 4)",
                lambda su, w, h, spp, extra=None: scenes.cornell(su, w, h, sphere_subdivisions=6, tonemap=True, spp=spp,
                                                                  integrator=extra),
                (512, 512, 64), None),
    "wavefront": ("400 instances of a 5,000-tri displaced sphere (2,000,000 tris, Substitute roughness U[0.05,1], "
                  "metallic Bernoulli(0.3)), 4,096 emissive tris of log-uniform radiance [0.1, 100] via the light "
                  "tree, PTMIS max depth 12 (Russian roulette from depth 4); the props kept as instances of one "
                  "mesh under a top-level tree",
                  lambda su, w, h, spp, extra=None: scenes.wavefront(su, w, h, spp, integrator=extra),
                  (1920, 1080, 256), (960, 540, 16)),
    "wavefront_flat": ("the same scene with every prop flattened into one 2,004,098-triangle tree "
                       "(\"instancing\": false)",
                       lambda su, w, h, spp, extra=None: scenes.wavefront(su, w, h, spp,
                                                                           integrator={"instancing": False, **(extra or {})}),
                       (1920, 1080, 256), None),
}


def rel_mse(x, r):
    """Mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2)."""
    return float(np.mean((x - r) ** 2 / (r * r + 1e-2)))


def measure(scene="cornell", width=None, height=None, spp=None, frames=3, convergence=False,
            cpu_reference=False, tuning_frames=6, integrator=None):
    """Times `frames` steady-state frames of a scene (device time from the renderer's events;
    end to end by the wall clock).  integrator: further PTMIS keys (e.g. "cuda_graphs": false)."""
    config, build, (w0, h0, spp0), cpu_frame = SCENES[scene]
    width, height, spp = width or w0, height or h0, spp or spp0
    lib = _lib.load()
    stats = _lib.RenderStats()
    su = capi.SuLibrary()
    out = {"workload": scene, "config": f"{config}, {width}x{height}, {spp} spp"}
    assert su.su_init(False) == 0
    try:
        build(su, width, height, spp, integrator)
        t0 = time.perf_counter()
        assert su.su_start_render_frame(0) == 0, su.messages  # scene upload + BVH build
        out["prepare_s"] = round(time.perf_counter() - t0, 3)
        assert su.su_render_frame(0) == 0, su.messages  # warm-up (autotuner)
        out["first_frame_s"] = round(time.perf_counter() - t0, 3)
        # The autotuner tries wave sizes, then lower occupancies, one full wave each, and keeps
        # the best for later frames: warm up until two frames in a row end on the same launch
        # shape (the tuned one), so that timed frames are steady-state frames.
        shape = None
        for _ in range(tuning_frames):
            assert lib.spb_render_last_stats(ctypes.byref(stats)) == 0
            now = (stats.wave_paths, stats.trace_blocks_per_sm)
            if now == shape:
                break
            shape = now
            assert su.su_render_frame(0) == 0, su.messages
        out["launch_shape"] = {"wave_paths": stats.wave_paths, "trace_blocks_per_sm": stats.trace_blocks_per_sm}
        dev, wall = [], []
        for _ in range(frames):
            t0 = time.perf_counter()
            assert su.su_render_frame(0) == 0
            assert su.su_postprocess() == 0
            su.framebuffer(width, height)
            wall.append(time.perf_counter() - t0)
            assert lib.spb_render_last_stats(ctypes.byref(stats)) == 0
            dev.append(stats.device_seconds)
        dev_s = statistics.median(dev)
        rays = stats.extension_rays + stats.shadow_rays
        samples = width * height * spp
        out.update({"instances": stats.instances, "device_triangles": stats.device_triangles,
                    "graph_waves": stats.graph_waves,
                    "msamples_s": round(samples / dev_s / 1e6, 3), "mrays_s": round(rays / dev_s / 1e6, 3),
                    "ms_per_frame": round(1e3 * dev_s, 3), "rays_per_sample": round(rays / samples, 3),
                    "e2e_msamples_s": round(samples / statistics.median(wall) / 1e6, 3),
                    "e2e_note": "su_render_frame + su_postprocess + su_copy_framebuffer to host, wall clock"})
        if convergence:
            assert su.su_create_sampler(4096) == 0
            assert su.su_render_frame(0) == 0 and su.su_postprocess() == 0
            ref = su.framebuffer(width, height)[0][:, :, :3].copy()
            k, reached = 1, None
            while k <= 1024:
                assert su.su_create_sampler(k) == 0
                assert su.su_render_frame(0) == 0 and su.su_postprocess() == 0
                lib.spb_render_last_stats(ctypes.byref(stats))
                e = rel_mse(su.framebuffer(width, height)[0][:, :, :3], ref)
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
            cw, ch, cspp = cpu_frame or (width, height, spp)
            _, timing = oracle.reference_render(lambda r: build(r, cw, ch, cspp), cw, ch, 0, progressive=False,
                                                prepare=True)
            what = "full frame" if cpu_frame is None else f"{cw}x{ch}, {cspp} spp frame of the same scene"
            out["cpu_baseline"] = {"msamples_s": round(cw * ch * cspp / timing["render_s"] / 1e6, 4),
                                   "seconds": round(timing["render_s"], 3), "cores": os.cpu_count(),
                                   "prepare_seconds": round(timing["prepare_s"], 3),
                                   "kind": "reference",
                                   "sample": f"{what}, the reference's su_render_frame (batch) on all host "
                                             "threads; its mesh BVH builds and first scene compile run before, "
                                             "timed apart (prepare_seconds)"}
    return out


VOLUME_CONFIG = ("2 m cube of 256^3 fBm density (5 octaves, seed 4), mu_t 20 per metre at density 1, albedo 0.9, "
                 "HG g 0.6, lit by a sphere light of radius 0.25 and a uniform environment; PTMIS max depth 32; "
                 "RGB delta/ratio tracking (the reference's transport; no hero wavelengths)")


def measure_phase_guiding(side=256, spp=128, ref_spp=8192, fractions=(0.5,)):
    """The phase guide of the spectral mode on the volume workload's first view (side x side):
    plain and guided renders of spp samples per pixel against a plain render of ref_spp, each
    with its relMSE (mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2)) and device
    seconds; efficiency = (relMSE x seconds) of plain / that of guided (above 1: guiding pays).
    fractions: the guide's shares of the continuation to try (PTMIS "guiding": {"fraction"})."""
    lib = _lib.load()
    stats = _lib.RenderStats()
    density = scenes.fbm_density(256)
    position, _ = scenes.volume_views()[0]
    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    out = {"workload": "volume, spectral mode, phase guiding",
           "config": f"{VOLUME_CONFIG.split('; RGB')[0]}; hero-wavelength spectral mode; first view at "
                     f"{side}x{side}, {spp} spp; reference {ref_spp} spp plain"}
    try:
        scenes.volume(su, side, side, spp, density, position=position)

        def frame(n, guiding):
            ptmis = {"min_bounces": 4, "max_bounces": 32, "spectral": True}
            if guiding is not None:
                ptmis["guiding"] = guiding
            assert su.su_create_integrators(json.dumps({"surface": {"PTMIS": ptmis}}).encode()) == 0
            assert su.su_create_sampler(n) == 0
            assert su.su_render_frame(0) == 0, su.messages
            assert su.su_postprocess() == 0
            img = su.framebuffer(side, side)[0][:, :, :3].copy()
            assert lib.spb_render_last_stats(ctypes.byref(stats)) == 0
            return img, stats.device_seconds

        ref, ref_s = frame(ref_spp, None)
        frame(spp, None)  # warm-up
        plain, plain_s = frame(spp, None)
        e_plain = rel_mse(plain, ref)
        out["plain"] = {"rel_mse": round(e_plain, 6), "device_seconds": round(plain_s, 4)}
        out["reference_device_seconds"] = round(ref_s, 3)
        for f in fractions:
            img, sec = frame(spp, {"fraction": f})
            e = rel_mse(img, ref)
            out[f"guided_{f}"] = {"rel_mse": round(e, 6), "device_seconds": round(sec, 4),
                                  "mean_ratio": [round(float(x), 4) for x in img.mean((0, 1)) / ref.mean((0, 1))],
                                  "efficiency": round(e_plain * plain_s / (e * sec), 3)}
    finally:
        su.su_release()
    return out


def measure_volume(views=4, spp=128, cpu_reference=False, batch=True, spectral=True, density_side=256):
    """The heterogeneous-volume workload: the first `views` of scenes.volume_views() (seeded
    camera positions, image sides U[256, 1024]) of one scene, built and uploaded once; each
    view moves the camera and sets its resolution, then renders one frame.  Samples/s over the
    device time of all views; the end-to-end rate includes, per view, su_render_frame +
    su_postprocess + framebuffer copy, and the scene's one-time upload.  With batch, the same
    views are also rendered together in one spb_render_views call (after one untimed call),
    timed on the device and end to end (the call, with every view's image copied to the host).
    With spectral, the same batch once more in the hero-wavelength spectral mode (4 wavelengths
    per path in [380, 720] nm; every view and sample in one persistent launch).  density_side:
    the density grid's side (256 for the workload; smaller for profiling runs)."""
    lib = _lib.load()
    stats = _lib.RenderStats()
    density = scenes.fbm_density(density_side)
    chosen = scenes.volume_views()[:views]
    samples, seconds, rays, wall = 0, 0.0, 0, 0.0
    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        position, side = chosen[0]
        cam = scenes.volume(su, side, side, spp, density, position=position)
        for position, side in chosen:
            t0 = time.perf_counter()
            assert su.su_camera_set_resolution(side, side) == 0
            su.set_transformation(cam, scenes._look_at(position))
            assert su.su_render_frame(0) == 0, su.messages
            assert su.su_postprocess() == 0
            su.framebuffer(side, side)
            wall += time.perf_counter() - t0
            assert lib.spb_render_last_stats(ctypes.byref(stats)) == 0
            seconds += stats.device_seconds
            samples += side * side * spp
            rays += stats.extension_rays + stats.shadow_rays
        if batch:
            cams = [(side, side, scenes.VOLUME_FOV, scenes._look_at(position)) for position, side in chosen]
            su.render_views(cams, spp)  # warm-up: the autotuner's probes
            t0 = time.perf_counter()
            su.render_views(cams, spp)
            batch_wall = time.perf_counter() - t0
            assert lib.spb_render_last_stats(ctypes.byref(stats)) == 0
            batch_out = {"msamples_s": round(samples / stats.device_seconds / 1e6, 3),
                         "mrays_s": round((stats.extension_rays + stats.shadow_rays) / stats.device_seconds / 1e6, 3),
                         "device_seconds": round(stats.device_seconds, 3),
                         "e2e_msamples_s": round(samples / batch_wall / 1e6, 3),
                         "wave_paths": stats.wave_paths,
                         "note": f"all {views} views in one spb_render_views call: their paths share the waves; "
                                 "e2e = the call, every view's image copied to the host"}
        if spectral:
            assert su.su_create_integrators(json.dumps({"surface": {"PTMIS": {
                "min_bounces": 4, "max_bounces": 32, "spectral": True}}}).encode()) == 0
            su.render_views(cams, spp)  # warm-up
            t0 = time.perf_counter()
            su.render_views(cams, spp)
            spectral_wall = time.perf_counter() - t0
            assert lib.spb_render_last_stats(ctypes.byref(stats)) == 0
            spectral_out = {"msamples_s": round(samples / stats.device_seconds / 1e6, 3),
                            "device_seconds": round(stats.device_seconds, 3),
                            "e2e_msamples_s": round(samples / spectral_wall / 1e6, 3),
                            "segments_per_sample": round(stats.extension_rays / stats.paths, 3),
                            "shadow_rays_per_sample": round(stats.shadow_rays / stats.paths, 3),
                            "note": f"hero-wavelength spectral mode (4 wavelengths in [380, 720] nm per path), "
                                    f"all {views} views and samples in one persistent launch"}
    finally:
        su.su_release()
    grid = "" if density_side == 256 else f" [density grid {density_side}^3 instead of 256^3]"
    out = {"workload": "volume", "config": f"{VOLUME_CONFIG}{grid}, {views} of 64 views (sides "
                                           f"{[v[1] for v in chosen]}), {spp} spp",
           "msamples_s": round(samples / seconds / 1e6, 3), "mrays_s": round(rays / seconds / 1e6, 3),
           "device_seconds": round(seconds, 3),
           "e2e_msamples_s": round(samples / wall / 1e6, 3),
           "e2e_note": "per view: camera move + su_render_frame + su_postprocess + su_copy_framebuffer to "
                       "host, wall clock (the scene's one-time upload and majorant build in the first view)"}
    if batch:
        out["batch"] = batch_out
        if spectral:
            out["spectral_batch"] = spectral_out
    if cpu_reference:
        import oracle  # test/baseline infrastructure: times the reference renderer

        if oracle.REF_RENDER.exists():
            position, _ = chosen[0]
            cw, cspp = 256, 32
            _, timing = oracle.reference_render(
                lambda r: scenes.volume(r, cw, cw, cspp, density, position=position), cw, cw, 0, progressive=False,
                prepare=True)
            out["cpu_baseline"] = {"msamples_s": round(cw * cw * cspp / timing["render_s"] / 1e6, 4),
                                   "seconds": round(timing["render_s"], 3), "cores": os.cpu_count(),
                                   "prepare_seconds": round(timing["prepare_s"], 3),
                                   "kind": "reference",
                                   "sample": f"first view at {cw}x{cw}, {cspp} spp, the reference's su_render_frame "
                                             "(batch) on all host threads; the majorant tree (built when the "
                                             "material is created), the mesh BVH builds and the first scene compile "
                                             "run before it, timed apart (prepare_seconds)"}
    return out


GUIDING_CONFIG = ("doorway interior (sprout_b200.scenes.doorway): 6 x 6 x 3 m room lit only through a 1 x 2 m "
                  "doorway by a uniform environment of radiance 5; 96 icospheres (491,520 tris) and 160 boxes, 70 % "
                  "diffuse / 30 % GGX conductors alpha U[0.1, 0.6]; PTMIS max depth 8 (Russian roulette from 4)")


def doorway_frame(width, height, spp, guiding=None, seed=0, stats_out=None):
    """One frame of the doorway interior through the su_* API: (RGB image as float64, device
    seconds of the render, wall seconds of su_render_frame + su_postprocess + framebuffer copy).
    The scene is built and uploaded before the timed frame (su_start_render_frame); a guided
    frame starts from an untrained network all the same (the first frame of the engine).
    stats_out (a dict), when given, receives the frame's spb_render_stats fields."""
    lib = _lib.load()
    stats = _lib.RenderStats()
    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        scenes.doorway(su, width, height, spp, guiding=guiding, render_seed=seed)
        assert su.su_start_render_frame(0) == 0, su.messages  # scene flattening, BVH build, upload
        t0 = time.perf_counter()
        assert su.su_render_frame(0) == 0, su.messages
        assert su.su_postprocess() == 0
        img = su.framebuffer(width, height)[0][:, :, :3].astype(np.float64)
        wall = time.perf_counter() - t0
        assert lib.spb_render_last_stats(ctypes.byref(stats)) == 0
        if stats_out is not None:
            stats_out.update({name: getattr(stats, name) for name, _ in stats._fields_})
        return img, stats.device_seconds, wall
    finally:
        su.su_release()


# Algorithmic FLOPs of the guiding network (32 -> 64 x 4 -> 40): forward per vertex; a training
# sample adds dW of every layer (as many again) and dA of layers 1..4.
GUIDE_FORWARD_FLOP = 2 * (32 * 64 + 3 * 64 * 64 + 64 * 40)  # 33,792
GUIDE_TRAIN_FLOP = 2 * GUIDE_FORWARD_FLOP + 2 * (3 * 64 * 64 + 64 * 40)  # 97,280


def network_roofline(stats):
    """The network's share of a guided frame against the tensor-core roofline: achieved
    algorithmic TFLOP/s of inference (input encoding included) and of training (batch gathering
    and Adam included) over their device time, as a fraction of the measured sustained BF16
    GEMM rate (MEASURED_PEAKS.json; the fallback figure when the file is absent)."""
    import pathlib

    peaks = pathlib.Path(__file__).resolve().parent.parent / "MEASURED_PEAKS.json"
    peak, kind = 1400.0, "fallback"
    if peaks.exists():
        peak, kind = float(json.loads(peaks.read_text())["bf16_tflops_sustained"]), "measured"
    out = {"peak_tflops": peak, "peak_kind": f"{kind}, sustained bf16", "unit": "TFLOP/s",
           "flop_per_vertex": GUIDE_FORWARD_FLOP, "flop_per_training_sample": GUIDE_TRAIN_FLOP}
    if stats.get("guide_inference_seconds", 0) > 0:
        a = stats["guide_vertices"] * GUIDE_FORWARD_FLOP / stats["guide_inference_seconds"] / 1e12
        out["inference"] = {"vertices": stats["guide_vertices"],
                            "seconds": round(stats["guide_inference_seconds"], 4),
                            "achieved": round(a, 2), "frac": round(a / peak, 4)}
    if stats.get("guide_training_seconds", 0) > 0:
        a = stats["guide_training_samples"] * GUIDE_TRAIN_FLOP / stats["guide_training_seconds"] / 1e12
        out["training"] = {"samples": stats["guide_training_samples"],
                           "seconds": round(stats["guide_training_seconds"], 4),
                           "achieved": round(a, 2), "frac": round(a / peak, 4)}
    return out


REFERENCE_64K = pathlib.Path(__file__).resolve().parent.parent / "tests" / "golden" / "doorway_reference_64k.npz"

# Training schedules of the guided integrator ("guiding" key of the PTMIS integrator): this
# renderer's defaults (passes of 1 spp, 16 Adam steps of 65,536 records, learning rate 1e-2,
# training until 16 spp), and the configuration's own (batches of 2^18 records, learning rate
# 1e-3, the rest as the defaults).
GUIDING_SCHEDULES = {
    "tuned": True,
    "config": {"batch": 1 << 18, "learning_rate": 1e-3},
}


def measure_guiding(width=1280, height=720, target=0.01):
    """Time to relMSE `target` on the doorway interior: plain MIS against learned guiding under
    each training schedule.

    relMSE is the mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2), r the converged
    image tests/golden/doorway_reference_64k.npz (65,536 spp of plain MIS at 1280x720, summed in
    float64 over 64 frames of independent seeds; tests/golden/make_doorway_reference.py), with no
    rescaling and nothing subtracted (its own error adds about 0.01 * s / 65536 at s spp).  For
    each integrator a probe render predicts the sample count that reaches the target (relMSE
    falls as 1 / spp), renders at that count (raised until the target is met) give the reported
    count, and the frame at that count is rendered three times; the median device and wall
    times are reported, so that one host stall on a shared machine does not set the ratio."""
    if not REFERENCE_64K.exists():
        raise FileNotFoundError(f"{REFERENCE_64K} missing: make it with tests/golden/make_doorway_reference.py")
    data = np.load(REFERENCE_64K)
    ref = data["image"].astype(np.float64)
    meta = json.loads(bytes(data["meta"]).decode())
    assert ref.shape == (height, width, 3), ref.shape

    def rel(img):
        return float(np.mean((img - ref) ** 2 / (ref * ref + 1e-2)))

    out = {"workload": "doorway", "config": f"{GUIDING_CONFIG}, {width}x{height}",
           "rel_mse": "mean over pixels and channels of (x - r)^2 / (r^2 + 0.01), no rescaling",
           "reference": {"spp": meta["spp"], "integrator": "plain MIS, float64 sum of 64 frames of independent "
                                                           "seeds (tests/golden/doorway_reference_64k.npz)",
                         "mean": [round(x, 6) for x in meta["mean"]]},
           "target": target}

    last_stats = {}

    def reach(first, guiding):
        """The smallest multiple of 8 spp whose frame meets the target: up from the prediction
        until it is met, then down while it still is."""
        spp, runs = first, []
        met = None
        for _ in range(12):
            img, dev, wall = doorway_frame(width, height, spp, guiding, stats_out=last_stats)
            err = rel(img)
            runs.append({"spp": spp, "rel_mse": round(err, 5), "device_seconds": round(dev, 4),
                         "wall_seconds": round(wall, 3)})
            if err <= target:
                met = runs[-1]
                if spp <= 8 or (len(runs) > 1 and runs[-2]["spp"] < spp):
                    break  # came up to it: the count below missed
                spp -= 8
            elif met is not None:
                break  # went down past it
            else:
                spp = max(spp + 8, int(np.ceil(spp * err / target / 8.0)) * 8)
        last = met if met is not None else runs[-1]
        spp  = last["spp"]
        devs, walls = [last["device_seconds"]], [last["wall_seconds"]]
        for _ in range(2):
            _, dev, wall = doorway_frame(width, height, spp, guiding, stats_out=last_stats)
            devs.append(round(dev, 4))
            walls.append(round(wall, 3))
        last["device_seconds"], last["wall_seconds"] = float(np.median(devs)), float(np.median(walls))
        last["device_seconds_frames"], last["wall_seconds_frames"] = devs, walls
        runs.remove(last)
        runs.append(last)
        return runs

    def predicted(guiding, probe):
        img, _, _ = doorway_frame(width, height, probe, guiding)
        return max(8, int(np.ceil(probe * rel(img) / target / 8.0)) * 8)

    plain = reach(predicted(None, 256), None)
    out["plain"] = plain[-1]
    out["runs"] = {"plain": plain}
    out["schedules"] = {}
    for name, guiding in GUIDING_SCHEDULES.items():
        runs = reach(predicted(guiding, 128), guiding)
        entry = {"guiding": guiding, "result": runs[-1], "network": network_roofline(last_stats)}
        if plain[-1]["rel_mse"] <= target and runs[-1]["rel_mse"] <= target:
            entry["guided_over_plain_device_time"] = round(runs[-1]["device_seconds"] / plain[-1]["device_seconds"], 4)
            entry["guided_over_plain_wall_time"] = round(runs[-1]["wall_seconds"] / plain[-1]["wall_seconds"], 4)
        out["schedules"][name] = entry
        out["runs"][name] = runs
    tuned = out["schedules"]["tuned"]
    out["guided"] = tuned["result"]
    out["network"] = tuned["network"]
    for key in ("guided_over_plain_device_time", "guided_over_plain_wall_time"):
        if key in tuned:
            out[key] = tuned[key]
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--scene", choices=sorted(SCENES) + ["volume", "guiding", "doorway"], default="cornell",
                   help="doorway: one frame of the guiding workload (plain MIS, or --guided)")
    p.add_argument("--guided", action="store_true", help="doorway: learned path guiding")
    p.add_argument("--views", type=int, default=4, help="volume workload: number of views")
    p.add_argument("--density", type=int, default=256, help="volume workload: the density grid's side")
    p.add_argument("--width", type=int)
    p.add_argument("--height", type=int)
    p.add_argument("--spp", type=int)
    p.add_argument("--frames", type=int, default=3)
    p.add_argument("--convergence", action="store_true")
    p.add_argument("--cpu-reference", action="store_true")
    a = p.parse_args()
    if a.scene == "volume":
        print(json.dumps(measure_volume(a.views, a.spp or 128, a.cpu_reference, density_side=a.density)))
    elif a.scene == "guiding":
        print(json.dumps(measure_guiding(a.width or 1280, a.height or 720)))
    elif a.scene == "doorway":
        w, h, spp = a.width or 1280, a.height or 720, a.spp or 64
        st = {}
        img, dev, wall = doorway_frame(w, h, spp, True if a.guided else None, stats_out=st)
        print(json.dumps({"workload": "doorway", "guided": a.guided, "config": f"{GUIDING_CONFIG}, {w}x{h}, {spp} spp",
                          "device_seconds": round(dev, 4), "wall_seconds": round(wall, 4),
                          "msamples_s": round(w * h * spp / dev / 1e6, 3), "mean": float(img.mean()),
                          "stats": st, "network": network_roofline(st) if a.guided else None}))
    else:
        print(json.dumps(measure(a.scene, a.width, a.height, a.spp, a.frames, a.convergence, a.cpu_reference)))


if __name__ == "__main__":
    main()
