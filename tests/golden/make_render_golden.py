"""Generates tests/golden/cornell_reference.npz with the compiled reference renderer.

Renders the Cornell-box scene of sprout_b200.scenes.cornell through the reference's own C API
(oracle/_ref/ref_render replaying the su_* calls; batch mode, su_create_defaults, i.e. the
Linear tonemapper to linear sRGB) at sizes the tests can compare against.

    python tests/golden/make_render_golden.py [case ...]   (default: all cases; named cases
                                                            are re-rendered into the existing file)
"""

from __future__ import annotations

import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from sprout_b200 import scenes  # noqa: E402

# A homogeneous scattering sphere in place of the metal one (Volumetric material).
MEDIUM = {"color": [0.8, 0.8, 0.8], "attenuation_distance": 0.05, "anisotropy": 0.5}
# An optically thin one, seen through: with max_bounces 1 the image is the direct light of the
# surfaces behind it, reached through two null (boundary) vertices that must not count as
# bounces.
THIN_MEDIUM = {"color": [0.8, 0.8, 0.8], "attenuation_distance": 0.5, "anisotropy": 0.5}
# A rotated, scaled cube filled with a density grid (Volumetric material with "density"),
# colour-dependent attenuation so that spectral MIS matters.
GRID_MEDIUM = {"color": [0.9, 0.6, 0.4], "attenuation_distance": 0.03, "anisotropy": 0.3}

# An emissive homogeneous sphere that is not a light: the camera sees its emission (absorption
# events, each adding the emitted radiance), its scattered light stays dark beyond the camera
# segment, and it absorbs and scatters the room's light.
EMISSIVE_MEDIUM = {"color": [0.8, 0.8, 0.8], "subsurface_color": [0.3, 0.3, 0.3], "attenuation_distance": 0.1,
                   "anisotropy": 0.3, "emission": [6.0, 3.0, 1.0]}

# The volume workload's density grid emitting (a Grid_emission: emission per unit absorption,
# the absorption scaling with density), grey absorption; and with colour-dependent absorption,
# where the light's normalisation by the largest absorption coefficient matters.
GLOW = {"emission": [3.0, 1.5, 0.6]}
GLOW_COLOR = {"emission": [3.0, 1.5, 0.6], "attenuation_color": [0.6, 0.4, 0.25]}
# A thin homogeneous emitting medium.
HAZE = {"attenuation_color": [0.5, 0.5, 0.5], "subsurface_color": [0.7, 0.7, 0.7], "attenuation_distance": 1.0,
        "anisotropy": 0.3, "emission": [2.0, 1.0, 0.5]}

# name -> (width, height, spp, scenes.cornell keyword arguments, density grid or None)
CASES = {
    "cornell64_sub3": (64, 64, 4096, {"sphere_subdivisions": 3}, None),
    "cornell128_sub6": (128, 128, 2048, {"sphere_subdivisions": 6}, None),
    "cornell64_medium": (64, 64, 4096, {"sphere_subdivisions": 4, "medium": MEDIUM}, None),
    "cornell64_thin_direct": (64, 64, 4096, {"sphere_subdivisions": 4, "medium": THIN_MEDIUM,
                                             "max_bounces": 1, "min_bounces": 1}, None),
    "cornell64_emissive": (64, 64, 4096, {"sphere_subdivisions": 4, "medium": EMISSIVE_MEDIUM}, None),
    "cornell64_grid": (64, 64, 4096, {"sphere_subdivisions": 2, "medium": GRID_MEDIUM},
                       scenes.density_grid()),
    # 66 emitters of different radiance and orientation, two of them two-sided (light tree)
    "cornell64_lights": (64, 64, 4096, {"sphere_subdivisions": 3, "many_lights": True}, None),
    # 400 instanced displaced spheres (rotated, scaled props sharing one mesh), 4,096 emitters
    "wavefront96": (96, 54, 2048, {"scene": "wavefront"}, None),
    # Disk, Sphere, Cube and Rectangle built-in shapes under an Infinite_sphere light
    "builtins96": (96, 72, 4096, {"scene": "builtins"}, None),
    # the same with the environment seen by the camera only (not a light)
    "builtins96_backdrop": (96, 72, 4096, {"scene": "builtins", "environment_light": False}, None),
    # a 2 m Cube of 32^3 fBm density (mu_t 20 per metre at density 1, albedo 0.9, g 0.6) lit
    # by a Sphere light and the environment, max depth 32
    "volume64": (64, 64, 2048, {"scene": "volume"}, scenes.fbm_density(32)),
    # the volume's grid emitting: seen by the camera only (the cube is not a light) ...
    "volume64_glow": (64, 64, 2048, {"scene": "volume", "medium": GLOW}, scenes.fbm_density(32)),
    # ... and as a light (Volume_image: next-event samples drawn from the emission distribution,
    # MIS against absorption events), with grey and with coloured absorption
    "volume64_glow_light": (64, 64, 2048, {"scene": "volume", "medium": GLOW, "medium_light": True},
                            scenes.fbm_density(32)),
    "volume64_glow_color_light": (64, 64, 2048, {"scene": "volume", "medium": GLOW_COLOR, "medium_light": True},
                                  scenes.fbm_density(32)),
    # a homogeneous emitting cube as a light (Volume: uniform points inside it)
    "volume64_haze_light": (64, 64, 2048, {"scene": "volume", "medium": HAZE, "medium_light": True}, None),
    # an emitting grid with a temperature grid (emission x black-body colour by temperature) as a
    # light; temperatures of 4250-5000 K, where this renderer's black-body colours (from a fit of
    # the CIE observer) agree with the reference's (from its 5 nm table) within 0.5 %
    "volume64_fire_light": (64, 64, 2048, {"scene": "volume", "medium": GLOW, "medium_light": True,
                                           "temperature_seed": 9}, scenes.fbm_density(32)),
    # a two-channel density: the second channel scales the emission (camera and light)
    "volume64_glow2_light": (64, 64, 2048, {"scene": "volume", "medium": GLOW, "medium_light": True,
                                            "emission_scale_seed": 11}, scenes.fbm_density(32)),
    # a colour grid (Grid_color): RGBA voxels, the coefficients from the colour times alpha
    "volume64_color": (64, 64, 2048, {"scene": "volume", "color_grid_seed": 21}, scenes.fbm_density(32)),
    # ... emitting, as a light (a Volume light: uniform points, the absorption at the point)
    "volume64_color_glow_light": (64, 64, 2048, {"scene": "volume", "color_grid_seed": 21, "medium": GLOW,
                                                 "medium_light": True}, scenes.fbm_density(32)),
    # the emitting grid in a Sphere as a light: next-event estimation cannot sample its inside,
    # so its emission counts on every segment
    "volume64_glow_sphere_light": (64, 64, 2048, {"scene": "volume", "medium": GLOW, "medium_light": True,
                                                  "medium_shape": scenes.SHAPE_SPHERE}, scenes.fbm_density(32)),
    # the guiding workload's room (plain MIS): lit only through a doorway by the environment
    "doorway96": (96, 54, 8192, {"scene": "doorway"}, None),
    # a take file (tests/golden/takes/room.take, written for these tests in the reference's take
    # and scene format) loaded by su_load_take: panels of a mesh file rotated by Euler angles,
    # built-in Sphere and Cube props, a Sphere lamp, a look_at camera; the sample count is set
    # after the take
    "take_room96": (96, 72, 4096, {"scene": "take", "take": "room.take"}, None),
    # the Cornell workload at its configured size: 512x512, the 81,920-triangle sphere
    "cornell512": (512, 512, 2048, {"sphere_subdivisions": 6}, None),
    # texture maps: a checker colour map repeated by uv scale 2, a roughness / metallic surface
    # map, a nearest-filtered colour map on a rotated block (byte and float images by id)
    "textured96": (96, 72, 4096, {"scene": "textured"}, None),
    # the guiding workload's room at 320x180 (plain MIS), the image the guided integrator is
    # compared with at a size where its network sees realistic training passes
    "doorway320": (320, 180, 4096, {"scene": "doorway"}, None),
}
# Cases stored as float16 (the large images; the tests' bounds are far above its rounding).
HALF = {"cornell512", "doorway320"}
TAKES = HERE / "takes"
PATH = HERE / "cornell_reference.npz"
# Block size of the block-mean comparison where 8 is too small: many small, bright emitters
# leave the 2048-spp reference image with 4 % noise in single 8x8 blocks (its 1024- and
# 2048-spp images differ by that much), 1.6 % in 16x16 blocks; the dense medium 1.7 % and
# 0.6 %.
BLOCK = {"wavefront96": 16, "volume64": 16, "doorway96": 16, "doorway320": 20, "volume64_glow": 16,
         "volume64_glow_light": 16, "volume64_glow_color_light": 16, "volume64_haze_light": 16,
         "volume64_glow_sphere_light": 16, "volume64_fire_light": 16, "volume64_glow2_light": 16,
         "volume64_color": 16, "volume64_color_glow_light": 16}


def build(su, w, h, spp, kwargs, density=None):
    """Issues a case's scene calls: {"scene": "wavefront"} -> scenes.wavefront,
    {"scene": "builtins", ...} -> scenes.builtin_shapes with the other keys, else
    scenes.cornell with the keyword arguments."""
    kwargs = dict(kwargs)
    name = kwargs.pop("scene", "cornell")
    if name == "wavefront":
        return scenes.wavefront(su, w, h, spp, **kwargs)
    if name == "builtins":
        return scenes.builtin_shapes(su, w, h, spp, **kwargs)
    if name == "volume":
        return scenes.volume(su, w, h, spp, density, **kwargs)
    if name == "doorway":
        return scenes.doorway(su, w, h, spp, **kwargs)
    if name == "textured":
        return scenes.textured_room(su, w, h, spp, **kwargs)
    if name == "take":
        su.su_mount(str(TAKES) + "/")
        su.load_take(str(TAKES / kwargs["take"]), w, h)
        su.su_create_sampler(spp)
        return su.su_create_defaults()
    return scenes.cornell(su, w, h, tonemap=True, spp=spp, density=density, **kwargs)


def main(names):
    out, meta = {}, {"generator": "oracle/_ref/ref_render (reference su_* C API, batch mode)", "cases": {}}
    if names and PATH.exists():
        old = np.load(PATH)
        out = {k: old[k] for k in old.files if k != "meta"}
        meta = json.loads(bytes(old["meta"]).decode())
    for name in names or CASES:
        w, h, spp, kwargs, density = CASES[name]
        img, timing = oracle.reference_render(lambda su: build(su, w, h, spp, kwargs, density), w, h, 0,
                                              progressive=False)
        if timing["status"] != 0:
            raise RuntimeError(f"{name}: reference status {timing['status']}")
        out[name] = img.astype(np.float16 if name in HALF else np.float32)
        if density is not None:
            out[name + "_density"] = density
        meta["cases"][name] = {"width": w, "height": h, "spp": spp, "scene": kwargs,
                               "density": None if density is None else name + "_density",
                               "block": BLOCK.get(name, 8),
                               "render_s": timing["render_s"], "mean": [float(x) for x in img.mean(axis=(0, 1))]}
        print(name, meta["cases"][name], flush=True)
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    np.savez_compressed(PATH, **out)


if __name__ == "__main__":
    main(sys.argv[1:])
