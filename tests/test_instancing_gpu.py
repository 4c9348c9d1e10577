"""Instancing: props that share a mesh kept as instances of one object-space tree under a
top-level tree over the props (two-level traversal: the ray transformed into each instance's
object space, hits transformed back), against the same scenes flattened into one world-space
tree and against the reference renderer's images (tests/golden/cornell_reference.npz, whose
props the reference itself keeps as instances under its prop BVH, prop_bvh_wrapper.cpp).

The two ways of building the scene sample identical paths in expectation but not sample for
sample (the trees differ, so rounding of hit points does), so images are compared with the
statistical bounds of the plain parity test."""

import ctypes
import json
import pathlib

import numpy as np
import pytest

from sprout_b200 import _lib, capi, scenes

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "cornell_reference.npz"


def block_means(img, b):
    h, w, c = img.shape
    return img[: h - h % b, : w - w % b].reshape(h // b, b, w // b, b, c).mean(axis=(1, 3))


def render(build, width, height):
    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        build(su)
        assert su.su_render_frame(0) == 0, su.messages
        assert su.su_postprocess() == 0
        img = su.framebuffer(width, height)[0][:, :, :3].astype(np.float64)
        stats = _lib.RenderStats()
        assert _lib.load().spb_render_last_stats(ctypes.byref(stats)) == 0
        return img, {name: getattr(stats, name) for name, _ in stats._fields_}
    finally:
        su.su_release()


def assert_close(img, ref, block, mean_tol=0.005, block_tol=0.02):
    m_ref, m_img = ref.mean(axis=(0, 1)), img.mean(axis=(0, 1))
    assert np.all(np.abs(m_img - m_ref) <= mean_tol * m_ref), (m_img, m_ref)
    bi, br = block_means(img, block), block_means(ref, block)
    worst = np.max(np.abs(bi - br) / (np.abs(br) + 0.01))
    assert worst < block_tol, f"worst {block}x{block} block deviation {worst:.4f}"


def golden(case):
    data = np.load(GOLDEN)
    meta = json.loads(bytes(data["meta"]).decode())["cases"][case]
    return data[case].astype(np.float64), meta


def test_many_instances_are_kept_as_instances_and_match_the_reference():
    """The 400-instance scene: by default (flattening would hold 2 M triangles for 9,096
    distinct ones) the props stay instances; forced flat, one 2 M-triangle tree.  Both match the
    reference's image."""
    ref, meta = golden("wavefront96")
    w, h, spp = meta["width"], meta["height"], 4 * meta["spp"]
    inst, st_inst = render(lambda su: scenes.wavefront(su, w, h, spp), w, h)
    flat, st_flat = render(lambda su: scenes.wavefront(su, w, h, spp, integrator={"instancing": False}), w, h)
    assert st_inst["instances"] == 402 and st_flat["instances"] == 0  # ground, 400 spheres, emitters
    assert st_inst["device_triangles"] < 20000 < 2_000_000 <= st_flat["device_triangles"]
    assert st_inst["overflow"] == 0 and st_flat["overflow"] == 0
    for img in (inst, flat):
        assert np.all(np.isfinite(img))
        assert_close(img, ref, meta["block"])


@pytest.mark.parametrize("case", ["cornell64_sub3", "cornell64_lights", "cornell64_medium", "cornell64_grid"])
def test_forced_instancing_matches_the_reference(case):
    """Scenes with a few props, forced through the two-level path: an area light and its
    room; 66 emitters through the light tree; a homogeneous medium (boundaries skipped by
    shadow rays, walked for transmittance); a density-grid medium in a rotated, scaled cube."""
    ref, meta = golden(case)
    w, h = meta["width"], meta["height"]
    data = np.load(GOLDEN)
    density = data[meta["density"]] if meta.get("density") else None
    kwargs = dict(meta["scene"])
    img, st = render(lambda su: scenes.cornell(su, w, h, tonemap=True, spp=4 * meta["spp"], density=density,
                                               integrator={"instancing": True}, **kwargs), w, h)
    assert st["instances"] > 0 and st["overflow"] == 0 and st["tracking_capped"] == 0
    assert np.all(np.isfinite(img))
    assert_close(img, ref, meta.get("block", 8))


def test_forced_instancing_volume_matches_the_reference():
    ref, meta = golden("volume64")
    w, h = meta["width"], meta["height"]
    density = np.load(GOLDEN)[meta["density"]]
    img, st = render(lambda su: scenes.volume(su, w, h, 4 * meta["spp"], density, integrator={"instancing": True}),
                     w, h)
    assert st["instances"] > 0 and st["tracking_capped"] == 0
    assert_close(img, ref, meta["block"])
