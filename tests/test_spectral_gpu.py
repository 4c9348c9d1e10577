"""Hero-wavelength spectral mode (the PTMIS "spectral" key; no counterpart in the reference,
which renders RGB): checked against its FP64 CPU restatement (oracle/spectral_oracle.c, an
independent estimator of the same image: one wavelength per path, global-majorant tracking,
its own light choice), against the RGB renderer on a grey scene (where the upsampling basis
reads back exactly), and for the view batch (each view traces the paths it traces alone); also
with the phase guide at medium vertices.

Statistical bounds: image means per channel within 1 %; 4x4-pixel block means within 5 %
(the oracle's own noise at 16,384 samples per pixel is about 2 %); relMSE (mean over pixels and
channels of (x - r)^2 / (r^2 + 1e-2)) below 1e-3.
"""

import ctypes
import math

import numpy as np
import pytest

import oracle
from sprout_b200 import _lib, capi, scenes

pytestmark = pytest.mark.gpu

W, H = 32, 24


def blocks(img, b):
    h, w, c = img.shape
    return img[: h - h % b, : w - w % b].reshape(h // b, b, w // b, b, c).mean(axis=(1, 3))


def rel_mse(x, r):
    return float(np.mean((x - r) ** 2 / (r * r + 1e-2)))


def render(spp, **scene):
    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        _, desc = scenes.spectral_box(su, W, H, spp, scenes.fbm_density(12), **scene)
        assert su.su_render_frame(0) == 0, su.messages
        assert su.su_postprocess() == 0
        img, status = su.framebuffer(W, H)
        assert status == 0
        st = _lib.RenderStats()
        assert _lib.load().spb_render_last_stats(ctypes.byref(st)) == 0
        assert st.overflow == 0 and st.tracking_capped == 0
        return img[:, :, :3].copy(), desc
    finally:
        su.su_release()


def assert_close(img, ref):
    assert np.all(np.isfinite(img))
    m_img, m_ref = img.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
    assert np.all(np.abs(m_img - m_ref) <= 0.01 * m_ref), (m_img, m_ref)
    dev = np.abs(blocks(img, 4) - blocks(ref, 4)) / (np.abs(blocks(ref, 4)) + 0.01)
    assert dev.max() < 0.05, dev.max()
    assert rel_mse(img, ref) < 1e-3


def test_spectral_mode_matches_its_oracle():
    """A chromatic density-grid medium, a coloured sphere light and a blue environment."""
    img, desc = render(16384)
    ref = oracle.spectral_render(desc, 16384)
    assert_close(img, ref)


def test_phase_guided_spectral_mode_matches_its_oracle():
    """The same scene with the phase guide (PTMIS "guiding" in spectral mode): the first 16 spp
    train it, the rest draw continuations from its lobes or the phase function (one-sample MIS),
    so the image still matches the oracle's."""
    img, desc = render(16384, integrator={"guiding": True})
    ref = oracle.spectral_render(desc, 16384)
    assert_close(img, ref)


def test_grey_scene_renders_as_in_rgb_mode():
    """With grey colours every upsampled spectrum is flat and reads back as its RGB value, so
    the spectral and the RGB renderer estimate the same image."""
    grey = {"medium": {"attenuation_color": [0.6, 0.6, 0.6], "attenuation_distance": 0.5,
                       "subsurface_color": [0.7, 0.7, 0.7], "anisotropy": 0.4},
            "emission": [25.0, 25.0, 25.0], "environment": [0.3, 0.3, 0.3]}
    spectral, _ = render(16384, **grey)
    rgb, _ = render(16384, integrator={"spectral": False}, **grey)
    assert_close(spectral, rgb)


def test_spectral_views_render_together_as_alone():
    """Spectral mode through spb_render_views: two views in one launch; each view's samples use
    its own pixel streams, so it matches its single-view render up to the order of the film's
    atomic sums."""
    views = [(W, H, math.radians(45.0), scenes._look_at((2.6, 1.6, -3.0))),
             (20, 20, math.radians(45.0), scenes._look_at((-2.4, 1.0, -3.1)))]
    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        cam, _ = scenes.spectral_box(su, W, H, 256, scenes.fbm_density(12))
        assert su.su_render_frame(0) == 0, su.messages
        batch = su.render_views(views, 256)
        alone = []
        for w, h, _, m in views:
            assert su.su_camera_set_resolution(w, h) == 0
            su.set_transformation(cam, m)
            assert su.su_render_frame(0) == 0, su.messages
            assert su.su_postprocess() == 0
            alone.append(su.framebuffer(w, h)[0].copy())
    finally:
        su.su_release()
    for b, a in zip(batch, alone):
        assert a[:, :, :3].mean() > 0.1
        np.testing.assert_allclose(b[:, :, :3], a[:, :, :3], rtol=1e-4, atol=1e-5)
