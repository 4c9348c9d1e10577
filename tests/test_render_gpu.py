"""Path-tracer parity: the B200 wavefront renderer, driven through the su_* C API, against
the reference renderer's converged images of the same scene (tests/golden/cornell_reference.npz,
made by the reference's own C API).

Monte Carlo images agree only in expectation, so the checks are statistical: the image means
per channel within 0.5%, 8x8-pixel block means within 2% (16x16 for the many-emitter scene,
whose reference image is noisier; plus a small absolute floor), and
the relative MSE of the whole image (mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2))
below a bound that the reference's own noise at its sample count dominates.  One case replaces
the metal sphere by a homogeneous scattering medium (Volumetric material: delta tracking,
Henyey-Greenstein phase function, transmittance along shadow rays).
"""

import ctypes
import json
import pathlib

import numpy as np
import pytest

from sprout_b200 import _lib, capi, scenes

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "cornell_reference.npz"


def rel_mse(x, r):
    return float(np.mean((x - r) ** 2 / (r * r + 1e-2)))


def block_means(img, b):
    h, w, c = img.shape
    return img[: h - h % b, : w - w % b].reshape(h // b, b, w // b, b, c).mean(axis=(1, 3))


def render(width, height, spp, progressive=False, iterations=0, stats=None, **scene):
    """Renders a scene through the su_* API; stats (a dict) receives the render's counters."""
    su = capi.SuLibrary()
    assert su.su_init(progressive) == 0
    try:
        scene = dict(scene)
        name = scene.pop("scene", "cornell")
        density = scene.pop("density", None)  # Cornell cases only
        if name == "wavefront":
            scenes.wavefront(su, width, height, spp, **scene)
        elif name == "builtins":
            scenes.builtin_shapes(su, width, height, spp, **scene)
        elif name == "volume":
            scenes.volume(su, width, height, spp, density, **scene)
        elif name == "doorway":
            scenes.doorway(su, width, height, spp, **scene)
        elif name == "textured":
            scenes.textured_room(su, width, height, spp, **scene)
        elif name == "take":
            takes = GOLDEN.parent / "takes"
            assert su.su_mount((str(takes) + "/").encode()) == 0
            assert su.su_load_take(str(takes / scene["take"]).encode()) == 0, su.messages
            assert su.su_create_sampler(spp) == 0
            assert su.su_create_defaults() == 0
        else:
            scenes.cornell(su, width, height, tonemap=True, spp=spp, density=density, **scene)
        if progressive:
            assert su.su_start_render_frame(0) == 0, su.messages
            for _ in range(iterations):
                assert su.su_render_iteration() == 0, su.messages
        else:
            assert su.su_render_frame(0) == 0, su.messages
        assert su.su_postprocess() == 0
        img, status = su.framebuffer(width, height)
        assert status == 0
        if stats is not None:
            st = _lib.RenderStats()
            assert _lib.load().spb_render_last_stats(ctypes.byref(st)) == 0
            stats.update({f: getattr(st, f) for f, _ in st._fields_})
        return img[:, :, :3].copy()
    finally:
        su.su_release()


CASES = ["cornell64_sub3", "cornell128_sub6", "cornell64_medium", "cornell64_emissive", "cornell64_thin_direct",
         "cornell64_grid",
         "cornell64_lights", "wavefront96", "builtins96", "builtins96_backdrop", "volume64",
         "doorway96", "take_room96", "cornell512", "doorway320", "textured96",
         "volume64_glow", "volume64_glow_light", "volume64_glow_color_light", "volume64_haze_light",
         "volume64_glow_sphere_light", "volume64_fire_light", "volume64_glow2_light", "volume64_color",
         "volume64_color_glow_light"]


@pytest.mark.parametrize("name", CASES)
def test_converged_image_matches_reference(name):
    data = np.load(GOLDEN)
    meta = json.loads(bytes(data["meta"]).decode())["cases"][name]
    ref = data[name].astype(np.float32)
    density = data[meta["density"]] if meta.get("density") else None
    img = render(meta["width"], meta["height"], 4 * meta["spp"], density=density, **meta["scene"])
    assert np.all(np.isfinite(img))
    m_ref = ref.mean(axis=(0, 1))
    m_img = img.mean(axis=(0, 1))
    assert np.all(np.abs(m_img - m_ref) <= 0.005 * m_ref), (m_img, m_ref)
    b = meta.get("block", 8)  # larger where the reference image is noisier (see the generator)
    bi, br = block_means(img, b), block_means(ref, b)
    worst = np.max(np.abs(bi - br) / (np.abs(br) + 0.01))
    assert worst < 0.02, f"worst {b}x{b} block deviation {worst:.4f}"
    assert rel_mse(img, ref) < 2e-3


@pytest.mark.parametrize("name", ["cornell64_lights", "wavefront96", "builtins96"])
def test_split_light_selection_matches_reference(name):
    """Split light selection (Adaptive light sampling, Tree::random_light with splitting) with a
    splitting threshold of 1, so that every light-tree node the walk passes above the split
    depth is split: at each of the first three vertices the environment and up to 64 emitters
    get a shadow ray each, where single selection sends one.  The estimator stays unbiased, so
    the image matches the reference's converged image (rendered with its default selection) as
    closely as the default does, while casting more shadow rays per sample."""
    data = np.load(GOLDEN)
    meta = json.loads(bytes(data["meta"]).decode())["cases"][name]
    ref = data[name].astype(np.float32)
    w, h, spp = meta["width"], meta["height"], 4 * meta["spp"]
    counts = {}
    images = {}
    for mode in ("Single", "split"):
        ls = {"strategy": "Single"} if mode == "Single" else {"strategy": "Adaptive", "splitting_threshold": 1.0}
        scene = dict(meta["scene"])
        scene["integrator"] = dict(scene.get("integrator") or {}, light_sampling=ls)
        st = {}
        images[mode] = render(w, h, spp if mode == "split" else meta["spp"], stats=st, **scene)
        counts[mode] = st["shadow_rays"] / st["paths"]
        assert st["overflow"] == 0
    img = images["split"]
    assert np.all(np.isfinite(img))
    m_ref = ref.mean(axis=(0, 1))
    m_img = img.mean(axis=(0, 1))
    assert np.all(np.abs(m_img - m_ref) <= 0.005 * m_ref), (m_img, m_ref)
    b = meta.get("block", 8)
    worst = np.max(np.abs(block_means(img, b) - block_means(ref, b)) / (np.abs(block_means(ref, b)) + 0.01))
    assert worst < 0.02, f"worst {b}x{b} block deviation {worst:.4f}"
    assert rel_mse(img, ref) < 2e-3
    assert counts["split"] > 1.2 * counts["Single"], counts


def test_progressive_iterations_converge_to_batch():
    """su_start_render_frame + su_render_iteration accumulate one sample per pixel per call."""
    a = render(32, 32, 1, progressive=True, iterations=256, sphere_subdivisions=2)
    b = render(32, 32, 1024, sphere_subdivisions=2)
    assert abs(a.mean() - b.mean()) < 0.02 * b.mean()


def test_api_errors_and_lifecycle():
    su = capi.SuLibrary()
    assert su.su_init(True) == 0
    try:
        assert su.su_init(True) == -1          # one engine only
        assert su.su_render_iteration() == -2  # nothing to render yet
        assert su.su_create_prop(3, 0, None) == capi.SU_RESOURCE_NULL  # Distant_sphere is not supported
        assert su.su_create_material(b"{not json") == capi.SU_RESOURCE_NULL
        assert su.su_load_take(b"x.take") == -2
    finally:
        assert su.su_release() == 0
    assert su.su_render() == -1  # no engine


def test_graph_replay_matches_direct_launches():
    """Waves replayed from a captured CUDA graph (small, recurring wave shapes) give the image
    that launching every kernel directly gives, bit for bit."""
    import ctypes

    from sprout_b200 import _lib

    lib = _lib.load()
    shape = {"wave_paths": 1 << 16, "trace_blocks_per_sm": 4}
    images, graph_waves = [], []
    for graphs in (True, False):
        su = capi.SuLibrary()
        assert su.su_init(False) == 0
        try:
            scenes.doorway(su, 96, 54, 64, integrator=dict(shape, cuda_graphs=graphs))
            assert su.su_render_frame(0) == 0, su.messages
            assert su.su_postprocess() == 0
            images.append(su.framebuffer(96, 54)[0][:, :, :3].copy())
            stats = _lib.RenderStats()
            assert lib.spb_render_last_stats(ctypes.byref(stats)) == 0
            graph_waves.append(stats.graph_waves)
        finally:
            su.su_release()
    assert graph_waves[0] > 0 and graph_waves[1] == 0
    assert np.array_equal(images[0], images[1])


def test_density_file_renders_like_the_image(tmp_path):
    """The density grid read from a SUB file (dense, and sparse behind a topology) renders the
    image the same grid given as an in-memory image renders, bit for bit."""
    from sprout_b200.sub import write_sub

    dens = scenes.density_grid()
    write_sub(tmp_path / "dense.sub", dens)
    write_sub(tmp_path / "sparse.sub", dens, sparse=True)
    medium = {"color": [0.9, 0.6, 0.4], "attenuation_distance": 0.03, "anisotropy": 0.3}
    kw = {"sphere_subdivisions": 2, "medium": medium}
    ref = render(48, 48, 64, density=dens, **kw)
    for name in ("dense.sub", "sparse.sub"):
        img = render(48, 48, 64, density=str(tmp_path / name), **kw)
        assert np.array_equal(img, ref), name


def test_render_exports_png(tmp_path, monkeypatch):
    """su_render renders frame 0 and exports it as the reference's default exporter does:
    output_000000.png, the 8-bit sRGB framebuffer."""
    from PIL import Image

    monkeypatch.chdir(tmp_path)
    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        scenes.cornell(su, 40, 30, sphere_subdivisions=2, tonemap=True, spp=16)
        assert su.su_render() == 0, su.messages
        rgb = np.zeros((30, 40, 3), np.uint8)
        assert su.su_copy_framebuffer(capi.SU_UINT8, 40, 30, 3, rgb.ctypes.data) == 0
        assert su.su_export_frame(3) == 0
    finally:
        su.su_release()
    png = np.asarray(Image.open(tmp_path / "output_000000.png"))
    assert png.shape == (30, 40, 3) and np.array_equal(png, rgb)
    assert np.array_equal(np.asarray(Image.open(tmp_path / "output_000003.png")), rgb)


def test_camera_move_renders_like_a_fresh_scene():
    """Moving the camera and changing the resolution between frames re-applies the camera
    without rebuilding the scene; the frame equals the one a freshly built scene with that
    camera renders, bit for bit."""
    def fresh(w, h, position):
        su = capi.SuLibrary()
        assert su.su_init(False) == 0
        try:
            cam = scenes.cornell(su, w, h, sphere_subdivisions=2, tonemap=True, spp=16)
            su.set_transformation(cam, scenes.translation(*position))
            assert su.su_render_frame(0) == 0
            assert su.su_postprocess() == 0
            return su.framebuffer(w, h)[0][:, :, :3].copy()
        finally:
            su.su_release()

    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        cam = scenes.cornell(su, 48, 40, sphere_subdivisions=2, tonemap=True, spp=16)
        assert su.su_render_frame(0) == 0
        assert su.su_camera_set_resolution(40, 32) == 0
        su.set_transformation(cam, scenes.translation(0.2, 1.1, -3.0))
        assert su.su_render_frame(0) == 0
        assert su.su_postprocess() == 0
        moved = su.framebuffer(40, 32)[0][:, :, :3].copy()
    finally:
        su.su_release()
    assert np.array_equal(moved, fresh(40, 32, (0.2, 1.1, -3.0)))


def test_golden_ratio_sampling_lowers_the_error():
    """Batch frames sample the camera and the first three vertices of each path from per-pixel
    golden ratio sequences, as the reference's batch mode does (sampler_golden_ratio.cpp); a
    progressive frame samples independently at random.  Both are unbiased (the parity cases
    above render in batch mode); at 16 spp, summed over three seeds, the batch image's relMSE
    against the reference's converged image is below 0.9 of the progressive image's."""
    data = np.load(GOLDEN)
    ref = data["cornell64_sub3"].astype(np.float32)
    e_batch = e_random = 0.0
    for seed in (1, 2, 3):
        batch = render(64, 64, 16, sphere_subdivisions=3, integrator={"seed": seed})
        random = render(64, 64, 1, progressive=True, iterations=16, sphere_subdivisions=3,
                        integrator={"seed": seed})
        e_batch += rel_mse(batch, ref)
        e_random += rel_mse(random, ref)
    assert e_batch < 0.9 * e_random, (e_batch, e_random)


def test_take_postprocessors_and_exporters(tmp_path, monkeypatch):
    """A take's "post" pipeline and "export" writers (take_loader.cpp:817-951): frames rendered
    with the Linear tonemapper and with ACES differ exactly by the tonemappers' curves (checked
    here per pixel from the Linear frame, which is AP1 -> sRGB of the film), and the EXR and RGBE
    exporters write output_000000.exr / .hdr holding the postprocessed frame."""
    import json

    takes = GOLDEN.parent / "takes"
    base = json.loads((takes / "room.take").read_text())
    base["sampler"] = {"Random": {"samples_per_pixel": 16}}

    def frame(post=None, export=None):
        take = dict(base)
        if post is not None:
            take["post"] = post
        if export is not None:
            take["export"] = export
        path = tmp_path / "t.take"
        path.write_text(json.dumps(take))
        su = capi.SuLibrary()
        assert su.su_init(False) == 0
        try:
            assert su.su_mount((str(takes) + "/").encode()) == 0
            assert su.su_load_take(str(path).encode()) == 0, su.messages
            assert su.su_render() == 0, su.messages
            img, _ = su.framebuffer(96, 72)
            return img[:, :, :3].astype(np.float64)
        finally:
            su.su_release()

    monkeypatch.chdir(tmp_path)
    linear = frame()
    aces = frame(post=[{"tonemapper": {"ACES": {"exposure": 0.5}}}],
                 export={"Image": {"format": "EXR"}})
    assert (tmp_path / "output_000000.exr").exists()
    # ACES of 2^0.5 * film, from the Linear frame (linear sRGB = AP1_to_sRGB(film))
    to_ap1 = np.linalg.inv(np.array([[1.70505155, -0.62179068, -0.08325840],
                                     [-0.13025714, 1.14080289, -0.01054853],
                                     [-0.02400328, -0.12896877, 1.15297171]]))
    film = linear @ to_ap1.T * 2 ** 0.5
    rrt = film @ np.array([[0.970889, 0.026963, 0.002148], [0.010889, 0.986963, 0.002148],
                           [0.010889, 0.026963, 0.962148]]).T
    odt = (rrt * (rrt + 0.0245786) - 0.000090537) / (rrt * (0.983729 * rrt + 0.4329510) + 0.238081)
    want = odt @ np.array([[1.60475, -0.53108, -0.07367], [-0.10208, 1.10813, -0.00605],
                           [-0.00327, -0.07276, 1.07602]]).T
    assert np.allclose(aces, want, rtol=1e-3, atol=1e-5)
    frame(export={"Image": {"format": "RGBE"}})
    assert (tmp_path / "output_000000.hdr").read_bytes().startswith(b"#?RADIANCE")


def test_views_render_together_as_alone():
    """spb_render_views: three views of different sizes and positions rendered in one call.  A
    view's sample streams depend on its own pixels only, so each traces the paths it traces when
    rendered alone through su_render_frame; only the order in which the film sums the samples
    differs (the waves group them differently), so the images agree to float rounding."""
    import math

    views = [(64, 48, scenes.translation(0.0, 1.0, -3.4)),
             (40, 40, scenes.translation(0.3, 0.9, -3.0)),
             (96, 24, scenes.translation(-0.2, 1.2, -3.6))]
    fov = math.radians(40.0)
    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        cam = scenes.cornell(su, 64, 48, sphere_subdivisions=3, spp=16)
        assert su.su_render_frame(0) == 0, su.messages  # uploads the scene
        batch = su.render_views([(w, h, fov, m) for w, h, m in views], 16)
        st = _lib.RenderStats()
        assert _lib.load().spb_render_last_stats(ctypes.byref(st)) == 0
        assert st.paths == 16 * sum((w + 2) * (h + 2) for w, h, _ in views)
        alone = []
        for w, h, m in views:
            assert su.su_camera_set_resolution(w, h) == 0
            su.set_transformation(cam, m)
            assert su.su_render_frame(0) == 0, su.messages
            assert su.su_postprocess() == 0
            img, status = su.framebuffer(w, h)
            assert status == 0
            alone.append(img.copy())
    finally:
        su.su_release()
    for (w, h, _), b, a in zip(views, batch, alone):
        assert b.shape == (h, w, 4) and np.all(np.isfinite(b))
        assert a[:, :, :3].mean() > 0.05
        np.testing.assert_allclose(b[:, :, :3], a[:, :, :3], rtol=1e-4, atol=1e-6)
