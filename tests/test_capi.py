"""The C ABI: every symbol declared in include/*.h is exported, and argument errors are
reported with the documented codes without touching a GPU."""

import ctypes
import pathlib
import re
import subprocess

import numpy as np

import sprout_b200 as sb
from sprout_b200 import _lib

INCLUDE = pathlib.Path(__file__).resolve().parent.parent / "include"


def declared_symbols():
    names = set()
    for header in INCLUDE.glob("*.h"):
        text = header.read_text()
        names |= set(re.findall(r"SPB_API\s+[\w\s\*]+?\b(spb_\w+)\s*\(", text))
        names |= set(re.findall(r"SU_LIBRARY_API\s+[\w\s\*]+?\b(su_\w+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"spb_tree_create", "spb_tree_build", "spb_intersect_device", "spb_intersect_p_device",
            "spb_intersect_host", "spb_intersect_p_host"} <= names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIBRARY_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = declared_symbols() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    for name in declared_symbols():
        assert hasattr(lib, name)
    # the ctypes prototypes cover both headers
    from sprout_b200 import capi

    assert {n for n in declared_symbols() if n.startswith("spb_")} <= set(_lib.PROTOTYPES)
    assert {n for n in declared_symbols() if n.startswith("su_")} == set(capi.PROTOTYPES)


def test_c_api_has_the_reference_entry_points():
    """include/sprout.h declares the reference's 35 su_* functions (source/capi/sprout.h:39-122)."""
    names = {n for n in declared_symbols() if n.startswith("su_")}
    assert len(names) == 35


def test_c_api_without_gpu_state():
    """Engine lifecycle calls that need no device work return the reference's codes."""
    from sprout_b200 import capi

    su = capi.SuLibrary()
    assert su.su_render() == -1 and su.su_release() == 0
    assert su.su_init(False) == 0
    assert su.su_init(False) == -1
    assert su.su_create_material(b'{"rendering": {"Substitute": {"color": [1, 0, 0]}}}') == 0
    assert su.su_create_material(b'{"rendering": {"Glass": {}}}') == capi.SU_RESOURCE_NULL
    assert su.su_render_iteration() == -2
    assert su.su_create_light(5) == -2
    assert su.su_release() == 0


def test_density_images_and_grid_materials():
    """su_create_image ids count from 0; a Volumetric "density" must name a one-channel image;
    "emission" is taken by homogeneous media and by density grids (Grid_emission), a
    "temperature" image of the density's dimensions beside a density grid, a two-channel
    density (density, emission scale), and a four-channel byte "color" image without a density
    (a colour grid; a float one leaves the medium homogeneous, as in the reference)."""
    import json

    import numpy as np

    from sprout_b200 import capi

    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        grid = np.linspace(0, 1, 4 * 3 * 2, dtype=np.float32).reshape(2, 3, 4)
        assert su.image(grid) == 0
        rgb = np.zeros((2, 2, 3), np.uint8)
        assert su.su_create_image(0, 3, 2, 2, 1, 0, 3, rgb.ctypes.data) == 1
        assert su.su_create_image(1, 1, 2, 2, 1, 0, 2, rgb.ctypes.data) == capi.SU_RESOURCE_NULL

        def volumetric(**p):
            return su.su_create_material(json.dumps({"rendering": {"Volumetric": p}}).encode())

        assert volumetric(density={"id": 0}, attenuation_distance=0.1) == 0
        assert volumetric(density={"id": 0}, sampler={"filter": "Nearest", "address": "Repeat"}) == 1
        assert volumetric(density={"id": 1}) == capi.SU_RESOURCE_NULL  # three channels
        assert volumetric(density={"id": 7}) == capi.SU_RESOURCE_NULL  # no such image
        assert volumetric(density={"file": "smoke.sub"}) == capi.SU_RESOURCE_NULL
        assert volumetric(density={"id": 0}, emission=[1, 1, 1]) == 2  # an emitting grid
        assert volumetric(emission=[1, 0.5, 0.2], attenuation_distance=0.2) == 3  # homogeneous
        assert volumetric(density={"id": 0}, temperature={"id": 0}, emission=[1, 1, 1]) == 4
        other = np.ones((3, 3, 4), np.float32)
        assert su.image(other) == 2
        assert volumetric(density={"id": 0}, temperature={"id": 2}) == capi.SU_RESOURCE_NULL  # other size
        assert volumetric(temperature={"id": 0}) == capi.SU_RESOURCE_NULL  # no density
        two = np.ones((2, 3, 4, 2), np.float32)  # density and emission scale
        assert su.image(two) == 3
        assert volumetric(density={"id": 3}, emission=[1, 1, 1]) == 5
        rgba = np.full((2, 3, 4, 4), 128, np.uint8)  # a colour grid (Grid_color): sRGB bytes and alpha
        assert su.image(rgba) == 4
        assert volumetric(color={"id": 4}, attenuation_distance=0.1) == 6
        assert volumetric(color={"id": 3}) == capi.SU_RESOURCE_NULL  # two channels
        assert volumetric(color={"id": 4}, density={"id": 0}) == 7  # the density wins, as in the reference
        floats = np.full((2, 3, 4, 4), 0.5, np.float32)  # not a colour texture in the reference
        assert su.image(floats) == 5
        assert volumetric(color={"id": 5}) == 8  # homogeneous, with a warning
    finally:
        assert su.su_release() == 0


def test_materials_and_meshes_from_files(tmp_path):
    """su_create_material_from_file reads a material JSON file and su_create_triangle_mesh_from_file
    a mesh JSON file, both found under the mounted folders; unreadable files give
    SU_RESOURCE_NULL."""
    import json

    from sprout_b200 import capi

    (tmp_path / "red.json").write_text(json.dumps({"rendering": {"Substitute": {"color": [1, 0, 0]}}}))
    (tmp_path / "quad.json").write_text(json.dumps({"geometry": {
        "parts": [{"start_index": 0, "num_indices": 6, "material_index": 0}],
        "vertices": {"positions": [0, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 0], "normals": [0, 0, 1] * 4},
        "indices": [0, 1, 2, 0, 2, 3]}}))
    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        assert su.su_create_material_from_file(b"red.json") == capi.SU_RESOURCE_NULL  # not mounted yet
        assert su.su_mount(str(tmp_path).encode()) == 0
        assert su.su_create_material_from_file(b"red.json") == 0
        mesh = su.su_create_triangle_mesh_from_file(b"quad.json")
        assert mesh != capi.SU_RESOURCE_NULL
        assert su.su_create_prop(mesh, 1, (ctypes.c_uint32 * 1)(0)) != capi.SU_RESOURCE_NULL
        assert su.su_create_triangle_mesh_from_file(b"missing.json") == capi.SU_RESOURCE_NULL
        assert su.su_create_material_from_file(b"missing.json") == capi.SU_RESOURCE_NULL
    finally:
        assert su.su_release() == 0


def test_ggx_albedo_table_matches_reference_table():
    """The energy-compensation table computed by this project against the reference's
    generated table (material/ggx/ggx_integral.inl), kept as a fixture made by
    tests/golden/make_ggx_golden.py."""
    import pathlib

    ref = np.load(pathlib.Path(__file__).resolve().parent / "golden" / "ggx_integral_reference.npz")["E"].reshape(1024)
    mine = np.zeros(1024, np.float32)
    assert _lib.load().spb_ggx_albedo_table(mine.ctypes.data) == 0
    assert np.max(np.abs(mine - ref)) < 5e-5


def test_argument_errors_use_documented_codes():
    lib = _lib.load()
    assert lib.spb_tree_create(None) == _lib.SPB_ERROR_ARGUMENT
    assert b"null" in lib.spb_last_error()
    assert lib.spb_tree_build(None, 3, 1, None, None, 0) == _lib.SPB_ERROR_ARGUMENT
    assert lib.spb_intersect_device(None, None, 0, None, None, None, None) == _lib.SPB_ERROR_ARGUMENT
    assert lib.spb_intersect_p_host(None, None, 0, None) == _lib.SPB_ERROR_ARGUMENT
    assert lib.spb_tree_release(None) == _lib.SPB_ERROR_ARGUMENT
    nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
    assert lib.spb_synth_sphere_mesh(0, 0.1, 1, ctypes.byref(nv), ctypes.byref(nt), None, None) == \
        _lib.SPB_ERROR_ARGUMENT


def test_no_silent_cpu_fallback_without_gpu():
    """Creating a tree needs CUDA; without a usable GPU the call fails loudly."""
    import torch

    if torch.cuda.is_available():
        return
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.spb_tree_create(ctypes.byref(h)) == _lib.SPB_ERROR_CUDA
    try:
        sb.Tree()
    except sb.SproutError as e:
        assert e.code == _lib.SPB_ERROR_CUDA
    else:
        raise AssertionError("Tree() must fail without a GPU")


def test_synthetic_mesh_is_closed_and_deterministic():
    pos, idx = sb.sphere_mesh(16, 0.1, 1)
    assert idx.shape == (4 * 16 * 16, 3) and pos.shape == (2 * 16 * 16 + 2, 3)
    pos2, idx2 = sb.sphere_mesh(16, 0.1, 1)
    assert np.array_equal(pos, pos2) and np.array_equal(idx, idx2)
    edges = np.sort(np.concatenate([idx[:, [0, 1]], idx[:, [1, 2]], idx[:, [2, 0]]]), axis=1)
    _, counts = np.unique(edges, axis=0, return_counts=True)
    assert (counts == 2).all()  # every edge shared by exactly two triangles
    valence = np.bincount(idx.ravel(), minlength=len(pos))
    assert valence.max() <= 6
    r = np.linalg.norm(pos, axis=1)
    assert 0.85 < r.min() and r.max() < 1.15


def test_synthetic_rays():
    rays = sb.random_rays(100000, seed=1)
    assert np.all(np.abs(rays[:, :3]) <= 2.0)
    assert np.allclose(np.linalg.norm(rays[:, 4:7], axis=1), 1.0, atol=1e-6)
    assert np.all(rays[:, 3] == 0) and np.all(rays[:, 7] == np.float32(3.4027715434167032e38))
    # the stream of ray i does not depend on the batch it is generated in
    part = sb.random_rays(100, seed=1, first=500)
    assert np.array_equal(part, rays[500:600])
    # directions are isotropic: mean close to zero
    assert np.abs(rays[:, 4:7].mean(axis=0)).max() < 0.01


def test_builtin_shapes_accepted():
    """Cube, Disk, Infinite_sphere, Rectangle and Sphere props are created by shape id; Canopy,
    Distant_sphere and Plane are not supported and return SU_RESOURCE_NULL."""
    import numpy as np

    from sprout_b200 import capi

    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        mat = su.su_create_material(b'{"rendering": {"Light": {"emission": [1, 1, 1]}}}')
        ids = np.array([mat], np.uint32)
        for shape in (1, 2, 4, 6, 7):
            assert su.su_create_prop(shape, 1, ids.ctypes.data) != capi.SU_RESOURCE_NULL, shape
        for shape in (0, 3, 5):
            assert su.su_create_prop(shape, 1, ids.ctypes.data) == capi.SU_RESOURCE_NULL, shape
    finally:
        assert su.su_release() == 0


def test_take_files_load(tmp_path):
    """su_load_take reads a take and its scene (tests/golden/takes: a take written in the
    reference's format) on the host, resolving names through su_mount folders; unreadable
    files, unknown material names and bad transformations give -2."""
    import json

    from sprout_b200 import capi

    takes = pathlib.Path(__file__).resolve().parent / "golden" / "takes"
    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        assert su.su_load_take(b"room.take") == -2  # not found before the folder is mounted
        assert su.su_mount((str(takes) + "/").encode()) == 0
        assert su.su_load_take(b"room.take") == 0
        assert su.su_load_take(b"missing.take") == -2
        assert su.su_load_take(b'{"scene": "missing.scene"}') == -2
        assert su.su_load_take(b"{not json") == -2
        scene = json.loads((takes / "room.scene").read_text())
        scene["entities"][0]["materials"] = ["no_such_material"]
        (tmp_path / "bad.scene").write_text(json.dumps(scene))
        assert su.su_load_take(json.dumps({"scene": str(tmp_path / "bad.scene")}).encode()) == -2
        scene = json.loads((takes / "room.scene").read_text())
        scene["entities"][0]["transformation"] = [1, 0, 0]
        (tmp_path / "bad_trafo.scene").write_text(json.dumps(scene))
        assert su.su_load_take(json.dumps({"scene": str(tmp_path / "bad_trafo.scene")}).encode()) == -2
    finally:
        assert su.su_release() == 0


def test_density_from_sub_files(tmp_path):
    """A Volumetric material's "density": {"file": ...} reads the reference's SUB format
    (dense or sparse, Float1 or Byte1; sprout_b200.sub.write_sub), resolved under su_mount
    folders; missing, foreign or truncated files give SU_RESOURCE_NULL."""
    import json

    from sprout_b200 import capi, scenes
    from sprout_b200.sub import write_sub

    dens = scenes.density_grid(8, 6, 5)
    for name, kw in {"dense.sub": {}, "sparse.sub": {"sparse": True}, "bytes.sub": {"byte": True},
                     "sparse_bytes.sub": {"byte": True, "sparse": True}}.items():
        write_sub(tmp_path / name, dens, **kw)
    (tmp_path / "truncated.sub").write_bytes((tmp_path / "dense.sub").read_bytes()[:-7])
    (tmp_path / "foreign.sub").write_bytes(b"PNG\0" + b"\0" * 64)

    su = capi.SuLibrary()
    assert su.su_init(False) == 0
    try:
        def volumetric(file):
            return su.su_create_material(json.dumps({"rendering": {"Volumetric": {"density": {"file": file}}}}).encode())

        assert volumetric(str(tmp_path / "dense.sub")) != capi.SU_RESOURCE_NULL
        assert volumetric("sparse.sub") == capi.SU_RESOURCE_NULL  # not mounted yet
        assert su.su_mount(str(tmp_path).encode()) == 0
        for name in ("sparse.sub", "bytes.sub", "sparse_bytes.sub"):
            assert volumetric(name) != capi.SU_RESOURCE_NULL, name
        for name in ("missing.sub", "truncated.sub", "foreign.sub"):
            assert volumetric(name) == capi.SU_RESOURCE_NULL, name
    finally:
        assert su.su_release() == 0
