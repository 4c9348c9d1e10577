"""Checkers for the sprout_b200 ray cast.  TEST INFRASTRUCTURE ONLY.

* :func:`restated_cast` -- the C restatement in ``cast_oracle.c`` (libcast_oracle.so).
* :func:`reference_cast` -- the reference's own Builder_SAH + Tree::intersect/intersect_p,
  compiled from the reference sources into ``_ref/ref_cast`` by ``Makefile``.
* :func:`synth_sphere_mesh`, :func:`synth_rays` -- the cast benchmark's inputs, restated in C
  (``synth_oracle.c``), so the reference can be timed without loading the product library.
* :func:`classify_mismatches` -- sorts closest-hit disagreements into rounding-level
  edge/tie cases and unexplained ones.

Only tests, the smoke check and the bench's CPU-baseline leg use this package.
"""

from __future__ import annotations

import ctypes
import json
import os
import pathlib
import subprocess
import tempfile

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ORACLE_LIB = HERE / "libcast_oracle.so"
REF_CAST = HERE / "_ref" / "ref_cast"

MODE_CLOSEST = 1
MODE_ANY = 2
MODE_BRUTE = 4

_lib = None


def _load():
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            raise ImportError(f"{ORACLE_LIB} missing: run sprout_b200.build.build_oracle()")
        lib = ctypes.CDLL(str(ORACLE_LIB))
        lib.oracle_cast.restype = ctypes.c_int32
        lib.oracle_cast.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int32]
        lib.oracle_triangle_test.restype = ctypes.c_int32
        lib.oracle_triangle_test.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_float, ctypes.c_void_p]
        lib.oracle_synth_sphere_mesh.restype = ctypes.c_int32
        lib.oracle_synth_sphere_mesh.argtypes = [ctypes.c_uint32, ctypes.c_float, ctypes.c_uint32,
                                                 ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_synth_rays.restype = ctypes.c_int32
        lib.oracle_synth_rays.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_float,
                                          ctypes.c_void_p, ctypes.c_uint32]
        lib.oracle_spectral_render.restype = ctypes.c_int32
        lib.oracle_spectral_render.argtypes = (
            [ctypes.c_uint32] + [ctypes.c_void_p] * 4 + [ctypes.c_uint32] * 3 + [ctypes.c_void_p] * 3 +
            [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p] +
            [ctypes.c_uint32] * 3 + [ctypes.c_uint64] + [ctypes.c_void_p] * 4)
        _lib = lib
    return _lib


def triangle_test(ray, a, b, c, tmax=None):
    """One restated Möller-Trumbore test: (passes, t, u, v)."""
    lib = _load()
    r = np.ascontiguousarray(ray, np.float32).reshape(8)
    pa, pb, pc = (np.ascontiguousarray(x, np.float32).reshape(3) for x in (a, b, c))
    out = np.zeros(3, np.float32)
    tm = float(r[7]) if tmax is None else float(tmax)
    ok = lib.oracle_triangle_test(r.ctypes.data, pa.ctypes.data, pb.ctypes.data, pc.ctypes.data, tm,
                                  out.ctypes.data)
    return bool(ok), float(out[0]), float(out[1]), float(out[2])


def restated_cast(positions, indices, rays, closest=True, any_hit=True, brute=False, threads=0):
    """Returns dict with ids, t, uv (closest) and occluded (any hit)."""
    lib = _load()
    pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    idx = np.ascontiguousarray(indices, np.uint32).reshape(-1, 3)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = r.shape[0]
    ids = np.empty(n, np.uint32)
    ts = np.empty(n, np.float32)
    uv = np.empty((n, 2), np.float32)
    occ = np.empty(n, np.uint8)
    mode = (MODE_CLOSEST if closest else 0) | (MODE_ANY if any_hit else 0) | (MODE_BRUTE if brute else 0)
    threads = threads or os.cpu_count() or 1
    st = lib.oracle_cast(pos.shape[0], idx.shape[0], pos.ctypes.data, idx.ctypes.data, n, r.ctypes.data,
                         ids.ctypes.data, ts.ctypes.data, uv.ctypes.data, occ.ctypes.data, threads, mode)
    if st != 0:
        raise ValueError("oracle_cast rejected its arguments")
    out = {}
    if closest:
        out.update(ids=ids, t=ts, uv=uv)
    if any_hit:
        out["occluded"] = occ
    return out


def synth_sphere_mesh(n: int, amplitude: float = 0.1, seed: int = 1):
    """The cast benchmark's displaced tetra-sphere, restated in C (synth_oracle.c)."""
    lib = _load()
    pos = np.empty((2 * n * n + 2, 3), np.float32)
    idx = np.empty((4 * n * n, 3), np.uint32)
    if lib.oracle_synth_sphere_mesh(n, amplitude, seed, pos.ctypes.data, idx.ctypes.data) != 0:
        raise ValueError("oracle_synth_sphere_mesh rejected its arguments")
    return pos, idx


def synth_rays(count: int, seed: int = 1, first: int = 0, extent: float = 2.0, threads: int = 0):
    """The cast benchmark's rays, restated in C (synth_oracle.c): (count, 8) float32."""
    lib = _load()
    rays = np.empty((count, 8), np.float32)
    if lib.oracle_synth_rays(first, count, seed, extent, rays.ctypes.data, threads or os.cpu_count() or 1) != 0:
        raise ValueError("oracle_synth_rays rejected its arguments")
    return rays


def reference_available() -> bool:
    return REF_CAST.exists()


def write_mesh(path, positions, indices):
    pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    idx = np.ascontiguousarray(indices, np.uint32).reshape(-1, 3)
    with open(path, "wb") as f:
        f.write(np.array([pos.shape[0], idx.shape[0]], np.uint32).tobytes())
        f.write(pos.tobytes())
        f.write(idx.tobytes())


def write_rays(path, rays):
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    with open(path, "wb") as f:
        f.write(np.array([r.shape[0]], np.uint64).tobytes())
        f.write(r.tobytes())


def reference_cast(positions, indices, rays, threads=0, mode="both", workdir=None):
    """Runs the compiled reference; returns dict(ids, t, occluded, timing)."""
    if not REF_CAST.exists():
        raise FileNotFoundError(f"{REF_CAST} missing: build it with `make -C oracle`")
    n = int(np.asarray(rays).reshape(-1, 8).shape[0])
    with tempfile.TemporaryDirectory(dir=workdir) as tmp:
        mesh_p = os.path.join(tmp, "mesh.bin")
        rays_p = os.path.join(tmp, "rays.bin")
        out_p = os.path.join(tmp, "out.bin")
        write_mesh(mesh_p, positions, indices)
        write_rays(rays_p, rays)
        res = subprocess.run([str(REF_CAST), mesh_p, rays_p, out_p, str(threads), mode],
                             capture_output=True, text=True, check=True)
        timing = json.loads(res.stdout.strip().splitlines()[-1])
        raw = np.fromfile(out_p, np.uint8)
    ids = raw[: 4 * n].view(np.uint32)
    ts = raw[4 * n: 8 * n].view(np.float32)
    occ = raw[8 * n: 9 * n]
    return {"ids": ids.copy(), "t": ts.copy(), "occluded": occ.copy(), "timing": timing}


MISS = 0xFFFFFFFF


def classify_mismatches(positions, indices, rays, ids_a, t_a, ids_b, t_b, test=None):
    """Splits the rays on which two closest-hit results disagree into those explained by
    rounding at a triangle edge or an equal-t tie and the unexplained rest.  ``test(ray, a, b,
    c)`` is the restated triangle test returning (pass, t, u, v) (default: :func:`triangle_test`).
    Returns (explained, unexplained) lists of ray indices."""
    test = test or triangle_test
    pos = np.asarray(positions, np.float32)
    idx = np.asarray(indices, np.uint32)
    explained, unexplained = [], []
    for i in np.nonzero(np.asarray(ids_a) != np.asarray(ids_b))[0]:
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


def id_parity(positions, indices, rays, ref_ids, ref_t, ids, t):
    """Summary of a closest-hit result against the reference's on the same rays: mismatching
    ids, split into edge/tie cases and unexplained ones, and the largest t difference in ulps
    where the ids agree (on hits)."""
    ref_ids = np.asarray(ref_ids, np.uint32)
    ids = np.asarray(ids, np.uint32)
    explained, unexplained = classify_mismatches(positions, indices, rays, ref_ids, ref_t, ids, t)
    same = (ref_ids == ids) & (ids != MISS)
    ulps = np.abs(np.asarray(ref_t, np.float32)[same].view(np.int32).astype(np.int64)
                  - np.asarray(t, np.float32)[same].view(np.int32).astype(np.int64))
    hist = np.bincount(np.minimum(ulps, 4), minlength=5) if ulps.size else np.zeros(5, np.int64)
    return {"rays": int(ids.size), "hits": int((ids != MISS).sum()),
            "mismatches": len(explained) + len(unexplained),
            "explained_edge_tie": len(explained), "unexplained": len(unexplained),
            "unexplained_rays": unexplained[:16],
            "t_max_ulp_on_equal_ids": int(ulps.max()) if ulps.size else 0,
            "t_ulp_histogram_0_1_2_3_4plus": [int(x) for x in hist]}


# ---- renderer oracle: the reference's C API in its own process ----------------------------

REF_RENDER = HERE / "_ref" / "ref_render"


class ScriptRecorder:
    """Records su_* calls (the subset the scene builders use) for _ref/ref_render to replay."""

    def __init__(self):
        self.lines = []
        self.data = bytearray()
        self.n = {"material": 0, "mesh": 0, "prop": 0, "image": 0}

    def _blob(self, array):
        while len(self.data) % 16:
            self.data.append(0)
        off = len(self.data)
        self.data += np.ascontiguousarray(array).tobytes()
        return off

    def su_create_camera_perspective(self, w, h, fov):
        self.lines.append(f"camera {w} {h} {float(fov):.9g}")
        return 4000

    def set_transformation(self, entity, matrix):
        m = np.asarray(matrix, np.float32).reshape(16)
        self.lines.append(f"trafo {entity} " + " ".join(f"{float(x):.9g}" for x in m))
        return 0

    def su_create_integrators(self, desc):
        self.lines.append("integrators " + (desc.decode() if isinstance(desc, bytes) else desc))
        return 0

    def su_create_sampler(self, spp):
        self.lines.append(f"sampler {int(spp)}")
        return 0

    def su_create_defaults(self):
        self.lines.append("defaults")
        return 0

    def su_mount(self, folder):
        self.lines.append(f"mount {folder.decode() if isinstance(folder, bytes) else folder}")
        return 0

    def load_take(self, path, width, height):
        """su_load_take of a take file whose camera renders width x height."""
        self.lines.append(f"take {int(width)} {int(height)} {path}")
        return 0

    def su_create_material(self, desc):
        self.lines.append("material " + (desc.decode() if isinstance(desc, bytes) else desc))
        self.n["material"] += 1
        return 1000 + self.n["material"] - 1

    def image(self, pixels):
        """su_create_image of an array (depth, height, width) or (height, width): one channel;
        (depth, height, width, channels): several; uint8 as Byte, anything else as Float.
        Returns the image id the reference assigns (images are numbered from 0)."""
        a = np.ascontiguousarray(pixels)
        kind = 0 if a.dtype == np.uint8 else 2
        a = a if a.dtype == np.uint8 else a.astype(np.float32)
        c = a.shape[3] if a.ndim == 4 else 1
        d, h, w = (a.shape[:3] if a.ndim >= 3 else (1,) + a.shape)
        off = self._blob(a)
        self.lines.append(f"image {kind} {c} {w} {h} {d} {off}")
        self.n["image"] += 1
        return self.n["image"] - 1

    def image2d(self, pixels):
        """su_create_image of a 2-D image (height, width, channels), uint8 (Byte) or float32."""
        a = np.ascontiguousarray(pixels)
        h, w, c = a.shape
        kind = 0 if a.dtype == np.uint8 else 2
        a = a if a.dtype == np.uint8 else a.astype(np.float32)
        self.lines.append(f"image {kind} {c} {w} {h} 1 {self._blob(a)}")
        self.n["image"] += 1
        return self.n["image"] - 1

    def mesh(self, positions, normals, indices, parts=None, uvs=None):
        pos = np.asarray(positions, np.float32).reshape(-1, 3)
        nrm = np.asarray(normals, np.float32).reshape(-1, 3)
        idx = np.asarray(indices, np.uint32).reshape(-1, 3)
        op, on, oi = self._blob(pos), self._blob(nrm), self._blob(idx)
        line = f"mesh {idx.shape[0]} {pos.shape[0]} {op} {on} {oi}"
        if parts is not None or uvs is not None:
            if parts is not None:
                prt = np.asarray(parts, np.uint32).reshape(-1, 3)
                line += f" {prt.shape[0]} {self._blob(prt)}"
            else:
                line += " 0 0"
        if uvs is not None:
            line += f" {self._blob(np.asarray(uvs, np.float32).reshape(-1, 2))}"
        self.lines.append(line)
        self.n["mesh"] += 1
        return 2000 + self.n["mesh"] - 1

    def prop(self, shape, materials):
        self.lines.append(f"prop {shape} {len(materials)} " + " ".join(str(int(m)) for m in materials))
        self.n["prop"] += 1
        return 3000 + self.n["prop"] - 1

    def su_create_light(self, prop):
        self.lines.append(f"light {prop}")
        return 0


def reference_render(build_scene, width, height, iterations, progressive=True, workdir=None, prepare=False):
    """Renders with the compiled reference: build_scene(recorder) issues the scene's calls.
    With prepare (batch mode), su_start_render_frame runs first and is timed apart
    (timing["prepare_s"]): it joins the asynchronous mesh BVH builds and compiles the scene, so
    timing["render_s"] covers the frame itself.  Returns (rgb image (H, W, 3) float32, timing)."""
    if not REF_RENDER.exists():
        raise FileNotFoundError(f"{REF_RENDER} missing: build it with `make -C oracle`")
    rec = ScriptRecorder()
    build_scene(rec)
    head = [f"init {1 if progressive else 0}"]
    tail = [f"progressive {iterations}"] if progressive else (["prepare", "frame 0"] if prepare else ["frame 0"])
    with tempfile.TemporaryDirectory(dir=workdir) as tmp:
        sp, dp, op = (os.path.join(tmp, n) for n in ("script.txt", "data.bin", "out.bin"))
        with open(sp, "w") as f:
            f.write("\n".join(head + rec.lines + tail) + "\n")
        with open(dp, "wb") as f:
            f.write(bytes(rec.data))
        res = subprocess.run([str(REF_RENDER), sp, dp, op], capture_output=True, text=True, check=True)
        timing = json.loads(res.stdout.strip().splitlines()[-1])
        img = np.fromfile(op, np.float32).reshape(height, width, 4)
    return img[:, :, :3].copy(), timing


# ---- the spectral mode's image (spectral_oracle.c) ----

SRGB_TO_AP1 = np.array([[0.61309732, 0.33952285, 0.04737928],
                        [0.07019422, 0.91635557, 0.01345259],
                        [0.02061560, 0.10956983, 0.86981512]])


def volumetric_coefficients(attenuation_color, attenuation_distance, subsurface_color, anisotropy):
    """(mu_a, mu_s) in ACEScg of a Volumetric material as su_create_material reads it: colours
    converted from sRGB, then the reference's attenuation() and scattering() mappings
    (collision_coefficients.inl:50-71; the library's capi.cpp restates them the same way)."""
    ac = SRGB_TO_AP1 @ np.asarray(attenuation_color, np.float64)
    ssc = SRGB_TO_AP1 @ np.asarray(subsurface_color, np.float64)
    g = float(np.clip(anisotropy, -0.999, 0.999))
    mu_t = -np.log(np.clip(ac, 0.01, 0.991102)) / attenuation_distance
    root = np.sqrt(9.59217 + 41.6808 * ssc + 17.7126 * ssc * ssc)
    factor = np.clip(4.097125 + 4.20863 * ssc - root, 0.0, 1.0)
    pss = (1.0 - factor * factor) / (1.0 - g * factor * factor)
    mu_a = mu_t * (1.0 - pss)
    return mu_a, mu_t - mu_a


def spectral_render(scene, spp, seed=1, runs=None):
    """The FP64 image (height, width, 3) of a scene described as sprout_b200.scenes.spectral_box
    returns it: `runs` independent renders of spp / runs samples per pixel on parallel threads,
    averaged."""
    import concurrent.futures
    import os

    lib = _load()
    tris = np.ascontiguousarray(scene["triangles"], np.float64)
    roles = np.ascontiguousarray(scene["roles"], np.int32)  # 0 lamp, 1 medium boundary
    mu_a, mu_s = volumetric_coefficients(**scene["medium"])
    g = float(np.clip(scene["medium"]["anisotropy"], -0.999, 0.999))
    emission = SRGB_TO_AP1 @ np.asarray(scene["emission"], np.float64)
    mats = np.ascontiguousarray(np.array([list(emission) + [0.0] * 5,
                                          list(mu_a) + list(mu_s) + [g, 1.0]], np.float64))
    types = np.array([0, 1], np.int32)
    density = np.ascontiguousarray(scene["density"], np.float64)
    nz, ny, nx = density.shape
    w2uvw = np.ascontiguousarray(scene["world_to_uvw"], np.float64)
    env = np.ascontiguousarray(SRGB_TO_AP1 @ np.asarray(scene["environment"], np.float64))
    cam = scene["camera"]
    m = np.asarray(cam["matrix"], np.float64)
    rot = np.ascontiguousarray(m[:3, :3] / np.linalg.norm(m[:3, :3], axis=1, keepdims=True))
    pos = np.ascontiguousarray(m[3, :3])
    w, h = cam["width"], cam["height"]
    runs = runs or max(1, min(os.cpu_count() or 1, spp))
    per = max(1, spp // runs)

    def one(k):
        out = np.zeros((h, w, 3), np.float64)
        weight = np.zeros((h, w), np.float64)
        light_tri = np.zeros(len(tris), np.uint32)
        light_cdf = np.zeros(len(tris), np.float64)
        lib.oracle_spectral_render(len(tris), tris.ctypes.data, roles.ctypes.data, types.ctypes.data,
                                   mats.ctypes.data, nx, ny, nz, density.ctypes.data, w2uvw.ctypes.data,
                                   env.ctypes.data, 1, w, h, float(cam["fov"]), rot.ctypes.data, pos.ctypes.data,
                                   per, scene["min_bounces"], scene["max_bounces"], seed * 7919 + k,
                                   light_tri.ctypes.data, light_cdf.ctypes.data, out.ctypes.data, weight.ctypes.data)
        return out

    with concurrent.futures.ThreadPoolExecutor(runs) as ex:
        images = list(ex.map(one, range(runs)))
    return np.mean(images, axis=0)
