"""Synthetic scenes for the path tracer, built through the su_* C API.

``cornell(su, ...)`` issues the same sequence of su_* calls against whichever library ``su``
binds (this package's or the reference's), so both render the identical scene:

* a Cornell box: floor, ceiling and back wall white (albedo 0.75), left wall red
  (0.75, 0.05, 0.05), right wall green (0.05, 0.75, 0.05) -- Substitute, roughness 1,
  metallic 0 (the reference has no pure Lambert material);
* a 0.5 x 0.5 m ceiling quad light (0.25 m^2), radiance 17, one-sided, facing down;
* an icosphere of radius 0.3 subdivided 6 times (81,920 triangles) with a GGX conductor,
  alpha 0.3 (roughness sqrt(0.3)), F0 = (0.95, 0.64, 0.54);
* a pinhole camera with a 40 degree horizontal field of view;
* PTMIS, max_bounces 8 (min_bounces 4, the reference default).
Colours are given in sRGB; both libraries map them to ACEScg.

Variants replace the metal sphere by a participating medium: a homogeneous Volumetric sphere,
or a rotated, scaled cube filled with a density grid (an in-memory 3-D image).
"""

from __future__ import annotations

import json
import math
import pathlib

import numpy as np


def icosphere(subdivisions: int):
    """Unit icosphere: 20 * 4^subdivisions triangles, vertex valence 5 or 6."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts, np.float32), np.array(faces, np.uint32)


def _quad(p0, p1, p2, p3, normal):
    """Two triangles p0 p1 p2, p0 p2 p3 wound so that cross(b - a, c - a) points along normal."""
    pos = np.array([p0, p1, p2, p3], np.float32)
    idx = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    n = np.array(normal, np.float32)
    g = np.cross(pos[1] - pos[0], pos[2] - pos[0])
    if np.dot(g, n) < 0:
        idx = idx[:, ::-1].copy()
    return pos, np.tile(n, (4, 1)), idx


def box():
    """Cube [-0.5, 0.5]^3 with outward faces: 12 triangles, 24 vertices (flat normals)."""
    pos, nrm, idx = [], [], []
    for axis in range(3):
        for sign in (-1.0, 1.0):
            n = np.zeros(3, np.float32)
            n[axis] = sign
            u, v = np.zeros(3, np.float32), np.zeros(3, np.float32)
            u[(axis + 1) % 3], v[(axis + 2) % 3] = 0.5, 0.5
            c = 0.5 * n
            qp, qn, qi = _quad(c - u - v, c + u - v, c + u + v, c - u + v, n)
            idx.append(qi + len(pos) * 4)
            pos.append(qp)
            nrm.append(qn)
    return np.concatenate(pos), np.concatenate(nrm), np.concatenate(idx)


def density_grid(nx: int = 24, ny: int = 20, nz: int = 28, seed: int = 4):
    """Deterministic density image (nz, ny, nx) in [0, 1]: a smooth blob times seeded
    low-frequency waves, exactly 0 near the corners (empty majorant cells)."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid((np.arange(nz) + 0.5) / nz, (np.arange(ny) + 0.5) / ny,
                          (np.arange(nx) + 0.5) / nx, indexing="ij")
    d = np.zeros_like(x)
    for _ in range(4):
        f = rng.uniform(1.0, 4.0, 3)
        ph = rng.uniform(0.0, 2.0 * np.pi, 3)
        d += np.sin(2 * np.pi * f[0] * x + ph[0]) * np.sin(2 * np.pi * f[1] * y + ph[1]) * \
            np.sin(2 * np.pi * f[2] * z + ph[2])
    r = np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2)
    d = np.clip(0.55 + 0.35 * d, 0.0, 1.0) * np.clip(1.6 - 2.6 * r, 0.0, 1.0)
    return d.astype(np.float32)


def grid_box_transformation(angle_degrees: float = 30.0, scale: float = 0.7,
                            position=(0.05, 0.45, 0.1)):
    """Row-major object-to-world matrix of the medium cube: uniform scale, rotation about y,
    translation."""
    a = math.radians(angle_degrees)
    c, s = math.cos(a), math.sin(a)
    m = np.eye(4, dtype=np.float32)
    m[:3, :3] = scale * np.array([[c, 0.0, -s], [0.0, 1.0, 0.0], [s, 0.0, c]], np.float32)
    m[3, :3] = position
    return m


def light_panel(n: int = 8, seed: int = 5, extent: float = 0.6, height: float = 1.98):
    """An n x n grid of small one-sided emitting quads under the ceiling (one mesh, one part per
    quad), plus two two-sided vertical quads near the side walls.  Returns (positions, normals,
    indices, parts, emissions): parts are (first index, index count, material slot) triples and
    emissions[k] the sRGB radiance of slot k -- log-uniform in [1, 40] times a random tint.
    Quad sizes, offsets, heights and tilts are jittered.  (The reference's light-tree builder
    recurses without end on many emitters with identical normals, so every quad is tilted.)"""
    rng = np.random.default_rng(seed)
    cell = 2.0 * extent / n
    pos, nrm, idx, parts = [], [], [], []
    for j in range(n):
        for i in range(n):
            cx = -extent + (i + 0.5 + rng.uniform(-0.15, 0.15)) * cell
            cz = -extent + (j + 0.5 + rng.uniform(-0.15, 0.15)) * cell
            hx, hz = rng.uniform(0.2, 0.33, 2) * cell
            y = height - rng.uniform(0.0, 0.05)
            sx, sz = rng.uniform(-0.3, 0.3, 2)  # slopes
            corners = [(cx + u * hx, y + sx * u * hx + sz * v * hz, cz + v * hz)
                       for u, v in ((-1, -1), (1, -1), (1, 1), (-1, 1))]
            g = np.cross(np.subtract(corners[1], corners[0]), np.subtract(corners[2], corners[0]))
            g = g / np.linalg.norm(g)
            qp, qn, qi = _quad(*corners, g if g[1] < 0 else -g)
            parts.append((3 * 2 * len(pos), 6, len(pos)))
            idx.append(qi + 4 * len(pos))
            pos.append(qp)
            nrm.append(qn)
    for x, z in ((-0.85, -0.07), (0.83, 0.11)):
        qp, qn, qi = _quad((x, 0.6, z - 0.2), (x, 0.6, z + 0.2), (x, 1.03, z + 0.2), (x, 1.03, z - 0.2),
                           (1, 0, 0))
        parts.append((3 * 2 * len(pos), 6, len(pos)))
        idx.append(qi + 4 * len(pos))
        pos.append(qp)
        nrm.append(qn)
    k = len(pos)
    radiance = np.exp(rng.uniform(np.log(1.0), np.log(40.0), k))
    tint = rng.uniform(0.5, 1.0, (k, 3))
    emissions = (radiance[:, None] * tint).astype(np.float32)
    return (np.concatenate(pos), np.concatenate(nrm), np.concatenate(idx),
            np.array(parts, np.uint32), emissions)


def cornell_geometry(sphere_subdivisions: int = 6):
    """name -> (positions, normals, indices) in world space (y up, box x, z in [-1, 1], y in [0, 2])."""
    g = {}
    g["floor"] = _quad((-1, 0, -1), (1, 0, -1), (1, 0, 1), (-1, 0, 1), (0, 1, 0))
    g["ceiling"] = _quad((-1, 2, -1), (-1, 2, 1), (1, 2, 1), (1, 2, -1), (0, -1, 0))
    g["back"] = _quad((-1, 0, 1), (1, 0, 1), (1, 2, 1), (-1, 2, 1), (0, 0, -1))
    g["left"] = _quad((-1, 0, -1), (-1, 0, 1), (-1, 2, 1), (-1, 2, -1), (1, 0, 0))
    g["right"] = _quad((1, 0, -1), (1, 2, -1), (1, 2, 1), (1, 0, 1), (-1, 0, 0))
    g["light"] = _quad((-0.25, 1.98, -0.25), (0.25, 1.98, -0.25), (0.25, 1.98, 0.25), (-0.25, 1.98, 0.25),
                       (0, -1, 0))
    v, f = icosphere(sphere_subdivisions)
    g["sphere"] = ((0.3 * v + np.array([0.0, 0.3, 0.0], np.float32)).astype(np.float32), v.copy(), f)
    return g


def _material(su, kind, **params):
    return su.su_create_material(json.dumps({"rendering": {kind: params}}).encode())


def translation(x, y, z):
    m = np.eye(4, dtype=np.float32)
    m[3, :3] = (x, y, z)
    return m


def cornell(su, width: int, height: int, sphere_subdivisions: int = 6, max_bounces: int = 8,
            min_bounces: int = 4, fov_degrees: float = 40.0, camera_position=(0.0, 1.0, -3.4),
            spp: int = 64, tonemap: bool = False, medium=None, density=None, many_lights=False, guiding=None,
            integrator=None):
    """Issues the scene's su_* calls on an initialised engine; returns the camera entity.

    medium: optional dict of Volumetric material parameters (e.g. color, attenuation_distance,
    anisotropy); the sphere then becomes a homogeneous participating medium instead of metal.
    density: optional (nz, ny, nx) float array, or the name of a SUB image file (sub.write_sub);
    with medium, the sphere is replaced by the cube of grid_box_transformation() filled with
    this density grid.
    many_lights: the ceiling light is replaced by light_panel(): 66 emitters of different
    radiance, two of them two-sided (a light-tree test).
    guiding: None for plain MIS, else True or a dict of guide settings (this renderer's
    "guiding" integrator key).
    integrator: further PTMIS keys (e.g. this renderer's "instancing").
    """
    cam = su.su_create_camera_perspective(width, height, math.radians(fov_degrees))
    su.set_transformation(cam, translation(*camera_position))
    ptmis = {"min_bounces": min_bounces, "max_bounces": max_bounces}
    if guiding is not None:
        ptmis["guiding"] = guiding
    ptmis.update(integrator or {})
    su.su_create_integrators(json.dumps({"surface": {"PTMIS": ptmis}}).encode())
    su.su_create_sampler(spp)
    if tonemap:
        su.su_create_defaults()

    white = _material(su, "Substitute", color=[0.75, 0.75, 0.75], roughness=1.0, metallic=0.0)
    red = _material(su, "Substitute", color=[0.75, 0.05, 0.05], roughness=1.0, metallic=0.0)
    green = _material(su, "Substitute", color=[0.05, 0.75, 0.05], roughness=1.0, metallic=0.0)
    if medium is None:
        metal = _material(su, "Substitute", color=[0.95, 0.64, 0.54], roughness=math.sqrt(0.3), metallic=1.0)
    elif density is None:
        metal = _material(su, "Volumetric", **medium)
    elif isinstance(density, (str, pathlib.Path)):
        metal = _material(su, "Volumetric", density={"file": str(density)}, **medium)
    else:
        image = su.image(density)
        metal = _material(su, "Volumetric", density={"id": int(image)}, **medium)
    light = _material(su, "Light", emission=[17.0, 17.0, 17.0])

    geo = cornell_geometry(sphere_subdivisions)
    if many_lights:
        del geo["light"]
    trafo = {}
    if density is not None:
        geo["sphere"] = box()
        trafo["sphere"] = grid_box_transformation()
    assign = {"floor": white, "ceiling": white, "back": white, "left": red, "right": green,
              "light": light, "sphere": metal}
    for name, (pos, nrm, idx) in geo.items():
        shape = su.mesh(pos, nrm, idx)
        prop = su.prop(shape, [assign[name]])
        # props carry no default world transformation in the reference: always set one
        su.set_transformation(prop, trafo.get(name, np.eye(4, dtype=np.float32)))
        if name == "light":
            su.su_create_light(prop)
    if many_lights:
        pos, nrm, idx, parts, emissions = light_panel()
        slots = []
        for k, e in enumerate(emissions):
            two_sided = k >= len(emissions) - 2
            slots.append(_material(su, "Light", emission=[float(x) for x in e], two_sided=two_sided))
        prop = su.prop(su.mesh(pos, nrm, idx, parts=parts), slots)
        su.set_transformation(prop, np.eye(4, dtype=np.float32))
        su.su_create_light(prop)
    return cam


def render_progressive(su, width: int, height: int, iterations: int, **scene):
    """Progressive rendering through the C API: returns the (H, W, 3) mean image."""
    assert su.su_init(True) == 0
    try:
        cornell(su, width, height, **scene)
        assert su.su_start_render_frame(0) == 0, su.messages
        for _ in range(iterations):
            assert su.su_render_iteration() == 0
        assert su.su_postprocess() == 0
        img, _status = su.framebuffer(width, height)
        return img[:, :, :3].copy()
    finally:
        su.su_release()


# ---- many instances and many lights: the 1920x1080 wavefront workload ----

def value_noise(p, seed: int):
    """Smooth 3-D value noise in [-1, 1] at points p (n, 3): hashed lattice values, quintic
    fade, trilinear blend."""
    p = np.asarray(p, np.float64)
    i = np.floor(p).astype(np.int64)
    f = p - i
    u = f * f * f * (f * (f * 6.0 - 15.0) + 10.0)

    def lattice(ix, iy, iz):
        h = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791) ^ (seed * 2654435761)
        h = (h ^ (h >> 13)) * 1274126177
        h = h ^ (h >> 16)
        return (h & 0xFFFF).astype(np.float64) / 32767.5 - 1.0

    out = 0.0
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = (np.where(dx, u[:, 0], 1 - u[:, 0]) * np.where(dy, u[:, 1], 1 - u[:, 1]) *
                     np.where(dz, u[:, 2], 1 - u[:, 2]))
                out = out + w * lattice(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz)
    return out


def displaced_sphere(segments: int = 50, rings: int = 51, amplitude: float = 0.1, octaves: int = 6,
                     seed: int = 2):
    """Unit UV sphere of 2 * segments * (rings - 2) + 2 * segments triangles (5,000 with the
    defaults), radius 1 + amplitude * fBm (lacunarity 2, gain 0.5); smooth vertex normals."""
    theta = np.pi * np.arange(1, rings) / rings
    phi = 2.0 * np.pi * np.arange(segments) / segments
    st, ct = np.sin(theta), np.cos(theta)
    ring = np.stack([np.outer(st, np.cos(phi)), np.repeat(ct[:, None], segments, 1),
                     np.outer(st, np.sin(phi))], -1).reshape(-1, 3)
    v = np.concatenate([[[0.0, 1.0, 0.0]], ring, [[0.0, -1.0, 0.0]]])
    fbm, amp, freq = np.zeros(len(v)), 1.0, 2.0
    for o in range(octaves):
        fbm += amp * value_noise(v * freq, seed + o)
        amp, freq = amp * 0.5, freq * 2.0
    v = v * (1.0 + amplitude * fbm)[:, None]
    faces = []
    top, bottom = 0, len(v) - 1
    for s in range(segments):
        s1 = (s + 1) % segments
        faces.append((top, 1 + s1, 1 + s))
        for r in range(rings - 2):
            a, b = 1 + r * segments + s, 1 + r * segments + s1
            c, d = a + segments, b + segments
            faces += [(a, b, d), (a, d, c)]
        last = 1 + (rings - 2) * segments
        faces.append((bottom, last + s, last + s1))
    f = np.array(faces, np.uint32)
    fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    if np.mean(np.einsum("ij,ij->i", fn, v[f[:, 0]])) < 0:  # wind outwards
        f = f[:, ::-1].copy()
        fn = -fn
    n = np.zeros_like(v)
    for k in range(3):
        np.add.at(n, f[:, k], fn)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    return v.astype(np.float32), n.astype(np.float32), f


def _rotation(rng):
    """Uniformly random rotation matrix (3x3, rows are the rotated axes)."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)],
                     [2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x)],
                     [2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)]])


def emitter_cloud(count: int = 4096, seed: int = 2, size: float = 0.25):
    """count small emissive triangles above the instances, facing roughly down with random
    tilt (one mesh, one part per triangle).  Returns (positions, normals, indices, parts,
    radiance): the brightest channel log-uniform in [0.1, 100], the others a random tint of it."""
    rng = np.random.default_rng(seed + 1000)
    centre = np.stack([rng.uniform(-12, 12, count), rng.uniform(6.0, 9.0, count),
                       rng.uniform(-12, 12, count)], 1)
    pos = np.zeros((count, 3, 3))
    for k in range(3):
        a = 2.0 * np.pi * (k / 3.0) + rng.uniform(-0.3, 0.3, count)
        pos[:, k] = centre + size * np.stack([np.cos(a), rng.uniform(-0.4, 0.4, count), np.sin(a)], 1)
    g = np.cross(pos[:, 1] - pos[:, 0], pos[:, 2] - pos[:, 0])
    flip = g[:, 1] > 0  # face down
    pos[flip] = pos[flip][:, ::-1]
    g[flip] = -g[flip]
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    idx = np.arange(3 * count, dtype=np.uint32).reshape(count, 3)
    parts = np.stack([3 * np.arange(count), np.full(count, 3), np.arange(count)], 1).astype(np.uint32)
    radiance = np.exp(rng.uniform(np.log(0.1), np.log(100.0), count))
    tint = rng.uniform(0.6, 1.0, (count, 3))
    tint /= tint.max(axis=1, keepdims=True)
    return (pos.reshape(-1, 3).astype(np.float32), np.repeat(g, 3, 0).astype(np.float32), idx, parts,
            (radiance[:, None] * tint).astype(np.float32))


def wavefront(su, width: int = 1920, height: int = 1080, spp: int = 256, max_bounces: int = 12,
              min_bounces: int = 4, instances: int = 400, emitters: int = 4096, seed: int = 2,
              tonemap: bool = True, integrator=None):
    """The many-instances, many-lights scene: a ground plane; `instances` randomly placed,
    scaled and rotated copies of one 5,000-triangle displaced sphere (props sharing a mesh, so
    2,000,000 triangles for 400), each with a random Substitute material (roughness U[0.05, 1],
    metallic Bernoulli(0.3), colour U[0, 1]^3); `emitters` emissive triangles with their own
    Light materials; PTMIS, max depth 12; a pinhole camera with a 60 degree field of view.
    integrator: further PTMIS keys (e.g. this renderer's "instancing")."""
    rng = np.random.default_rng(seed)
    cam = su.su_create_camera_perspective(width, height, math.radians(60.0))
    m = np.eye(4, dtype=np.float32)
    # rows: camera x, y, z axes in world space; pitched down by 0.25 rad
    m[1, 1], m[1, 2], m[2, 1], m[2, 2] = math.cos(0.25), math.sin(0.25), -math.sin(0.25), math.cos(0.25)
    m[3, :3] = (0.0, 6.0, -17.0)
    su.set_transformation(cam, m)
    ptmis = {"min_bounces": min_bounces, "max_bounces": max_bounces}
    ptmis.update(integrator or {})
    su.su_create_integrators(json.dumps({"surface": {"PTMIS": ptmis}}).encode())
    su.su_create_sampler(spp)
    if tonemap:
        su.su_create_defaults()
    ground = _material(su, "Substitute", color=[0.6, 0.6, 0.6], roughness=0.9, metallic=0.0)
    pos, nrm, idx = _quad((-30, 0, -30), (30, 0, -30), (30, 0, 30), (-30, 0, 30), (0, 1, 0))
    prop = su.prop(su.mesh(pos, nrm, idx), [ground])
    su.set_transformation(prop, np.eye(4, dtype=np.float32))
    v, n, f = displaced_sphere(seed=seed)
    sphere = su.mesh(v, n, f)
    for _ in range(instances):
        mat = _material(su, "Substitute", color=[float(c) for c in rng.uniform(0.0, 1.0, 3)],
                        roughness=float(rng.uniform(0.05, 1.0)), metallic=float(rng.random() < 0.3))
        t = np.eye(4, dtype=np.float32)
        t[:3, :3] = float(rng.uniform(0.3, 1.0)) * _rotation(rng)
        t[3, :3] = (rng.uniform(-11, 11), rng.uniform(1.0, 4.5), rng.uniform(-11, 11))
        prop = su.prop(sphere, [mat])
        su.set_transformation(prop, t)
    if emitters:
        pos, nrm, idx, parts, radiance = emitter_cloud(emitters, seed)
        slots = [_material(su, "Light", emission=[float(x) for x in e]) for e in radiance]
        prop = su.prop(su.mesh(pos, nrm, idx, parts=parts), slots)
        su.set_transformation(prop, np.eye(4, dtype=np.float32))
        su.su_create_light(prop)
    return cam


# ---- built-in shapes under an environment light ----

SHAPE_CUBE, SHAPE_DISK, SHAPE_INFINITE_SPHERE, SHAPE_RECTANGLE, SHAPE_SPHERE = 1, 2, 4, 6, 7


def _trafo(scale, rows, position):
    """Row-major object-to-world matrix: rows are the object's x, y, z axes in world space,
    each times the scale (a number or three), then the position."""
    m = np.eye(4, dtype=np.float32)
    m[:3, :3] = np.asarray(rows, np.float32) * np.broadcast_to(np.asarray(scale, np.float32), (3,))[:, None]
    m[3, :3] = position
    return m


def builtin_shapes(su, width: int = 64, height: int = 48, spp: int = 64, environment=(0.4, 0.5, 0.7),
                   environment_light: bool = True, max_bounces: int = 8, min_bounces: int = 4,
                   lamp: bool = True, integrator=None):
    """Built-in analytic shapes created by id (su_create_prop with SU_SHAPE_*): a Disk of
    radius 3 as the ground, a metal Sphere, a rotated Cube, a Rectangle light of 0.6 x 0.6
    facing down (radiance 20), and an Infinite_sphere of uniform radiance `environment` (a
    light unless environment_light is False, then only seen by the camera).  lamp=False leaves
    the Rectangle light out.  integrator: further PTMIS keys."""
    cam = su.su_create_camera_perspective(width, height, math.radians(45.0))
    m = np.eye(4, dtype=np.float32)
    m[1, 1], m[1, 2], m[2, 1], m[2, 2] = math.cos(0.25), math.sin(0.25), -math.sin(0.25), math.cos(0.25)
    m[3, :3] = (0.0, 1.5, -4.0)
    su.set_transformation(cam, m)
    ptmis = {"min_bounces": min_bounces, "max_bounces": max_bounces}
    ptmis.update(integrator or {})
    su.su_create_integrators(json.dumps({"surface": {"PTMIS": ptmis}}).encode())
    su.su_create_sampler(spp)
    su.su_create_defaults()
    ground = _material(su, "Substitute", color=[0.7, 0.7, 0.7], roughness=0.8, metallic=0.0)
    metal = _material(su, "Substitute", color=[0.9, 0.8, 0.5], roughness=0.4, metallic=1.0)
    red = _material(su, "Substitute", color=[0.8, 0.1, 0.1], roughness=0.6, metallic=0.0)
    lamp_mat = _material(su, "Light", emission=[20.0, 20.0, 20.0])
    sky = _material(su, "Light", emission=[float(x) for x in environment])
    a = math.radians(30.0)
    props = [
        (SHAPE_DISK, ground, _trafo(3.0, [[1, 0, 0], [0, 0, -1], [0, 1, 0]], (0.0, 0.0, 0.0)), False),
        (SHAPE_SPHERE, metal, _trafo(0.5, np.eye(3), (-0.7, 0.5, 0.3)), False),
        (SHAPE_CUBE, red, _trafo(0.4, [[math.cos(a), 0, -math.sin(a)], [0, 1, 0], [math.sin(a), 0, math.cos(a)]],
                                 (0.8, 0.4, -0.1)), False),
        (SHAPE_RECTANGLE, lamp_mat, _trafo(0.3, [[1, 0, 0], [0, 0, 1], [0, -1, 0]], (0.0, 2.5, 0.0)), True),
        (SHAPE_INFINITE_SPHERE, sky, np.eye(4, dtype=np.float32), environment_light),
    ]
    if not lamp:
        del props[3]
    for shape, mat, trafo, light in props:
        prop = su.prop(shape, [mat])
        su.set_transformation(prop, trafo)
        if light:
            su.su_create_light(prop)
    return cam


# ---- a heterogeneous medium lit by a sphere light and the environment ----

# Volumetric colours for the medium: attenuation colour 0.5 over 0.034657 m gives
# mu_t = -ln(0.5) / 0.034657 = 20 per metre at density 1; subsurface colour 0.32297 gives a
# single-scattering albedo of 0.9 at anisotropy 0.6 through the reference's scattering()
# mapping (collision_coefficients.inl:50-71).
VOLUME_FOV = math.radians(40.0)  # horizontal field of view of the volume views

VOLUME_MEDIUM = {"attenuation_color": [0.5, 0.5, 0.5], "attenuation_distance": 0.0346574,
                 "subsurface_color": [0.322972, 0.322972, 0.322972], "anisotropy": 0.6}


def fbm_density(n: int = 256, octaves: int = 5, seed: int = 4):
    """(n, n, n) float32 density in [0, 1] with maximum exactly 1: fBm of seeded value noise
    (random lattices of 4 * 2^o cells per axis, trilinearly upsampled; gain 0.5), shifted and
    clipped so that about a fifth of the cube is empty."""
    from scipy import ndimage

    rng = np.random.default_rng(seed)
    f = np.zeros((n, n, n), np.float32)
    amp = 1.0
    for o in range(octaves):
        cells = 4 << o
        lattice = rng.uniform(-1.0, 1.0, (cells + 1,) * 3).astype(np.float32)
        f += amp * ndimage.zoom(lattice, n / (cells + 1), order=1, mode="nearest", grid_mode=True)[:n, :n, :n]
        amp *= 0.5
    f = (f - f.mean()) / f.std()
    d = np.clip(0.5 + 0.4 * f, 0.0, None)
    return (d / d.max()).astype(np.float32)


def volume_views(count: int = 64, seed: int = 4):
    """Seeded camera views of the medium: (position on a sphere of radius 5 around the
    cube's centre, image side U[256, 1024] px)."""
    rng = np.random.default_rng(seed + 100)
    out = []
    for _ in range(count):
        z = rng.uniform(-0.3, 0.8)
        phi = rng.uniform(0.0, 2.0 * np.pi)
        r = math.sqrt(1.0 - z * z)
        out.append(((5.0 * r * math.cos(phi), 5.0 * z, 5.0 * r * math.sin(phi)), int(rng.integers(256, 1025))))
    return out


def _look_at(position, target=(0.0, 0.0, 0.0)):
    """Camera-to-world matrix (rows: camera x, y, z axes, then the position): z towards the
    target, x horizontal (world up cross z), y = z cross x."""
    p = np.asarray(position, np.float64)
    zc = np.asarray(target, np.float64) - p
    zc /= np.linalg.norm(zc)
    xc = np.cross([0.0, 1.0, 0.0], zc)
    xc /= np.linalg.norm(xc)
    yc = np.cross(zc, xc)
    m = np.eye(4, dtype=np.float32)
    m[0, :3], m[1, :3], m[2, :3], m[3, :3] = xc, yc, zc, p
    return m


def volume(su, width: int, height: int, spp: int, density, position=(3.0, 2.0, -3.2),
           max_bounces: int = 32, min_bounces: int = 4, environment=(0.3, 0.35, 0.4), integrator=None,
           medium=None, medium_light: bool = False, medium_shape: int = SHAPE_CUBE, temperature_seed=None,
           emission_scale_seed=None, color_grid_seed=None):
    """A 2 m Cube (built-in, [-1, 1]^3) filled with a density grid (VOLUME_MEDIUM), lit by a
    Sphere light of radius 0.25 (radiance 60) and a uniform Infinite_sphere environment; a
    pinhole camera at `position` looking at the centre with a 40 degree field of view; PTMIS
    with max depth 32.  integrator: further PTMIS keys (e.g. this renderer's "instancing").
    medium: Volumetric keys replacing VOLUME_MEDIUM's (e.g. "emission"); density None for a
    homogeneous medium; medium_light: the medium's prop is a light too (su_create_light);
    medium_shape: the built-in shape holding the medium (a Sphere has radius 1); temperature_seed:
    give the density grid a temperature grid of its size, 0.9 + 0.3 x fBm of that seed (about
    4250-5000 K on the emission's black-body scale); emission_scale_seed: make the density a
    two-channel image whose second channel, 0.5 + fBm of that seed, scales the emission;
    color_grid_seed: a colour grid instead (Grid_color, from a four-channel byte image as the
    reference takes it: sRGB colour and alpha): the density as alpha, each colour channel
    0.35 + 0.6 x fBm of seeds from that one."""
    cam = su.su_create_camera_perspective(width, height, VOLUME_FOV)
    su.set_transformation(cam, _look_at(position))
    ptmis = {"min_bounces": min_bounces, "max_bounces": max_bounces}
    ptmis.update(integrator or {})
    su.su_create_integrators(json.dumps({"surface": {"PTMIS": ptmis}}).encode())
    su.su_create_sampler(spp)
    su.su_create_defaults()
    params = dict(VOLUME_MEDIUM)
    params.update(medium or {})
    if density is not None and color_grid_seed is not None:
        n = density.shape[0]
        rgb = [0.35 + 0.6 * fbm_density(n, seed=color_grid_seed + k) for k in range(3)]
        rgba = np.rint(255.0 * np.clip(np.stack(rgb + [density], axis=-1), 0.0, 1.0)).astype(np.uint8)
        params["color"] = {"id": int(su.image(rgba))}
    elif density is not None:
        if emission_scale_seed is not None:
            # a two-channel density: the grid, and 0.5 + fBm of that seed scaling the emission
            scale = 0.5 + fbm_density(density.shape[0], seed=emission_scale_seed)
            density = np.stack([density, scale.astype(np.float32)], axis=-1)
        params["density"] = {"id": int(su.image(density))}
        if temperature_seed is not None:
            heat = 0.9 + 0.3 * fbm_density(density.shape[0], seed=temperature_seed)
            params["temperature"] = {"id": int(su.image(heat.astype(np.float32)))}
    fill = _material(su, "Volumetric", **params)
    lamp = _material(su, "Light", emission=[60.0, 60.0, 60.0])
    sky = _material(su, "Light", emission=[float(x) for x in environment])
    for shape, mat, trafo in ((medium_shape, fill, np.eye(4, dtype=np.float32)),
                              (SHAPE_SPHERE, lamp, _trafo(0.25, np.eye(3), (1.8, 2.2, -1.6))),
                              (SHAPE_INFINITE_SPHERE, sky, np.eye(4, dtype=np.float32))):
        prop = su.prop(shape, [mat])
        su.set_transformation(prop, trafo)
        if mat != fill or medium_light:
            su.su_create_light(prop)
    return cam


# ---- an interior lit through a doorway: the path-guiding workload ----

def _box_mesh(lo, hi):
    """Axis-aligned box from corner lo to corner hi, outward faces (12 triangles)."""
    p, n, f = box()
    lo, hi = np.asarray(lo, np.float32), np.asarray(hi, np.float32)
    return (p + 0.5) * (hi - lo) + lo, n, f


def doorway(su, width: int = 1280, height: int = 720, spp: int = 64, seed: int = 3, spheres: int = 96,
            boxes: int = 160, sphere_subdivisions: int = 4, max_bounces: int = 8, min_bounces: int = 4,
            environment: float = 5.0, guiding=None, render_seed: int = 0, integrator=None):
    """A 6 x 6 x 3 m room (x, z in [-3, 3], y in [0, 3]) whose only opening is a 1 x 2 m doorway
    in the wall z = 3, outside a uniform environment of radiance `environment` (an
    Infinite_sphere light).  Inside: `spheres` icospheres (20 * 4^subdivisions triangles each:
    491,520 with the defaults) and `boxes` boxes at seeded random places; 70 % of the objects
    Lambertian-like (Substitute, roughness 1, metallic 0), 30 % GGX conductors with alpha
    U[0.1, 0.6].  Walls, floor and ceiling are grey Substitute (roughness 1).  A pinhole camera
    in the room's far corner looks towards the doorway with a 60 degree field of view.
    guiding: None for plain MIS, else True or a dict of guide settings (this renderer's
    "guiding" integrator key; the reference ignores it).  render_seed: the sample streams' seed
    (this renderer's "seed" integrator key), for independent renders.  integrator: further
    PTMIS keys (e.g. this renderer's fixed launch shapes "wave_paths", "trace_blocks_per_sm")."""
    rng = np.random.default_rng(seed)
    eye = np.array([-2.4, 1.5, -2.7])
    cam = su.su_create_camera_perspective(width, height, math.radians(60.0))
    su.set_transformation(cam, _look_at(eye, (0.6, 0.9, 2.0)))
    ptmis = {"min_bounces": min_bounces, "max_bounces": max_bounces}
    if guiding is not None:
        ptmis["guiding"] = guiding
    if render_seed:
        ptmis["seed"] = render_seed
    ptmis.update(integrator or {})

    def clear(c, r):
        """Keeps objects off the camera and out of the doorway."""
        return (np.linalg.norm(np.asarray(c) - eye) > r + 1.0 and
                not (abs(c[0]) < 0.5 + r + 0.3 and c[2] > 2.0 - r))
    su.su_create_integrators(json.dumps({"surface": {"PTMIS": ptmis}}).encode())
    su.su_create_sampler(spp)
    su.su_create_defaults()
    wall = _material(su, "Substitute", color=[0.7, 0.7, 0.7], roughness=1.0, metallic=0.0)

    def add(pos, nrm, idx, mat):
        prop = su.prop(su.mesh(pos, nrm, idx), [mat])
        su.set_transformation(prop, np.eye(4, dtype=np.float32))

    # Room shell: quads facing inwards; the wall z = 3 is split around the doorway.
    quads = [((-3, 0, -3), (3, 0, -3), (3, 0, 3), (-3, 0, 3), (0, 1, 0)),      # floor
             ((-3, 3, -3), (-3, 3, 3), (3, 3, 3), (3, 3, -3), (0, -1, 0)),     # ceiling
             ((-3, 0, -3), (-3, 3, -3), (3, 3, -3), (3, 0, -3), (0, 0, 1)),    # wall z = -3
             ((-3, 0, -3), (-3, 0, 3), (-3, 3, 3), (-3, 3, -3), (1, 0, 0)),    # wall x = -3
             ((3, 0, -3), (3, 3, -3), (3, 3, 3), (3, 0, 3), (-1, 0, 0)),       # wall x = 3
             ((-3, 0, 3), (-0.5, 0, 3), (-0.5, 3, 3), (-3, 3, 3), (0, 0, -1)),  # z = 3, left of door
             ((0.5, 0, 3), (3, 0, 3), (3, 3, 3), (0.5, 3, 3), (0, 0, -1)),     # z = 3, right of door
             ((-0.5, 2, 3), (0.5, 2, 3), (0.5, 3, 3), (-0.5, 3, 3), (0, 0, -1))]  # above the door
    for q in quads:
        add(*_quad(*q), wall)

    def material():
        if rng.random() < 0.7:
            return _material(su, "Substitute", color=[float(c) for c in rng.uniform(0.2, 0.9, 3)],
                             roughness=1.0, metallic=0.0)
        alpha = rng.uniform(0.1, 0.6)
        return _material(su, "Substitute", color=[float(c) for c in rng.uniform(0.5, 1.0, 3)],
                         roughness=float(math.sqrt(alpha)), metallic=1.0)

    v, f = icosphere(sphere_subdivisions)
    placed = 0
    while placed < spheres:
        r = rng.uniform(0.08, 0.3)
        c = (rng.uniform(-2.7, 2.7), rng.uniform(r, 2.6), rng.uniform(-2.7, 2.7))
        if clear(c, r):
            add(r * v + np.array(c, np.float32), v, f, material())
            placed += 1
    placed = 0
    while placed < boxes:
        size = rng.uniform(0.1, 0.5, 3)
        lo = np.array([rng.uniform(-2.9, 2.9 - size[0]),
                       0.0 if rng.random() < 0.5 else rng.uniform(0.0, 2.9 - size[1]),
                       rng.uniform(-2.9, 2.9 - size[2])])
        if clear(lo + 0.5 * size, 0.5 * float(np.linalg.norm(size))):
            add(*_box_mesh(lo, lo + size), material())
            placed += 1
    sky = _material(su, "Light", emission=[environment] * 3)
    prop = su.prop(SHAPE_INFINITE_SPHERE, [sky])
    su.set_transformation(prop, np.eye(4, dtype=np.float32))
    su.su_create_light(prop)
    return cam


def checker_image(size: int = 64, checks: int = 8, colors=((200, 40, 30), (30, 60, 210))):
    """A size x size RGB byte image of checks x checks squares of two colours."""
    y, x = np.mgrid[0:size, 0:size]
    odd = ((x * checks // size) + (y * checks // size)) % 2 == 1
    img = np.empty((size, size, 3), np.uint8)
    img[~odd] = colors[0]
    img[odd] = colors[1]
    return img


def surface_image(size: int = 32, stripes: int = 4):
    """A size x size two-channel byte image: roughness (X) in stripes of 0.1 and 0.9 along x,
    metallic (Y) 1 in the lower half of the rows, else 0.  (Bytes, because the reference
    renderer returns NaN for float images used as surface or roughness maps.)"""
    y, x = np.mgrid[0:size, 0:size]
    img = np.empty((size, size, 2), np.uint8)
    img[..., 0] = np.where((x * stripes // size) % 2 == 0, 26, 230)
    img[..., 1] = np.where(y >= size // 2, 255, 0)
    return img


def textured_room(su, width: int, height: int, spp: int, max_bounces: int = 8, integrator=None):
    """The Cornell box with texture maps instead of the sphere's metal: the back wall's colour
    from a checker image (byte sRGB, uv scale 2, so the image repeats twice), the floor's
    roughness and metallic from a two-channel byte image (Surface use), and a rotated block
    whose colour comes from the checker image through a "textures" entry, sampled with the
    Nearest filter; every quad carries texture coordinates over [0, 1]^2."""
    cam = su.su_create_camera_perspective(width, height, math.radians(40.0))
    su.set_transformation(cam, translation(0.0, 1.0, -3.4))
    ptmis = {"min_bounces": 4, "max_bounces": max_bounces}
    ptmis.update(integrator or {})
    su.su_create_integrators(json.dumps({"surface": {"PTMIS": ptmis}}).encode())
    su.su_create_sampler(spp)
    su.su_create_defaults()
    checker = su.image2d(checker_image())
    surface = su.image2d(surface_image())
    back = _material(su, "Substitute", color={"id": int(checker), "scale": 2.0}, roughness=1.0)
    floor = _material(su, "Substitute", color=[0.8, 0.8, 0.75], surface={"id": int(surface)})
    white = _material(su, "Substitute", color=[0.75, 0.75, 0.75], roughness=1.0, metallic=0.0)
    red = _material(su, "Substitute", color=[0.75, 0.05, 0.05], roughness=1.0, metallic=0.0)
    green = _material(su, "Substitute", color=[0.05, 0.75, 0.05], roughness=1.0, metallic=0.0)
    block = _material(su, "Substitute", textures=[{"id": int(checker), "usage": "Color"}], roughness=0.6,
                      sampler={"filter": "Nearest"})
    light = _material(su, "Light", emission=[17.0, 17.0, 17.0])
    geo = cornell_geometry(1)
    del geo["sphere"]
    quad_uv = np.array([[0, 1], [1, 1], [1, 0], [0, 0]], np.float32)
    assign = {"floor": floor, "ceiling": white, "back": back, "left": red, "right": green, "light": light}
    for name, (pos, nrm, idx) in geo.items():
        prop = su.prop(su.mesh(pos, nrm, idx, uvs=quad_uv), [assign[name]])
        su.set_transformation(prop, np.eye(4, dtype=np.float32))
        if name == "light":
            su.su_create_light(prop)
    # a textured block: the unit box with per-face texture coordinates
    pos, nrm, idx = box()
    uv = np.tile(quad_uv, (len(pos) // 4, 1))
    prop = su.prop(su.mesh(pos, nrm, idx, uvs=uv), [block])
    m = np.diag([0.6, 0.6, 0.6, 1.0]).astype(np.float32)
    c, sn = math.cos(0.4), math.sin(0.4)
    m[:3, :3] = np.array([[0.6 * c, 0, -0.6 * sn], [0, 0.6, 0], [0.6 * sn, 0, 0.6 * c]], np.float32)
    m[3, :3] = (0.2, 0.3, 0.2)
    su.set_transformation(prop, m)
    return cam


# ---- a chromatic medium for the spectral mode ----

def spectral_box(su, width: int, height: int, spp: int, density, position=(2.6, 1.6, -3.0),
                 max_bounces: int = 12, min_bounces: int = 4, integrator=None, medium=None, emission=None,
                 environment=None):
    """The spectral mode's check scene: a [-1, 1]^3 box (a mesh with outward faces) filled with
    a density grid of a chromatic medium (attenuation colour [0.4, 0.6, 0.8] over 0.5 m,
    subsurface colour 0.7, anisotropy 0.4), a sphere light of radius 0.3 (an icosphere mesh,
    radiance [30, 22, 14]) beside it and a uniform environment [0.2, 0.3, 0.5]; PTMIS with the
    renderer's "spectral" key.  Returns the camera entity and the scene as data (world-space
    triangles, per-triangle roles, material parameters as given to su_create_material, the
    density and its world-to-texture map, the camera), from which the oracle renders the same
    image.  medium (Volumetric parameters), emission and environment replace the colours."""
    fov = math.radians(45.0)
    cam = su.su_create_camera_perspective(width, height, fov)
    view = _look_at(position)
    su.set_transformation(cam, view)
    ptmis = {"min_bounces": min_bounces, "max_bounces": max_bounces, "spectral": True}
    ptmis.update(integrator or {})
    su.su_create_integrators(json.dumps({"surface": {"PTMIS": ptmis}}).encode())
    su.su_create_sampler(spp)
    medium = medium or {"attenuation_color": [0.4, 0.6, 0.8], "attenuation_distance": 0.5,
                        "subsurface_color": [0.7, 0.7, 0.7], "anisotropy": 0.4}
    emission = emission or [30.0, 22.0, 14.0]
    environment = environment or [0.2, 0.3, 0.5]
    image = su.image(density)
    m_medium = _material(su, "Volumetric", density={"id": int(image)}, **medium)
    m_lamp = _material(su, "Light", emission=emission)
    m_sky = _material(su, "Light", emission=environment)
    bp, bn, bi = _box_mesh((-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))
    v, f = icosphere(1)
    lp = (0.3 * v + np.array([1.5, 1.4, -1.3], np.float32)).astype(np.float32)
    box_prop = su.prop(su.mesh(bp, bn, bi), [m_medium])
    su.set_transformation(box_prop, np.eye(4, dtype=np.float32))
    lamp_prop = su.prop(su.mesh(lp, v, f), [m_lamp])
    su.set_transformation(lamp_prop, np.eye(4, dtype=np.float32))
    su.su_create_light(lamp_prop)
    sky_prop = su.prop(SHAPE_INFINITE_SPHERE, [m_sky])
    su.set_transformation(sky_prop, np.eye(4, dtype=np.float32))
    su.su_create_light(sky_prop)
    tris = np.concatenate([bp[bi].reshape(-1, 9), lp[f].reshape(-1, 9)]).astype(np.float64)
    roles = np.concatenate([np.ones(len(bi), np.int32), np.zeros(len(f), np.int32)])
    scene = {"triangles": tris, "roles": roles, "medium": medium, "emission": emission,
             "environment": environment, "density": np.asarray(density, np.float64),
             "world_to_uvw": [[0.5, 0.0, 0.0, 0.5], [0.0, 0.5, 0.0, 0.5], [0.0, 0.0, 0.5, 0.5]],
             "camera": {"width": width, "height": height, "fov": fov, "matrix": view},
             "min_bounces": min_bounces, "max_bounces": max_bounces}
    return cam, scene
