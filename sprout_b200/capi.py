"""ctypes binding of the sprout C API (include/sprout.h), for any library that exports it.

``SuLibrary(path)`` binds the su_* functions of a shared library: this package's
libsprout_b200.so (the B200 path tracer) or, in tests, the reference's own libsprout.so --
the same calls drive both, which is what makes one a drop-in for the other.
"""

from __future__ import annotations

import ctypes
import pathlib

import numpy as np

from . import _lib

u32, i32, f32, vp = ctypes.c_uint32, ctypes.c_int32, ctypes.c_float, ctypes.c_void_p
SU_RESOURCE_NULL = 0xFFFFFFFF
SU_UINT8 = 0
SU_FLOAT32 = 2

LOG_FUNC = ctypes.CFUNCTYPE(None, ctypes.c_uint32, ctypes.c_char_p)

PROTOTYPES = {
    "su_platform_revision": (ctypes.c_char_p, []),
    "su_init": (i32, [ctypes.c_bool]),
    "su_release": (i32, []),
    "su_mount": (i32, [ctypes.c_char_p]),
    "su_clear": (i32, []),
    "su_load_take": (i32, [ctypes.c_char_p]),
    "su_create_defaults": (i32, []),
    "su_create_camera": (u32, [ctypes.c_char_p]),
    "su_create_camera_perspective": (u32, [u32, u32, f32]),
    "su_camera_set_resolution": (i32, [u32, u32]),
    "su_create_sampler": (i32, [u32]),
    "su_create_integrators": (i32, [ctypes.c_char_p]),
    "su_create_image": (u32, [u32, u32, u32, u32, u32, u32, u32, vp]),
    "su_create_material": (u32, [ctypes.c_char_p]),
    "su_create_material_from_file": (u32, [ctypes.c_char_p]),
    "su_create_triangle_mesh_async": (u32, [u32, u32, u32, vp, u32, vp, u32, vp, u32, vp, vp, u32, vp]),
    "su_create_triangle_mesh_from_file": (u32, [ctypes.c_char_p]),
    "su_create_prop": (u32, [u32, u32, vp]),
    "su_create_light": (i32, [u32]),
    "su_camera_entity": (u32, []),
    "su_camera_sensor_dimensions": (i32, [vp]),
    "su_entity_allocate_frames": (i32, [u32]),
    "su_entity_transformation": (i32, [u32, vp]),
    "su_entity_set_transformation": (i32, [u32, vp]),
    "su_entity_set_transformation_frame": (i32, [u32, u32, vp]),
    "su_render": (i32, []),
    "su_render_frame": (i32, [u32]),
    "su_export_frame": (i32, [u32]),
    "su_start_render_frame": (i32, [u32]),
    "su_set_expected_iterations": (i32, [u32]),
    "su_render_iteration": (i32, []),
    "su_postprocess": (i32, []),
    "su_copy_framebuffer": (i32, [u32, u32, u32, u32, vp]),
    "su_register_log": (i32, [LOG_FUNC]),
    "su_register_progress": (i32, [vp, vp]),
}


class SuLibrary:
    """The su_* entry points of one shared library."""

    def __init__(self, path=None, log=True):
        path = pathlib.Path(path) if path else _lib.LIBRARY_PATH
        if path == _lib.LIBRARY_PATH:
            self.lib = _lib.load()
        else:
            self.lib = ctypes.CDLL(str(path))
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(self.lib, name)
            fn.restype = res
            fn.argtypes = args
        self.messages = []
        self._log = LOG_FUNC(lambda t, m: self.messages.append((int(t), m.decode(errors="replace"))))
        if log:
            self.lib.su_register_log(self._log)
        self._keep = []  # buffers handed to the library stay alive as long as it might read them

    def __getattr__(self, name):
        return getattr(self.lib, name)

    def mesh(self, positions, normals, indices, parts=None, uvs=None):
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        nrm = np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        idx = np.ascontiguousarray(indices, np.uint32).reshape(-1, 3)
        prt = None if parts is None else np.ascontiguousarray(parts, np.uint32).reshape(-1, 3)
        tex = None if uvs is None else np.ascontiguousarray(uvs, np.float32).reshape(-1, 2)
        self._keep += [pos, nrm, idx, prt, tex]
        return self.lib.su_create_triangle_mesh_async(
            idx.shape[0], pos.shape[0], 3, pos.ctypes.data, 3, nrm.ctypes.data, 0, None,
            0 if tex is None else 2, None if tex is None else tex.ctypes.data,
            idx.ctypes.data, 0 if prt is None else prt.shape[0], None if prt is None else prt.ctypes.data)

    def image(self, pixels):
        """su_create_image of pixels (depth, height, width) or (height, width) for one channel,
        (depth, height, width, channels) for several: uint8 as Byte, anything else as Float."""
        a = np.ascontiguousarray(pixels)
        kind, size = (0, 1) if a.dtype == np.uint8 else (2, 4)
        a = a if a.dtype == np.uint8 else a.astype(np.float32)
        self._keep.append(a)
        c = a.shape[3] if a.ndim == 4 else 1
        d, h, w = a.shape[:3] if a.ndim >= 3 else (1,) + a.shape
        return self.lib.su_create_image(kind, c, w, h, d, 0, size * c, a.ctypes.data)

    def image2d(self, pixels):
        """su_create_image of a 2-D image (height, width, channels): uint8 pixels as Byte (sRGB
        encoded where used as colour), float32 pixels as Float."""
        a = np.ascontiguousarray(pixels)
        h, w, c = a.shape
        kind, size = (0, 1) if a.dtype == np.uint8 else (2, 4)
        a = a if a.dtype == np.uint8 else a.astype(np.float32)
        self._keep.append(a)
        return self.lib.su_create_image(kind, c, w, h, 1, 0, size * c, a.ctypes.data)

    def prop(self, shape, materials):
        mats = np.ascontiguousarray(materials, np.uint32)
        self._keep.append(mats)
        return self.lib.su_create_prop(shape, len(mats), mats.ctypes.data)

    def set_transformation(self, entity, matrix):
        m = np.ascontiguousarray(matrix, np.float32).reshape(16)
        return self.lib.su_entity_set_transformation(entity, m.ctypes.data)

    def render_views(self, views, spp):
        """Renders the engine's scene from several cameras in one call (spb_render_views of the
        sprout_b200 library): views are (width, height, fov_radians, 4x4 row-major
        camera-to-world matrix) tuples; returns one (height, width, 4) float32 image per view."""
        arr = (_lib.View * len(views))()
        total = 0
        for v, (w, h, fov, m) in zip(arr, views):
            v.width, v.height, v.fov = int(w), int(h), float(fov)
            v.transformation[:] = [float(x) for x in np.asarray(m, np.float32).reshape(16)]
            total += int(w) * int(h)
        out = np.zeros(total * 4, np.float32)
        _lib.check(self.lib.spb_render_views(len(views), arr, int(spp), out.ctypes.data))
        images, at = [], 0
        for w, h, _, _ in views:
            images.append(out[at * 4:(at + w * h) * 4].reshape(h, w, 4))
            at += w * h
        return images

    def framebuffer(self, width, height):
        out = np.zeros((height, width, 4), np.float32)
        status = self.lib.su_copy_framebuffer(SU_FLOAT32, width, height, 4, out.ctypes.data)
        return out, status
