"""Host-side mirror of the reference's triangle-mesh tree for batched GPU casts.

The reference traverses one ray at a time on the CPU through
``scene::shape::triangle::bvh::Tree`` (source/core/scene/shape/triangle/bvh/triangle_bvh_tree.hpp):
``Builder_SAH(16, 64, 4).build(tree, ...)`` builds it, ``Tree::intersect`` returns the closest
hit (index, u, v, and the ray's max_t shrunk to the hit t) and ``Tree::intersect_p`` answers
occlusion.  :class:`Tree` keeps those names and meanings for batches of rays:

* ``Tree.build(positions, indices)``           -- Builder_SAH::build
* ``Tree.intersect(rays) -> (ids, t, uv)``      -- Tree::intersect per ray
* ``Tree.intersect_p(rays) -> occluded``        -- Tree::intersect_p per ray

``rays`` is an (n, 8) float32 array in the reference's math::ray order
(origin.xyz, min_t, direction.xyz, max_t).  Hit ids are the caller's triangle indices
(0xFFFFFFFF = miss).  Host numpy arrays go through the copying entry points; CUDA torch
tensors go through the device entry points on the current torch stream.

Errors raise :class:`SproutError` with the library's message; a missing native library
raises ImportError.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

MISS = _lib.SPB_MISS


def _ptr(a) -> int:
    return a.ctypes.data if isinstance(a, np.ndarray) else int(a.data_ptr())


def _is_cuda(a) -> bool:
    return hasattr(a, "is_cuda") and a.is_cuda


class Tree:
    """A BVH over one triangle mesh, resident on the current CUDA device."""

    def __init__(self):
        self._lib = _lib.load()
        handle = ctypes.c_void_p()
        _lib.check(self._lib.spb_tree_create(ctypes.byref(handle)))
        self._handle = handle

    def close(self) -> None:
        if getattr(self, "_handle", None) and self._handle.value:
            _lib.check(self._lib.spb_tree_release(self._handle))
            self._handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def build(self, positions, indices, num_threads: int = 0) -> "Tree":
        pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        idx = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3)
        _lib.check(self._lib.spb_tree_build(self._handle, pos.shape[0], idx.shape[0],
                                            pos.ctypes.data, idx.ctypes.data, num_threads))
        return self

    def info(self) -> dict:
        info = _lib.TreeInfo()
        _lib.check(self._lib.spb_tree_info_get(self._handle, ctypes.byref(info)))
        return {name: getattr(info, name) for name, _ in info._fields_}

    def status(self) -> int:
        """Rays dropped by the kernel's stack guard since the tree was created (normally 0)."""
        out = ctypes.c_uint32()
        _lib.check(self._lib.spb_tree_status(self._handle, ctypes.byref(out)))
        return out.value

    # ---- closest hit -------------------------------------------------------------------
    def intersect(self, rays, out=None, want_uv: bool = False):
        """Closest hit per ray: (ids uint32, t float32[, uv float32 (n, 2)])."""
        if _is_cuda(rays):
            return self._intersect_device(rays, out, want_uv)
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = r.shape[0]
        if out is None:
            ids = np.empty(n, np.uint32)
            ts = np.empty(n, np.float32)
            uv = np.empty((n, 2), np.float32) if want_uv else None
        else:
            ids, ts, uv = out
        _lib.check(self._lib.spb_intersect_host(self._handle, r.ctypes.data, n, ids.ctypes.data,
                                                ts.ctypes.data, uv.ctypes.data if uv is not None else None))
        return (ids, ts, uv) if want_uv else (ids, ts)

    def _intersect_device(self, rays, out, want_uv):
        import torch

        assert rays.dtype == torch.float32 and rays.is_contiguous(), "rays: contiguous float32"
        n = rays.numel() // 8
        if out is None:
            ids = torch.empty(n, dtype=torch.int32, device=rays.device)
            ts = torch.empty(n, dtype=torch.float32, device=rays.device)
            uv = torch.empty((n, 2), dtype=torch.float32, device=rays.device) if want_uv else None
        else:
            ids, ts, uv = out
        stream = torch.cuda.current_stream(rays.device).cuda_stream
        _lib.check(self._lib.spb_intersect_device(self._handle, rays.data_ptr(), n, ids.data_ptr(),
                                                  ts.data_ptr(), uv.data_ptr() if uv is not None else None,
                                                  stream))
        return (ids, ts, uv) if want_uv else (ids, ts)

    def traversal_stats(self, rays) -> dict:
        """Closest-hit cast of a CUDA tensor of rays that also counts the traversal's work:
        {"rays", "node_steps", "triangle_steps"} summed over the batch (nodes visited are 80 B
        each, triangles tested 48 B each)."""
        import torch

        assert _is_cuda(rays) and rays.dtype == torch.float32 and rays.is_contiguous()
        n = rays.numel() // 8
        ids = torch.empty(n, dtype=torch.int32, device=rays.device)
        ts = torch.empty(n, dtype=torch.float32, device=rays.device)
        nodes = ctypes.c_uint64()
        tris = ctypes.c_uint64()
        stream = torch.cuda.current_stream(rays.device).cuda_stream
        _lib.check(self._lib.spb_cast_stats_device(self._handle, rays.data_ptr(), n, ids.data_ptr(),
                                                   ts.data_ptr(), stream, ctypes.byref(nodes),
                                                   ctypes.byref(tris)))
        return {"rays": n, "node_steps": nodes.value, "triangle_steps": tris.value}

    # ---- any hit -------------------------------------------------------------------------
    def intersect_p(self, rays, out=None):
        """Occlusion per ray: uint8 1 if any triangle is hit within [min_t, max_t]."""
        if _is_cuda(rays):
            import torch

            assert rays.dtype == torch.float32 and rays.is_contiguous(), "rays: contiguous float32"
            n = rays.numel() // 8
            occ = out if out is not None else torch.empty(n, dtype=torch.uint8, device=rays.device)
            stream = torch.cuda.current_stream(rays.device).cuda_stream
            _lib.check(self._lib.spb_intersect_p_device(self._handle, rays.data_ptr(), n,
                                                        occ.data_ptr(), stream))
            return occ
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = r.shape[0]
        occ = out if out is not None else np.empty(n, np.uint8)
        _lib.check(self._lib.spb_intersect_p_host(self._handle, r.ctypes.data, n, occ.ctypes.data))
        return occ


# ---- synthetic inputs of the cast benchmark ---------------------------------------------

def sphere_mesh(n: int, amplitude: float = 0.1, seed: int = 1):
    """Displaced tetra-sphere: 4 n^2 triangles (n = 512 gives 1,048,576)."""
    lib = _lib.load()
    nv = ctypes.c_uint32()
    nt = ctypes.c_uint32()
    _lib.check(lib.spb_synth_sphere_mesh(n, amplitude, seed, ctypes.byref(nv), ctypes.byref(nt), None, None))
    pos = np.empty((nv.value, 3), np.float32)
    idx = np.empty((nt.value, 3), np.uint32)
    _lib.check(lib.spb_synth_sphere_mesh(n, amplitude, seed, ctypes.byref(nv), ctypes.byref(nt),
                                         pos.ctypes.data, idx.ctypes.data))
    return pos, idx


def random_rays(count: int, seed: int = 1, first: int = 0, extent: float = 2.0,
                out=None, num_threads: int = 0):
    """Rays with origins uniform in [-extent, extent]^3 and uniform directions, (count, 8)."""
    lib = _lib.load()
    rays = out if out is not None else np.empty((count, 8), np.float32)
    _lib.check(lib.spb_synth_rays(first, count, seed, extent, rays.ctypes.data, num_threads))
    return rays
