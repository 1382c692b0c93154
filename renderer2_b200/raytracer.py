"""Python view of the path tracer entry points (C ABI in include/r2.h).

Mirrors rt::Raytracer (raytracer/raytracer.hpp:29-72): a scene is committed
once (LBVH built on the device) and renderFrame produces the linear radiance
buffer of SFrame::data (3 floats per pixel, row 0 = bottom) before tonemapping.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class Camera(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("fov_deg", C.c_float), ("pos", C.c_float * 3),
                ("look_at", C.c_float * 3), ("up", C.c_float * 3)]


class RenderParams(C.Structure):
    _fields_ = [("spp", C.c_uint32), ("max_depth", C.c_uint32), ("seed", C.c_uint32), ("flags", C.c_uint32)]


BVH_AUTO, BVH_PLOC, BVH_KARRAS = -1, 0, 1


def set_bvh_method(method: int):
    """Hierarchy of the BVHs built from now on, process-wide (r2_set_bvh_method):
    BVH_AUTO (default: PLOC for render scenes, Karras for filter scenes), BVH_PLOC or BVH_KARRAS."""
    N.check(N.lib.r2_set_bvh_method(int(method)))


def bvh_method() -> int:
    return int(N.lib.r2_get_bvh_method())


def camera(width, height, fov_deg=45.0, pos=(0, 0, 3), look_at=(0, 0, 0), up=(0, 1, 0)) -> Camera:
    c = Camera()
    c.width, c.height, c.fov_deg = int(width), int(height), float(fov_deg)
    c.pos[:] = list(map(float, pos))
    c.look_at[:] = list(map(float, look_at))
    c.up[:] = list(map(float, up))
    return c


BRICK_GRID = 1  # R2_RENDER_BRICK_GRID ("UseBrickGrid")


def params(spp=16, max_depth=8, seed=0, brick_grid=False) -> RenderParams:
    p = RenderParams()
    p.spp, p.max_depth, p.seed = int(spp), int(max_depth), int(seed)
    p.flags = BRICK_GRID if brick_grid else 0
    return p


SPHERE, CIRCLE = 0, 1


class Tuning(C.Structure):
    """Launch tuning (r2_render_tuning); 0 fields select the defaults; images never depend on it."""
    _fields_ = [("track_steps", C.c_uint32), ("trav_visits", C.c_uint32), ("trav_refill", C.c_uint32),
                ("wave_paths", C.c_uint32), ("media_rounds", C.c_uint32), ("track_blocks", C.c_uint32),
                ("track_limit", C.c_uint32), ("top_nodes", C.c_uint32), ("sort_rays", C.c_uint32)]
    NAMES = ("track_steps", "trav_visits", "trav_refill", "wave_paths", "media_rounds", "track_blocks",
             "track_limit", "top_nodes", "sort_rays")

    def as_tuple(self):
        return tuple(getattr(self, n) for n in self.NAMES)

    def as_dict(self):
        return dict(zip(self.NAMES, self.as_tuple()))


def tuning(track_steps=0, trav_visits=0, trav_refill=0, wave_paths=0, media_rounds=0, track_blocks=0,
           track_limit=0, top_nodes=0, sort_rays=0) -> Tuning:
    return Tuning(track_steps, trav_visits, trav_refill, wave_paths, media_rounds, track_blocks, track_limit,
                  top_nodes, sort_rays)


class Scene:
    """Device-resident render scene (r2_scene_*)."""

    def __init__(self):
        h = C.c_void_p()
        N.check(N.lib.r2_scene_create(C.byref(h)))
        self.handle = h
        self._keep = []

    def close(self):
        if self.handle:
            N.check(N.lib.r2_scene_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_mesh(self, mesh, material, model_to_world=None, mask=255):
        pos = np.ascontiguousarray(mesh.positions, np.float32)
        idx = np.ascontiguousarray(mesh.indices, np.uint32)
        nrm = np.ascontiguousarray(mesh.normals, np.float32)
        m2w = np.ascontiguousarray(N.identity43() if model_to_world is None else model_to_world, np.float32)
        N.check(N.lib.r2_scene_add_mesh(self.handle, N.ptr(pos), pos.shape[0], N.ptr(idx), idx.shape[0], N.ptr(nrm),
                                        C.byref(material), N.ptr(m2w), mask))

    def add_mesh_textured(self, mesh, material, uv, model_to_world=None, mask=255, albedo=None, specular=None,
                          normal=None, alpha=None):
        """Mesh with texture coordinates (n, 2) and PNG texture maps (r2_scene_add_mesh_textured)."""
        pos = np.ascontiguousarray(mesh.positions, np.float32)
        idx = np.ascontiguousarray(mesh.indices, np.uint32)
        nrm = np.ascontiguousarray(mesh.normals, np.float32)
        uvs = np.ascontiguousarray(uv, np.float32)
        assert uvs.shape == (pos.shape[0], 2)
        m2w = np.ascontiguousarray(N.identity43() if model_to_world is None else model_to_world, np.float32)
        enc = [str(p).encode() if p else None for p in (albedo, specular, normal, alpha)]
        maps = N.MaterialMaps(*enc)
        N.check(N.lib.r2_scene_add_mesh_textured(self.handle, N.ptr(pos), pos.shape[0], N.ptr(idx), idx.shape[0],
                                                 N.ptr(nrm), N.ptr(uvs), C.byref(material), C.byref(maps), N.ptr(m2w),
                                                 mask))

    def add_mesh_asset(self, mesh, material, uv=None, albedo=None, specular=None, normal=None, alpha=None) -> int:
        """A mesh kept in model space with its own BVH, placed by add_mesh_instance (r2_scene_add_mesh_asset)."""
        pos = np.ascontiguousarray(mesh.positions, np.float32)
        idx = np.ascontiguousarray(mesh.indices, np.uint32)
        nrm = np.ascontiguousarray(mesh.normals, np.float32)
        uvs = None if uv is None else np.ascontiguousarray(uv, np.float32)
        maps = None
        if uvs is not None:
            assert uvs.shape == (pos.shape[0], 2)
            maps = N.MaterialMaps(*[str(p).encode() if p else None for p in (albedo, specular, normal, alpha)])
        a = C.c_uint32()
        N.check(N.lib.r2_scene_add_mesh_asset(self.handle, N.ptr(pos), pos.shape[0], N.ptr(idx), idx.shape[0],
                                              N.ptr(nrm), N.ptr(uvs) if uvs is not None else None, C.byref(material),
                                              C.byref(maps) if maps is not None else None, C.byref(a)))
        return a.value

    def add_mesh_instance(self, asset: int, model_to_world=None, mask=255):
        m2w = np.ascontiguousarray(N.identity43() if model_to_world is None else model_to_world, np.float32)
        N.check(N.lib.r2_scene_add_mesh_instance(self.handle, int(asset), N.ptr(m2w), mask))

    def add_shape(self, kind, center, radius, normal, material, mask=255):
        c = np.ascontiguousarray(center, np.float32)
        n = np.ascontiguousarray(normal, np.float32)
        N.check(N.lib.r2_scene_add_shape(self.handle, int(kind), N.ptr(c), float(radius), N.ptr(n), C.byref(material),
                                         mask))

    def add_medium(self, path, sigma_a, sigma_s, pos=(0, 0, 0), orientation=(0, 1, 0), scaling=(1, 1, 1), mask=255,
                   g=None):
        """Medium "Path" of scenedescription.json: loads <path>.nvdb and <path>.brickgrid.
        g (the "G" key) selects the Henyey-Greenstein phase function."""
        arrs = [np.ascontiguousarray(v, np.float32) for v in (sigma_a, sigma_s, pos, orientation, scaling)]
        p = [N.ptr(a) for a in arrs]
        if g is None:
            N.check(N.lib.r2_scene_add_medium(self.handle, str(path).encode(), *p, mask))
        else:
            N.check(N.lib.r2_scene_add_medium_hg(self.handle, str(path).encode(), p[0], p[1], float(g), p[2], p[3],
                                                 p[4], mask))

    def set_envmap(self, rgb: np.ndarray):
        rgb = np.ascontiguousarray(rgb, np.float32)
        h, w, _ = rgb.shape
        N.check(N.lib.r2_scene_set_envmap(self.handle, N.ptr(rgb), w, h))

    def commit(self):
        N.check(N.lib.r2_scene_commit(self.handle))

    def set_vertices(self, positions, normals=None, stream: int = 0, nverts: int = 0):
        """Replace the world-space vertex positions (and normals) of the committed scene, in mesh order: numpy
        arrays, or host addresses (e.g. of pinned tensors, which make the copy asynchronous) with nverts."""
        def addr(a):
            if a is None:
                return None
            if isinstance(a, int):
                return C.c_void_p(a)
            assert a.flags["C_CONTIGUOUS"] and a.dtype == np.float32
            return C.c_void_p(a.ctypes.data)
        n = nverts or positions.size // 3
        N.check(N.lib.r2_scene_set_vertices(self.handle, addr(positions), addr(normals), n,
                                            C.c_void_p(stream or None)))

    def rebuild(self, stream: int = 0):
        """Rebuild the triangle BVH on the device from the resident triangles (waits for the build)."""
        N.check(N.lib.r2_scene_rebuild(self.handle, C.c_void_p(stream or None)))

    def bvh_info(self):
        """(inner nodes, height, kernels launched by the last build) of the surface BVH."""
        v = [C.c_uint32() for _ in range(3)]
        N.check(N.lib.r2_scene_bvh_info(self.handle, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def render_device(self, cam: Camera, prm: RenderParams, d_rgb: int, stream: int = 0, stats=None):
        st = np.zeros(8, np.float64)
        N.check(N.lib.r2_render_device(self.handle, C.byref(cam), C.byref(prm), C.c_void_p(d_rgb),
                                       C.c_void_p(stream or None), N.ptr(st)))
        if stats is not None:
            stats[:] = st
        return st

    def set_tuning(self, t: Tuning):
        N.check(N.lib.r2_scene_set_tuning(self.handle, C.byref(t)))

    def get_tuning(self) -> Tuning:
        t = Tuning()
        N.check(N.lib.r2_scene_get_tuning(self.handle, C.byref(t)))
        return t

    def wave_samples(self, cam: Camera, prm: RenderParams) -> int:
        """Samples of every pixel one wave of this frame renders (r2_scene_wave_samples)."""
        n = C.c_uint32()
        N.check(N.lib.r2_scene_wave_samples(self.handle, C.byref(cam), C.byref(prm), C.byref(n)))
        return n.value

    def autotune(self, cam: Camera, prm: RenderParams) -> Tuning:
        """Times one wave of this frame per candidate setting and keeps the fastest (see r2_scene_autotune)."""
        t = Tuning()
        N.check(N.lib.r2_scene_autotune(self.handle, C.byref(cam), C.byref(prm), C.byref(t)))
        return t

    def render(self, cam: Camera, prm: RenderParams, out_ptr: int = 0) -> np.ndarray:
        """Frame in host memory (r2_render_host): a new array, or the width*height*3 floats at host address out_ptr
        (e.g. a pinned buffer; None is returned then)."""
        if out_ptr:
            N.check(N.lib.r2_render_host(self.handle, C.byref(cam), C.byref(prm), C.c_void_p(out_ptr)))
            return None
        out = np.zeros((cam.height, cam.width, 3), np.float32)
        N.check(N.lib.r2_render_host(self.handle, C.byref(cam), C.byref(prm), N.ptr(out)))
        return out


class RenderBatch:
    """Frames of several committed scenes rendered by one captured CUDA graph
    (r2_render_batch_*); frames are device pointers of width*height*3 floats."""

    def __init__(self, scenes, cams, prms, d_frames):
        n = len(scenes)
        assert len(cams) == n and len(prms) == n and len(d_frames) == n and n > 0
        self._keep = (list(scenes), (Camera * n)(*cams), (RenderParams * n)(*prms))
        sh = (C.c_void_p * n)(*[s.handle for s in scenes])
        fr = (C.c_void_p * n)(*[int(p) for p in d_frames])
        h = C.c_void_p()
        N.check(N.lib.r2_render_batch_create(sh, self._keep[1], self._keep[2], fr, n, C.byref(h)))
        self.handle = h

    def run(self, stream: int = 0, timing: bool = True) -> float:
        """Renders every frame; with timing, waits and returns the device milliseconds."""
        ms = C.c_double(0.0)
        N.check(N.lib.r2_render_batch_run(self.handle, C.c_void_p(stream or None), C.byref(ms) if timing else None))
        return ms.value

    def close(self):
        if self.handle:
            N.check(N.lib.r2_render_batch_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
