"""Python view of the pipeline entry points (config.json in, files and frames
out), mirroring CPipeline (raytracer/pipeline.cu:18-90): load a config, run
the filter over its FILTER mesh, render a frame, write the output image.

Also writes the input files of a pipeline run (OBJ/MTL meshes, Radiance .hdr
environment maps, scene description and config JSON) for synthetic workloads.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from . import _native as N
from .raytracer import Camera


class ConfigInfo(C.Structure):
    _fields_ = [("frame_width", C.c_uint32), ("frame_height", C.c_uint32), ("channels", C.c_uint32),
                ("samples", C.c_uint32), ("gamma", C.c_float), ("use_brick_grid", C.c_uint32),
                ("filter_active", C.c_uint32), ("filter", N.FilterParams), ("camera", Camera),
                ("env_width", C.c_uint32), ("env_height", C.c_uint32), ("n_shapes", C.c_uint32),
                ("n_meshes", C.c_uint32), ("n_media", C.c_uint32), ("n_triangles", C.c_uint32)]


class RenderOpts(C.Structure):
    _fields_ = [("spp", C.c_uint32), ("max_depth", C.c_uint32), ("seed", C.c_uint32), ("flags", C.c_uint32)]


class Config:
    """r2_config: a loaded config.json with its scene description and assets."""

    def __init__(self, path):
        h = C.c_void_p()
        N.check(N.lib.r2_config_load(str(path).encode(), C.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            N.check(N.lib.r2_config_free(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> ConfigInfo:
        i = ConfigInfo()
        N.check(N.lib.r2_config_info_get(self.handle, C.byref(i)))
        return i

    def filter_run(self, out_root=None):
        st = np.zeros(4)
        N.check(N.lib.r2_filter_run(self.handle, None if out_root is None else str(out_root).encode(), N.ptr(st)))
        return st

    def render(self, spp=0, max_depth=0, seed=0, want_bytes=True):
        """Returns (linear (H, W, 3) float32 with row 0 at the bottom, bytes (H, W, 3) uint8 or None)."""
        i = self.info()
        o = RenderOpts(spp, max_depth, seed, 0)
        lin = np.zeros((i.frame_height, i.frame_width, 3), np.float32)
        by = np.zeros((i.frame_height, i.frame_width, 3), np.uint8) if want_bytes else None
        N.check(N.lib.r2_render(self.handle, C.byref(o), N.ptr(lin), N.ptr(by) if want_bytes else None))
        return lin, by


def tonemap(linear: np.ndarray, gamma: float):
    """r2_tonemap on host arrays: (tonemapped floats, bytes)."""
    lin = np.ascontiguousarray(linear, np.float32)
    h, w = lin.shape[:2]
    out = np.zeros_like(lin)
    by = np.zeros(lin.shape, np.uint8)
    N.check(N.lib.r2_tonemap(N.ptr(lin), w, h, float(gamma), N.ptr(out), N.ptr(by)))
    return out, by


def write_png(path, rgb: np.ndarray, flip_vertical=False):
    a = np.ascontiguousarray(rgb, np.uint8)
    N.check(N.lib.r2_write_png(str(path).encode(), N.ptr(a), a.shape[1], a.shape[0], int(flip_vertical)))


def write_jpg(path, rgb: np.ndarray, flip_vertical=False, quality=100):
    a = np.ascontiguousarray(rgb, np.uint8)
    N.check(N.lib.r2_write_jpg(str(path).encode(), N.ptr(a), a.shape[1], a.shape[0], int(flip_vertical),
                               int(quality)))


def read_png(path):
    """(H, W, 4) uint8 RGBA texels and the file's channel count."""
    w, h, c = C.c_uint32(), C.c_uint32(), C.c_int()
    N.check(N.lib.r2_read_png(str(path).encode(), None, 0, C.byref(w), C.byref(h), C.byref(c)))
    out = np.zeros((h.value, w.value, 4), np.uint8)
    N.check(N.lib.r2_read_png(str(path).encode(), N.ptr(out), out.size, None, None, None))
    return out, c.value


def read_hdr(path) -> np.ndarray:
    w, h = C.c_uint32(), C.c_uint32()
    N.check(N.lib.r2_read_hdr(str(path).encode(), None, 0, C.byref(w), C.byref(h)))
    out = np.zeros((h.value, w.value, 3), np.float32)
    N.check(N.lib.r2_read_hdr(str(path).encode(), N.ptr(out), out.size, None, None))
    return out


def write_hdr(path, rgb: np.ndarray):
    a = np.ascontiguousarray(rgb, np.float32)
    N.check(N.lib.r2_write_hdr(str(path).encode(), N.ptr(a), a.shape[1], a.shape[0]))


def obj_info(directory, filename):
    ns, nv, nt = C.c_uint32(), C.c_uint32(), C.c_uint32()
    m = N.Material()
    N.check(N.lib.r2_obj_info(str(directory).encode(), str(filename).encode(), C.byref(ns), C.byref(nv),
                              C.byref(nt), C.byref(m)))
    return ns.value, nv.value, nt.value, m


# ---------------------------------------------------------------- input files

def write_obj(directory, name, parts):
    """parts: list of (Mesh, kd, ks, ns, ni).  Writes <name>.obj + <name>.mtl
    (one material per part, vertex normals included)."""
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, name + ".mtl"), "w") as f:
        for i, (_, kd, ks, ns, ni) in enumerate(parts):
            f.write(f"newmtl m{i}\nKd {kd[0]:.9g} {kd[1]:.9g} {kd[2]:.9g}\nKs {ks[0]:.9g} {ks[1]:.9g} {ks[2]:.9g}\n"
                    f"Ns {ns:.9g}\nNi {ni:.9g}\n")
    lines = [f"mtllib {name}.mtl"]
    base = 0
    for i, (mesh, *_rest) in enumerate(parts):
        p = np.asarray(mesh.positions, np.float32)
        n = np.asarray(mesh.normals, np.float32)
        lines += ["v %.9g %.9g %.9g" % tuple(map(float, v)) for v in p]
        lines += ["vn %.9g %.9g %.9g" % tuple(map(float, v)) for v in n]
        lines.append(f"usemtl m{i}")
        for t in np.asarray(mesh.indices, np.int64) + 1 + base:
            lines.append("f %d//%d %d//%d %d//%d" % (t[0], t[0], t[1], t[1], t[2], t[2]))
        base += p.shape[0]
    with open(os.path.join(directory, name + ".obj"), "w") as f:
        f.write("\n".join(lines) + "\n")


def write_config(path, scene_objects, envmap, scenedescription, width, height, samples, fov=45.0,
                 cam_pos=(0, 0, 3), look_at=(0, 0, 0), up=(0, 1, 0), gamma=2.0, use_brick_grid=True,
                 filter_active=False, min_voxel_size=1.0, lods=1, samples_per_voxel=100, sigma_t=10.0,
                 iterations=20, alpha=0.1, clip_rays=True):
    """config.json and scenedescription.json with the reference's keys."""
    with open(scenedescription, "w") as f:
        f.write("// scene description\n" + json.dumps(scene_objects, indent=2))
    cfg = {
        "General": {"FrameWidth": width, "FrameHeight": height, "ChannelsPerPixel": 3, "Samples": samples,
                    "Gamma": gamma, "UseBrickGrid": use_brick_grid, "DebugMode": "NONE"},
        "Filtering": {"Active": filter_active, "MinVoxelSize": min_voxel_size, "LODs": lods,
                      "SamplesPerVoxel": samples_per_voxel, "Debug": False, "DebugSamples": 100, "SigmaT": sigma_t,
                      "EstimationIterations": iterations, "Alpha": alpha, "ClipRays": clip_rays},
        "Camera": {"Fov": fov, "Pos": list(cam_pos), "LookAt": list(look_at), "Up": list(up)},
        "Scene": {"Envmap": envmap, "Scenedescription": scenedescription},
    }
    with open(path, "w") as f:
        f.write("/* pipeline config */\n" + json.dumps(cfg, indent=2))
