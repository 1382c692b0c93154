"""Python view of the filter entry points (C ABI in include/r2.h).

Mirrors the reference's filter interface, filter::CFilter(const SConfig&) and
CFilter::runFiltering() (raytracer/filter.hpp:13-44): a scene is prepared
once (BVH built on the device) and each LOD is filtered into the 32-byte
SFilteredDataCompact layout indexed x + y*nx + z*nx*ny.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _native as N


@dataclass
class Mesh:
    positions: np.ndarray  # (nverts, 3) float32, model space
    indices: np.ndarray    # (ntris, 3) uint32
    normals: np.ndarray    # (nverts, 3) float32

    @property
    def nverts(self) -> int:
        return int(self.positions.shape[0])

    @property
    def ntris(self) -> int:
        return int(self.indices.shape[0])


def material(diffuse=(0.8, 0.8, 0.8), specular=(1.0, 1.0, 1.0), alpha=0.3, ior=1.5, diffuse_roughness=0.0):
    """CMaterial from MTL keys (raytracer/src/material/material.cu:80-148)."""
    m = N.Material()
    m.diffuse[:] = list(diffuse)
    m.specular[:] = list(specular)
    m.alpha_x = m.alpha_y = float(alpha)
    m.eta_i = 1.0
    m.eta_t = float(ior)
    m.diffuse_roughness = float(diffuse_roughness)
    return m


def params(samples_per_voxel=64, iterations=10, sigma_t=10.0, alpha=0.1, clip_rays=True, seed=0,
           min_voxel_size=1.0, lods=1, sggx_projection=False, sggx_floor=0.0):
    """Filter parameters (r2_filter_params); sggx_projection replaces each voxel's mean S by its FP64
    eigendecomposition with eigenvalues floored at sggx_floor times the largest."""
    p = N.FilterParams()
    p.min_voxel_size = float(min_voxel_size)
    p.lods = int(lods)
    p.samples_per_voxel = int(samples_per_voxel)
    p.sigma_t = float(sigma_t)
    p.estimation_iterations = int(iterations)
    p.alpha = float(alpha)
    p.clip_rays = 1 if clip_rays else 0
    p.seed = int(seed)
    p.sggx_projection = 1 if sggx_projection else 0
    p.sggx_floor = float(sggx_floor)
    return p


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class FilterScene:
    """Device-resident FILTER mesh (r2_filter_scene_*)."""

    def __init__(self, mesh: Mesh, mat, model_to_world=None, tex=None):
        """tex (nullable): dict(uv=(nverts, 2), albedo / specular / normal / alpha = PNG paths)."""
        self.mesh = mesh
        self._pos = _c(mesh.positions, np.float32)
        self._idx = _c(mesh.indices, np.uint32)
        self._nrm = _c(mesh.normals, np.float32)
        self._m2w = _c(N.identity43() if model_to_world is None else model_to_world, np.float32)
        self._mat = mat
        h = C.c_void_p()
        if tex is None:
            N.check(N.lib.r2_filter_scene_create(N.ptr(self._pos), mesh.nverts, N.ptr(self._idx), mesh.ntris,
                                                 N.ptr(self._nrm), C.byref(mat), N.ptr(self._m2w), C.byref(h)))
        else:
            self._uv = _c(tex["uv"], np.float32)
            maps = N.MaterialMaps(*[str(tex[k]).encode() if tex.get(k) else None
                                    for k in ("albedo", "specular", "normal", "alpha")])
            N.check(N.lib.r2_filter_scene_create_textured(N.ptr(self._pos), mesh.nverts, N.ptr(self._idx), mesh.ntris,
                                                          N.ptr(self._nrm), N.ptr(self._uv), C.byref(mat),
                                                          C.byref(maps), N.ptr(self._m2w), C.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            N.check(N.lib.r2_filter_scene_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def grid(self, voxel_size: float) -> N.FilterGrid:
        g = N.FilterGrid()
        N.check(N.lib.r2_filter_scene_grid(self.handle, float(voxel_size), C.byref(g)))
        return g

    def run(self, grid, prm, d_out: int, d_wide: int = 0, d_fp16: int = 0, stream: int = 0, stats=None):
        st = np.zeros(4, np.float64)
        N.check(N.lib.r2_filter_scene_run(self.handle, C.byref(grid), C.byref(prm), C.c_void_p(d_out),
                                          C.c_void_p(d_wide or None), C.c_void_p(d_fp16 or None),
                                          C.c_void_p(stream or None), N.ptr(st) if stats is not None else None))
        if stats is not None:
            stats[:] = st[:3]

    def run_eig(self, grid, prm, d_out: int, d_eig: int, d_wide: int = 0, stream: int = 0):
        """The same LOD with the FP64 eigendecomposition of each voxel's mean S in d_eig (12 floats per voxel)."""
        N.check(N.lib.r2_filter_scene_run_eig(self.handle, C.byref(grid), C.byref(prm), C.c_void_p(d_out),
                                              C.c_void_p(d_wide or None), None, C.c_void_p(d_eig),
                                              C.c_void_p(stream or None), None))

    def count(self, grid, prm, d_out: int):
        """Counting build of the same LOD: (rays traced, inner nodes visited, triangles tested)."""
        c = np.zeros(3, np.uint64)
        N.check(N.lib.r2_filter_scene_count(self.handle, C.byref(grid), C.byref(prm), C.c_void_p(d_out), N.ptr(c)))
        return tuple(int(x) for x in c)

    def bvh(self):
        nn = C.c_uint32()
        ht = C.c_uint32()
        N.check(N.lib.r2_filter_scene_bvh(self.handle, None, 0, None, 0, C.byref(nn), C.byref(ht)))
        nodes = np.zeros((nn.value, 16), np.int32)
        order = np.zeros(self.mesh.ntris, np.uint32)
        N.check(N.lib.r2_filter_scene_bvh(self.handle, N.ptr(nodes), nodes.size, N.ptr(order), order.size,
                                          None, None))
        return nodes, order, ht.value


def filter_mesh(mesh: Mesh, mat, prm, voxel_size: float, model_to_world=None, wide=False, out_ptr: int = 0,
                out_capacity: int = 0):
    """One LOD through the host-buffer entry point r2_filter_mesh (upload, BVH
    build, filter, download).  Returns (grid, voxels[, wide]); with out_ptr the
    payloads go to that host address (e.g. a pinned buffer of out_capacity
    voxels) and (grid, None) is returned."""
    pos = _c(mesh.positions, np.float32)
    idx = _c(mesh.indices, np.uint32)
    nrm = _c(mesh.normals, np.float32)
    m2w = _c(N.identity43() if model_to_world is None else model_to_world, np.float32)
    g = N.FilterGrid()
    # grid first, to size the output
    lo = mesh.positions.min(axis=0).astype(np.float32)
    hi = mesh.positions.max(axis=0).astype(np.float32)
    N.check(N.lib.r2_filter_setup_grid(N.ptr(lo), N.ptr(hi), N.ptr(m2w), float(voxel_size), C.byref(g)))
    nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
    if out_ptr:
        assert out_capacity >= nvox and not wide
        N.check(N.lib.r2_filter_mesh(N.ptr(pos), mesh.nverts, N.ptr(idx), mesh.ntris, N.ptr(nrm), C.byref(mat),
                                     N.ptr(m2w), C.byref(prm), float(voxel_size), C.byref(g), C.c_void_p(out_ptr),
                                     None, out_capacity))
        return g, None
    out = np.zeros(nvox, N.VOXEL_DTYPE)
    w = np.zeros((nvox, 20), np.float32) if wide else None
    N.check(N.lib.r2_filter_mesh(N.ptr(pos), mesh.nverts, N.ptr(idx), mesh.ntris, N.ptr(nrm), C.byref(mat),
                                 N.ptr(m2w), C.byref(prm), float(voxel_size), C.byref(g), N.ptr(out), N.ptr(w),
                                 nvox))
    return (g, out, w) if wide else (g, out)


def run_filtering(mesh: Mesh, mat, prm, out_root, model, pos=(0, 0, 0), orientation=(0, 1, 0), scaling=(1, 1, 1)):
    """All LODs of one FILTER object with file outputs (CFilter::runFiltering,
    filter.cu:74-123): <out_root>/<model>/filtered_mesh_<vs>.nvdb and
    .brickgrid per LOD plus <out_root>/volume_description.json.  Returns the
    medium paths (without extension) and the stats
    [lods, voxels, active voxels, kernel ms]."""
    p = _c(mesh.positions, np.float32)
    ix = _c(mesh.indices, np.uint32)
    nr = _c(mesh.normals, np.float32)
    pos3, ori3, sc3 = (_c(v, np.float32) for v in (pos, orientation, scaling))
    st = np.zeros(4)
    N.check(N.lib.r2_filter_run_mesh(N.ptr(p), mesh.nverts, N.ptr(ix), mesh.ntris, N.ptr(nr), C.byref(mat),
                                     N.ptr(pos3), N.ptr(ori3), N.ptr(sc3), C.byref(prm), str(out_root).encode(),
                                     str(model).encode(), N.ptr(st)))
    vs = np.float32(prm.min_voxel_size)
    paths = []
    for _ in range(int(st[0])):
        paths.append(os.path.join(str(out_root), str(model), "filtered_mesh_%f" % float(vs)))
        vs = np.float32(vs * np.float32(2.0))
    return paths, st
