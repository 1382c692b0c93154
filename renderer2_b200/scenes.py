"""Seeded synthetic inputs of the benchmark configurations.

The reference's thesis assets (Xfrog OBJ trees, 4k HDR maps) are not
available, so each configuration is a seeded generator with the stated shapes
and value distributions; the generators run natively (r2_gen_*).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .filter import Mesh


def icosphere(subdiv: int = 4, amplitude: float = 0.05, seed: int = 1) -> Mesh:
    """Icosphere (20*4^subdiv triangles, radius 1) displaced radially by
    1 + amplitude * valuenoise(4p)."""
    nv = C.c_uint32()
    nt = C.c_uint32()
    N.check(N.lib.r2_gen_icosphere(subdiv, amplitude, seed, None, 0, None, 0, None, C.byref(nv), C.byref(nt)))
    pos = np.zeros((nv.value, 3), np.float32)
    nrm = np.zeros((nv.value, 3), np.float32)
    idx = np.zeros((nt.value, 3), np.uint32)
    N.check(N.lib.r2_gen_icosphere(subdiv, amplitude, seed, N.ptr(pos), pos.size, N.ptr(idx), idx.size,
                                   N.ptr(nrm), None, None))
    return Mesh(pos, idx, nrm)


def foliage(n_quads: int = 500_000, n_branches: int = 20, clustered: float = 0.7, seed: int = 4) -> Mesh:
    """Leaf quads in the unit cube, `clustered` of them around Bezier branches."""
    pos = np.zeros((4 * n_quads, 3), np.float32)
    nrm = np.zeros((4 * n_quads, 3), np.float32)
    idx = np.zeros((2 * n_quads, 3), np.uint32)
    N.check(N.lib.r2_gen_foliage(n_quads, n_branches, clustered, seed, N.ptr(pos), pos.size, N.ptr(idx), idx.size,
                                 N.ptr(nrm), None, None))
    return Mesh(pos, idx, nrm)


def voxel_size_for(mesh: Mesh, n: int) -> float:
    """MinVoxelSize giving n voxels along the longest extent (maxExtent / n)."""
    ext = mesh.positions.max(axis=0) - mesh.positions.min(axis=0)
    return float(np.float32(ext.max()) / np.float32(n))
