"""Seeded synthetic inputs of the benchmark configurations.

The reference's thesis assets (Xfrog OBJ trees, 4k HDR maps) are not
available, so each configuration is a seeded generator with the stated shapes
and value distributions.  The generators are plain numpy (no native code), so
that the CPU baseline builds the same inputs without loading the GPU library.
Random values come from Philox4x32-10 (Salmon et al., SC 2011) keyed by the
seed, one counter block per lattice point or per quad, so every output is a
pure function of the parameters.
"""
from __future__ import annotations

import numpy as np

from .filter import Mesh

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
_LO = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32 with 10 rounds over arrays of counters (uint32); returns 4 uint32 arrays."""
    c0, c1, c2, c3 = (np.asarray(x, np.uint32) for x in (c0, c1, c2, c3))
    c0, c1, c2, c3 = np.broadcast_arrays(c0, c1, c2, c3)
    c0, c1, c2, c3 = (x.copy() for x in (c0, c1, c2, c3))
    k0, k1 = np.uint32(k0), np.uint32(k1)
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = c0.astype(np.uint64) * _M0
            p1 = c2.astype(np.uint64) * _M1
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & _LO).astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & _LO).astype(np.uint32)
            c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
            k0 = np.uint32(k0 + _W0)
            k1 = np.uint32(k1 + _W1)
    return c0, c1, c2, c3


def _u53(a, b):
    """Uniform doubles in [0, 1) with 53 random bits from two uint32 words."""
    return ((a >> np.uint32(5)).astype(np.float64) * 67108864.0 + (b >> np.uint32(6)).astype(np.float64)) * (
        1.0 / 9007199254740992.0)


def value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Value noise at points p (n x 3, float64): smoothstep interpolation of hashed lattice values in [-1, 1]."""
    f = np.floor(p)
    i = f.astype(np.int64)
    t = p - f
    t = t * t * (3.0 - 2.0 * t)
    c = np.empty((p.shape[0], 2, 2, 2))
    for dz in range(2):
        for dy in range(2):
            for dx in range(2):
                h, _, _, _ = philox4x32_10((i[:, 0] + dx).astype(np.uint32), (i[:, 1] + dy).astype(np.uint32),
                                           (i[:, 2] + dz).astype(np.uint32), 0x9E37, seed, 0x7F4A7C15)
                c[:, dz, dy, dx] = h.astype(np.float64) * (2.0 / 4294967295.0) - 1.0
    tx, ty, tz = t[:, 0], t[:, 1], t[:, 2]
    x00 = c[:, 0, 0, 0] + (c[:, 0, 0, 1] - c[:, 0, 0, 0]) * tx
    x10 = c[:, 0, 1, 0] + (c[:, 0, 1, 1] - c[:, 0, 1, 0]) * tx
    x01 = c[:, 1, 0, 0] + (c[:, 1, 0, 1] - c[:, 1, 0, 0]) * tx
    x11 = c[:, 1, 1, 0] + (c[:, 1, 1, 1] - c[:, 1, 1, 0]) * tx
    y0 = x00 + (x10 - x00) * ty
    y1 = x01 + (x11 - x01) * ty
    return y0 + (y1 - y0) * tz


def smooth_normals(pos: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """Area-weighted vertex normals: the sum of the adjacent faces' cross products, normalised."""
    p = pos.astype(np.float64)
    e1 = p[idx[:, 1]] - p[idx[:, 0]]
    e2 = p[idx[:, 2]] - p[idx[:, 0]]
    n = np.cross(e1, e2)
    acc = np.zeros_like(p)
    for k in range(3):
        np.add.at(acc, idx[:, k], n)
    ln = np.sqrt((acc * acc).sum(axis=1))
    ln[ln == 0.0] = 1.0
    return (acc / ln[:, None]).astype(np.float32)


_ICO_FACES = np.array([0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1,
                       8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1],
                      np.int64).reshape(20, 3)


def icosphere(subdiv: int = 4, amplitude: float = 0.05, seed: int = 1) -> Mesh:
    """Icosphere (20*4^subdiv triangles, radius 1) displaced radially by
    1 + amplitude * valuenoise(4p).  Each subdivision splits every face into
    four; an edge's midpoint vertex is numbered in the order the faces first
    reach the edge."""
    if subdiv > 9:
        raise ValueError("subdivision level above 9")
    t = (1.0 + np.sqrt(5.0)) / 2.0
    P = np.array([-1, t, 0, 1, t, 0, -1, -t, 0, 1, -t, 0, 0, -1, t, 0, 1, t, 0, -1, -t, 0, 1, -t, t, 0, -1, t, 0, 1,
                  -t, 0, -1, -t, 0, 1], np.float64).reshape(12, 3)
    P /= np.sqrt((P * P).sum(axis=1))[:, None]
    F = _ICO_FACES.copy()
    for _ in range(subdiv):
        a, b, c = F[:, 0], F[:, 1], F[:, 2]
        e = np.stack([np.stack([a, b], 1), np.stack([b, c], 1), np.stack([c, a], 1)], 1).reshape(-1, 2)
        e.sort(axis=1)
        key = e[:, 0] * np.int64(P.shape[0]) + e[:, 1]
        uk, first, inv = np.unique(key, return_index=True, return_inverse=True)
        order = np.argsort(first, kind="stable")  # unique edges in first-encounter order
        rank = np.empty_like(order)
        rank[order] = np.arange(order.size)
        ev = e[first[order]]
        mid = 0.5 * (P[ev[:, 0]] + P[ev[:, 1]])
        mid /= np.sqrt((mid * mid).sum(axis=1))[:, None]
        m = (P.shape[0] + rank[inv]).reshape(-1, 3)
        ab, bc, ca = m[:, 0], m[:, 1], m[:, 2]
        F = np.stack([a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca], 1).reshape(-1, 3)
        P = np.concatenate([P, mid])
    r = 1.0 + float(amplitude) * value_noise(4.0 * P, seed)
    pos = (P * r[:, None]).astype(np.float32)
    idx = F.astype(np.uint32)
    return Mesh(pos, idx, smooth_normals(pos, idx))


def foliage(n_quads: int = 500_000, n_branches: int = 20, clustered: float = 0.7, seed: int = 4) -> Mesh:
    """Leaf quads in the unit cube: a fraction `clustered` Gaussian (sigma 0.02)
    around n_branches cubic Bezier curves (control points U[0.1, 0.9]^3), the
    rest uniform; random orientation (normal uniform on the sphere, in-plane
    rotation uniform), edge U[0.005, 0.02].  Quad q draws its values from
    Philox blocks (q, slot) under key (seed, 1)."""
    q = np.arange(n_quads, dtype=np.uint64)

    def draws(slot):  # two uniforms per Philox block
        a, b, c, d = philox4x32_10((q & _LO).astype(np.uint32), (q >> np.uint64(32)).astype(np.uint32),
                                   np.uint32(slot), 0x51A7, seed, 1)
        return _u53(a, b), _u53(c, d)

    cc, _ = philox4x32_10(np.arange(3 * max(n_branches, 1) * 4, dtype=np.uint32), 0, 0, 0xB7A9, seed, 2)[:2]
    ctrl = 0.1 + 0.8 * (cc.astype(np.float64) / 4294967296.0)
    ctrl = ctrl.reshape(max(n_branches, 1), 4, 3)
    u_cl, u_br = draws(0)
    u_t, u_n0 = draws(1)
    u_n1, u_n2 = draws(2)
    u_n3, u_n4 = draws(3)
    u_n5, u_x = draws(4)
    u_y, u_z = draws(5)
    u_zn, u_phi = draws(6)
    u_rot, u_h = draws(7)
    is_cl = (u_cl < clustered) & (n_branches > 0)
    br = np.minimum((u_br * n_branches).astype(np.int64), max(n_branches - 1, 0))
    it = 1.0 - u_t
    w = np.stack([it * it * it, 3 * u_t * it * it, 3 * u_t * u_t * it, u_t * u_t * u_t], 1)
    curve = np.einsum("qj,qjk->qk", w, ctrl[br])

    def gauss(a, b):  # Box-Muller
        a = np.maximum(a, 1e-300)
        return np.sqrt(-2.0 * np.log(a)) * np.cos(2.0 * np.pi * b)

    jit = np.stack([gauss(u_n0, u_n1), gauss(u_n2, u_n3), gauss(u_n4, u_n5)], 1)
    c = np.where(is_cl[:, None], curve + 0.02 * jit, np.stack([u_x, u_y, u_z], 1))
    c = np.clip(c, 0.0, 1.0)
    z = 1.0 - 2.0 * u_zn
    phi = 2.0 * np.pi * u_phi
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    n = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    big = np.abs(n[:, 0]) > 0.9
    a = np.stack([np.where(big, 0.0, 1.0), np.where(big, 1.0, 0.0), np.zeros(n_quads)], 1)
    t1 = np.cross(n, a)
    t1 /= np.sqrt((t1 * t1).sum(axis=1))[:, None]
    t2 = np.cross(n, t1)
    rot = 2.0 * np.pi * u_rot
    cr, sr = np.cos(rot)[:, None], np.sin(rot)[:, None]
    u = cr * t1 + sr * t2
    v = -sr * t1 + cr * t2
    h = (0.5 * (0.005 + 0.015 * u_h))[:, None]
    sgn = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], np.float64)
    pos = c[:, None, :] + h[:, None, :] * (sgn[None, :, 0:1] * u[:, None, :] + sgn[None, :, 1:2] * v[:, None, :])
    pos = pos.reshape(-1, 3).astype(np.float32)
    nrm = np.repeat(n, 4, axis=0).astype(np.float32)
    base = (4 * np.arange(n_quads, dtype=np.uint32))[:, None]
    idx = (base + np.array([0, 1, 2, 0, 2, 3], np.uint32)[None, :]).reshape(-1, 3)
    return Mesh(pos, idx.astype(np.uint32), nrm)


def voxel_size_for(mesh: Mesh, n: int) -> float:
    """MinVoxelSize giving n voxels along the longest extent (maxExtent / n)."""
    ext = mesh.positions.max(axis=0) - mesh.positions.min(axis=0)
    return float(np.float32(ext.max()) / np.float32(n))
