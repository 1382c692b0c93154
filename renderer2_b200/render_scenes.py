"""Seeded synthetic render scenes of the benchmark configurations."""
from __future__ import annotations

import numpy as np

from . import filter as F
from . import raytracer as R
from . import scenes


def white_env(w: int = 4, h: int = 2) -> np.ndarray:
    """Constant white environment (radiance 1 in every direction)."""
    return np.ones((h, w, 3), np.float32)


def lognormal_env(w: int = 512, h: int = 256, sigma: float = 1.5, seed: int = 3) -> np.ndarray:
    """Procedural HDR map: every channel of every texel ~ lognormal(0, sigma)."""
    rng = np.random.default_rng(seed)
    return rng.lognormal(0.0, sigma, size=(h, w, 3)).astype(np.float32)


def translate43(x, y, z):
    m = np.zeros(12, np.float32)
    m[0] = m[4] = m[8] = 1.0
    m[9:12] = (x, y, z)
    return m


def icosphere_scene():
    """Small plain scene: icosphere sub 4 (5,120 tris), GGX roughness 0.3 albedo 0.8, constant white env;
    camera (0,0,3) -> origin, fov 45."""
    mesh = scenes.icosphere(4, 0.05, 1)
    mat = F.material(diffuse=(0.8, 0.8, 0.8), specular=(1.0, 1.0, 1.0), alpha=0.3, ior=1.5)
    desc = {"meshes": [(mesh, mat, translate43(0, 0, 0))], "shapes": [], "env": white_env()}
    cam = R.camera(256, 256, 45.0, (0, 0, 3), (0, 0, 0), (0, 1, 0))
    return desc, cam


def icosphere_grid_scene():
    """Surface path-tracing scene: 8x8 grid of displaced icospheres (64 x 5,120 = 327,680 tris), per-object GGX
    roughness U[0.05, 1] and albedo U[0.2, 0.9] (seed 2), lognormal(0, 1.5) 512x256 env (seed 3)."""
    rng = np.random.default_rng(2)
    meshes = []
    for k in range(64):
        i, j = k % 8, k // 8
        mesh = scenes.icosphere(4, 0.05, k + 1)
        a = float(rng.uniform(0.05, 1.0))
        alb = float(rng.uniform(0.2, 0.9))
        mat = F.material(diffuse=(alb, alb, alb), specular=(1.0, 1.0, 1.0), alpha=a, ior=1.5)
        meshes.append((mesh, mat, translate43(-8.75 + 2.5 * i, -8.75 + 2.5 * j, 0.0)))
    desc = {"meshes": meshes, "shapes": [], "env": lognormal_env()}
    cam = R.camera(1024, 1024, 45.0, (0, 0, 24), (0, 0, 0), (0, 1, 0))
    return desc, cam


def volume_scene(work_dir, index: int = 0, grid: int = 256, n_quads: int = 200_000, ico_subdiv: int = 6,
                 width: int = 1920, height: int = 1080, filter_spv: int = 64, filter_iters: int = 10):
    """Batched-volume scene `index` (seed 5 + index): a foliage grid filtered on the GPU
    (LOD 0 NanoVDB + brick grid written under work_dir, grid^3 voxels) as an
    SGGX medium scaled to a 4-unit cube, a displaced icosphere (20 * 4^ico_subdiv
    triangles) beside it, a ground disc and a lognormal(0, 1.5) environment;
    1920x1080 camera, fov 60.  sigma_s = 10 (the filter's SigmaT), sigma_a = 0."""
    seed = 5 + index
    leaves = scenes.foliage(n_quads, 20, 0.7, seed)
    mat = F.material(diffuse=(0.15, 0.55, 0.1), specular=(0.05, 0.05, 0.05), alpha=0.45, ior=1.5)
    prm = F.params(samples_per_voxel=filter_spv, iterations=filter_iters,
                   min_voxel_size=scenes.voxel_size_for(leaves, grid), lods=1)
    paths, _ = F.run_filtering(leaves, mat, prm, work_dir, f"foliage{index}")
    ico = scenes.icosphere(ico_subdiv, 0.08, seed)
    m2w = np.zeros(12, np.float32)
    m2w[0] = m2w[4] = m2w[8] = 1.5
    m2w[9:12] = (6.5, 1.5, 2.0)
    desc = {
        "meshes": [(ico, F.material(diffuse=(0.7, 0.6, 0.5), specular=(1, 1, 1), alpha=0.25, ior=1.5), m2w)],
        "shapes": [(R.CIRCLE, (0.0, -0.01, 0.0), 1000.0, (0, 1, 0),
                    F.material(diffuse=(0.4, 0.35, 0.3), specular=(0.2, 0.2, 0.2), alpha=0.8, ior=1.3,
                               diffuse_roughness=0.5))],
        "media": [(paths[0], (0.0, 0.0, 0.0), (10.0, 10.0, 10.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), (4.0, 4.0, 4.0))],
        "env": lognormal_env(512, 256, 1.5, seed),
    }
    cam = R.camera(width, height, 60.0, (3.0, 3.0, 13.0), (3.5, 1.8, 2.0), (0, 1, 0))
    return desc, cam


def build_scene(desc) -> R.Scene:
    sc = R.Scene()
    for entry in desc.get("meshes", []):
        mesh, mat, m2w = entry[:3]
        tex = entry[3] if len(entry) > 3 else None
        if tex is None:
            sc.add_mesh(mesh, mat, m2w)
        else:
            sc.add_mesh_textured(mesh, mat, tex["uv"], m2w, albedo=tex.get("albedo"), specular=tex.get("specular"),
                                 normal=tex.get("normal"), alpha=tex.get("alpha"))
    for kind, c, r, n, mat in desc.get("shapes", []):
        sc.add_shape(kind, c, r, n, mat)
    for med in desc.get("media", []):
        path, sa, ss, pos, ori, scl = med[:6]
        g = med[6] if len(med) > 6 else None
        sc.add_medium(path, sa, ss, pos, ori, scl, g=g)
    sc.set_envmap(desc["env"])
    sc.commit()
    return sc
