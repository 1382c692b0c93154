"""Seeded synthetic render scenes of the benchmark configurations."""
from __future__ import annotations

import json
import os

import numpy as np

from . import filter as F
from . import forest as FO
from . import pipeline as P
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


def trs43(pos, axis_angle=(0.0, 1.0, 0.0, 0.0), scale=(1.0, 1.0, 1.0)):
    """T * R * S as 12 floats (glm mat4x3 column order); R rotates by angle
    (radians) about the axis."""
    ax = np.asarray(axis_angle[:3], np.float64)
    ax = ax / np.linalg.norm(ax)
    a = float(axis_angle[3])
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    Rm = np.eye(3) + np.sin(a) * K + (1 - np.cos(a)) * K @ K
    M = Rm @ np.diag(np.asarray(scale, np.float64))
    m = np.zeros(12, np.float32)
    m[0:3], m[3:6], m[6:9] = M[:, 0], M[:, 1], M[:, 2]
    m[9:12] = pos
    return m


def instanced_scene(n_side: int = 3, width: int = 64, height: int = 64):
    """Two-level scene: one displaced icosphere (sub 3) placed n_side^2 times
    with rotations and non-uniform scales (one asset, one material), a second
    icosphere as a world-space mesh, a ground disc and a lognormal(0, 1.5)
    environment."""
    ico = scenes.icosphere(3, 0.08, 7)
    mat = F.material(diffuse=(0.7, 0.5, 0.3), specular=(1.0, 1.0, 1.0), alpha=0.35, ior=1.5)
    rng = np.random.default_rng(17)
    meshes = []
    for k in range(n_side * n_side):
        i, j = k % n_side, k // n_side
        axis = rng.normal(size=3)
        meshes.append((ico, mat, trs43((-2.2 * (n_side - 1) / 2 + 2.2 * i, -2.2 * (n_side - 1) / 2 + 2.2 * j, 0.0),
                                       (*axis, float(rng.uniform(0, np.pi))), tuple(rng.uniform(0.6, 1.1, 3)))))
    other = scenes.icosphere(2, 0.05, 9)
    meshes.append((other, F.material(diffuse=(0.2, 0.6, 0.8), specular=(0.5, 0.5, 0.5), alpha=0.2, ior=1.5),
                   trs43((0.0, 0.0, 2.0), scale=(0.7, 0.7, 0.7))))
    ground = F.material(diffuse=(0.5, 0.5, 0.5), specular=(0.04, 0.04, 0.04), alpha=0.8, ior=1.5)
    desc = {"meshes": meshes, "shapes": [(R.CIRCLE, (0.0, -3.6, 0.0), 50.0, (0.0, 1.0, 0.0), ground)],
            "env": lognormal_env(64, 32, 1.5, 4)}
    cam = R.camera(width, height, 50.0, (0.5, 1.0, 9.0), (0, 0, 0), (0, 1, 0))
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


def world_vertices(desc):
    """World-space vertex positions and normals of the scene's meshes in the order build_scene adds them (the
    layout r2_scene_set_vertices takes), transformed with the library's float operation order."""
    P, Nn = [], []
    for entry in desc.get("meshes", []):
        mesh, _, m2w = entry[:3]
        m = np.asarray(m2w, np.float32).reshape(4, 3)
        p = mesh.positions.astype(np.float32)
        n = mesh.normals.astype(np.float32)
        wp = (((m[0] * p[:, :1] + m[1] * p[:, 1:2]) + m[2] * p[:, 2:3]) + m[3] * np.float32(1.0)).astype(np.float32)
        wn = (((m[0] * n[:, :1] + m[1] * n[:, 1:2]) + m[2] * n[:, 2:3]) + m[3] * np.float32(0.0)).astype(np.float32)
        P.append(wp)
        Nn.append(wn)
    return np.ascontiguousarray(np.concatenate(P)), np.ascontiguousarray(np.concatenate(Nn))


def mesh_groups(desc):
    """Indices of desc["meshes"] entries that share one mesh object and one
    material object (instances of one asset), for the groups of two or more."""
    groups = {}
    for k, entry in enumerate(desc.get("meshes", [])):
        groups.setdefault((id(entry[0]), id(entry[1])), []).append(k)
    return [g for g in groups.values() if len(g) > 1]


def build_scene(desc, instancing: bool = True) -> R.Scene:
    """The scene of a description; with instancing, meshes that share their mesh
    and material objects become one asset with an instance each (two-level BVH)."""
    sc = R.Scene()
    grouped = {}
    if instancing:
        for g in mesh_groups(desc):
            for k in g:
                grouped[k] = g[0]
    assets = {}
    for k, entry in enumerate(desc.get("meshes", [])):
        mesh, mat, m2w = entry[:3]
        tex = entry[3] if len(entry) > 3 else None
        if k in grouped:
            first = grouped[k]
            if first not in assets:
                t = tex or {}
                assets[first] = sc.add_mesh_asset(mesh, mat, uv=t.get("uv"), albedo=t.get("albedo"),
                                                  specular=t.get("specular"), normal=t.get("normal"),
                                                  alpha=t.get("alpha"))
            sc.add_mesh_instance(assets[first], m2w)
        elif tex is None:
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


# ---------------------------------------------------------------- forests

# (name, size class, expected height, seed) of the synthetic tree library
TREE_SPECS = (("FA01", "Large", 20.0, 11), ("FB02", "Medium", 8.0, 12), ("FC03", "Small", 2.5, 13))
# the forest generator's camera (generate_random_forest.py:257): pos, look-at, up, fov
FOREST_CAMERA = ((-680.0, 35.1, 680.0), (-675.0, 31.5, 675.0), (0.0, 1.0, 0.0), 90.0)
FOREST_SIGMA_A = (0.0, 0.0, 0.0)
FOREST_SIGMA_S = (10.0, 10.0, 10.0)  # the generator's media (toFile, common_functions.py:88-89)


def tree_mesh(seed: int, n_quads: int) -> F.Mesh:
    """A slender synthetic tree: foliage quads squeezed to 0.3 x 1 x 0.3."""
    m = scenes.foliage(n_quads, 8, 0.7, seed)
    sc = np.array([0.3, 1.0, 0.3], np.float32)
    nrm = m.normals / sc
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    return F.Mesh((m.positions * sc).astype(np.float32), m.indices, nrm.astype(np.float32))


def forest_library(work_dir, n_quads: int = 20_000, grid: int = 64, lods: int = 4, filter_spv: int = 32,
                   filter_iters: int = 10) -> dict:
    """Synthetic tree models for forest scenes: per TREE_SPECS entry a tree
    mesh written as an OBJ asset and filtered on the GPU into `lods` LODs
    (finest: grid voxels along the height), with the volume description the
    filter writes.  Returns {relevant_models, volume_descriptions, assets_root,
    filtering_root, meshes}."""
    work_dir = str(work_dir)
    filtering_root = os.path.join(work_dir, "filtering")
    assets_root = os.path.join(work_dir, "assets")
    relevant = {"Large": [], "Medium": [], "Small": []}
    meshes = {}
    mat = F.material(diffuse=(0.15, 0.55, 0.1), specular=(0.05, 0.05, 0.05), alpha=0.45, ior=1.5)
    for name, group, height, seed in TREE_SPECS:
        mesh = tree_mesh(seed, n_quads)
        prm = F.params(samples_per_voxel=filter_spv, iterations=filter_iters,
                       min_voxel_size=scenes.voxel_size_for(mesh, grid), lods=lods)
        F.run_filtering(mesh, mat, prm, filtering_root, name)
        P.write_obj(os.path.join(assets_root, "Synthetic", name), name,
                    [(mesh, (0.15, 0.55, 0.1), (0.05, 0.05, 0.05), 8.0, 1.5)])
        ext = mesh.positions.max(axis=0) - mesh.positions.min(axis=0)
        relevant[group].append({"Name": name, "Path": f"Synthetic/{name}", "Dimensions": [float(x) for x in ext],
                                "ExpectedHeight": height, "Orientation": [0.0, 1.0, 0.0]})
        meshes[name] = mesh
    with open(os.path.join(filtering_root, "volume_description.json")) as f:
        volumes = json.load(f)
    return {"relevant_models": relevant, "volume_descriptions": volumes, "assets_root": assets_root,
            "filtering_root": filtering_root, "meshes": meshes}


def forest_trees(lib: dict, attempts: int, radius: float, width: int, height: int, min_lod: float = 0.0,
                 covered_pixels: float = 1.0, camera=FOREST_CAMERA, seed: int = 0, placed: list = None) -> list:
    """The generator's scene list for a forest of the library's trees: dart
    throwing in a disc of `radius` (or the trees `placed` earlier), LODs
    chosen on the GPU for a width x height sensor at `camera`."""
    pos, look, up, fov = camera
    cam = FO.lod_camera(pos, look, up, width, height, fov)
    return FO.generate_forest(lib["relevant_models"], lib["volume_descriptions"], cam, False, min_lod,
                              covered_pixels, attempts, seed, radius, assets_root=lib["assets_root"] + "/",
                              filtering_root=lib["filtering_root"] + "/", placed=placed)


def forest_ground():
    """The generator's ground disc (toFile, common_functions.py:92-104)."""
    m = F.material(diffuse=(0.07, 0.07, 0.01), specular=(0.9, 0.9, 0.9), alpha=0.99, ior=1.2,
                   diffuse_roughness=0.999)
    m.eta_i = 1.00029
    return (R.CIRCLE, (0.0, 0.0, 0.0), 3.402823466e+38, (0.0, 1.0, 0.0), m)


def forest_desc(lib: dict, trees: list, env_seed: int = 3, media_only: bool = False) -> dict:
    """Scene description of a forest scene list: a medium instance per
    medium tree (files shared by path), the tree mesh per mesh tree (or, with
    media_only, its finest LOD instead), the ground disc and a lognormal
    environment."""
    mat = F.material(diffuse=(0.15, 0.55, 0.1), specular=(0.05, 0.05, 0.05), alpha=0.45, ior=1.5)
    finest = {name: sorted(lods, key=float)[0] for name, lods in lib["volume_descriptions"].items()}
    desc = {"meshes": [], "media": [], "shapes": [forest_ground()], "env": lognormal_env(512, 256, 1.5, env_seed)}
    for kind, directory, filename, pos, ori, scl in trees:
        assert tuple(ori) == (0.0, 1.0, 0.0), "synthetic trees stand upright"
        if kind == "Mesh":
            name = filename[:-4]
            if media_only:
                kind, directory, filename = "Medium", lib["filtering_root"] + "/" + name + "/", \
                    "filtered_mesh_" + finest[name]
            else:
                m2w = np.zeros(12, np.float32)
                m2w[0], m2w[4], m2w[8] = scl
                m2w[9:12] = pos
                desc["meshes"].append((lib["meshes"][name], mat, m2w))
                continue
        desc["media"].append((directory + "/" + filename, FOREST_SIGMA_A, FOREST_SIGMA_S, tuple(pos), tuple(ori),
                              tuple(scl)))
    return desc


def forest_config(lib: dict, trees: list, work_dir, width: int, height: int, samples: int,
                  camera=FOREST_CAMERA) -> str:
    """config.json + scenedescription.json (the generator's object format) and
    the environment map for a forest scene list; returns the config path."""
    work_dir = str(work_dir)
    env = os.path.join(work_dir, "forest_env.hdr")
    P.write_hdr(env, lognormal_env(512, 256, 1.5, 3))
    sd = os.path.join(work_dir, "scenedescription_forest.json")
    cfg = os.path.join(work_dir, "config_forest.json")
    pos, look, up, fov = camera
    P.write_config(cfg, FO.scene_objects(trees), env, sd, width, height, samples, fov=fov, cam_pos=pos,
                   look_at=look, up=up, use_brick_grid=True)
    return cfg
