"""Many-instance forest scenes with screen-space LOD selection.

Restates the reference's forest generator
(raytracer/src/filtering/generate_random_forest.py, common_functions.py):
trees are placed by dart throwing in a disc with a collision test over
distance classes (generateRandomForest 250-300, sampleModelPosition 48-71,
uniformSampleCircle 14-17, checkCollision 227-231,
getRelevantAccelerationClasses 235-247), and each placed tree gets the LOD
whose voxels best match the pixels it covers (selectLOD 179-225).  The
selection runs for all trees in one GPU launch (``r2_select_lods``); the
placement draws the same random numbers in the same order as the generator
(numpy's legacy generator, seed 0 by default), so the same inputs give the
same forest.  The scene list and the file written by ``write_scene`` have the
generator's format (toFile, common_functions.py:69-106).
"""
from __future__ import annotations

import ctypes as C
import json
import math

import numpy as np

from . import _native as N

RADIUS = 1000
ACCEL_CLASSES = 10
TREE_CDF = (0.9, 0.98, 1.0)  # large, medium, small


def look_at(eye, center, up) -> np.ndarray:
    """World-to-view matrix (common_functions.py:20-39)."""
    eye = np.array(eye)
    center = np.array(center)
    up = np.array(up)
    g = center - eye
    w = -g / np.linalg.norm(g)
    u = np.cross(up, w)
    u /= np.linalg.norm(u)
    v = np.cross(w, u)
    m1 = np.array([[u[0], u[1], u[2], 0], [v[0], v[1], v[2], 0], [w[0], w[1], w[2], 0], [0, 0, 0, 1]])
    m2 = np.array([[1, 0, 0, -eye[0]], [0, 1, 0, -eye[1]], [0, 0, 1, -eye[2]], [0, 0, 0, 1]])
    return np.matmul(m1, m2)


def far_scale() -> float:
    """intersectBB's far-distance factor 1 + 2 * gamma(3), gamma(n) = n eps / (1 - n eps)
    with float32 eps (generate_random_forest.py:132-133, 147)."""
    eps = np.finfo(np.float32).eps
    g = (3 * eps) / (1 - 3 * eps)
    return float(1 + 2 * g)


def lod_camera(pos, lookat, up, sensor_width: int, sensor_height: int, fov: float) -> dict:
    """The generator's camera (getCamera, common_functions.py:41-67) plus its
    native record for r2_select_lods."""
    w2v = look_at(pos, lookat, up)
    pixel_size = 1.e-5
    near = (sensor_width * pixel_size) / (2.0 * math.tan(math.radians(fov) / 2.0))
    cam = {"Pos": np.array(pos), "LookAt": np.array(lookat), "Up": np.array(up), "WorldToView": w2v,
           "SensorWidth": sensor_width, "SensorHeight": sensor_height, "Fov": fov, "NearPlaneDistance": near,
           "PixelSize": pixel_size}
    rec = np.zeros(1, N.LOD_CAMERA_DTYPE)
    rec["world_to_view"][0] = np.asarray(w2v, np.float64).reshape(16)
    rec["pos"][0] = np.asarray(cam["Pos"], np.float64)
    rec["near_plane_distance"] = near
    rec["pixel_size"] = pixel_size
    rec["pixel_area"] = pixel_size ** 2
    rec["sensor_width"] = sensor_width
    rec["sensor_height"] = sensor_height
    rec["far_scale"] = far_scale()
    cam["native"] = rec
    return cam


def max_bounds(volume_descriptions: dict) -> dict:
    """Per model the union of its LODs' boxes (getMaxBounds, common_functions.py:5-17)."""
    out = {}
    for name, values in volume_descriptions.items():
        first = values[list(values.keys())[0]]
        bbmin, bbmax = list(first["BBMin"]), list(first["BBMax"])
        for lod in values.values():
            bbmin = [min(bbmin[k], lod["BBMin"][k]) for k in range(3)]
            bbmax = [max(bbmax[k], lod["BBMax"][k]) for k in range(3)]
        out[name] = {"BBMin": bbmin, "BBMax": bbmax}
    return out


class LodTable:
    """The volume descriptions of some models as the native LOD table: model
    m's LODs in the order selectLOD walks them (sorted keys)."""

    def __init__(self, volume_descriptions: dict, models):
        self.models = list(models)
        self.keys = []  # (model name, key) per table index
        recs = []
        self.first = np.zeros(len(self.models), np.uint32)
        self.count = np.zeros(len(self.models), np.uint32)
        for m, name in enumerate(self.models):
            lods = volume_descriptions[name]
            self.first[m] = len(recs)
            for key in sorted(lods):
                d = lods[key]
                r = np.zeros((), N.LOD_VOLUME_DTYPE)
                r["voxel_size"] = float(key)
                r["bb_min"] = d["BBMin"]
                r["bb_max"] = d["BBMax"]
                r["num_voxels"] = d["NumVoxels"]
                r["corners"] = [d[f"P{k}"] for k in range(8)]
                recs.append(r)
                self.keys.append((name, key))
            self.count[m] = len(recs) - self.first[m]
        self.lods = np.array(recs, N.LOD_VOLUME_DTYPE) if recs else np.zeros(1, N.LOD_VOLUME_DTYPE)
        self.index = {name: m for m, name in enumerate(self.models)}


def select_lods(camera: dict, table: LodTable, tree_pos, tree_scaling, tree_model, min_lod: float = 0.1,
                covered_pixels: float = 1.0) -> np.ndarray:
    """LOD index per tree (into table.keys; -1: the mesh), on the GPU."""
    pos = np.ascontiguousarray(np.asarray(tree_pos, np.float64).reshape(-1, 3))
    sc = np.ascontiguousarray(np.asarray(tree_scaling, np.float64).reshape(-1))
    mdl = np.ascontiguousarray(np.asarray(tree_model, np.uint32).reshape(-1))
    n = len(sc)
    assert pos.shape[0] == n and mdl.shape[0] == n
    out = np.zeros(n, np.int32)
    N.check(N.lib.r2_select_lods(N.ptr(camera["native"]), N.ptr(table.lods), N.ptr(table.first),
                                 N.ptr(table.count), len(table.models), N.ptr(pos), N.ptr(sc), N.ptr(mdl), n,
                                 C.c_double(min_lod), C.c_double(covered_pixels), N.ptr(out)))
    return out


def _sample_circle(rs, radius):
    r = math.sqrt(rs.uniform()) * radius
    theta = 2 * math.pi * rs.uniform()
    return np.array([r * math.cos(theta), 0, r * math.sin(theta)])


def _sample_position(rs, relevant_models, index, bounds, radius):
    model = relevant_models[index]
    height = rs.normal(model["ExpectedHeight"], model["ExpectedHeight"] * 0.01)
    scaling = height / model["Dimensions"][1]
    circle = _sample_circle(rs, radius)
    bbmin = np.array(bounds[model["Name"]]["BBMin"])
    bbmax = np.array(bounds[model["Name"]]["BBMax"])
    pos = (2.0 * circle - scaling * (bbmin + bbmax)) * 0.5
    pos[1] = 0
    dims = scaling * (bbmax - bbmin)
    return {"Model": model, "Pos": pos, "BoundingCirclePos": circle, "Scaling": scaling,
            "BoundingRadius": math.sqrt((dims[0] / 2) ** 2 + (dims[2] / 2) ** 2)}


def _classes(p, radius):
    pos = p["BoundingCirclePos"]
    distance = np.sqrt(np.dot(pos, pos))
    upper = distance + p["BoundingRadius"]
    lower = distance - p["BoundingRadius"]
    sq = radius ** 2
    lo = int(ACCEL_CLASSES * lower ** 2 / sq)
    hi = int(ACCEL_CLASSES * upper ** 2 / sq)
    return list(range(lo, min(hi + 1, ACCEL_CLASSES)))


class _ClassSet:
    """Placed trees of one distance class: circle centres and radii."""

    def __init__(self):
        self.c = np.zeros((64, 3))
        self.r = np.zeros(64)
        self.n = 0

    def add(self, c, r):
        if self.n == len(self.r):
            self.c = np.concatenate([self.c, np.zeros_like(self.c)])
            self.r = np.concatenate([self.r, np.zeros_like(self.r)])
        self.c[self.n] = c
        self.r[self.n] = r
        self.n += 1

    def collides(self, c, r):
        # checkCollision: |c_i - c| <= r_i + r + 0.0001 (the generator takes the
        # length with np.dot, which may round the last bit of the sum differently)
        if self.n == 0:
            return False
        d = self.c[:self.n] - c
        dist = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
        return bool(np.any(dist <= self.r[:self.n] + r + 0.0001))


def place_trees(relevant_models: dict, volume_descriptions: dict, attempts: int = 100_000, seed: int = 0,
                radius: float = RADIUS) -> list:
    """Dart throwing of generateRandomForest (generate_random_forest.py:250-300):
    per attempt a size class (TREE_CDF), a model of the class, a height
    ~ N(expected, 1 %) and a disc position; kept unless its bounding circle
    meets one already placed in a distance class it overlaps."""
    rs = np.random.RandomState(seed)
    bounds = max_bounds(volume_descriptions)
    classes = [_ClassSet() for _ in range(ACCEL_CLASSES)]
    placed = []
    for _ in range(attempts):
        u = rs.uniform()
        group = "Large" if u < TREE_CDF[0] else ("Medium" if u < TREE_CDF[1] else "Small")
        models = relevant_models[group]
        index = int(rs.uniform() * len(models))
        p = _sample_position(rs, models, index, bounds, radius)
        cls = _classes(p, radius)
        if any(classes[k].collides(p["BoundingCirclePos"], p["BoundingRadius"]) for k in cls):
            continue
        placed.append(p)
        for k in cls:
            classes[k].add(p["BoundingCirclePos"], p["BoundingRadius"])
    return placed


def generate_forest(relevant_models: dict, volume_descriptions: dict, camera: dict, generate_gt: bool = False,
                    min_lod: float = 0.1, covered_pixels: float = 1.0, attempts: int = 100_000, seed: int = 0,
                    radius: float = RADIUS, assets_root: str = "../../raytracer/assets/",
                    filtering_root: str = "./filtering/", placed: list = None) -> list:
    """The forest as the generator's scene list: (type, directory, filename,
    pos, orientation, scaling) per tree, a Mesh for LOD "0" and a Medium for
    the others (getTreeDescription, generate_random_forest.py:19-46).
    `placed` (optional): the trees of an earlier place_trees call."""
    if placed is None:
        placed = place_trees(relevant_models, volume_descriptions, attempts, seed, radius)
    names = sorted({p["Model"]["Name"] for p in placed})
    table = LodTable(volume_descriptions, names)
    if generate_gt or not placed:
        choice = np.full(len(placed), -1, np.int32)
    else:
        choice = select_lods(camera, table, [p["Pos"] for p in placed], [p["Scaling"] for p in placed],
                             [table.index[p["Model"]["Name"]] for p in placed], min_lod, covered_pixels)
    scene = []
    for p, c in zip(placed, choice):
        model = p["Model"]
        s = p["Scaling"]
        if c < 0:
            scene.append(("Mesh", assets_root + model["Path"], model["Name"] + ".obj", tuple(p["Pos"]),
                          tuple(model["Orientation"]), (s, s, s)))
        else:
            scene.append(("Medium", filtering_root + model["Name"] + "/", "filtered_mesh_" + table.keys[c][1],
                          tuple(p["Pos"]), tuple(model["Orientation"]), (s, s, s)))
    return scene


def scene_objects(scene: list) -> list:
    """The scene list as scenedescription.json objects plus the ground disc
    (toFile, common_functions.py:69-106)."""
    out = []
    for kind, directory, filename, pos, ori, sc in scene:
        pos = [float(x) for x in pos]
        ori = [float(x) for x in ori]
        sc = [float(x) for x in sc]
        if kind == "Mesh":
            out.append({"Type": "Mesh", "Directory": directory, "Filename": filename, "Pos": pos,
                        "Orientation": ori, "Scaling": sc, "Mask": ["RENDER"]})
        else:
            out.append({"Type": "Medium", "Path": directory + "/" + filename, "SigmaA": [0.0, 0.0, 0.0],
                        "SigmaS": [10.0, 10.0, 10.0], "Pos": pos, "Orientation": ori, "Scaling": sc,
                        "Mask": ["RENDER"]})
    out.append({"Type": "Circle", "Pos": [0.0, 0.0, 0.0], "Radius": 3.402823466e+38, "Normal": [0.0, 1.0, 0.0],
                "DiffuseReflection": [0.07, 0.07, 0.01], "DiffuseRoughness": 0.999,
                "SpecularReflection": [0.9, 0.9, 0.9], "AlphaX": 0.99, "AlphaY": 0.99, "EtaI": 1.00029,
                "EtaT": 1.2})
    return out


def write_scene(scene: list, path) -> None:
    with open(path, "w") as f:
        json.dump(scene_objects(scene), f, indent=True)
