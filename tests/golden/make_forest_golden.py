"""Generates tests/golden/forest_lod.json with the reference's own forest generator.

Imports generate_random_forest.py and common_functions.py from the
reference tree (raytracer/src/filtering) and runs its functions on a
synthetic model library: the dart-throwing placement of generateRandomForest
for a bounded number of attempts (seed 0), and selectLOD for the placed trees
plus trees scattered in front of the camera, under several settings.  Run in
the build container, where the reference tree is mounted:

    python tests/golden/make_forest_golden.py [/path/to/reference/raytracer/src/filtering]

The JSON holds inputs and the reference's outputs; tests/test_forest_*.py
check the oracle, the placement restatement and the GPU selection against it
without needing the reference.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "forest_lod.json")

ATTEMPTS = 1500
SETTINGS = [(0.1, 1.0), (0.5, 4.0), (0.0, 0.25), (2.0, 1.0)]


def bounding_points(mn, mx):
    """P0..P7 in the order of CVolumeDescriptionManager::getBoundingPoints."""
    return [[mn[0], mn[1], mn[2]], [mx[0], mn[1], mn[2]], [mx[0], mn[1], mx[2]], [mn[0], mn[1], mx[2]],
            [mn[0], mx[1], mn[2]], [mx[0], mx[1], mn[2]], [mx[0], mx[1], mx[2]], [mn[0], mx[1], mx[2]]]


def synthetic_library():
    """Four models (sizes like the thesis' Xfrog plants, in model units) with
    LODs of doubling voxel size; one model's keys include "12.800000" so the
    string order of sorted(lods) differs from the numeric one."""
    rng = np.random.default_rng(11)
    specs = [("LA01", "Large", (64.0, 242.9, 65.9), 20.0, [0.5 * 2 ** k for k in range(6)]),
             ("LB02", "Large", (173.3, 222.6, 144.5), 20.5, [0.4 * 2 ** k for k in range(7)]),
             ("MC03", "Medium", (88.5, 120.0, 89.2), 8.0, [0.25 * 2 ** k for k in range(5)]),
             ("SD04", "Small", (30.0, 41.0, 28.0), 2.5, [0.1 * 2 ** k for k in range(4)])]
    relevant = {"Large": [], "Medium": [], "Small": []}
    volumes = {}
    for name, group, dims, height, sizes in specs:
        relevant[group].append({"Name": name, "Path": f"Synthetic/{name}/Models", "Dimensions": list(dims),
                                "ExpectedHeight": height, "Orientation": [0.0, 0.0, 1.0]})
        lods = {}
        for vs in sizes:
            # the filtered grid's box: the model box grown to whole voxels of the LOD
            ext = np.array(dims)
            mn = -0.5 * ext * np.array([1.0, 0.0, 1.0]) - rng.uniform(0.0, vs, 3)
            n = np.ceil((ext + rng.uniform(0.0, vs, 3)) / vs).astype(int)
            mx = mn + n * vs
            mn32 = [float(np.float32(x)) for x in mn]
            mx32 = [float(np.float32(x)) for x in mx]
            e = {"NumVoxels": [int(x) for x in n], "BBMin": mn32, "BBMax": mx32}
            for k, p in enumerate(bounding_points(mn32, mx32)):
                e[f"P{k}"] = p
            lods["%f" % vs] = e
        volumes[name] = dict(sorted(lods.items()))  # nlohmann::json writes keys in string order
    return relevant, volumes


def main(ref_dir: str) -> None:
    sys.path.insert(0, ref_dir)
    import generate_random_forest as G  # noqa: E402  (the reference's module)
    from common_functions import getCamera, getMaxBounds  # noqa: E402

    relevant, volumes = synthetic_library()
    cam_args = ([-680.0, 35.1, 680.0], [-675.0, 31.5, 675.0], [0.0, 1.0, 0.0], 1920, 1080, 90)
    camera = getCamera(*cam_args)
    bounds = getMaxBounds(volumes)

    # placement: the body of generateRandomForest for ATTEMPTS attempts
    np.random.seed(0)
    accel = [[] for _ in range(G.ACCEL_CLASSES)]
    placed = []
    tree_cdf = [0.9, 0.98, 1.0]
    for _ in range(ATTEMPTS):
        u = np.random.uniform()
        models = relevant["Large"] if u < tree_cdf[0] else (relevant["Medium"] if u < tree_cdf[1] else relevant["Small"])
        index = int(np.random.uniform() * len(models))
        p = G.sampleModelPosition(models, index, bounds)
        classes = G.getRelevantAccelerationClasses(p)
        collide = any(G.checkCollision(o, p) for c in classes for o in accel[c])
        if not collide:
            placed.append(p)
            for c in classes:
                accel[c].append(p)

    # selection inputs: the placed trees and trees in front of the camera
    rng = np.random.default_rng(5)
    trees = [{"model": p["Model"]["Name"], "pos": [float(x) for x in p["Pos"]], "scaling": float(p["Scaling"])}
             for p in placed]
    eye = np.array(cam_args[0])
    fwd = np.array(cam_args[1]) - eye
    fwd /= np.linalg.norm(fwd)
    side = np.cross(fwd, [0.0, 1.0, 0.0])
    side /= np.linalg.norm(side)
    names = [m["Name"] for g in relevant.values() for m in g]
    dims = {m["Name"]: m for g in relevant.values() for m in g}
    for _ in range(600):
        name = names[int(rng.integers(len(names)))]
        d = float(np.exp(rng.uniform(np.log(3.0), np.log(900.0))))
        lateral = float(rng.uniform(-1.2, 1.2)) * d
        back = -1.0 if rng.uniform() < 0.08 else 1.0
        pos = eye + back * fwd * d + side * lateral
        pos[1] = 0.0
        sc = dims[name]["ExpectedHeight"] * float(rng.uniform(0.9, 1.1)) / dims[name]["Dimensions"][1]
        trees.append({"model": name, "pos": [float(x) for x in pos], "scaling": float(sc)})
    choices = []
    for min_lod, cov in SETTINGS:
        choices.append([G.selectLOD(camera, np.array(t["pos"]), t["scaling"], volumes[t["model"]], False, min_lod, cov)
                        for t in trees])
    out = {
        "camera": {"pos": cam_args[0], "lookat": cam_args[1], "up": cam_args[2], "width": cam_args[3],
                   "height": cam_args[4], "fov": cam_args[5]},
        "relevant_models": relevant,
        "volume_descriptions": volumes,
        "placement": {"attempts": ATTEMPTS, "seed": 0,
                      "trees": [{"model": p["Model"]["Name"], "pos": [float(x) for x in p["Pos"]],
                                 "scaling": float(p["Scaling"]), "radius": float(p["BoundingRadius"]),
                                 "circle": [float(x) for x in p["BoundingCirclePos"]]} for p in placed]},
        "selection": {"trees": trees, "settings": [list(s) for s in SETTINGS], "choices": choices},
    }
    with open(OUT, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    counts = [{k: c.count(k) for k in sorted(set(c))} for c in choices]
    print(f"{len(placed)} placed of {ATTEMPTS}; {len(trees)} selection trees; {OUT}")
    for s, c in zip(SETTINGS, counts):
        print(s, c)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.environ["R2_REFERENCE_DIR"], "raytracer", "src",
                                                              "filtering"))
