"""Forest scenes on the CPU: the oracle's LOD selection and the placement
restatement against the reference generator's own outputs.

tests/golden/forest_lod.json was produced by tests/golden/make_forest_golden.py
from the reference's generate_random_forest.py: dart-throwing placement
(seed 0, 1,500 attempts) over a synthetic four-model library, and selectLOD
for 1,840 trees under four (min_lod, covered_pixels) settings.
"""
import json
import os

import numpy as np
import pytest

import oracle_lib as O
from renderer2_b200 import forest as FO

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "forest_lod.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _camera(g):
    c = g["camera"]
    return FO.lod_camera(c["pos"], c["lookat"], c["up"], c["width"], c["height"], c["fov"])


def _inputs(g, table):
    trees = g["selection"]["trees"]
    pos = np.array([t["pos"] for t in trees])
    sc = np.array([t["scaling"] for t in trees])
    mdl = np.array([table.index[t["model"]] for t in trees], np.uint32)
    return pos, sc, mdl


def _keys(table, choice):
    return ["0" if c < 0 else table.keys[c][1] for c in choice]


def test_golden_exercises_every_branch(golden):
    """Meshes, finest and coarsest LODs and trees outside the frustum all occur."""
    for choices in golden["selection"]["choices"]:
        assert choices.count("0") > 0
        assert len(set(choices)) >= 6
    assert len(golden["placement"]["trees"]) > 1000


def test_lod_table_walks_keys_in_string_order(golden):
    table = FO.LodTable(golden["volume_descriptions"], ["LB02"])
    keys = [k for _, k in table.keys]
    assert keys == sorted(keys)
    assert keys.index("12.800000") < keys.index("3.200000")  # string order, not numeric
    assert table.lods["voxel_size"].max() == pytest.approx(25.6)


def test_oracle_selection_matches_reference(golden):
    table = FO.LodTable(golden["volume_descriptions"], sorted(golden["volume_descriptions"]))
    cam = _camera(golden)
    pos, sc, mdl = _inputs(golden, table)
    for (min_lod, cov), want in zip(golden["selection"]["settings"], golden["selection"]["choices"]):
        got = O.select_lods(cam["native"], table.lods, table.first, table.count, pos, sc, mdl, min_lod, cov)
        assert _keys(table, got) == want, (min_lod, cov)


def test_camera_record_matches_generator(golden):
    cam = _camera(golden)
    rec = cam["native"][0]
    assert rec["near_plane_distance"] == pytest.approx(1920 * 1e-5 / 2.0)
    assert rec["pixel_area"] == 1.e-5 ** 2
    assert rec["far_scale"] == float(np.float32(1) + np.float32(2) * (np.float32(3) * np.finfo(np.float32).eps) /
                                     (np.float32(1) - np.float32(3) * np.finfo(np.float32).eps))
    w2v = rec["world_to_view"].reshape(4, 4)
    eye = np.array(golden["camera"]["pos"] + [1.0])
    assert np.allclose(w2v @ eye, [0, 0, 0, 1], atol=1e-9)


def test_placement_matches_reference(golden):
    placed = FO.place_trees(golden["relevant_models"], golden["volume_descriptions"],
                            golden["placement"]["attempts"], golden["placement"]["seed"])
    want = golden["placement"]["trees"]
    assert len(placed) == len(want)
    for p, w in zip(placed, want):
        assert p["Model"]["Name"] == w["model"]
        assert [float(x) for x in p["Pos"]] == w["pos"]
        assert float(p["Scaling"]) == w["scaling"]
        assert float(p["BoundingRadius"]) == w["radius"]
        assert [float(x) for x in p["BoundingCirclePos"]] == w["circle"]


def test_placement_keeps_circles_apart(golden):
    placed = FO.place_trees(golden["relevant_models"], golden["volume_descriptions"], 600, 3, radius=300.0)
    c = np.array([p["BoundingCirclePos"] for p in placed])
    r = np.array([p["BoundingRadius"] for p in placed])
    d = np.sqrt(((c[:, None, :] - c[None, :, :]) ** 2).sum(-1))
    close = d <= r[:, None] + r[None, :] + 0.0001
    np.fill_diagonal(close, False)
    # the distance classes only test neighbours in overlapping annuli; trees
    # in one class never overlap
    assert close.sum() <= 0.02 * len(placed) ** 2
    assert len(placed) > 100


def test_scene_objects_have_generator_format(golden):
    scene = [("Mesh", "../../raytracer/assets/Synthetic/LA01/Models", "LA01.obj", (1.0, 0.0, 2.0),
              (0.0, 0.0, 1.0), (0.1, 0.1, 0.1)),
             ("Medium", "./filtering/LA01/", "filtered_mesh_1.000000", (3.0, 0.0, 4.0), (0.0, 0.0, 1.0),
              (0.1, 0.1, 0.1))]
    objs = FO.scene_objects(scene)
    assert objs[0]["Type"] == "Mesh" and objs[0]["Filename"] == "LA01.obj" and objs[0]["Mask"] == ["RENDER"]
    assert objs[1]["Type"] == "Medium" and objs[1]["Path"] == "./filtering/LA01//filtered_mesh_1.000000"
    assert objs[1]["SigmaS"] == [10.0, 10.0, 10.0]
    assert objs[-1]["Type"] == "Circle" and objs[-1]["Radius"] == 3.402823466e+38
