"""Many-instance forest scenes on the GPU: LOD selection and rendering.

The selection kernel (r2_select_lods) is checked against the reference
generator's own choices (tests/golden/forest_lod.json) and against the
oracle's restatement on 200,000 random trees.  Forest frames (a hundred
medium instances of three filtered tree models sharing their files, walked
through the instance BVH) are checked against the oracle, which tests every
medium box of every ray in instance order; the config path (the generator's
scene description) renders the same frame as the scene built call by call.
"""
import json
import os

import numpy as np
import pytest

import oracle_lib as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from renderer2_b200 import _native as N  # noqa: E402
from renderer2_b200 import forest as FO  # noqa: E402
from renderer2_b200 import pipeline as P  # noqa: E402
from renderer2_b200 import raytracer as R  # noqa: E402
from renderer2_b200 import render_scenes as RS  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "forest_lod.json")
PIX_REL = 1e-4
# a small forest (disc of radius 60) seen from its edge
NEAR_CAMERA = ((0.0, 14.0, 85.0), (0.0, 4.0, 0.0), (0.0, 1.0, 0.0), 60.0)


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _golden_inputs(g):
    table = FO.LodTable(g["volume_descriptions"], sorted(g["volume_descriptions"]))
    c = g["camera"]
    cam = FO.lod_camera(c["pos"], c["lookat"], c["up"], c["width"], c["height"], c["fov"])
    trees = g["selection"]["trees"]
    pos = np.array([t["pos"] for t in trees])
    sc = np.array([t["scaling"] for t in trees])
    mdl = np.array([table.index[t["model"]] for t in trees], np.uint32)
    return table, cam, pos, sc, mdl


def test_gpu_selection_matches_reference(golden):
    table, cam, pos, sc, mdl = _golden_inputs(golden)
    for (min_lod, cov), want in zip(golden["selection"]["settings"], golden["selection"]["choices"]):
        got = FO.select_lods(cam, table, pos, sc, mdl, min_lod, cov)
        assert ["0" if c < 0 else table.keys[c][1] for c in got] == want, (min_lod, cov)


def test_gpu_selection_matches_oracle_at_scale(golden):
    table, cam, _, _, _ = _golden_inputs(golden)
    rng = np.random.default_rng(17)
    n = 200_000
    eye = np.array(golden["camera"]["pos"])
    pos = eye + np.stack([rng.uniform(-1500, 1500, n), np.zeros(n), rng.uniform(-1500, 1500, n)], axis=1)
    pos[:, 1] = 0.0
    sc = rng.uniform(0.01, 0.2, n)
    mdl = rng.integers(0, len(table.models), n).astype(np.uint32)
    for min_lod, cov in [(0.1, 1.0), (0.0, 3.0)]:
        got = FO.select_lods(cam, table, pos, sc, mdl, min_lod, cov)
        want = O.select_lods(cam["native"], table.lods, table.first, table.count, pos, sc, mdl, min_lod, cov)
        assert np.array_equal(got, want)
        assert len(np.unique(got)) >= 10


def test_selection_argument_errors(golden):
    table, cam, pos, sc, mdl = _golden_inputs(golden)
    bad = mdl.copy()
    bad[3] = len(table.models)
    with pytest.raises(N.R2Error) as e:
        FO.select_lods(cam, table, pos, sc, bad)
    assert e.value.status == 1  # R2_ERR_INVALID_ARGUMENT
    assert len(FO.select_lods(cam, table, pos[:0], sc[:0], mdl[:0])) == 0


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    return RS.forest_library(tmp_path_factory.mktemp("forest"), n_quads=3000, grid=24, lods=3, filter_spv=16,
                             filter_iters=6)


@pytest.fixture(scope="module")
def trees(lib):
    return RS.forest_trees(lib, attempts=400, radius=60.0, width=48, height=32, camera=NEAR_CAMERA)


def _cam(w, h, camera=NEAR_CAMERA):
    pos, look, up, fov = camera
    return R.camera(w, h, fov, pos, look, up)


def _agree(g, o):
    tol = PIX_REL * np.maximum(1.0, np.abs(o))
    return np.all(np.abs(g - o) <= tol, axis=1).mean()


def test_forest_has_many_instances_and_lods(lib, trees):
    kinds = [t[0] for t in trees]
    assert kinds.count("Medium") > 40
    lods = {t[2] for t in trees if t[0] == "Medium"}
    assert len(lods) >= 2


@pytest.mark.parametrize("dda", [True, False])
def test_forest_frame_matches_oracle(lib, trees, dda):
    desc = RS.forest_desc(lib, trees, media_only=True)
    assert len(desc["media"]) > 40  # the instance BVH path
    cam = _cam(48, 32)
    sc = RS.build_scene(desc)
    g = sc.render(cam, R.params(2, 5, 7, brick_grid=dda)).reshape(-1, 3)
    sc.close()
    o = O.render(desc, cam, 2, 5, 7, flags=1 if dda else 0)
    assert np.isfinite(g).all()
    # paths take identical decisions; values differ by the rounding of the
    # transcendental functions in the environment lookup and the Oren-Nayar
    # ground (at most 2e-4 relative on this frame)
    frac = _agree(g, o)
    assert frac >= 0.99, f"only {frac:.4f} of pixels agree to 1e-4"
    assert np.all(np.abs(g - o) <= 1e-3 * np.maximum(1.0, np.abs(o)))


def test_forest_rounds_never_change_the_frame(lib, trees):
    """Paths crossing many tree boxes: the boundaries a bounce queues in rounds
    and those it walks in the last pass give the same frame."""
    desc = RS.forest_desc(lib, trees, media_only=True)
    cam = _cam(40, 28)
    prm = R.params(2, 6, 11, brick_grid=True)
    sc = RS.build_scene(desc)
    ref = sc.render(cam, prm)
    for rounds in (1, 3, 12, 32):
        sc.set_tuning(R.tuning(media_rounds=rounds, track_steps=3))
        assert np.array_equal(sc.render(cam, prm), ref), rounds
    sc.close()


def test_instances_of_one_path_share_the_first_coefficients(lib, trees):
    desc = RS.forest_desc(lib, trees, media_only=True)
    path = desc["media"][0][0]
    same = [i for i, m in enumerate(desc["media"]) if m[0] == path]
    assert len(same) >= 2
    cam = _cam(32, 24)

    def frame(d):
        sc = RS.build_scene(d)
        img = sc.render(cam, R.params(1, 4, 3, brick_grid=True))
        sc.close()
        return img

    ref = frame(desc)
    changed = dict(desc)
    changed["media"] = list(desc["media"])
    k = same[1]
    changed["media"][k] = (path, (0.0, 0.0, 0.0), (2.0, 2.0, 2.0)) + tuple(desc["media"][k][3:])
    assert np.array_equal(frame(changed), ref)  # later instances take the first load's coefficients
    first = dict(desc)
    first["media"] = list(desc["media"])
    first["media"][same[0]] = (path, (0.0, 0.0, 0.0), (2.0, 2.0, 2.0)) + tuple(desc["media"][same[0]][3:])
    assert not np.array_equal(frame(first), ref)


def test_forest_config_renders_the_scene(lib, trees, tmp_path):
    media_trees = [t for t in trees if t[0] == "Medium"]
    cfg_path = RS.forest_config(lib, media_trees, tmp_path, 40, 24, 2, camera=NEAR_CAMERA)
    cfg = P.Config(cfg_path)
    info = cfg.info()
    assert info.n_media == len(media_trees) and info.n_shapes == 1
    lin, _ = cfg.render(spp=2, max_depth=4, seed=1)
    cfg.close()
    desc = RS.forest_desc(lib, media_trees)
    desc["env"] = P.read_hdr(os.path.join(str(tmp_path), "forest_env.hdr"))
    sc = RS.build_scene(desc)
    ref = sc.render(_cam(40, 24), R.params(2, 4, 1, brick_grid=True))
    sc.close()
    assert np.array_equal(lin, ref)


def test_forest_config_with_mesh_trees(lib, tmp_path):
    """Trees close to the camera are meshes (LOD "0"); every mesh tree of a
    model shares one OBJ load."""
    trees = RS.forest_trees(lib, attempts=400, radius=60.0, width=320, height=200, min_lod=0.0,
                            covered_pixels=64.0, camera=NEAR_CAMERA)
    meshes = [t for t in trees if t[0] == "Mesh"]
    assert meshes, "no tree close enough for its mesh"
    cfg = P.Config(RS.forest_config(lib, trees, tmp_path, 40, 24, 1, camera=NEAR_CAMERA))
    info = cfg.info()
    assert info.n_meshes == len(meshes)
    assert info.n_triangles == sum(lib["meshes"][t[2][:-4]].ntris for t in meshes)
    lin, _ = cfg.render(spp=1, max_depth=3, seed=0)
    cfg.close()
    assert np.isfinite(lin).all() and lin.mean() > 0.0
