"""Two-level scenes on the GPU: instanced mesh assets (top-level BVH over the
instances, bottom-level BVH per asset, rays taken to object space) against
the oracle's two-level scene with the same random streams."""
import numpy as np
import pytest

import oracle_lib as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from renderer2_b200 import raytracer as R  # noqa: E402
from renderer2_b200 import render_scenes as RS  # noqa: E402


def _agree(g, o, tol=1e-4):
    return (np.abs(g - o) <= tol * np.maximum(1.0, np.abs(o))).all(axis=1).mean()


@pytest.mark.parametrize("method", [R.BVH_PLOC, R.BVH_KARRAS], ids=["ploc", "karras"])
def test_instanced_scene_matches_oracle(method):
    R.set_bvh_method(method)
    O.lib.orc_set_bvh_method(method)
    try:
        desc, cam = RS.instanced_scene(3, 64, 64)
        sc = RS.build_scene(desc)
        nodes, height, launches = sc.bvh_info()
        g = sc.render(cam, R.params(4, 6, 3)).reshape(-1, 3)
        sc.close()
        o = O.render(desc, cam, 4, 6, 3)
    finally:
        R.set_bvh_method(R.BVH_AUTO)
        O.lib.orc_set_bvh_method(-1)
    frac = _agree(g, o)
    print(f"two-level ({nodes} nodes, height {height}, {launches} build launches): {frac:.5f} of pixels within 1e-4")
    assert frac >= 0.999
    assert np.abs(g.mean(0) - o.mean(0)).max() < 1e-5 * max(1.0, np.abs(o.mean(0)).max())


def test_instances_only_and_many_instances():
    """No world-space meshes (instances only), 49 instances of one asset, a shadowing disc."""
    desc, cam = RS.instanced_scene(7, 48, 48)
    desc = dict(desc, meshes=desc["meshes"][:49])
    sc = RS.build_scene(desc)
    g = sc.render(cam, R.params(4, 5, 11)).reshape(-1, 3)
    sc.close()
    o = O.render(desc, cam, 4, 5, 11)
    assert _agree(g, o) >= 0.999


def test_instanced_rebuild_and_tuning_invariance():
    """r2_scene_rebuild of a two-level scene and the launch tuning change no bit of the frame."""
    desc, cam = RS.instanced_scene(3, 48, 48)
    sc = RS.build_scene(desc)
    prm = R.params(4, 6, 9)
    a = sc.render(cam, prm)
    sc.rebuild()
    b = sc.render(cam, prm)
    sc.set_tuning(R.tuning(0, 7, 3, 4096))
    c = sc.render(cam, prm)
    sc.close()
    assert np.array_equal(a, b) and np.array_equal(a, c)
